// TEST INFRASTRUCTURE ONLY -- a C-ABI harness around the REFERENCE's vendored
// OpSparse (src/libopsparse), compiled from the reference sources where they
// lie (see oracle/Makefile, target `opsparse`) into
// oracle/_ref/libref_opsparse_{f64,f32}.so: one precision per library, as the
// reference builds it (USE_DOUBLE_PRECISION selects `mdouble`,
// src/libopsparse/include/opsparse/cuda_common.h).
//
// It runs what the reference's `opsparse` app runs (src/apps/opsparse.cu:24-44):
// operands uploaded with CSR::H2D, then `opsparse(A, B, C, meta, timing)`.
// Timing follows that app's `measure` lambda: steady_clock around one call
// plus a device synchronize; C is destroyed after the clock stops.
//
// Nothing here is part of the product; the product library never links it.

#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>

#include <opsparse/opsparse.h>

namespace {

thread_local std::string g_err;

// Fill a CSR the way the app's conversion does (conversion.cuh:7-21): host
// arrays owned by the CSR (released by its destructor), then H2D.
void fill(CSR& a, int32_t m, int32_t n, int32_t nnz, const int32_t* rpt, const int32_t* col,
          const mdouble* val) {
    a.M = m;
    a.N = n;
    a.nnz = nnz;
    a.rpt = new mint[m + 1];
    a.col = new mint[nnz > 0 ? nnz : 1];
    a.val = new mdouble[nnz > 0 ? nnz : 1];
    std::memcpy(a.rpt, rpt, sizeof(mint) * (m + 1));
    std::memcpy(a.col, col, sizeof(mint) * nnz);
    std::memcpy(a.val, val, sizeof(mdouble) * nnz);
    a.H2D();
}

}  // namespace

extern "C" {

const char* ops_last_error(void) { return g_err.c_str(); }

int ops_value_bytes(void) { return static_cast<int>(sizeof(mdouble)); }

void ops_free(void* p) { std::free(p); }

// C = A * B through OpSparse; C's arrays are malloc'd here (free with ops_free).
int ops_run(int32_t am, int32_t an, int32_t annz, const int32_t* arpt, const int32_t* acol,
            const mdouble* aval, int32_t bm, int32_t bn, int32_t bnnz, const int32_t* brpt,
            const int32_t* bcol, const mdouble* bval, int32_t* out_dims, int32_t** crpt,
            int32_t** ccol, mdouble** cval) {
    try {
        CSR A;
        CSR B;
        fill(A, am, an, annz, arpt, acol, aval);
        fill(B, bm, bn, bnnz, brpt, bcol, bval);
        CSR C;
        Meta meta;
        Timings timing;
        opsparse(A, B, C, meta, timing);
        C.D2H();
        out_dims[0] = C.M;
        out_dims[1] = C.N;
        out_dims[2] = C.nnz;
        *crpt = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (C.M + 1)));
        *ccol = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (C.nnz > 0 ? C.nnz : 1)));
        *cval = static_cast<mdouble*>(std::malloc(sizeof(mdouble) * (C.nnz > 0 ? C.nnz : 1)));
        std::memcpy(*crpt, C.rpt, sizeof(int32_t) * (C.M + 1));
        std::memcpy(*ccol, C.col, sizeof(int32_t) * C.nnz);
        std::memcpy(*cval, C.val, sizeof(mdouble) * C.nnz);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// Wall-clock seconds of `runs` calls after `warmups`, as the app's measure
// lambda takes them.
int ops_time(int32_t am, int32_t an, int32_t annz, const int32_t* arpt, const int32_t* acol,
             const mdouble* aval, int32_t bm, int32_t bn, int32_t bnnz, const int32_t* brpt,
             const int32_t* bcol, const mdouble* bval, int warmups, int runs, double* seconds) {
    using Clock = std::chrono::steady_clock;
    try {
        CSR A;
        CSR B;
        fill(A, am, an, annz, arpt, acol, aval);
        fill(B, bm, bn, bnnz, brpt, bcol, bval);
        // the clock stops before C is destroyed (it lives until the app's
        // measure lambda returns)
        auto once = [&]() -> double {
            const auto t0 = Clock::now();
            CSR C;
            Meta meta;
            Timings timing;
            opsparse(A, B, C, meta, timing);
            if (cudaDeviceSynchronize() != cudaSuccess) throw std::exception();
            return std::chrono::duration<double>(Clock::now() - t0).count();
        };
        for (int i = 0; i < warmups; i++) once();
        for (int i = 0; i < runs; i++) seconds[i] = once();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

}  // extern "C"
