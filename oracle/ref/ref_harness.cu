// TEST INFRASTRUCTURE ONLY -- a C-ABI harness around the REFERENCE's own
// GPU code, compiled from the reference sources where they lie (see
// oracle/Makefile, target `ref`) into oracle/_ref/libref_proposal.so.
//
// It lets tests/ and the golden-vector script run, on a B200, exactly what the
// reference's apps run:
//   - proposal::proposal_inner<T, Parameters<CC80>>   (src/libproposal/include/proposal/proposal.cuh:26-80)
//     The reference's dispatcher proposal::proposal() throws on CC 10.0
//     (proposal.cuh:108-123); CC80 is its largest parameter table
//     (<= 166,912 B of shared memory per block, which fits sm_100a).
//   - cusparse2<T>   (src/libcusparse/include/cusparse/cusparse.cuh:171-351),
//     the reference's `validate` oracle (src/apps/common.hpp:116-120).
//   - utils::get_nip (src/libutils/include/utils/nip.cuh:52-78).
// Timing follows the reference's `measure` lambda (src/apps/proposal.cu:28-35):
// steady_clock around the call plus cudaDeviceSynchronize; C is freed after
// the clock stops.
//
// Nothing here is part of the product; the product library never links it.

#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>

#include <proposal/proposal.cuh>
#include <cusparse/cusparse.cuh>
#include <utils/utils.cuh>

namespace {

thread_local std::string g_err;

template<typename T>
utils::HostCSR<T> make_host(int32_t m, int32_t n, int32_t nnz, const int32_t* rpt,
                            const int32_t* col, const T* val) {
    utils::HostCSR<T> h(nnz, m, n);
    std::memcpy(h.rpt, rpt, sizeof(int32_t) * (m + 1));
    std::memcpy(h.col, col, sizeof(int32_t) * nnz);
    std::memcpy(h.val, val, sizeof(T) * nnz);
    return h;
}

template<typename T>
void export_host(const utils::HostCSR<T>& c, int32_t* out_dims, int32_t** rpt, int32_t** col,
                 T** val) {
    out_dims[0] = c.m;
    out_dims[1] = c.n;
    out_dims[2] = c.nnz;
    *rpt = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (c.m + 1)));
    *col = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (c.nnz > 0 ? c.nnz : 1)));
    *val = static_cast<T*>(std::malloc(sizeof(T) * (c.nnz > 0 ? c.nnz : 1)));
    std::memcpy(*rpt, c.rpt, sizeof(int32_t) * (c.m + 1));
    std::memcpy(*col, c.col, sizeof(int32_t) * c.nnz);
    std::memcpy(*val, c.val, sizeof(T) * c.nnz);
}

template<typename T>
int run(int which, int32_t am, int32_t an, int32_t annz, const int32_t* arpt,
        const int32_t* acol, const T* aval, int32_t bm, int32_t bn, int32_t bnnz,
        const int32_t* brpt, const int32_t* bcol, const T* bval, int32_t* out_dims,
        int32_t** crpt, int32_t** ccol, T** cval) {
    try {
        const auto ha = make_host<T>(am, an, annz, arpt, acol, aval);
        const auto hb = make_host<T>(bm, bn, bnnz, brpt, bcol, bval);
        const auto da = ha.template to<utils::Location::Device>();
        const auto db = hb.template to<utils::Location::Device>();
        if (which == 0) {
            auto dc = proposal::proposal_inner<T, proposal::Parameters<proposal::CC80>>(da, db);
            utils::device_sync();
            export_host(dc.template to<utils::Location::Host>(), out_dims, crpt, ccol, cval);
        } else {
            auto dc = cusparse2<T>(da, db);
            utils::device_sync();
            export_host(dc.template to<utils::Location::Host>(), out_dims, crpt, ccol, cval);
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

template<typename T>
int time_calls(int which, int32_t am, int32_t an, int32_t annz, const int32_t* arpt,
               const int32_t* acol, const T* aval, int32_t bm, int32_t bn, int32_t bnnz,
               const int32_t* brpt, const int32_t* bcol, const T* bval, int warmups,
               int runs, double* seconds, int64_t* nip_out) {
    using Clock = std::chrono::steady_clock;
    try {
        const auto ha = make_host<T>(am, an, annz, arpt, acol, aval);
        const auto hb = make_host<T>(bm, bn, bnnz, brpt, bcol, bval);
        const auto da = ha.template to<utils::Location::Device>();
        const auto db = hb.template to<utils::Location::Device>();
        // the clock stops before C is destroyed, as in the app's measure
        // lambda, where C lives until the lambda returns
        auto once = [&]() -> double {
            Clock::time_point t0;
            Clock::time_point t1;
            if (which == 0) {
                t0 = Clock::now();
                auto c = proposal::proposal_inner<T, proposal::Parameters<proposal::CC80>>(da, db);
                utils::device_sync();
                t1 = Clock::now();
            } else {
                t0 = Clock::now();
                auto c = cusparse2<T>(da, db);
                utils::device_sync();
                t1 = Clock::now();
            }
            return std::chrono::duration<double>(t1 - t0).count();
        };
        for (int i = 0; i < warmups; i++) once();
        for (int i = 0; i < runs; i++) seconds[i] = once();
        if (nip_out) *nip_out = utils::get_nip(da, db);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

} // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

void ref_free(void* p) { std::free(p); }

#define REF_ARGS(T)                                                                      \
    int32_t am, int32_t an, int32_t annz, const int32_t *arpt, const int32_t *acol,      \
        const T *aval, int32_t bm, int32_t bn, int32_t bnnz, const int32_t *brpt,        \
        const int32_t *bcol, const T *bval
#define REF_FWD am, an, annz, arpt, acol, aval, bm, bn, bnnz, brpt, bcol, bval

int ref_proposal_f64(REF_ARGS(double), int32_t* out_dims, int32_t** crpt, int32_t** ccol,
                     double** cval) {
    return run<double>(0, REF_FWD, out_dims, crpt, ccol, cval);
}
int ref_proposal_f32(REF_ARGS(float), int32_t* out_dims, int32_t** crpt, int32_t** ccol,
                     float** cval) {
    return run<float>(0, REF_FWD, out_dims, crpt, ccol, cval);
}
int ref_cusparse2_f64(REF_ARGS(double), int32_t* out_dims, int32_t** crpt, int32_t** ccol,
                      double** cval) {
    return run<double>(1, REF_FWD, out_dims, crpt, ccol, cval);
}
int ref_cusparse2_f32(REF_ARGS(float), int32_t* out_dims, int32_t** crpt, int32_t** ccol,
                      float** cval) {
    return run<float>(1, REF_FWD, out_dims, crpt, ccol, cval);
}
int ref_time_f64(int which, REF_ARGS(double), int warmups, int runs, double* seconds,
                 int64_t* nip) {
    return time_calls<double>(which, REF_FWD, warmups, runs, seconds, nip);
}
int ref_time_f32(int which, REF_ARGS(float), int warmups, int runs, double* seconds,
                 int64_t* nip) {
    return time_calls<float>(which, REF_FWD, warmups, runs, seconds, nip);
}

} // extern "C"
