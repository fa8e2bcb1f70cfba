// Command-line driver with the reference apps' interface
// (src/apps/common.hpp:22-208 run_app, src/apps/proposal.cu), running the
// B200 library through its C++ drop-in (b200_proposal.hpp):
//
//   spgemm_app inputA inputB [--loglevel L] validate
//   spgemm_app inputA inputB [--loglevel L] save OUTPUT
//   spgemm_app inputA inputB [--loglevel L] benchmark [--runs N] [--warmups N] [--pause MS]
//
// Output lines match the reference's, so its tasks.py parser
// (`Run\s+(\d+): (.+)ns [|] (\d+[.]\d*) FLOPS`, tasks.py:104-107) reads them:
//   validate:  "Validation succeeded" / "Validation failed" + sizes   (common.hpp:123-135)
//   save:      "Saving result to <out>"                              (common.hpp:144)
//   benchmark: "A: m x n (nnz non-zero elements)", "B: ...", "NIP: ...", "C: ...",
//              "Run  i: <t>ns | <flops> FLOPS"                       (common.hpp:196-204)
// validate compares against cuSPARSE SpGEMM ALG2 with the reference's
// tolerance (structure equal; |l-r| <= 1e-8 + 1e-5 max(|l|,|r|), csr.cuh:218-239).
// Precision is chosen at build time like the reference (USE_DOUBLE_PRECISION).
#include <cuda_runtime.h>
#include <cusparse.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "b200_proposal.hpp"

#ifdef USE_DOUBLE_PRECISION
using Value = double;
#else
using Value = float;
#endif

namespace {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw std::runtime_error(std::string("CUDA error (") + what + "): " + cudaGetErrorString(e));
}

void sparse_check(cusparseStatus_t e, const char* what) {
    if (e != CUSPARSE_STATUS_SUCCESS)
        throw std::runtime_error(std::string("cuSPARSE error (") + what +
                                 "): " + cusparseGetErrorString(e));
}

struct HostCSR {
    int32_t nnz = 0, m = 0, n = 0;
    std::vector<int32_t> rpt, col;
    std::vector<Value> val;
};

// Device CSR with the layout and ownership of utils::CSR<T, Location::Device>
// (csr.cuh:22-63): public nnz/m/n/rpt/col/val, arrays released by cudaFree.
struct DeviceCSR {
    int32_t nnz = 0, m = 0, n = 0;
    int32_t* rpt = nullptr;
    int32_t* col = nullptr;
    Value* val = nullptr;
    DeviceCSR() = default;
    DeviceCSR(const DeviceCSR&) = delete;
    DeviceCSR& operator=(const DeviceCSR&) = delete;
    DeviceCSR(DeviceCSR&& o) noexcept { *this = std::move(o); }
    DeviceCSR& operator=(DeviceCSR&& o) noexcept {
        std::swap(nnz, o.nnz);
        std::swap(m, o.m);
        std::swap(n, o.n);
        std::swap(rpt, o.rpt);
        std::swap(col, o.col);
        std::swap(val, o.val);
        return *this;
    }
    ~DeviceCSR() {
        cudaFree(rpt);
        cudaFree(col);
        cudaFree(val);
    }
};

HostCSR load(const std::string& path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error("Failed to open file " + path);
    const auto size = static_cast<long long>(f.tellg());
    if (size < 12) throw std::runtime_error("File " + path + " is too small");
    f.seekg(0);
    HostCSR h;
    int32_t hdr[3];
    f.read(reinterpret_cast<char*>(hdr), sizeof hdr);
    h.nnz = hdr[0];
    h.m = hdr[1];
    h.n = hdr[2];
    const long long expect = 12 + 4LL * (h.m + 1) + 12LL * h.nnz;
    if (size < expect) throw std::runtime_error("Failed to read file " + path);
    if (size > expect) throw std::runtime_error("File " + path + " is too large");
    h.rpt.resize(h.m + 1);
    h.col.resize(h.nnz);
    std::vector<double> v(h.nnz);
    f.read(reinterpret_cast<char*>(h.rpt.data()), 4LL * (h.m + 1));
    f.read(reinterpret_cast<char*>(h.col.data()), 4LL * h.nnz);
    f.read(reinterpret_cast<char*>(v.data()), 8LL * h.nnz);
    if (!f) throw std::runtime_error("Failed to read file " + path);
    h.val.assign(v.begin(), v.end());  // values are always double on disk
    return h;
}

void save(const std::string& path, const HostCSR& h) {
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("Failed to open file " + path);
    const int32_t hdr[3] = {h.nnz, h.m, h.n};
    std::vector<double> v(h.val.begin(), h.val.end());
    f.write(reinterpret_cast<const char*>(hdr), sizeof hdr);
    f.write(reinterpret_cast<const char*>(h.rpt.data()), 4LL * (h.m + 1));
    f.write(reinterpret_cast<const char*>(h.col.data()), 4LL * h.nnz);
    f.write(reinterpret_cast<const char*>(v.data()), 8LL * h.nnz);
    if (!f) throw std::runtime_error("Failed to write to file");
}

DeviceCSR to_device(const HostCSR& h) {
    DeviceCSR d;
    d.nnz = h.nnz;
    d.m = h.m;
    d.n = h.n;
    cuda_check(cudaMalloc(&d.rpt, 4 * (size_t(h.m) + 1)), "malloc");
    cuda_check(cudaMalloc(&d.col, 4 * std::max<size_t>(h.nnz, 1)), "malloc");
    cuda_check(cudaMalloc(&d.val, sizeof(Value) * std::max<size_t>(h.nnz, 1)), "malloc");
    cuda_check(cudaMemcpy(d.rpt, h.rpt.data(), 4 * (size_t(h.m) + 1), cudaMemcpyHostToDevice), "copy");
    cuda_check(cudaMemcpy(d.col, h.col.data(), 4 * size_t(h.nnz), cudaMemcpyHostToDevice), "copy");
    cuda_check(cudaMemcpy(d.val, h.val.data(), sizeof(Value) * h.nnz, cudaMemcpyHostToDevice), "copy");
    return d;
}

HostCSR to_host(const DeviceCSR& d) {
    HostCSR h;
    h.nnz = d.nnz;
    h.m = d.m;
    h.n = d.n;
    h.rpt.resize(d.m + 1);
    h.col.resize(d.nnz);
    h.val.resize(d.nnz);
    cuda_check(cudaMemcpy(h.rpt.data(), d.rpt, 4 * (size_t(d.m) + 1), cudaMemcpyDeviceToHost), "copy");
    if (d.nnz > 0) {
        cuda_check(cudaMemcpy(h.col.data(), d.col, 4 * size_t(d.nnz), cudaMemcpyDeviceToHost), "copy");
        cuda_check(cudaMemcpy(h.val.data(), d.val, sizeof(Value) * d.nnz, cudaMemcpyDeviceToHost), "copy");
    }
    return h;
}

// cuSPARSE SpGEMM, ALG2: workEstimation -> estimateMemory -> compute -> copy;
// the reference's validation oracle is the same library call sequence
// (src/libcusparse/include/cusparse/cusparse.cuh:171-351).
DeviceCSR cusparse_alg2(const DeviceCSR& a, const DeviceCSR& b) {
    constexpr cudaDataType DT = sizeof(Value) == 8 ? CUDA_R_64F : CUDA_R_32F;
    const Value alpha = 1, beta = 0;
    cusparseHandle_t handle;
    sparse_check(cusparseCreate(&handle), "create");
    cusparseSpMatDescr_t da, db, dc;
    sparse_check(cusparseCreateCsr(&da, a.m, a.n, a.nnz, a.rpt, a.col, a.val, CUSPARSE_INDEX_32I,
                                   CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, DT), "csr A");
    sparse_check(cusparseCreateCsr(&db, b.m, b.n, b.nnz, b.rpt, b.col, b.val, CUSPARSE_INDEX_32I,
                                   CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, DT), "csr B");
    sparse_check(cusparseCreateCsr(&dc, a.m, b.n, 0, nullptr, nullptr, nullptr, CUSPARSE_INDEX_32I,
                                   CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, DT), "csr C");
    cusparseSpGEMMDescr_t sd;
    sparse_check(cusparseSpGEMM_createDescr(&sd), "descr");
    const auto op = CUSPARSE_OPERATION_NON_TRANSPOSE;
    const auto alg = CUSPARSE_SPGEMM_ALG2;
    size_t s1 = 0, s2 = 0, s3 = 0;
    void *b1 = nullptr, *b2 = nullptr, *b3 = nullptr;
    sparse_check(cusparseSpGEMM_workEstimation(handle, op, op, &alpha, da, db, &beta, dc, DT, alg,
                                               sd, &s1, nullptr), "work 1");
    cuda_check(cudaMalloc(&b1, s1), "malloc");
    sparse_check(cusparseSpGEMM_workEstimation(handle, op, op, &alpha, da, db, &beta, dc, DT, alg,
                                               sd, &s1, b1), "work 2");
    sparse_check(cusparseSpGEMM_estimateMemory(handle, op, op, &alpha, da, db, &beta, dc, DT, alg,
                                               sd, 0.2f, &s3, nullptr, nullptr), "estimate 1");
    cuda_check(cudaMalloc(&b3, s3), "malloc");
    sparse_check(cusparseSpGEMM_estimateMemory(handle, op, op, &alpha, da, db, &beta, dc, DT, alg,
                                               sd, 0.2f, &s3, b3, &s2), "estimate 2");
    cudaFree(b3);
    cuda_check(cudaMalloc(&b2, s2), "malloc");
    sparse_check(cusparseSpGEMM_compute(handle, op, op, &alpha, da, db, &beta, dc, DT, alg, sd,
                                        &s2, b2), "compute");
    int64_t m64, n64, nnz64;
    sparse_check(cusparseSpMatGetSize(dc, &m64, &n64, &nnz64), "size");
    DeviceCSR c;
    c.m = a.m;
    c.n = b.n;
    c.nnz = static_cast<int32_t>(nnz64);
    cuda_check(cudaMalloc(&c.rpt, 4 * (size_t(c.m) + 1)), "malloc");
    cuda_check(cudaMalloc(&c.col, 4 * std::max<size_t>(c.nnz, 1)), "malloc");
    cuda_check(cudaMalloc(&c.val, sizeof(Value) * std::max<size_t>(c.nnz, 1)), "malloc");
    sparse_check(cusparseCsrSetPointers(dc, c.rpt, c.col, c.val), "set");
    sparse_check(cusparseSpGEMM_copy(handle, op, op, &alpha, da, db, &beta, dc, DT, alg, sd),
                 "copy");
    cuda_check(cudaDeviceSynchronize(), "sync");
    cusparseSpGEMM_destroyDescr(sd);
    cusparseDestroySpMat(da);
    cusparseDestroySpMat(db);
    cusparseDestroySpMat(dc);
    cusparseDestroy(handle);
    cudaFree(b1);
    cudaFree(b2);
    return c;
}

bool reference_equal(const HostCSR& l, const HostCSR& r) {
    if (l.nnz != r.nnz || l.m != r.m || l.n != r.n) return false;
    if (l.rpt != r.rpt || l.col != r.col) return false;
    for (int32_t i = 0; i < l.nnz; i++) {
        const Value x = l.val[i], y = r.val[i];
        if (x == y) continue;
        if (!(std::fabs(x - y) <= Value(1e-8) + Value(1e-5) * std::max(std::fabs(x), std::fabs(y))))
            return false;
    }
    return true;
}

struct Args {
    std::string a, b, sub, output, loglevel = "info";
    int runs = 1, warmups = 0, pause = 50;
};

[[noreturn]] void usage(const char* prog, const std::string& msg) {
    std::fprintf(stderr,
                 "%s\nUsage: %s inputA inputB [--loglevel L] {validate | save OUTPUT | "
                 "benchmark [--runs N] [--warmups N] [--pause MS]}\n",
                 msg.c_str(), prog);
    std::exit(EXIT_FAILURE);
}

int to_nonneg(const char* prog, const std::string& opt, const std::string& v) {
    char* end = nullptr;
    const long x = std::strtol(v.c_str(), &end, 10);
    if (end == v.c_str() || *end != '\0' || x < 0) usage(prog, opt + ": not a non-negative number");
    return static_cast<int>(x);
}

Args parse(int argc, char** argv) {
    Args a;
    std::vector<std::string> pos;
    for (int i = 1; i < argc; i++) {
        std::string t = argv[i];
        std::string val;
        const auto eq = t.find('=');
        const bool is_opt = t.rfind("--", 0) == 0;
        if (is_opt && eq != std::string::npos) {
            val = t.substr(eq + 1);
            t = t.substr(0, eq);
        } else if (is_opt) {
            if (i + 1 >= argc) usage(argv[0], t + " needs a value");
            val = argv[++i];
        }
        if (t == "--loglevel") {
            a.loglevel = val;
        } else if (t == "--runs") {
            a.runs = to_nonneg(argv[0], t, val);
        } else if (t == "--warmups") {
            a.warmups = to_nonneg(argv[0], t, val);
        } else if (t == "--pause") {
            a.pause = to_nonneg(argv[0], t, val);
        } else if (is_opt) {
            usage(argv[0], "unknown option " + t);
        } else {
            pos.push_back(t);
        }
    }
    if (pos.size() < 3) usage(argv[0], "inputA, inputB and a subcommand are required");
    a.a = pos[0];
    a.b = pos[1];
    a.sub = pos[2];
    if (a.sub == "save") {
        if (pos.size() != 4) usage(argv[0], "save needs an output path");
        a.output = pos[3];
    } else if ((a.sub == "validate" || a.sub == "benchmark") && pos.size() == 3) {
    } else {
        usage(argv[0], "exactly one subcommand: validate, save or benchmark");
    }
    for (const std::string& p : {a.a, a.b})
        if (!std::ifstream(p)) usage(argv[0], "File does not exist: " + p);
    return a;
}

int run(int argc, char** argv) {
    using Clock = std::chrono::steady_clock;
    const Args args = parse(argc, argv);
    const HostCSR ha = load(args.a);
    const HostCSR hb = load(args.b);
    if (ha.n != hb.m) {
        std::fprintf(stderr, "Matrix A columns (%d) must match matrix B rows (%d)\n", ha.n, hb.m);
        return EXIT_FAILURE;
    }
    if (args.sub == "validate") {
        HostCSR hc, hr;
        {
            const DeviceCSR da = to_device(ha), db = to_device(hb);
            hc = to_host(b200::proposal(da, db));
        }
        {
            const DeviceCSR da = to_device(ha), db = to_device(hb);
            hr = to_host(cusparse_alg2(da, db));
        }
        if (reference_equal(hc, hr)) {
            std::printf("Validation succeeded\n");
        } else {
            std::printf("Validation failed\n");
            std::printf("Matrix C: %d x %d (%d non-zero elements)\n", hc.m, hc.n, hc.nnz);
            std::printf("Matrix C (cuSPARSE): %d x %d (%d non-zero elements)\n", hr.m, hr.n, hr.nnz);
        }
    }
    if (args.sub == "save") {
        std::printf("Saving result to %s\n", args.output.c_str());
        const DeviceCSR da = to_device(ha), db = to_device(hb);
        save(args.output, to_host(b200::proposal(da, db)));
    }
    if (args.sub == "benchmark") {
        const DeviceCSR da = to_device(ha), db = to_device(hb);
        const auto pause = std::chrono::milliseconds(args.pause);
        auto measure = [&]() {
            const auto t0 = Clock::now();
            { auto c = b200::proposal(da, db); }
            cuda_check(cudaDeviceSynchronize(), "sync");
            return Clock::now() - t0;
        };
        for (int i = 0; i < args.warmups; i++) {
            std::this_thread::sleep_for(pause);
            measure();
        }
        std::vector<Clock::duration> times(args.runs);
        for (int i = 0; i < args.runs; i++) {
            std::this_thread::sleep_for(pause);
            times[i] = measure();
        }
        const long long nip = b200::get_nip(da, db);
        const double flop = 2.0 * static_cast<double>(nip);
        const DeviceCSR c = b200::proposal(da, db);
        std::printf("A: %d x %d (%d non-zero elements)\n", ha.m, ha.n, ha.nnz);
        std::printf("B: %d x %d (%d non-zero elements)\n", hb.m, hb.n, hb.nnz);
        std::printf("NIP: %lld\n", nip);
        std::printf("C: %d x %d (%d non-zero elements)\n", c.m, c.n, c.nnz);
        for (int i = 0; i < args.runs; i++) {
            const double secs = std::chrono::duration<double>(times[i]).count();
            const long long ns = std::chrono::duration_cast<std::chrono::nanoseconds>(times[i]).count();
            std::printf("Run %2d: %lldns | %.3f FLOPS\n", i + 1, ns, flop / secs);
        }
    }
    return EXIT_SUCCESS;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        return run(argc, argv);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return EXIT_FAILURE;
    }
}
