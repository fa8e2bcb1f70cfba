// Allocation-free row-size pass: the exact nnz of every row of C = A*B,
// written into an array the caller owns.
//
// Who needs it: code that must not call cudaMalloc (or cudaMallocAsync, or a
// library routine that allocates) at the point where it sizes a product.
// Examples are a caller that has handed all device memory to its own pool
// allocator, a caller in a region where an allocation would synchronise the
// device, or a caller that plans a product before allocating C from its own
// memory.  Everything else in this library allocates: the handle owns scratch
// buffers and C is allocated for the caller.  This entry point instead uses a
// fixed scratch area compiled into the library's device image.
//
// The kernel is the global-bin count of the symbolic phase (a bitmap over B's
// columns per row in flight; atomicOr tells whether a column is new).  Its
// bitmaps live in g_noalloc_bitmaps: kSlots slots of SPGEMM_NOALLOC_MAX_COLS
// bits, 4 MiB on every GPU that loads the library, held until the process
// exits.
#include <mutex>
#include <string>

#include "../../include/spgemm.h"
#include "cta.cuh"

namespace b200 {
namespace {

constexpr int kNoAllocThreads = 1024;
constexpr int kSlots = 32;                       // CTAs in flight, one bitmap each
constexpr int kWordsPerSlot = SPGEMM_NOALLOC_MAX_COLS / 32;

static __device__ __align__(256) uint32_t g_noalloc_bitmaps[kSlots * kWordsPerSlot];

__global__ __launch_bounds__(kNoAllocThreads) void k_row_nnz_noalloc(
    const int32_t* __restrict__ a_rpt, const int32_t* __restrict__ a_col,
    const int32_t* __restrict__ b_rpt, const int32_t* __restrict__ b_col, int32_t m,
    int32_t n_cols, uint32_t* __restrict__ bitmaps, int32_t* __restrict__ nnz_out) {
    __shared__ CtaScratch<kNoAllocThreads> sc;
    uint32_t* bm = bitmaps + static_cast<size_t>(blockIdx.x) * kWordsPerSlot;
    for (int row = blockIdx.x; row < m; row += gridDim.x) {
        const int a0 = a_rpt[row];
        const int a1 = a_rpt[row + 1];
        int cnt = 0;
        int bad = 0;
        // a column outside [0, B.n) is skipped (it would index past this
        // slot) and the row's count becomes -1
        cta_for_products<kNoAllocThreads>(a_col, b_rpt, a0, a1, sc, [&](int qb, int) {
            const int32_t key = __ldg(b_col + qb);
            if (static_cast<uint32_t>(key) >= static_cast<uint32_t>(n_cols)) {
                bad = 1;
                return;
            }
            const uint32_t bit = 1u << (key & 31);
            const uint32_t old = atomicOr(bm + (key >> 5), bit);
            cnt += (old & bit) ? 0 : 1;
        });
        cnt = block_sum<kNoAllocThreads>(cnt, sc.warp_tot);
        bad = __syncthreads_or(bad);
        if (threadIdx.x == 0) nnz_out[row] = bad ? -1 : cnt;
        // every thread has read the warp totals of block_sum before the next
        // walk's scan writes them again
        __syncthreads();
        // leave the slot all-zero for the next row: clear exactly the words
        // this row touched (several keys may share a word; zero is idempotent)
        cta_for_products<kNoAllocThreads>(a_col, b_rpt, a0, a1, sc, [&](int qb, int) {
            const int32_t key = __ldg(b_col + qb);
            if (static_cast<uint32_t>(key) < static_cast<uint32_t>(n_cols)) bm[key >> 5] = 0u;
        });
    }
}

std::mutex g_noalloc_mu;
constexpr int kMaxDevices = 64;
void* g_noalloc_ptr[kMaxDevices] = {};  // device address of the slab, per device ordinal

}  // namespace

// Records the message spgemm_last_error_string() returns (defined beside it).
void set_last_error(const std::string& msg);

namespace {
spgemm_status noalloc_fail(spgemm_status st, const std::string& msg) {
    set_last_error(msg);
    return st;
}
}  // namespace
}  // namespace b200

using namespace b200;

extern "C" spgemm_status spgemm_row_nnz_noalloc(const spgemm_csr_view* A,
                                                const spgemm_csr_view* B,
                                                int32_t* c_row_nnz, void* stream) {
    if (A == nullptr || B == nullptr)
        return noalloc_fail(SPGEMM_ERR_INVALID_ARG, "A or B is NULL");
    if (A->m < 0 || A->n < 0 || A->nnz < 0 || B->m < 0 || B->n < 0 || B->nnz < 0)
        return noalloc_fail(SPGEMM_ERR_INVALID_ARG, "negative dimension");
    if (A->n != B->m)
        return noalloc_fail(SPGEMM_ERR_INVALID_ARG, "A.n must equal B.m");
    if (B->n > SPGEMM_NOALLOC_MAX_COLS)
        return noalloc_fail(SPGEMM_ERR_INVALID_ARG,
                            "B.n = " + std::to_string(B->n) +
                                " exceeds the allocation-free limit of " +
                                std::to_string(SPGEMM_NOALLOC_MAX_COLS) + " columns");
    if (A->m == 0) return SPGEMM_OK;
    if (c_row_nnz == nullptr || A->rpt == nullptr || B->rpt == nullptr ||
        (A->nnz > 0 && A->col == nullptr) || (B->nnz > 0 && B->col == nullptr))
        return noalloc_fail(SPGEMM_ERR_INVALID_ARG, "NULL array");
    int dev = 0;
    if (cudaError_t e = cudaGetDevice(&dev); e != cudaSuccess)
        return noalloc_fail(SPGEMM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return noalloc_fail(SPGEMM_ERR_UNSUPPORTED_DEVICE,
                            "device ordinal " + std::to_string(dev) +
                                " is beyond the allocation-free path's table of " +
                                std::to_string(kMaxDevices) + " devices");
    void* slab = nullptr;
    {
        // once per device, with that device current: the host-side name of a
        // __device__ array is not a device address, so look the address up
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (g_noalloc_ptr[dev] == nullptr) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_bitmaps);
            if (e != cudaSuccess || p == nullptr)
                return noalloc_fail(SPGEMM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") +
                                                         cudaGetErrorString(e));
            g_noalloc_ptr[dev] = p;
        }
        slab = g_noalloc_ptr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the slab keeps whatever the last call left; the words this call can
    // touch (the first ceil(B.n / 32) of each slot in use) must start at zero
    const int grid = A->m < kSlots ? A->m : kSlots;
    const size_t words = (static_cast<size_t>(B->n) + 31) / 32;
    cudaError_t e = cudaSuccess;
    if (words > 0)
        e = cudaMemset2DAsync(slab, sizeof(uint32_t) * kWordsPerSlot, 0, sizeof(uint32_t) * words,
                              static_cast<size_t>(grid), s);
    if (e == cudaSuccess) {
        k_row_nnz_noalloc<<<grid, kNoAllocThreads, 0, s>>>(A->rpt, A->col, B->rpt, B->col, A->m,
                                                          B->n, static_cast<uint32_t*>(slab),
                                                          c_row_nnz);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        return noalloc_fail(SPGEMM_ERR_CUDA, std::string("row nnz kernel: ") + cudaGetErrorString(e));
    return SPGEMM_OK;
}
