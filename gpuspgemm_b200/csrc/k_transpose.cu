// CSR transpose T = A^T with sorted columns in every row of T.
//
// The reference has no transpose: its Galerkin use (R = P^T for R*A*P) leaves
// the transpose to the caller.  Here it is a library call so that a chained
// product stays on the device:
//   1. column counts of A (warp-aggregated atomics) into T.rpt;
//   2. the product path's binning pass with the scan (k_bin.cu) turns the
//      counts into T.rpt and bins T's rows by length;
//   3. scatter: every entry (i, j) of A takes a slot of row j of T through an
//      atomic cursor and stores the 64-bit key (i << 32 | position in A);
//   4. per bin, sort each row's keys ascending (the row indices i are unique
//      within a row, so the order is fully determined) and write T.col = i,
//      T.val = A.val[position].
// Sorting uses the bitonic network in which every comparator sends the
// smaller key to the lower index; a row of len keys runs the network of the
// next power of two with the missing tail taken as +infinity, and every
// comparator that touches the tail is a no-op, so the tail is never stored.
#include "cta.cuh"
#include "kernels.hpp"

namespace b200 {

namespace {

constexpr uint64_t kKeyInf = ~0ull;

__device__ __forceinline__ void cas_asc(uint64_t* a, long long lo, long long hi) {
    const uint64_t x = a[lo];
    const uint64_t y = a[hi];
    if (x > y) {
        a[lo] = y;
        a[hi] = x;
    }
}

// Ascending sort of a[0, len) by the CTA (a in shared or global memory).
template<int THREADS>
__device__ void cta_sort_keys(uint64_t* a, long long len) {
    long long N = 1;
    while (N < len) N <<= 1;
    const long long pairs = N >> 1;
    for (long long k = 2; k <= N; k <<= 1) {
        const long long half = k >> 1;
        // flip: i <-> k-1-i inside every block of k
        for (long long p = threadIdx.x; p < pairs; p += THREADS) {
            const long long blk = (p / half) * k;
            const long long i = p & (half - 1);
            const long long hi = blk + k - 1 - i;
            if (hi < len) cas_asc(a, blk + i, hi);
        }
        __syncthreads();
        for (long long j = half >> 1; j > 0; j >>= 1) {
            for (long long p = threadIdx.x; p < pairs; p += THREADS) {
                const long long lo = 2 * p - (p & (j - 1));
                if (lo + j < len) cas_asc(a, lo, lo + j);
            }
            __syncthreads();
        }
    }
}

template<typename V>
__device__ __forceinline__ void store_entry(const ProductArgs& p, int32_t at, uint64_t key) {
    p.c_col[at] = static_cast<int32_t>(key >> 32);
    static_cast<V*>(p.c_val)[at] =
        __ldg(static_cast<const V*>(p.a_val) + static_cast<uint32_t>(key & 0xffffffffu));
}

// ---- 1. column counts -------------------------------------------------------
// A column index outside [0, n) is not counted; the host sees the total fall
// short of nnz and reports the operand as invalid.
__global__ __launch_bounds__(256) void k_col_count(const int32_t* __restrict__ col, int32_t nnz,
                                                   int32_t n, int32_t* __restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    // the loop bound is warp-uniform, so every lane joins each match
    for (long long base = static_cast<long long>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31);
         base < nnz; base += stride) {
        const long long e = base + lane;
        int32_t c = e < nnz ? __ldg(col + e) : -1;
        if (c >= n) c = -1;
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        if (c >= 0 && lane == __ffs(peers) - 1) atomicAdd(cnt + c, __popc(peers));
    }
}

// ---- 3. scatter of keys -----------------------------------------------------
// One warp per row of A; lanes over the row's entries.  Entries whose column
// is outside [0, n) were not counted and are skipped.
__global__ __launch_bounds__(256) void k_tr_scatter(const int32_t* __restrict__ a_rpt,
                                                    const int32_t* __restrict__ a_col, int32_t m,
                                                    int32_t n, const int32_t* __restrict__ t_rpt,
                                                    int32_t* __restrict__ cursor,
                                                    uint64_t* __restrict__ keys) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < m; r += warps) {
        const int s0 = __ldg(a_rpt + r);
        const int s1 = __ldg(a_rpt + r + 1);
        for (int e = s0 + lane; e < s1; e += 32) {
            const int c = __ldg(a_col + e);
            if (c < 0 || c >= n) continue;
            const int pos = __ldg(t_rpt + c) + atomicAdd(cursor + c, 1);
            keys[pos] = (static_cast<uint64_t>(static_cast<uint32_t>(r)) << 32) |
                        static_cast<uint32_t>(e);
        }
    }
}

// ---- 4. per-bin row sorts ---------------------------------------------------
// Rows of up to 32 keys: one warp per row, the network in registers.
template<typename V, int THREADS>
__global__ __launch_bounds__(THREADS) void k_tr_sort_warp(ProductArgs p) {
    const int lane = threadIdx.x & 31;
    const int rid = blockIdx.x * (THREADS / 32) + (threadIdx.x >> 5);
    if (rid >= p.nrows) return;  // warp-uniform
    const int row = p.rows[rid];
    const int t0 = p.c_rpt[row];
    const int len = p.c_rpt[row + 1] - t0;
    uint64_t v = lane < len ? p.keys[t0 + lane] : kKeyInf;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
        const int half = k >> 1;
        uint64_t o = __shfl_xor_sync(0xffffffffu, v, k - 1);
        v = (lane & half) ? (v > o ? v : o) : (v < o ? v : o);
#pragma unroll
        for (int j = half >> 1; j > 0; j >>= 1) {
            o = __shfl_xor_sync(0xffffffffu, v, j);
            v = (lane & j) ? (v > o ? v : o) : (v < o ? v : o);
        }
    }
    if (lane < len) store_entry<V>(p, t0 + lane, v);
}

// Rows of up to CAP keys: one CTA per row, the keys in shared memory.
template<typename V, int THREADS, int CAP>
__global__ __launch_bounds__(THREADS) void k_tr_sort_cta(ProductArgs p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* s = reinterpret_cast<uint64_t*>(smem_raw);
    const int row = p.rows[blockIdx.x];
    const int t0 = p.c_rpt[row];
    const int len = p.c_rpt[row + 1] - t0;
    if (len > CAP) {  // routed by its length: cannot happen
        if (threadIdx.x == 0) report(p.status, kStCapacity, row, len);
        return;
    }
    for (int i = threadIdx.x; i < len; i += THREADS) s[i] = p.keys[t0 + i];
    __syncthreads();
    cta_sort_keys<THREADS>(s, len);
    for (int i = threadIdx.x; i < len; i += THREADS) store_entry<V>(p, t0 + i, s[i]);
}

// Longer rows: one CTA per row, sorting the row's keys in place in global
// memory (the network's passes stay in L2 for rows of a few MB).
template<typename V, int THREADS>
__global__ __launch_bounds__(THREADS) void k_tr_sort_global(ProductArgs p) {
    for (int rid = blockIdx.x; rid < p.nrows; rid += gridDim.x) {
        const int row = p.rows[rid];
        const int t0 = p.c_rpt[row];
        const int len = p.c_rpt[row + 1] - t0;
        uint64_t* a = p.keys + t0;
        cta_sort_keys<THREADS>(a, len);
        for (int i = threadIdx.x; i < len; i += THREADS) store_entry<V>(p, t0 + i, a[i]);
        __syncthreads();
    }
}

template<typename V, int THREADS>
cudaError_t launch_warp(const ProductArgs& p, cudaStream_t s) {
    constexpr int R = THREADS / 32;
    k_tr_sort_warp<V, THREADS><<<(p.nrows + R - 1) / R, THREADS, 0, s>>>(p);
    return cudaGetLastError();
}

template<typename V, int THREADS, int CAP>
cudaError_t launch_cta(const ProductArgs& p, cudaStream_t s) {
    k_tr_sort_cta<V, THREADS, CAP><<<p.nrows, THREADS, sizeof(uint64_t) * CAP, s>>>(p);
    return cudaGetLastError();
}

template<typename V, int THREADS>
cudaError_t launch_global(const ProductArgs& p, cudaStream_t s) {
    const int grid = p.nrows < 2 * 148 ? p.nrows : 2 * 148;
    k_tr_sort_global<V, THREADS><<<grid, THREADS, 0, s>>>(p);
    return cudaGetLastError();
}

template<typename V>
struct TransposeLadder {
    static const BinLauncher bins[4];
};

template<typename V>
const BinLauncher TransposeLadder<V>::bins[4] = {
    {BinKind::Team, 32, 8, 256, 0, "tr_sort_warp32", launch_warp<V, 256>},
    {BinKind::Cta, 2048, 1, 256, sizeof(uint64_t) * 2048, "tr_sort_cta2048",
     launch_cta<V, 256, 2048>},
    {BinKind::Cta, 16384, 1, 1024, sizeof(uint64_t) * 16384, "tr_sort_cta16384",
     launch_cta<V, 1024, 16384>},
    {BinKind::Global, INT32_MAX, 1, 1024, 0, "tr_sort_global", launch_global<V, 1024>},
};

template<typename V>
cudaError_t prepare_ladder() {
    cudaError_t e = cudaFuncSetAttribute(k_tr_sort_cta<V, 1024, 16384>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(sizeof(uint64_t) * 16384));
    return e;
}

}  // namespace

int transpose_ladder_f64(const BinLauncher** out) {
    *out = TransposeLadder<double>::bins;
    return 4;
}

int transpose_ladder_f32(const BinLauncher** out) {
    *out = TransposeLadder<float>::bins;
    return 4;
}

cudaError_t transpose_prepare() {
    cudaError_t e = prepare_ladder<double>();
    if (e != cudaSuccess) return e;
    return prepare_ladder<float>();
}

cudaError_t launch_col_count(const int32_t* col, int32_t nnz, int32_t n, int32_t* cnt,
                             cudaStream_t s) {
    if (nnz <= 0) return cudaSuccess;
    long long g = (static_cast<long long>(nnz) + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    k_col_count<<<static_cast<int>(g), 256, 0, s>>>(col, nnz, n, cnt);
    return cudaGetLastError();
}

cudaError_t launch_tr_scatter(const int32_t* a_rpt, const int32_t* a_col, int32_t m, int32_t n,
                              const int32_t* t_rpt, int32_t* cursor, uint64_t* keys,
                              cudaStream_t s) {
    if (m <= 0) return cudaSuccess;
    long long g = (static_cast<long long>(m) + 7) / 8;
    if (g > 148 * 16) g = 148 * 16;
    k_tr_scatter<<<static_cast<int>(g), 256, 0, s>>>(a_rpt, a_col, m, n, t_rpt, cursor, keys);
    return cudaGetLastError();
}

}  // namespace b200
