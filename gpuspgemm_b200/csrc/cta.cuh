// CTA-wide building blocks: block scan / reduction, the CTA-flattened product
// walk, in-place compaction and bitonic sorts of shared-memory tables.
#pragma once

#include "common.cuh"

namespace b200 {

// Shared scratch a CTA needs to flatten one chunk of THREADS A entries.
template<int THREADS>
struct CtaScratch {
    int32_t exc[THREADS];  // exclusive prefix of B-row lengths within the chunk
    int32_t bs[THREADS];   // B-row start of each A entry of the chunk
    int32_t warp_tot[THREADS / kWarp];
    int32_t total;
    int32_t aux[3];  // per-row words of the kernels (e.g. the fill's Dmax)
};

// Inclusive scan of one int per thread over the CTA.  Contains two
// __syncthreads; `warp_tot` must not be touched by the caller until after the
// next barrier.
template<int THREADS>
__device__ __forceinline__ int block_inclusive_scan(int v, int32_t* warp_tot) {
    static_assert(THREADS % kWarp == 0 && THREADS / kWarp <= kWarp, "block size");
    constexpr int NW = THREADS / kWarp;
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == kWarp - 1) warp_tot[w] = v;
    __syncthreads();
    if (w == 0) {
        int x = lane < NW ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < kWarp; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        if (lane < NW) warp_tot[lane] = x;
    }
    __syncthreads();
    if (w > 0) v += warp_tot[w - 1];
    return v;
}

// Sum over the CTA; every thread gets the result.  Two barriers.
template<int THREADS>
__device__ __forceinline__ int block_sum(int v, int32_t* warp_tot) {
    constexpr int NW = THREADS / kWarp;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) warp_tot[w] = v;
    __syncthreads();
    int t = 0;
#pragma unroll
    for (int i = 0; i < NW; i++) t += warp_tot[i];
    return t;
}

// Walk the intermediate products of the A-row segment [a0, a1) with the whole
// CTA.  Chunks of THREADS A entries are scanned once; then every thread takes
// products q = tid, tid + THREADS, ... of the chunk and finds its A entry by a
// binary search of the chunk's prefix.  Calls f(q_b, a_index, q_row) with
// q_row the product's place in the row's flattened sequence (products of A
// entry a0 first, each B row in order).  All threads must call it (it
// contains barriers).
template<int THREADS, typename F>
__device__ __forceinline__ void cta_for_products_at(const int32_t* __restrict__ a_col,
                                                    const int32_t* __restrict__ b_rpt, int a0,
                                                    int a1, CtaScratch<THREADS>& sc, F&& f) {
    const int tid = threadIdx.x;
    int off = 0;  // products of the chunks before this one
    for (int base = a0; base < a1; base += THREADS) {
        const int e = base + tid;
        int bs = 0;
        int len = 0;
        if (e < a1) {
            const int c = __ldg(a_col + e);
            bs = __ldg(b_rpt + c);
            len = __ldg(b_rpt + c + 1) - bs;
        }
        const int inc = block_inclusive_scan<THREADS>(len, sc.warp_tot);
        sc.exc[tid] = inc - len;
        sc.bs[tid] = bs;
        if (tid == THREADS - 1) sc.total = inc;
        __syncthreads();
        const int total = sc.total;
        const int nvalid = min(THREADS, a1 - base);
        for (int q = tid; q < total; q += THREADS) {
            int lo = 0;
            int n = nvalid;
            while (n > 1) {
                const int half = n >> 1;
                lo = (sc.exc[lo + half] <= q) ? lo + half : lo;
                n -= half;
            }
            f(sc.bs[lo] + q - sc.exc[lo], base + lo, off + q);
        }
        off += total;
        __syncthreads();
    }
}

// The same walk with U products per thread in flight: each thread takes
// products q, q + THREADS, ..., q + (U-1) THREADS together, runs their U
// binary searches interleaved (one shared trip count), issues every
// `load(q_b, a_index, q_row)` -- the product's global reads, returning a value
// -- and only then every `use(value, q_b, a_index, q_row)`.  A walk whose
// work is a dependent global read followed by a shared-memory update thus
// keeps U reads outstanding per thread instead of one.  Same products, same
// arguments as cta_for_products_at.
//
// With CONVERGED set, whole warps take products together (lane l of a warp
// takes the warp's base + l) and every lane calls
// `use(value, q_b, a_index, q_row, valid)`, valid telling whether the lane holds
// a product, so `use` may contain warp-wide operations on the full mask.
template<int THREADS, int U, bool CONVERGED = false, typename L, typename F>
__device__ __forceinline__ void cta_for_products_mlp(const int32_t* __restrict__ a_col,
                                                     const int32_t* __restrict__ b_rpt, int a0,
                                                     int a1, CtaScratch<THREADS>& sc, L&& load,
                                                     F&& use) {
    using Val = decltype(load(0, 0, 0));
    const int tid = threadIdx.x;
    int off = 0;
    for (int base = a0; base < a1; base += THREADS) {
        const int e = base + tid;
        int bs = 0;
        int len = 0;
        if (e < a1) {
            const int c = __ldg(a_col + e);
            bs = __ldg(b_rpt + c);
            len = __ldg(b_rpt + c + 1) - bs;
        }
        const int inc = block_inclusive_scan<THREADS>(len, sc.warp_tot);
        sc.exc[tid] = inc - len;
        sc.bs[tid] = bs;
        if (tid == THREADS - 1) sc.total = inc;
        __syncthreads();
        const int total = sc.total;
        const int nvalid = min(THREADS, a1 - base);
        // CONVERGED: the loop bound is the warp's first lane's, so a warp
        // enters and leaves together
        const int tid0 = CONVERGED ? (tid & ~(kWarp - 1)) : tid;
        for (int q0 = tid, w0 = tid0; w0 < total; q0 += THREADS * U, w0 += THREADS * U) {
            int lo[U];
#pragma unroll
            for (int u = 0; u < U; u++) lo[u] = 0;
            for (int n = nvalid; n > 1;) {
                const int half = n >> 1;
#pragma unroll
                for (int u = 0; u < U; u++)
                    lo[u] = (sc.exc[lo[u] + half] <= q0 + u * THREADS) ? lo[u] + half : lo[u];
                n -= half;
            }
            Val v[U];
            int qb[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int q = q0 + u * THREADS;
                qb[u] = sc.bs[lo[u]] + q - sc.exc[lo[u]];
                if (q < total) v[u] = load(qb[u], base + lo[u], off + q);
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int q = q0 + u * THREADS;
                if constexpr (CONVERGED) {
                    use(v[u], qb[u], base + lo[u], off + q, q < total);
                } else {
                    if (q < total) use(v[u], qb[u], base + lo[u], off + q);
                }
            }
        }
        off += total;
        __syncthreads();
    }
}

// The same walk for callers that need no product position: f(q_b, a_index).
template<int THREADS, typename F>
__device__ __forceinline__ void cta_for_products(const int32_t* __restrict__ a_col,
                                                 const int32_t* __restrict__ b_rpt, int a0,
                                                 int a1, CtaScratch<THREADS>& sc, F&& f) {
    cta_for_products_at<THREADS>(a_col, b_rpt, a0, a1, sc,
                                 [&](int qb, int ai, int) { f(qb, ai); });
}

// Column window of one row of C: the smallest first column and the largest
// last column over the B rows that the A entries [a0, a1) select, clamped to
// [0, n_cols).  When B's rows are sorted every key of the row lies inside it;
// callers that depend on that check each key and fall back to [0, n_cols).
// Returns (lo, hi); lo > hi for a row with no products.  All threads must call
// it (three barriers; it reuses sc.exc / sc.bs).
template<int THREADS>
__device__ __forceinline__ int2 cta_col_window(const int32_t* __restrict__ a_col,
                                               const int32_t* __restrict__ b_rpt,
                                               const int32_t* __restrict__ b_col, int a0, int a1,
                                               int n_cols, CtaScratch<THREADS>& sc) {
    constexpr int NW = THREADS / kWarp;
    int lo = INT32_MAX;
    int hi = -1;
    for (int e = a0 + threadIdx.x; e < a1; e += THREADS) {
        const int r = __ldg(a_col + e);
        const int s0 = __ldg(b_rpt + r);
        const int s1 = __ldg(b_rpt + r + 1);
        if (s0 < s1) {
            lo = min(lo, __ldg(b_col + s0));
            hi = max(hi, __ldg(b_col + s1 - 1));
        }
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    __syncthreads();  // the previous user of exc / bs is done
    if (lane == 0) {
        sc.exc[w] = lo;
        sc.bs[w] = hi;
    }
    __syncthreads();
    lo = INT32_MAX;
    hi = -1;
#pragma unroll
    for (int i = 0; i < NW; i++) {
        lo = min(lo, sc.exc[i]);
        hi = max(hi, sc.bs[i]);
    }
    __syncthreads();  // exc / bs are free again for the product walk
    return make_int2(max(lo, 0), min(hi, n_cols - 1));
}

// Move the non-empty slots of table[0, T) to its front, in slot order.
// Returns the number of keys.  Reads of a chunk complete (barrier inside the
// scan) before any write, and writes land at or before the slot they came
// from, so the in-place move is safe.
template<int THREADS>
__device__ __forceinline__ int cta_compact(int32_t* table, int T, int32_t* warp_tot) {
    int base = 0;
    for (int c = 0; c < T; c += THREADS) {
        const int idx = c + threadIdx.x;
        const int32_t k = idx < T ? table[idx] : kEmpty;
        const int flag = (k != kEmpty) ? 1 : 0;
        const int inc = block_inclusive_scan<THREADS>(flag, warp_tot);
        if (flag) table[base + inc - 1] = k;
        // after the scan warp_tot holds the inclusive warp totals: the last
        // one is the chunk's key count
        const int tot = warp_tot[THREADS / kWarp - 1];
        __syncthreads();
        base += tot;
    }
    return base;
}

// Ascending bitonic sort of s[0, N) (N a power of two) by the whole CTA.
template<int THREADS>
__device__ __forceinline__ void cta_bitonic_sort(int32_t* s, int N) {
    for (int k = 2; k <= N; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < (N >> 1); i += THREADS) {
                const int lo = 2 * i - (i & (j - 1));
                const int hi = lo + j;
                const bool up = (lo & k) == 0;
                const int32_t a = s[lo];
                const int32_t b = s[hi];
                if ((a > b) == up) {
                    s[lo] = b;
                    s[hi] = a;
                }
            }
            __syncthreads();
        }
    }
}

// Move the non-empty slots of table[0, T) to its front, in slot order, by a
// team of G lanes (T a multiple of G).  Returns the number of keys.  Every
// lane has read its slot of a chunk before the ballot, and a chunk's writes
// land below the next chunk's first slot, so the in-place move is safe.
template<int G>
__device__ __forceinline__ int team_compact(int32_t* table, int T, unsigned mask, int lane) {
    const unsigned below = (1u << (threadIdx.x & 31u)) - 1u;
    int out = 0;
    for (int base = 0; base < T; base += G) {
        const int32_t k = table[base + lane];
        const bool flag = k != kEmpty;
        const unsigned bits = __ballot_sync(mask, flag) & mask;
        if (flag) table[out + __popc(bits & below)] = k;
        out += __popc(bits);
    }
    team_sync<G>(mask);
    return out;
}

// Ascending bitonic sort of s[0, N) (N a power of two) by a team of G lanes.
template<int G>
__device__ __forceinline__ void team_bitonic_sort(int32_t* s, int N, unsigned mask, int lane) {
    for (int k = 2; k <= N; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < (N >> 1); i += G) {
                const int lo = 2 * i - (i & (j - 1));
                const int hi = lo + j;
                const bool up = (lo & k) == 0;
                const int32_t a = s[lo];
                const int32_t b = s[hi];
                if ((a > b) == up) {
                    s[lo] = b;
                    s[hi] = a;
                }
            }
            team_sync<G>(mask);
        }
    }
}

__host__ __device__ constexpr int next_pow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

}  // namespace b200
