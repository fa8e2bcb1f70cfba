// Device-side building blocks shared by every kernel of the B200 SpGEMM path.
//
// Teams: a "team" is G consecutive lanes of one warp (G in {4, 8, 16, 32})
// that cooperate on one row of C, or a whole CTA (see cta.cuh).  Every team
// walks a row's intermediate products as ONE flattened sequence
//     q = 0 .. NIP(row)-1,  product q = (A entry e, B entry bs_e + q - exc_e)
// so that consecutive lanes read consecutive B entries (coalesced) and every
// lane gets the same amount of work whatever the B-row lengths are.  The
// reference instead gives each lane of a partial warp one A entry and walks
// that B row serially (sym1.cuh:77-94, num.cuh:106-116).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace b200 {

constexpr int kWarp = 32;
// Empty hash slot.  Larger than every column index, so a sorted table puts the
// empties last (the reference uses -1 read as uint32, sym2.cuh:104-113).
constexpr int32_t kEmpty = 0x7fffffff;

// Device status word, written by kernels that hit a bounded limit.  Nothing
// traps: the kernel records the flag, skips the work and returns, and the host
// turns the flag into SPGEMM_ERR_INTERNAL.
enum : unsigned {
    kStProbeLimit = 1u,   // a hash probe sequence ran past its bound
    kStCapacity = 2u,     // a row did not fit the bin it was routed to
    kStBadInput = 4u,     // checked mode found an invalid operand
    kStNipOverflow = 8u,  // a row's NIP does not fit int32
    kStClusterFail = 16u, // (diagnostic) a cluster row spilled to the global bin
    kStIndex = 32u,       // a computed shared-memory index or alignment failed its check
    kStWait = 64u         // a bounded wait on another CTA's result ran out
};

struct DevStatus {
    unsigned flags;
    int32_t row;
    int32_t detail;
    int32_t pad;
};

__device__ __forceinline__ void report(DevStatus* st, unsigned flag, int32_t row,
                                       int32_t detail = 0) {
    atomicOr(&st->flags, flag);
    st->row = row;
    st->detail = detail;
}

// Multiplicative (Fibonacci) hash reduced to [0, T) by the high half of a
// 32x32 product; T need not be a power of two.  The reference uses
// (key * 107) mod T (parameters.cuh:14, sym1.cuh:82).  Which hash is used does
// not change any result: only the distinct count and the sorted key set leave
// the table.
__device__ __forceinline__ uint32_t hash_slot(int32_t key, uint32_t T) {
    return __umulhi(static_cast<uint32_t>(key) * 0x9E3779B1u, T);
}

// ---- team (sub-warp) primitives -------------------------------------------

template<int G>
__device__ __forceinline__ unsigned team_mask() {
    if constexpr (G == 32) {
        return 0xffffffffu;
    } else {
        const unsigned lane = threadIdx.x & 31u;
        return ((1u << G) - 1u) << (lane & ~static_cast<unsigned>(G - 1));
    }
}

template<int G>
__device__ __forceinline__ int team_lane() {
    return static_cast<int>(threadIdx.x & (G - 1));
}

template<int G>
__device__ __forceinline__ int team_inclusive_scan(unsigned mask, int v, int lane) {
#pragma unroll
    for (int o = 1; o < G; o <<= 1) {
        const int t = __shfl_up_sync(mask, v, o, G);
        if (lane >= o) v += t;
    }
    return v;
}

template<int G, typename T>
__device__ __forceinline__ T team_sum(unsigned mask, T v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
    return v;
}

template<int G>
__device__ __forceinline__ void team_sync(unsigned mask) {
    if constexpr (G == 32) {
        __syncwarp();
    } else {
        __syncwarp(mask);
    }
}

// Walk the intermediate products of the A-row segment [a0, a1) with a team of
// G lanes.  For every product, calls f(q_b, a_index, q) where q_b is the
// position of the B entry in B.col / B.val, a_index the position of the A
// entry and q the product's place in the row's flattened sequence (products
// of A entry a0 first, each B row in order).  All lanes of the team must call
// this together (the shuffles are team-wide).
template<int G, typename F>
__device__ __forceinline__ void team_for_products_at(const int32_t* __restrict__ a_col,
                                                     const int32_t* __restrict__ b_rpt, int a0,
                                                     int a1, F&& f) {
    const unsigned mask = team_mask<G>();
    const int lane = team_lane<G>();
    int off = 0;
    for (int base = a0; base < a1; base += G) {
        const int e = base + lane;
        int bs = 0;
        int len = 0;
        if (e < a1) {
            const int c = __ldg(a_col + e);
            bs = __ldg(b_rpt + c);
            len = __ldg(b_rpt + c + 1) - bs;
        }
        const int inc = team_inclusive_scan<G>(mask, len, lane);
        const int total = __shfl_sync(mask, inc, G - 1, G);
        const int exc = inc - len;
        for (int q0 = 0; q0 < total; q0 += G) {
            const int q = q0 + lane;
            // largest source lane s with exc_s <= q (lanes with len 0 share exc
            // with their successor, so the result always has len_s > 0)
            int s = 0;
#pragma unroll
            for (int step = G / 2; step > 0; step >>= 1) {
                const int cand = __shfl_sync(mask, exc, s + step, G);
                if (cand <= q) s += step;
            }
            const int sbs = __shfl_sync(mask, bs, s, G);
            const int sexc = __shfl_sync(mask, exc, s, G);
            if (q < total) f(sbs + q - sexc, base + s, off + q);
        }
        off += total;
    }
}

// The same walk with up to U products per lane in flight: a lane takes
// products q, q + G, ..., q + (U-1) G of the chunk together, runs their
// shuffle searches interleaved, issues every `load(q_b, a_index, q_row)` (the
// product's global reads, returning a value), then every
// `use(value, q_b, a_index, q_row)`.  Same products, same arguments as
// team_for_products_at.
//
// With CONVERGED set every lane of the team calls
// `use(value, q_b, a_index, q_row, valid)` together, valid telling whether the
// lane holds a product, so `use` may contain operations on the team's mask.
template<int G, int U, bool CONVERGED = false, typename L, typename F>
__device__ __forceinline__ void team_for_products_mlp(const int32_t* __restrict__ a_col,
                                                      const int32_t* __restrict__ b_rpt, int a0,
                                                      int a1, L&& load, F&& use) {
    if constexpr (U == 1 && !CONVERGED) {
        // one product per lane: the plain walk (fewer registers)
        team_for_products_at<G>(a_col, b_rpt, a0, a1,
                                [&](int qb, int ai, int q) { use(load(qb, ai, q), qb, ai, q); });
        return;
    }
    using Val = decltype(load(0, 0, 0));
    const unsigned mask = team_mask<G>();
    const int lane = team_lane<G>();
    int off = 0;
    for (int base = a0; base < a1; base += G) {
        const int e = base + lane;
        int bs = 0;
        int len = 0;
        if (e < a1) {
            const int c = __ldg(a_col + e);
            bs = __ldg(b_rpt + c);
            len = __ldg(b_rpt + c + 1) - bs;
        }
        const int inc = team_inclusive_scan<G>(mask, len, lane);
        const int total = __shfl_sync(mask, inc, G - 1, G);
        const int exc = inc - len;
        for (int q0 = 0; q0 < total; q0 += G * U) {
            // steps of this round that hold products (uniform over the team)
            const int nu = min(U, (total - q0 + G - 1) / G);
            int s[U];
#pragma unroll
            for (int u = 0; u < U; u++) s[u] = 0;
#pragma unroll
            for (int step = G / 2; step > 0; step >>= 1) {
#pragma unroll
                for (int u = 0; u < U; u++) {
                    if (u < nu) {
                        const int cand = __shfl_sync(mask, exc, s[u] + step, G);
                        if (cand <= q0 + u * G + lane) s[u] += step;
                    }
                }
            }
            Val v[U];
            int qb[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (u < nu) {
                    const int q = q0 + u * G + lane;
                    const int sbs = __shfl_sync(mask, bs, s[u], G);
                    const int sexc = __shfl_sync(mask, exc, s[u], G);
                    qb[u] = sbs + q - sexc;
                    if (q < total) v[u] = load(qb[u], base + s[u], off + q);
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int q = q0 + u * G + lane;
                if constexpr (CONVERGED) {
                    if (u < nu) use(v[u], qb[u], base + s[u], off + q, q < total);
                } else {
                    if (u < nu && q < total) use(v[u], qb[u], base + s[u], off + q);
                }
            }
        }
        off += total;
    }
}

// The same walk for callers that need no product position: f(q_b, a_index).
template<int G, typename F>
__device__ __forceinline__ void team_for_products(const int32_t* __restrict__ a_col,
                                                  const int32_t* __restrict__ b_rpt, int a0,
                                                  int a1, F&& f) {
    team_for_products_at<G>(a_col, b_rpt, a0, a1, [&](int qb, int ai, int) { f(qb, ai); });
}

// lower_bound over a sorted int array of length n (n >= 1); the key is known to
// be present.  Branch-free loop with a uniform trip count.  Mirrors the
// reference's find_key (num.cuh:28-41).
__device__ __forceinline__ int lower_bound_present(const int32_t* cols, int n, int32_t key) {
    int lo = 0;
    int len = n;
    while (len > 1) {
        const int half = len >> 1;
        lo = (cols[lo + half - 1] < key) ? lo + half : lo;
        len -= half;
    }
    return lo;
}

// Insert `key` into a linear-probing table of T slots.  Returns 1 if the key
// was new, 0 if already present.  The probe loop is bounded by T; if it runs
// out (table full -- impossible for rows routed by their bound) the status
// word is flagged and the key dropped.
__device__ __forceinline__ int table_insert(int32_t* table, uint32_t T, int32_t key,
                                            DevStatus* st, int32_t row) {
    uint32_t h = hash_slot(key, T);
    for (uint32_t probe = 0; probe < T; probe++) {
        const int32_t old = atomicCAS(table + h, kEmpty, key);
        if (old == kEmpty) return 1;
        if (old == key) return 0;
        h = (h + 1 == T) ? 0u : h + 1;
    }
    report(st, kStProbeLimit, row);
    return 0;
}

}  // namespace b200
