// Register bitonic sort of a team's keys (the fill bins' sort step).
//
// A team of G lanes sorts N = G * E keys, E per lane in registers.  The lanes
// may load any E keys each -- a sort does not care where its input starts --
// so they load striped (key e * G + lane), which is free of shared-memory bank
// conflicts.  The network then runs on the BLOCKED order: lane L's register e
// is element L * E + e.  Compare-exchange steps closer than E stay inside a
// lane's registers; wider steps pair lane L with lane L ^ (j / E) through a
// shuffle of width G.  At the end lane L holds ranks L * E .. L * E + E - 1.
//
// The sorted keys go back to shared memory under the swizzle
//     swz(i) = i ^ ((i >> 5) & 31),
// which makes the blocked write (lane L, element L * E + e), the striped read
// (element e * 32 + L) and single-index reads (the numeric phase's binary
// search) all bank-conflict free within a 32-lane team.
#pragma once

#include "cta.cuh"

namespace b200 {

__device__ __forceinline__ int swz(int i) { return i ^ ((i >> 5) & 31); }

// Lower bound of a key known to be present in the swizzled sorted keys[0, n).
__device__ __forceinline__ int lower_bound_present_swz(const int32_t* keys, int n, int32_t key) {
    int lo = 0;
    int len = n;
    while (len > 1) {
        const int half = len >> 1;
        lo = (keys[swz(lo + half - 1)] < key) ? lo + half : lo;
        len -= half;
    }
    return lo;
}

template<int G, int E>
__device__ __forceinline__ void team_sort_regs(int32_t* keys, int n, unsigned mask, int lane) {
    constexpr int N = G * E;
    int32_t r[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
        const int i = e * G + lane;
        r[e] = i < n ? keys[i] : kEmpty;
    }
#pragma unroll
    for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j < E) {
                // partners inside the lane: elements e and e + j
#pragma unroll
                for (int e = 0; e < E; e++) {
                    if ((e & j) == 0) {
                        // ascending iff bit k of the element's index is clear;
                        // for k < E that bit comes from e, else from the lane
                        const bool up = k < E ? ((e & k) == 0) : (((lane * E) & k) == 0);
                        const int32_t a = r[e];
                        const int32_t b = r[e + j];
                        r[e] = up ? min(a, b) : max(a, b);
                        r[e + j] = up ? max(a, b) : min(a, b);
                    }
                }
            } else {
                // partner lane L ^ (j / E), same register
                const int d = j / E;
                const bool lower = (lane & d) == 0;
                const bool up = ((lane * E) & k) == 0;
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const int32_t o = __shfl_xor_sync(mask, r[e], d, G);
                    r[e] = (lower == up) ? min(r[e], o) : max(r[e], o);
                }
            }
        }
    }
    team_sync<G>(mask);  // every lane has read its input keys
#pragma unroll
    for (int e = 0; e < E; e++) keys[swz(lane * E + e)] = r[e];
    team_sync<G>(mask);
}

// Sort keys[0, n) (n <= T, T = G * EMAX) of a team into swizzled order.
template<int G, int EMAX>
__device__ __forceinline__ void team_sort_swz(int32_t* keys, int n, unsigned mask, int lane) {
    const int e = (n + G - 1) / G;
    if (e <= 1) {
        team_sort_regs<G, 1>(keys, n, mask, lane);
    } else if (e <= 2) {
        if constexpr (EMAX >= 2) team_sort_regs<G, 2>(keys, n, mask, lane);
    } else if (e <= 4) {
        if constexpr (EMAX >= 4) team_sort_regs<G, 4>(keys, n, mask, lane);
    } else if (e <= 8) {
        if constexpr (EMAX >= 8) team_sort_regs<G, 8>(keys, n, mask, lane);
    } else if (e <= 16) {
        if constexpr (EMAX >= 16) team_sort_regs<G, 16>(keys, n, mask, lane);
    } else {
        if constexpr (EMAX >= 32) team_sort_regs<G, 32>(keys, n, mask, lane);
    }
}

// In-lane steps j < E of stage k: elements e and e + j; ascending iff bit k of
// the element's index (lane * E + e) is clear.
template<int E>
__device__ __forceinline__ void lane_steps(int32_t (&r)[E], int k, int base) {
#pragma unroll
    for (int j = E / 2; j > 0; j >>= 1) {
        if (j < k) {
#pragma unroll
            for (int e = 0; e < E; e++) {
                if ((e & j) == 0) {
                    const bool up = ((base + e) & k) == 0;
                    const int32_t a = r[e];
                    const int32_t b = r[e + j];
                    r[e] = up ? min(a, b) : max(a, b);
                    r[e + j] = up ? max(a, b) : min(a, b);
                }
            }
        }
    }
}

// The same network over a whole CTA: THREADS threads with E keys each.
// Steps closer than E stay in registers, steps up to 32 * E pair lanes of one
// warp through shuffles, and only the wider steps (log2(THREADS / 32) levels,
// a handful of stages) exchange through shared memory, in swizzled order.
// Unlike the team network, the stage loops run at run time: the CTA kernels
// run beside the team kernels, and fully unrolled copies of this network for
// every E measured slower on the 1M power-law product (code size and
// registers).  keys[] must hold at least THREADS * E slots.  All threads must
// call it.
template<int THREADS, int E>
__device__ __forceinline__ void cta_sort_regs(int32_t* keys, int n) {
    constexpr int N = THREADS * E;
    const int tid = threadIdx.x;
    int32_t r[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
        const int i = e * THREADS + tid;
        r[e] = i < n ? keys[i] : kEmpty;
    }
    __syncthreads();  // every thread has read its input keys
#pragma unroll 1
    for (int k = 2; k <= N; k <<= 1) {
        const bool up = ((tid * E) & k) == 0;
#pragma unroll 1
        for (int j = k >> 1; j >= E; j >>= 1) {
            const int d = j / E;
            const bool keep_min = ((tid & d) == 0) == up;
            if (d < 32) {
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const int32_t o = __shfl_xor_sync(0xffffffffu, r[e], d);
                    r[e] = keep_min ? min(r[e], o) : max(r[e], o);
                }
            } else {
#pragma unroll
                for (int e = 0; e < E; e++) keys[swz(tid * E + e)] = r[e];
                __syncthreads();
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const int32_t o = keys[swz((tid ^ d) * E + e)];
                    r[e] = keep_min ? min(r[e], o) : max(r[e], o);
                }
                __syncthreads();
            }
        }
        lane_steps<E>(r, k, tid * E);
    }
#pragma unroll
    for (int e = 0; e < E; e++) keys[swz(tid * E + e)] = r[e];
    __syncthreads();
}

// Sort keys[0, n) of a CTA into swizzled order.  Rows of up to THREADS * 16
// keys use the register network; longer ones (the largest CTA bins) run the
// shared-memory bitonic network on keys[0, next_pow2(n)) and are then
// swizzled in place -- swz only permutes inside 32-key blocks and is its own
// inverse, so each warp swaps within its blocks with no CTA barrier between
// its read and its write.  keys[] must hold next_pow2(n) and THREADS * 16 slots.
template<int THREADS>
__device__ __forceinline__ void cta_sort_swz(int32_t* keys, int n) {
    const int e = (n + THREADS - 1) / THREADS;
    if (e <= 1) {
        cta_sort_regs<THREADS, 1>(keys, n);
    } else if (e <= 2) {
        cta_sort_regs<THREADS, 2>(keys, n);
    } else if (e <= 4) {
        cta_sort_regs<THREADS, 4>(keys, n);
    } else if (e <= 8) {
        cta_sort_regs<THREADS, 8>(keys, n);
    } else if (e <= 16) {
        cta_sort_regs<THREADS, 16>(keys, n);
    } else {
        const int pn = next_pow2(n);
        for (int i = n + threadIdx.x; i < pn; i += THREADS) keys[i] = kEmpty;
        __syncthreads();
        cta_bitonic_sort<THREADS>(keys, pn);
        const int lane = threadIdx.x & 31;
        for (int b = (threadIdx.x >> 5) * 32; b < pn; b += THREADS) {
            const int32_t v = keys[b + lane];
            __syncwarp();
            keys[swz(b + lane)] = v;
        }
        __syncthreads();
    }
}

// Stable CTA radix sort of keys[0, n) by their bits [lo_bit, lo_bit + nbits),
// in place, 7 bits per pass.  Warp w owns the segment [w S, (w + 1) S),
// S = 32 ceil(n / THREADS) <= 32 RMAX; in round i lane l holds key
// w S + 32 i + l, so rounds, then lanes, follow the keys' order.  Per pass:
// every thread loads its keys into registers (so the pass may scatter over
// the array it read); each warp ranks its keys per digit -- lanes with the
// same digit in a round find one another through 7 ballots and the lowest of
// them adds their count to the warp's counter -- then one block scan over
// (digit, warp) gives every key its place.  `hist` holds 128 * THREADS / 32
// ints.  All threads must call it.  Equal digits keep their order, so keys
// whose low bits hold their input position come out ordered by the sort bits
// and then by position.
template<int THREADS, int RMAX>
__device__ __forceinline__ void cta_radix_sort(uint32_t* keys, int n, int lo_bit, int nbits,
                                               int32_t* hist, int32_t* warp_tot) {
    constexpr int NW = THREADS / kWarp;
    constexpr int DIGITS = 128;
    static_assert(NW * DIGITS == 4 * THREADS, "four counters per thread in the scan");
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int w = tid >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int S = kWarp * ((n + THREADS - 1) / THREADS);
    const int R = S / kWarp;  // <= RMAX
    int32_t* wh = hist + w * DIGITS;
    for (int bit = lo_bit; bit < lo_bit + nbits; bit += 7) {
        uint32_t k[RMAX];
        int rk[RMAX];
#pragma unroll
        for (int i = 0; i < RMAX; i++) {
            const int idx = w * S + kWarp * i + lane;
            k[i] = (i < R && idx < n) ? keys[idx] : 0u;
        }
#pragma unroll
        for (int c = 0; c < DIGITS / kWarp; c++) wh[c * kWarp + lane] = 0;
        __syncthreads();  // every key is in registers; the counters are clear
#pragma unroll
        for (int i = 0; i < RMAX; i++) {
            if (i < R) {
                const bool valid = w * S + kWarp * i + lane < n;
                const unsigned d = (k[i] >> bit) & (DIGITS - 1);
                unsigned peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
                for (int b = 0; b < 7; b++) {
                    const unsigned m = __ballot_sync(0xffffffffu, (d >> b) & 1u);
                    peers &= ((d >> b) & 1u) ? m : ~m;
                }
                const int pre = wh[d];
                rk[i] = pre + __popc(peers & lt);
                __syncwarp();
                if (valid && (peers & lt) == 0u) wh[d] = pre + __popc(peers);
                __syncwarp();
            }
        }
        __syncthreads();
        // exclusive scan of the counters in (digit, warp) order
        int v[4];
        int sum = 0;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int L = 4 * tid + c;
            v[c] = hist[(L & (NW - 1)) * DIGITS + (L / NW)];
            sum += v[c];
        }
        int run = block_inclusive_scan<THREADS>(sum, warp_tot) - sum;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int L = 4 * tid + c;
            hist[(L & (NW - 1)) * DIGITS + (L / NW)] = run;
            run += v[c];
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < RMAX; i++) {
            if (i < R && w * S + kWarp * i + lane < n) {
                const unsigned d = (k[i] >> bit) & (DIGITS - 1);
                keys[wh[d] + rk[i]] = k[i];
            }
        }
        __syncthreads();
    }
}

}  // namespace b200
