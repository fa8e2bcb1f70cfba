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

#include "common.cuh"

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

}  // namespace b200
