// Row binning and the row-pointer scan.
//
// The reference bins rows three times (by NIP for sym1, by nnz for sym2 and
// for num), each time with two kernels and two host round-trips
// (binning.cuh:146-205), plus a CUB max + scan (binning.cuh:208-243).  Here a
// binning pass is three kernels with no host round-trip in between:
//   hist     per-CTA bin histogram (+ NIP per row, or + per-CTA nnz sums)
//   offsets  one CTA scans the histograms (bin-major) and the CTA sums
//   scatter  stable scatter of row ids (+ the exclusive scan into C.rpt)
// The scatter is stable: rows of a bin keep ascending row order, so the bin
// kernels read A and write C in order.
#include "cta.cuh"
#include "kernels.hpp"

namespace b200 {

namespace {

__device__ __forceinline__ int find_bin(const Ladder& lad, int32_t key) {
    int b = lad.nb - 1;
    for (int i = 0; i < lad.nb; i++) {
        if (key <= lad.limit[i]) {
            b = i;
            break;
        }
    }
    return b < lad.min_bin ? lad.min_bin : b;
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---- pass 1: NIP per row (setup.cuh:29-95) + histogram --------------------
__global__ __launch_bounds__(kBinThreads) void k_nip_hist(
    const int32_t* __restrict__ a_rpt, const int32_t* __restrict__ a_col,
    const int32_t* __restrict__ b_rpt, int32_t m, int32_t* __restrict__ c_rpt,
    int32_t* __restrict__ nip_copy, int32_t* __restrict__ hist, Plan* __restrict__ plan,
    DevStatus* __restrict__ st, const __grid_constant__ Ladder lad) {
    __shared__ int32_t s_hist[kMaxBins];
    __shared__ long long s_tot[kBinThreads / kWarp];
    __shared__ int32_t s_max[kBinThreads / kWarp];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int w = tid >> 5;
    if (tid < kMaxBins) s_hist[tid] = 0;
    __syncthreads();

    constexpr int kGroups = kBinRowsPerCta / kWarp / (kBinThreads / kWarp);  // per warp
    long long my_tot = 0;
    int32_t my_max = 0;
    for (int j = 0; j < kGroups; j++) {
        const int r = blockIdx.x * kBinRowsPerCta + (w * kGroups + j) * kWarp + lane;
        int s0 = 0;
        int s1 = 0;
        if (r < m) {
            s0 = a_rpt[r];
            s1 = a_rpt[r + 1];
        }
        const int len = s1 - s0;
        long long nip = 0;
        // short rows: a lane each, all at once; long rows (>= 32 entries): the
        // whole warp, one after another (setup.cuh:52-75 gives the warp every
        // row of a group that holds a long one)
        if (len < kWarp) {
#pragma unroll 4
            for (int p = s0; p < s1; p++) {
                const int c = __ldg(a_col + p);
                nip += __ldg(b_rpt + c + 1) - __ldg(b_rpt + c);
            }
        }
        for (unsigned longm = __ballot_sync(0xffffffffu, len >= kWarp); longm != 0u;
             longm &= longm - 1u) {
            const int i = __ffs(longm) - 1;
            const int rs = __shfl_sync(0xffffffffu, s0, i);
            const int re = __shfl_sync(0xffffffffu, s1, i);
            // 8 entries per lane in flight: all their columns first, then all
            // the B-row bounds (the longest rows set the kernel's duration)
            constexpr int U = 8;
            long long part = 0;
            for (int p0 = rs + lane; p0 < re; p0 += U * kWarp) {
                int c[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const int p = p0 + u * kWarp;
                    c[u] = p < re ? __ldg(a_col + p) : -1;
                }
#pragma unroll
                for (int u = 0; u < U; u++)
                    if (c[u] >= 0) part += __ldg(b_rpt + c[u] + 1) - __ldg(b_rpt + c[u]);
            }
            part = warp_sum_ll(part);
            if (lane == i) nip = part;
        }
        if (r < m) {
            int32_t key;
            if (nip > INT32_MAX) {
                report(st, kStNipOverflow, r);
                key = INT32_MAX;
            } else {
                key = static_cast<int32_t>(nip);
            }
            c_rpt[r] = key;
            if (nip_copy != nullptr) nip_copy[r] = key;
            my_tot += nip;
            my_max = max(my_max, key);
            if (key > 0) atomicAdd(&s_hist[find_bin(lad, key)], 1);
        }
    }
    my_tot = warp_sum_ll(my_tot);
    my_max = __reduce_max_sync(0xffffffffu, my_max);
    if (lane == 0) {
        s_tot[w] = my_tot;
        s_max[w] = my_max;
    }
    __syncthreads();
    if (tid == 0) {
        long long t = 0;
        int32_t mx = 0;
        for (int i = 0; i < kBinThreads / kWarp; i++) {
            t += s_tot[i];
            mx = max(mx, s_max[i]);
        }
        atomicAdd(reinterpret_cast<unsigned long long*>(&plan->total_key),
                  static_cast<unsigned long long>(t));
        atomicMax(&plan->max_key, mx);
    }
    if (tid < kMaxBins) hist[blockIdx.x * kMaxBins + tid] = s_hist[tid];
}

// ---- pass 1': nnz histogram + per-CTA nnz sums ----------------------------
__global__ __launch_bounds__(kBinThreads) void k_nnz_hist(
    const int32_t* __restrict__ c_rpt, int32_t m, int32_t* __restrict__ hist,
    int64_t* __restrict__ cta_sum, Plan* __restrict__ plan, const __grid_constant__ Ladder lad,
    const Ladder* __restrict__ dlad) {
    // limits chosen on the device (nullptr: the launch's own)
    const Ladder& L = dlad != nullptr ? *dlad : lad;
    __shared__ int32_t s_hist[kMaxBins];
    __shared__ long long s_tot[kBinThreads / kWarp];
    __shared__ int32_t s_max[kBinThreads / kWarp];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int w = tid >> 5;
    if (tid < kMaxBins) s_hist[tid] = 0;
    __syncthreads();
    long long my_tot = 0;
    int32_t my_max = 0;
    for (int it = 0; it < kBinRowsPerCta / kBinThreads; it++) {
        const int r = blockIdx.x * kBinRowsPerCta + it * kBinThreads + tid;
        if (r < m) {
            const int32_t key = c_rpt[r];
            my_tot += key;
            my_max = max(my_max, key);
            if (key > 0) atomicAdd(&s_hist[find_bin(L, key)], 1);
        }
    }
    my_tot = warp_sum_ll(my_tot);
    my_max = __reduce_max_sync(0xffffffffu, my_max);
    if (lane == 0) {
        s_tot[w] = my_tot;
        s_max[w] = my_max;
    }
    __syncthreads();
    if (tid == 0) {
        long long t = 0;
        int32_t mx = 0;
        for (int i = 0; i < kBinThreads / kWarp; i++) {
            t += s_tot[i];
            mx = max(mx, s_max[i]);
        }
        cta_sum[blockIdx.x] = t;
        atomicMax(&plan->max_key, mx);
    }
    if (tid < kMaxBins) hist[blockIdx.x * kMaxBins + tid] = s_hist[tid];
}

// ---- pass 2: offsets (one CTA) ---------------------------------------------
constexpr int kOffThreads = 1024;

__global__ __launch_bounds__(kOffThreads) void k_bin_offsets(int32_t* __restrict__ hist,
                                                             int32_t nctas,
                                                             int64_t* __restrict__ cta_sum,
                                                             Plan* __restrict__ plan,
                                                             const __grid_constant__ Ladder lad) {
    __shared__ int32_t warp_tot[kOffThreads / kWarp];
    __shared__ long long warp_tot_ll[kOffThreads / kWarp];
    const int tid = threadIdx.x;
    int running = 0;
    for (int b = 0; b < lad.nb; b++) {
        const int start = running;
        for (int c = 0; c < nctas; c += kOffThreads) {
            const int i = c + tid;
            const int v = i < nctas ? hist[i * kMaxBins + b] : 0;
            const int inc = block_inclusive_scan<kOffThreads>(v, warp_tot);
            if (i < nctas) hist[i * kMaxBins + b] = running + inc - v;
            running += warp_tot[kOffThreads / kWarp - 1];
            __syncthreads();
        }
        if (tid == 0) {
            plan->bin_size[b] = running - start;
            plan->bin_off[b] = start;
        }
    }
    if (cta_sum != nullptr) {
        // exclusive scan of the per-CTA nnz sums (int64) -> row-pointer bases
        const int lane = tid & 31;
        const int w = tid >> 5;
        long long run = 0;
        for (int c = 0; c < nctas; c += kOffThreads) {
            const int i = c + tid;
            const long long v = i < nctas ? cta_sum[i] : 0;
            long long x = v;
#pragma unroll
            for (int o = 1; o < kWarp; o <<= 1) {
                const long long t = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += t;
            }
            if (lane == kWarp - 1) warp_tot_ll[w] = x;
            __syncthreads();
            long long before = 0;
            for (int k = 0; k < w; k++) before += warp_tot_ll[k];
            long long total = 0;
            for (int k = 0; k < kOffThreads / kWarp; k++) total += warp_tot_ll[k];
            if (i < nctas) cta_sum[i] = run + before + x - v;
            run += total;
            __syncthreads();
        }
        if (tid == 0) {
            plan->total_key = run;
            plan->overflow = run > INT32_MAX ? 1 : 0;
        }
    }
}

// ---- pass 3: stable scatter (+ exclusive scan into C.rpt) ------------------
__global__ __launch_bounds__(kBinThreads) void k_bin_scatter(
    int32_t* __restrict__ c_rpt, int32_t m, const int32_t* __restrict__ hist_off,
    const int64_t* __restrict__ cta_off, int32_t* __restrict__ bins,
    const Plan* __restrict__ plan, const __grid_constant__ Ladder lad, int scan,
    const Ladder* __restrict__ dlad) {
    const Ladder& L = dlad != nullptr ? *dlad : lad;  // limits chosen on the device, if any
    constexpr int NW = kBinThreads / kWarp;
    __shared__ int32_t s_base[kMaxBins];
    __shared__ int32_t s_off[kMaxBins];
    __shared__ int32_t s_wcnt[NW][kMaxBins];
    __shared__ long long s_wsum[NW];
    __shared__ long long s_run;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int w = tid >> 5;
    if (tid < kMaxBins) {
        s_base[tid] = 0;
        s_off[tid] = hist_off[blockIdx.x * kMaxBins + tid];
    }
    if (tid == 0) s_run = 0;
    const long long base_rpt = scan ? cta_off[blockIdx.x] : 0;
    const unsigned lt_mask = (1u << lane) - 1u;

    for (int it = 0; it < kBinRowsPerCta / kBinThreads; it++) {
        const int r = blockIdx.x * kBinRowsPerCta + it * kBinThreads + tid;
        const int32_t key = r < m ? c_rpt[r] : 0;
        const int bin = key > 0 ? find_bin(L, key) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, bin);
        const int lrank = __popc(peers & lt_mask);
        long long x = key;
        if (scan) {
#pragma unroll
            for (int o = 1; o < kWarp; o <<= 1) {
                const long long t = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += t;
            }
        }
        if (tid < NW * kMaxBins) (&s_wcnt[0][0])[tid] = 0;
        __syncthreads();
        if (lrank == 0 && bin >= 0) s_wcnt[w][bin] = __popc(peers);
        if (scan && lane == kWarp - 1) s_wsum[w] = x;
        __syncthreads();
        if (bin >= 0) {
            int rank = s_base[bin] + lrank;
            for (int k = 0; k < w; k++) rank += s_wcnt[k][bin];
            bins[s_off[bin] + rank] = r;
        }
        if (scan && r < m) {
            long long before = s_run;
            for (int k = 0; k < w; k++) before += s_wsum[k];
            c_rpt[r] = static_cast<int32_t>(base_rpt + before + x - key);
        }
        __syncthreads();
        if (tid < kMaxBins) {
            int add = 0;
            for (int k = 0; k < NW; k++) add += s_wcnt[k][tid];
            s_base[tid] += add;
        }
        if (scan && tid == 0) {
            long long add = 0;
            for (int k = 0; k < NW; k++) add += s_wsum[k];
            s_run += add;
        }
        __syncthreads();
    }
    if (scan && blockIdx.x == gridDim.x - 1 && tid == 0) {
        c_rpt[m] = static_cast<int32_t>(plan->total_key);
    }
}

// ---- one-pass fill: compaction of the rows into C ----------------------------
// Row r's entries sit at [off[r], off[r] + nnz_r) of the temporary arrays (its
// NIP-sized slot); copy them to [rpt[r], rpt[r+1]) of C.  One CTA per chunk
// of kCompactRows rows stages the chunk's row pointers and slot offsets in
// shared memory.  Its warps take tiles of 32 x kCompactUnroll consecutive
// OUTPUT entries; lane l copies entries tile + 32k + l (coalesced writes;
// reads coalesced within rows).  An entry's row is found by one binary search
// per tile and lane, then by stepping the row forward from one of the lane's
// entries to the next -- unless the chunk's rows average fewer than
// kCompactStepMin entries, where every entry does its own binary search.
constexpr int kCompactRows = 256;
constexpr int kCompactThreads = 256;
constexpr int kCompactUnroll = 8;    // entries per lane and tile, in flight together
constexpr int kCompactStepMin = 16;  // mean row length from which rows are stepped

template<typename W>
__global__ __launch_bounds__(kCompactThreads) void k_compact_rows(
    const int32_t* __restrict__ off, const int32_t* __restrict__ rpt, int32_t m,
    const int32_t* __restrict__ tmp_col, const W* __restrict__ tmp_val,
    int32_t* __restrict__ col, W* __restrict__ val) {
    constexpr int NW = kCompactThreads / kWarp;
    constexpr int U = kCompactUnroll;
    __shared__ int32_t s_rpt[kCompactRows + 1];
    __shared__ int32_t s_off[kCompactRows];
    const int r0 = blockIdx.x * kCompactRows;
    const int nr = min(kCompactRows, m - r0);
    for (int i = threadIdx.x; i <= nr; i += kCompactThreads) {
        s_rpt[i] = rpt[r0 + i];
        if (i < nr) s_off[i] = off[r0 + i];
    }
    __syncthreads();
    const int j0 = s_rpt[0];
    const int j1 = s_rpt[nr];
    const bool step = (j1 - j0) >= kCompactStepMin * nr;  // uniform over the CTA
    // the last row i of the chunk with s_rpt[i] <= j
    auto search = [&](int j) {
        int lo = 0;
        int len = nr;
        while (len > 1) {
            const int half = len >> 1;
            lo = s_rpt[lo + half] <= j ? lo + half : lo;
            len -= half;
        }
        return lo;
    };
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    for (int t0 = j0 + w * kWarp * U; t0 < j1; t0 += NW * kWarp * U) {
        int src[U];
        int lo = search(min(t0 + lane, j1 - 1));
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int j = min(t0 + u * kWarp + lane, j1 - 1);
            if (step) {
                while (s_rpt[lo + 1] <= j) lo++;
            } else {
                lo = search(j);
            }
            src[u] = s_off[lo] + (j - s_rpt[lo]);
        }
        int32_t c[U];
        W v[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            c[u] = __ldg(tmp_col + src[u]);
            v[u] = __ldg(tmp_val + src[u]);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int j = t0 + u * kWarp + lane;
            if (j < j1) {
                col[j] = c[u];
                val[j] = v[u];
            }
        }
    }
}

// ---- checked mode: operand validation --------------------------------------
__global__ void k_check_csr(const int32_t* __restrict__ rpt, const int32_t* __restrict__ col,
                            int32_t m, int32_t n, int32_t nnz, DevStatus* __restrict__ st) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r == 0 && (rpt[0] != 0 || rpt[m] != nnz)) report(st, kStBadInput, -1, 0);
    if (r >= m) return;
    const int s0 = rpt[r];
    const int s1 = rpt[r + 1];
    if (s0 > s1 || s0 < 0 || s1 > nnz) {
        report(st, kStBadInput, r, 1);
        return;
    }
    int prev = -1;
    for (int p = s0; p < s1; p++) {
        const int c = col[p];
        if (c < 0 || c >= n || c <= prev) {
            report(st, kStBadInput, r, 2);
            return;
        }
        prev = c;
    }
}

__global__ void k_total_nip(const int32_t* __restrict__ a_rpt, const int32_t* __restrict__ a_col,
                            const int32_t* __restrict__ b_rpt, int32_t m,
                            unsigned long long* __restrict__ out) {
    long long s = 0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x) {
        for (int p = a_rpt[r]; p < a_rpt[r + 1]; p++) {
            const int c = a_col[p];
            s += b_rpt[c + 1] - b_rpt[c];
        }
    }
    s = warp_sum_ll(s);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, static_cast<unsigned long long>(s));
}

}  // namespace

cudaError_t launch_nip_hist(const int32_t* a_rpt, const int32_t* a_col, const int32_t* b_rpt,
                            int32_t m, int32_t* c_rpt, int32_t* nip_copy, int32_t* hist,
                            Plan* plan, DevStatus* st, const Ladder& lad, cudaStream_t s) {
    const int g = bin_ctas(m);
    if (g == 0) return cudaSuccess;
    k_nip_hist<<<g, kBinThreads, 0, s>>>(a_rpt, a_col, b_rpt, m, c_rpt, nip_copy, hist, plan, st,
                                         lad);
    return cudaGetLastError();
}

cudaError_t launch_nnz_hist(const int32_t* c_rpt, int32_t m, int32_t* hist, int64_t* cta_sum,
                            Plan* plan, const Ladder& lad, cudaStream_t s, const Ladder* dlad) {
    const int g = bin_ctas(m);
    if (g == 0) return cudaSuccess;
    k_nnz_hist<<<g, kBinThreads, 0, s>>>(c_rpt, m, hist, cta_sum, plan, lad, dlad);
    return cudaGetLastError();
}

cudaError_t launch_bin_offsets(int32_t* hist, int32_t nctas, int64_t* cta_sum, Plan* plan,
                               const Ladder& lad, cudaStream_t s) {
    k_bin_offsets<<<1, kOffThreads, 0, s>>>(hist, nctas, cta_sum, plan, lad);
    return cudaGetLastError();
}

cudaError_t launch_bin_scatter(int32_t* c_rpt, int32_t m, const int32_t* hist_off,
                               const int64_t* cta_off, int32_t* bins, const Plan* plan,
                               const Ladder& lad, bool scan, cudaStream_t s, const Ladder* dlad) {
    const int g = bin_ctas(m);
    if (g == 0) return cudaSuccess;
    k_bin_scatter<<<g, kBinThreads, 0, s>>>(c_rpt, m, hist_off, cta_off, bins, plan, lad,
                                            scan ? 1 : 0, dlad);
    return cudaGetLastError();
}

cudaError_t launch_compact_rows(const int32_t* off, const int32_t* rpt, int32_t m,
                                const int32_t* tmp_col, const void* tmp_val, int32_t* col,
                                void* val, int value_bytes, cudaStream_t s) {
    if (m <= 0) return cudaSuccess;
    const int g = (m + kCompactRows - 1) / kCompactRows;
    if (value_bytes == 8)
        k_compact_rows<long long><<<g, kCompactThreads, 0, s>>>(
            off, rpt, m, tmp_col, static_cast<const long long*>(tmp_val), col,
            static_cast<long long*>(val));
    else
        k_compact_rows<int32_t><<<g, kCompactThreads, 0, s>>>(
            off, rpt, m, tmp_col, static_cast<const int32_t*>(tmp_val), col,
            static_cast<int32_t*>(val));
    return cudaGetLastError();
}

cudaError_t launch_check_csr(const int32_t* rpt, const int32_t* col, int32_t m, int32_t n,
                             int32_t nnz, DevStatus* st, cudaStream_t s) {
    const int g = (m + 255) / 256;
    k_check_csr<<<g > 0 ? g : 1, 256, 0, s>>>(rpt, col, m, n, nnz, st);
    return cudaGetLastError();
}

cudaError_t launch_total_nip(const int32_t* a_rpt, const int32_t* a_col, const int32_t* b_rpt,
                             int32_t m, long long* out, cudaStream_t s) {
    int g = (m + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    if (g == 0) return cudaSuccess;
    k_total_nip<<<g, 256, 0, s>>>(a_rpt, a_col, b_rpt, m,
                                  reinterpret_cast<unsigned long long*>(out));
    return cudaGetLastError();
}

}  // namespace b200
