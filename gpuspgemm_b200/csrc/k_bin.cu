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
constexpr int kNipThreads = 256;  // kBinRowsPerCta rows per CTA, as the other passes

__global__ __launch_bounds__(kNipThreads) void k_nip_hist(
    const int32_t* __restrict__ a_rpt, const int32_t* __restrict__ a_col,
    const int32_t* __restrict__ b_rpt, int32_t m, int32_t* __restrict__ c_rpt,
    int32_t* __restrict__ nip_copy, int32_t* __restrict__ hist, Plan* __restrict__ plan,
    DevStatus* __restrict__ st, const __grid_constant__ Ladder lad,
    int32_t* __restrict__ hist_fill, int64_t* __restrict__ cta_sum,
    const __grid_constant__ Ladder fill) {
    __shared__ int32_t s_hist[kMaxBins];
    __shared__ int32_t s_hist_fill[kMaxBins];
    __shared__ long long s_tot[kNipThreads / kWarp];
    __shared__ int32_t s_max[kNipThreads / kWarp];
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int w = tid >> 5;
    if (tid < kMaxBins) {
        s_hist[tid] = 0;
        s_hist_fill[tid] = 0;
    }
    __syncthreads();

    constexpr int kGroups = kBinRowsPerCta / kWarp / (kNipThreads / kWarp);  // per warp
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
            if (key > 0) {
                atomicAdd(&s_hist[find_bin(lad, key)], 1);
                if (hist_fill != nullptr) atomicAdd(&s_hist_fill[find_bin(fill, key)], 1);
            }
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
        for (int i = 0; i < kNipThreads / kWarp; i++) {
            t += s_tot[i];
            mx = max(mx, s_max[i]);
        }
        atomicAdd(reinterpret_cast<unsigned long long*>(&plan->total_key),
                  static_cast<unsigned long long>(t));
        atomicMax(&plan->max_key, mx);
        if (cta_sum != nullptr) cta_sum[blockIdx.x] = t;
    }
    if (tid < kMaxBins) {
        hist[blockIdx.x * kMaxBins + tid] = s_hist[tid];
        if (hist_fill != nullptr) hist_fill[blockIdx.x * kMaxBins + tid] = s_hist_fill[tid];
    }
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

// ---- pass 2, all bins at once (one CTA) ------------------------------------
// The per-CTA histograms src_hist[i][e] count rows by a source ladder `src`
// (e.g. the NIP pass's fill ladder, whose limits include every limit the
// device may choose); each source bin maps to the final ladder's bin (dlad
// when given, else lad) that holds its upper limit.  hist[i][b] receives CTA
// i's first position in final bin b RELATIVE to the bin's start (the scatter
// adds plan->bin_off), cta_sum (when given) its exclusive scan.  Per chunk of
// kOffMapChunk CTAs: every thread stages one CTA's final-bin counts in shared
// memory, then a warp per bin (and one for the CTA sums) scans them -- each
// lane 32 consecutive CTAs, one warp scan of the lanes' sums.  One pass over
// the histograms and two block barriers per chunk, where k_bin_offsets scans
// bin after bin with the whole CTA.
constexpr int kOffMapThreads = 1024;
constexpr int kOffMapChunk = kOffMapThreads;  // a CTA's count in a bin fits 16 bits

// staged element j of a chunk: one spare slot per 32 keeps the lanes' runs of
// 32 in distinct banks
__device__ __forceinline__ int offmap_pad(int j) { return j + (j >> 5); }

__global__ __launch_bounds__(kOffMapThreads) void k_bin_offsets_map(
    const int32_t* __restrict__ src_hist, int32_t* __restrict__ hist, int32_t nctas,
    const __grid_constant__ Ladder src, int64_t* __restrict__ cta_sum, Plan* __restrict__ plan,
    const __grid_constant__ Ladder lad, const Ladder* __restrict__ dlad,
    unsigned long long* __restrict__ zero, int32_t nzero) {
    constexpr int NW = kOffMapThreads / kWarp;
    constexpr int PADDED = kOffMapChunk + kOffMapChunk / kWarp;
    // words a later kernel of the product needs zeroed (the row pointer's
    // look-back state): cleared here instead of by a memset of their own
    for (int i = threadIdx.x; i < nzero; i += kOffMapThreads) zero[i] = 0ull;
    static_assert(NW > kMaxBins, "a warp per bin and one for the CTA sums");
    static_assert(kBinRowsPerCta < 65536, "16-bit counts");
    __shared__ uint16_t s_cnt[kMaxBins][PADDED + 1];
    __shared__ long long s_sum[PADDED];
    __shared__ int32_t s_map[kMaxBins];
    __shared__ int32_t s_e0[kMaxBins];
    __shared__ int32_t s_e1[kMaxBins];
    __shared__ int32_t s_tot[kMaxBins];
    const Ladder& L = dlad != nullptr ? *dlad : lad;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int w = tid >> 5;
    const int nb = L.nb;
    const int ne = src.nb;
    const bool sums = cta_sum != nullptr;
    if (tid < kMaxBins) {
        int b = nb - 1;
        if (tid < ne) {
            const int32_t u = src.limit[tid];
            for (int i = 0; i < nb; i++) {
                if (u <= L.limit[i]) {
                    b = i;
                    break;
                }
            }
            b = b < L.min_bin ? L.min_bin : b;
        }
        s_map[tid] = b;
        s_e0[tid] = ne;
        s_e1[tid] = ne;
    }
    __syncthreads();
    if (tid == 0) {
        // each final bin's range of source bins (the map is monotone; empty
        // ranges start at ne)
        for (int e = ne - 1; e >= 0; e--) s_e0[s_map[e]] = e;
        for (int e = 0; e < ne; e++) s_e1[s_map[e]] = e + 1;
        for (int b = 0; b < nb; b++)
            if (s_e1[b] < s_e0[b]) s_e1[b] = s_e0[b];
    }
    __syncthreads();
    const bool scans_bin = w < nb;
    const bool scans_sums = w == NW - 1 && sums;
    long long run = 0;  // this warp's bin (or the CTA sums) so far
    for (int c0 = 0; c0 < nctas; c0 += kOffMapChunk) {
        // stage: thread tid holds CTA c0 + tid
        {
            const int i = c0 + tid;
            for (int b = 0; b < nb; b++) {
                int32_t c = 0;
                if (i < nctas)
                    for (int e = s_e0[b]; e < s_e1[b]; e++) c += src_hist[i * kMaxBins + e];
                s_cnt[b][offmap_pad(tid)] = static_cast<uint16_t>(c);
            }
            if (sums) s_sum[offmap_pad(tid)] = i < nctas ? cta_sum[i] : 0;
        }
        __syncthreads();
        if (scans_bin || scans_sums) {
            // lane: CTAs [c0 + 32 lane, c0 + 32 lane + 32)
            long long part = 0;
#pragma unroll 8
            for (int k = 0; k < kWarp; k++) {
                const int j = offmap_pad(lane * kWarp + k);
                part += scans_bin ? static_cast<long long>(s_cnt[w][j]) : s_sum[j];
            }
            long long x = part;
#pragma unroll
            for (int o = 1; o < kWarp; o <<= 1) {
                const long long t = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += t;
            }
            long long acc = run + x - part;
            for (int k = 0; k < kWarp; k++) {
                const int i = c0 + lane * kWarp + k;
                if (i >= nctas) break;
                const int j = offmap_pad(lane * kWarp + k);
                if (scans_bin) {
                    hist[i * kMaxBins + w] = static_cast<int32_t>(acc);
                    acc += s_cnt[w][j];
                } else {
                    cta_sum[i] = acc;
                    acc += s_sum[j];
                }
            }
            run += __shfl_sync(0xffffffffu, x, kWarp - 1);
        }
        __syncthreads();
    }
    if (scans_bin && lane == 0) s_tot[w] = static_cast<int32_t>(run);
    if (scans_sums && lane == 0) {
        plan->total_key = run;
        plan->overflow = run > INT32_MAX ? 1 : 0;
    }
    __syncthreads();
    if (tid == 0) {
        int32_t off = 0;
        for (int b = 0; b < nb; b++) {
            plan->bin_size[b] = s_tot[b];
            plan->bin_off[b] = off;
            off += s_tot[b];
        }
    }
}

// ---- pass 3: stable scatter (+ exclusive scan into C.rpt) ------------------
__global__ __launch_bounds__(kBinThreads) void k_bin_scatter(
    int32_t* __restrict__ c_rpt, int32_t m, const int32_t* __restrict__ hist_off,
    const int64_t* __restrict__ cta_off, int32_t* __restrict__ bins,
    const Plan* __restrict__ plan, const __grid_constant__ Ladder lad, int scan,
    const Ladder* __restrict__ dlad, int bin_relative) {
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
        // offsets within each bin (k_bin_offsets_map) or of the row list
        s_off[tid] = hist_off[blockIdx.x * kMaxBins + tid] +
                     (bin_relative && tid < L.nb ? plan->bin_off[tid] : 0);
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

// ---- one-pass row pointer -----------------------------------------------------
// The rows' nnz become the row pointer in place, tile by tile (kScanTile rows
// a CTA): 8 bytes of traffic per row, where a one-bin pass of the binning
// kernels takes three launches and also writes a row list.
constexpr int kScanThreads = 256;
constexpr int kScanPer = kScanTile / kScanThreads;  // rows per thread
static_assert(kScanPer * kScanThreads == kScanTile, "tile");

// the tile in shared memory, one padding word per 32 (thread t reads its
// kScanPer consecutive rows without bank conflicts)
__device__ __forceinline__ int scan_pad(int i) { return i + (i >> 5); }

// One launch, the tiles chained by decoupled look-back.
// Each CTA takes the next tile from a ticket counter (state[0]), so every tile
// before its own belongs to a CTA that has already started; it scans its tile
// in shared memory and publishes the tile's sum in state[1 + tile].  Warp 0
// then reads the states of the tiles before it, 32 at a time, adding their
// sums back to the nearest tile that has published its prefix (the sum of the
// counts through that tile), and publishes its own prefix.  A state word holds
// its kind in the top two bits (0: nothing yet, kTileSum, kTilePrefix) and the
// value below them; the counter and states are zeroed before the launch.  The
// waits are bounded: past kLookbackSpins rounds the CTA reports kStWait and
// goes on with what it has, and the call fails on the status.  (It replaced a
// reduce launch plus a scan launch: 1M rows 0.021 -> 0.011 ms.)
constexpr unsigned long long kTileSum = 1ull << 62;
constexpr unsigned long long kTilePrefix = 2ull << 62;
constexpr unsigned long long kTileValue = (1ull << 62) - 1ull;
constexpr int kLookbackSpins = 1 << 20;

__global__ __launch_bounds__(kScanThreads) void k_rpt_scan1(int32_t* __restrict__ cnt, int32_t m,
                                                            int32_t ntiles,
                                                            unsigned long long* __restrict__ state,
                                                            Plan* __restrict__ plan,
                                                            DevStatus* __restrict__ st) {
    constexpr int NW = kScanThreads / kWarp;
    constexpr unsigned kAll = 0xffffffffu;
    __shared__ int32_t s_row[kScanTile + kScanTile / 32];
    __shared__ int32_t s_wtot[NW];
    __shared__ int32_t s_wmax[NW];
    __shared__ int32_t s_tile;
    __shared__ long long s_base;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int w = tid >> 5;
    if (tid == 0) s_tile = static_cast<int32_t>(atomicAdd(state, 1ull));
    __syncthreads();
    const int tile = s_tile;
    if (tile >= ntiles) {  // a counter left from an earlier launch: uniform over the CTA
        if (tid == 0) report(st, kStIndex, tile, ntiles);
        return;
    }
    const long long r0 = static_cast<long long>(tile) * kScanTile;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        const int j = k * kScanThreads + tid;
        s_row[scan_pad(j)] = r0 + j < m ? cnt[r0 + j] : 0;
    }
    __syncthreads();
    // thread tid: rows [tid * kScanPer, (tid + 1) * kScanPer) of the tile
    int v[kScanPer];
    int run = 0;
    int mx = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        v[k] = s_row[scan_pad(tid * kScanPer + k)];
        run += v[k];
        mx = max(mx, v[k]);
    }
    mx = __reduce_max_sync(kAll, mx);
    if (lane == 0) s_wmax[w] = mx;
    const int inc = block_inclusive_scan<kScanThreads>(run, s_wtot);
    __syncthreads();
    if (w == 0) {
        const long long tsum = static_cast<unsigned>(s_wtot[NW - 1]);  // counts: >= 0
        int tmax = lane < NW ? s_wmax[lane] : 0;
        tmax = __reduce_max_sync(kAll, tmax);
        if (lane == 0) {
            atomicMax(&plan->max_key, tmax);
            atomicExch(state + 1 + tile, (tile == 0 ? kTilePrefix : kTileSum) |
                                             min(static_cast<unsigned long long>(tsum), kTileValue));
        }
        long long excl = 0;
        int pred = tile - 1;
        int spins = 0;
        while (pred >= 0) {
            const int t = pred - lane;
            const unsigned long long f =
                t >= 0 ? static_cast<unsigned long long>(
                             *reinterpret_cast<volatile unsigned long long*>(state + 1 + t))
                       : kTilePrefix;
            const unsigned kind = static_cast<unsigned>(f >> 62);
            const unsigned pre = __ballot_sync(kAll, kind == 2u);
            // the lanes up to the nearest prefix (all 32 when there is none)
            const unsigned upto = pre != 0u ? ((pre & (0u - pre)) << 1) - 1u : kAll;
            if ((__ballot_sync(kAll, kind == 0u) & upto) != 0u) {
                if (++spins > kLookbackSpins) {
                    if (lane == 0) report(st, kStWait, tile, pred);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            const long long x = (upto >> lane) & 1u ? static_cast<long long>(f & kTileValue) : 0;
            excl += warp_sum_ll(x);
            if (pre != 0u) break;
            pred -= kWarp;
        }
        if (lane == 0) {
            if (tile > 0)
                atomicExch(state + 1 + tile,
                           kTilePrefix | min(static_cast<unsigned long long>(excl + tsum), kTileValue));
            s_base = excl;
        }
    }
    __syncthreads();
    const long long base = s_base;
    // int arithmetic inside the tile: it wraps only when the total leaves
    // int32, which the plan's int64 total flags
    int pos = static_cast<int>(base) + inc - run;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        s_row[scan_pad(tid * kScanPer + k)] = pos;
        pos += v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        const int j = k * kScanThreads + tid;
        if (r0 + j < m) cnt[r0 + j] = s_row[scan_pad(j)];
    }
    if (tile == ntiles - 1 && tid == 0) {
        const long long total = base + static_cast<unsigned>(s_wtot[NW - 1]);
        cnt[m] = static_cast<int32_t>(total);
        plan->total_key = total;
        plan->overflow = total > INT32_MAX ? 1 : 0;
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
// The slots are read once, with cache-streaming loads (evict first), so they
// do not push C's freshly written lines out of L2.  (On the 1M-row power-law
// product, FP64: 256-row chunks with plain loads 0.165 ms; streaming loads
// 0.143; with 64-row chunks as well, 0.136 -- more, shorter CTAs.)
constexpr int kCompactRows = 64;
constexpr int kCompactThreads = 256;
constexpr int kCompactUnroll = 8;    // entries per lane and tile, in flight together
constexpr int kCompactStepMin = 16;  // mean row length from which rows are stepped

template<typename W>
__global__ __launch_bounds__(kCompactThreads) void k_compact_rows(
    const int32_t* __restrict__ off, const int32_t* __restrict__ rpt, int32_t m,
    const int32_t* __restrict__ tmp_col, const W* __restrict__ tmp_val,
    int32_t* __restrict__ col, W* __restrict__ val, int32_t cap) {
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
    const int j1 = min(s_rpt[nr], cap);  // a count past C's capacity is reported by the host
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
            c[u] = __ldcs(tmp_col + src[u]);
            v[u] = __ldcs(tmp_val + src[u]);
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
                            Plan* plan, DevStatus* st, const Ladder& lad, cudaStream_t s,
                            int32_t* hist_fill, int64_t* cta_sum, const Ladder* fill) {
    const int g = bin_ctas(m);
    if (g == 0) return cudaSuccess;
    const Ladder none = {};
    k_nip_hist<<<g, kNipThreads, 0, s>>>(a_rpt, a_col, b_rpt, m, c_rpt, nip_copy, hist, plan, st,
                                         lad, fill != nullptr ? hist_fill : nullptr,
                                         fill != nullptr ? cta_sum : nullptr,
                                         fill != nullptr ? *fill : none);
    return cudaGetLastError();
}

cudaError_t launch_bin_offsets_map(const int32_t* src_hist, int32_t* hist, int32_t nctas,
                                   const Ladder& src, int64_t* cta_sum, Plan* plan,
                                   const Ladder& lad, const Ladder* dlad, cudaStream_t s,
                                   unsigned long long* zero, int32_t nzero) {
    k_bin_offsets_map<<<1, kOffMapThreads, 0, s>>>(src_hist, hist, nctas, src, cta_sum, plan, lad,
                                                   dlad, zero, nzero);
    return cudaGetLastError();
}

cudaError_t launch_rpt_scan1(int32_t* cnt, int32_t m, unsigned long long* state, Plan* plan,
                             DevStatus* st, cudaStream_t s) {
    if (m <= 0) return cudaSuccess;
    const int tiles = rpt_scan_tiles(m);
    k_rpt_scan1<<<tiles, kScanThreads, 0, s>>>(cnt, m, tiles, state, plan, st);
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
                               const Ladder& lad, bool scan, cudaStream_t s, const Ladder* dlad,
                               bool bin_relative) {
    const int g = bin_ctas(m);
    if (g == 0) return cudaSuccess;
    k_bin_scatter<<<g, kBinThreads, 0, s>>>(c_rpt, m, hist_off, cta_off, bins, plan, lad,
                                            scan ? 1 : 0, dlad, bin_relative ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_compact_rows(const int32_t* off, const int32_t* rpt, int32_t m,
                                const int32_t* tmp_col, const void* tmp_val, int32_t* col,
                                void* val, int value_bytes, cudaStream_t s, int32_t cap) {
    if (m <= 0) return cudaSuccess;
    const int g = (m + kCompactRows - 1) / kCompactRows;
    if (value_bytes == 8)
        k_compact_rows<long long><<<g, kCompactThreads, 0, s>>>(
            off, rpt, m, tmp_col, static_cast<const long long*>(tmp_val), col,
            static_cast<long long*>(val), cap);
    else
        k_compact_rows<int32_t><<<g, kCompactThreads, 0, s>>>(
            off, rpt, m, tmp_col, static_cast<const int32_t*>(tmp_val), col,
            static_cast<int32_t*>(val), cap);
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
