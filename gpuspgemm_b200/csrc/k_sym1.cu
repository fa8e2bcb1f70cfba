// Symbolic phase 1: exact nnz of every row of C (the count of distinct column
// keys among the row's intermediate products), one kernel per row bin.
// Replaces sym1.cuh:28-306 (k_sym1_smem_pwarp / k_sym1_smem / k_sym1_smem_max /
// k_sym1_global).  Output: c_rpt[row] = nnz(row).
//
// Ladder (key = NIP of the row; a table of T slots is never more than 80 %
// full, the reference's SYM1_RANGE_RATIO 1/1.2, parameters.cuh:12-16):
//   team bins   4/8/16/32 lanes per row, several rows per CTA
//   CTA bins    one row per CTA, tables up to 216 KB of shared memory
//   cluster bin the largest rows: one table spread over a thread-block
//               cluster's distributed shared memory; a row whose distinct
//               count outgrows it is appended to a fail list
//   global bin  fail-list rows: a bitmap over B's columns in global memory
#include <cooperative_groups.h>

#include "cluster_insert.cuh"
#include "cta.cuh"
#include "kernels.hpp"

namespace cg = cooperative_groups;

namespace b200 {

namespace {

template<int G, int THREADS, int T>
__global__ __launch_bounds__(THREADS) void k_sym1_team(ProductArgs p) {
    constexpr int R = THREADS / G;
    extern __shared__ int32_t smem[];
    const int team = threadIdx.x / G;
    const int lane = team_lane<G>();
    const unsigned mask = team_mask<G>();
    const int rid = blockIdx.x * R + team;
    if (rid >= p.nrows) return;  // whole team leaves together
    int32_t* table = smem + team * T;
    for (int i = lane; i < T; i += G) table[i] = kEmpty;
    team_sync<G>(mask);
    const int row = p.rows[rid];
    const int a0 = p.a_rpt[row];
    const int a1 = p.a_rpt[row + 1];
    int cnt = 0;
    team_for_products<G>(p.a_col, p.b_rpt, a0, a1, [&](int qb, int) {
        cnt += table_insert(table, T, __ldg(p.b_col + qb), p.status, row);
    });
    cnt = team_sum<G>(mask, cnt);
    if (lane == 0) p.c_rpt[row] = cnt;
}

template<int THREADS, int T>
__global__ __launch_bounds__(THREADS) void k_sym1_cta(ProductArgs p) {
    extern __shared__ int32_t smem[];
    auto& sc = *reinterpret_cast<CtaScratch<THREADS>*>(smem + T);
    const int row = p.rows[blockIdx.x];
    for (int i = threadIdx.x; i < T; i += THREADS) smem[i] = kEmpty;
    __syncthreads();
    const int a0 = p.a_rpt[row];
    const int a1 = p.a_rpt[row + 1];
    int cnt = 0;
    cta_for_products<THREADS>(p.a_col, p.b_rpt, a0, a1, sc, [&](int qb, int) {
        cnt += table_insert(smem, T, __ldg(p.b_col + qb), p.status, row);
    });
    cnt = block_sum<THREADS>(cnt, sc.warp_tot);
    if (threadIdx.x == 0) p.c_rpt[row] = cnt;
}

// Cluster bin: the row's table is split over the cluster's CTAs; slot h of the
// global table lives in CTA h / T of the cluster at local slot h % T, reached
// through distributed shared memory (ld/st/atom.shared::cluster; no TMA).
// The CTAs of the cluster share the row's products.  A row whose distinct
// count passes 80 % of the cluster capacity, or one of whose keys probes
// kClusterMaxProbes slots, stops and goes to the fail list (the reference's
// k_sym1_smem_max spills per CTA on its per-insert load test,
// sym1.cuh:171-245).  The insert and its bounds are cluster_insert.cuh's.
struct ClusterTableOps {
    cg::cluster_group cluster;
    int32_t* table;      // this CTA's T slots (the same offset in every CTA)
    int32_t* s_count;    // this CTA's new-key count
    int32_t* s_spill;    // this CTA's copy of the row's spill flag
    int32_t* s_total;    // the published total (read through CTA 0)
    uint32_t T;
    uint32_t nslots;
    int32_t load_limit;
    int32_t ncta;

    __device__ uint32_t slots() const { return nslots; }
    __device__ int32_t empty() const { return kEmpty; }
    __device__ int32_t limit() const { return load_limit; }
    __device__ int32_t csize() const { return ncta; }
    __device__ int32_t cas(uint32_t h, int32_t key) {
        int32_t* slot = cluster.map_shared_rank(table + (h % T), static_cast<int>(h / T));
        return atomicCAS(slot, kEmpty, key);
    }
    __device__ bool spilled() { return *reinterpret_cast<volatile int32_t*>(s_spill) != 0; }
    __device__ void spill() {
        for (int r = 0; r < ncta; r++) atomicExch(cluster.map_shared_rank(s_spill, r), 1);
    }
    __device__ int32_t count_local() { return atomicAdd(s_count, 1); }
    __device__ int32_t publish(int32_t add) {
        return atomicAdd(cluster.map_shared_rank(s_total, 0), add) + add;
    }
};

template<int THREADS, int T>
__global__ __launch_bounds__(THREADS) void k_sym1_cluster(ProductArgs p) {
    extern __shared__ int32_t smem[];
    auto& sc = *reinterpret_cast<CtaScratch<THREADS>*>(smem + T);
    __shared__ int32_t s_count;   // distinct keys inserted by this CTA
    __shared__ int32_t s_spill;   // the row's spill flag (every CTA holds a copy)
    __shared__ int32_t s_total;   // published count (used in CTA 0)
    cg::cluster_group cluster = cg::this_cluster();
    const int csize = static_cast<int>(cluster.num_blocks());
    const int crank = static_cast<int>(cluster.block_rank());
    const uint32_t total_slots = static_cast<uint32_t>(T) * static_cast<uint32_t>(csize);
    const int rid = blockIdx.x / csize;
    const int row = p.rows[rid];

    for (int i = threadIdx.x; i < T; i += THREADS) smem[i] = kEmpty;
    if (threadIdx.x == 0) {
        s_count = 0;
        s_spill = 0;
        s_total = 0;
    }
    cluster.sync();

    ClusterTableOps ops{cluster, smem, &s_count, &s_spill, &s_total, static_cast<uint32_t>(T),
                        total_slots, static_cast<int32_t>(0.8 * static_cast<double>(total_slots)),
                        csize};
    const int a0 = p.a_rpt[row];
    const int a1 = p.a_rpt[row + 1];
    // the cluster walks the row's A entries in slices of THREADS, CTA c taking
    // slices c, c + csize, ...
    for (int base = a0 + crank * THREADS; base < a1; base += csize * THREADS) {
        const int end = min(base + THREADS, a1);
        if (__syncthreads_or(ops.spilled() ? 1 : 0)) break;
        // lanes holding the same key elect one lane to probe the remote table
        // (each probe is a CAS in another CTA's shared memory)
        cta_for_products_mlp<THREADS, 2, true>(
            p.a_col, p.b_rpt, base, end, sc, [&](int qb, int, int) { return __ldg(p.b_col + qb); },
            [&](int32_t key, int, int, int, bool valid) {
                const unsigned peers = __match_any_sync(0xffffffffu, valid ? key : kEmpty);
                const bool leader =
                    (threadIdx.x & 31u) == static_cast<unsigned>(__ffs(peers) - 1);
                if (valid && leader && !ops.spilled()) cluster_insert(ops, key);
            });
    }
    cluster.sync();
    if (crank == 0 && threadIdx.x == 0) {
        if (s_spill != 0) {
            const int idx = atomicAdd(p.fail_count, 1);
            p.fail_rows[idx] = row;
            p.c_rpt[row] = 0;
        } else {
            int total = 0;
            for (int r = 0; r < csize; r++) total += *cluster.map_shared_rank(&s_count, r);
            p.c_rpt[row] = total;
        }
    }
    cluster.sync();  // no CTA leaves while another may still touch its table
}

// Global bin: a bitmap per row in flight (global scratch, B.n bits per CTA),
// of which only the row's column window [lo, hi] is cleared and used -- a
// row of a block-diagonal batch touches one block's columns, not all of B's.
// atomicOr tells whether a key is new; the count is exact.  A key outside
// the window (B rows not sorted) redoes the row over [0, B.n).
template<int THREADS>
__global__ __launch_bounds__(THREADS) void k_sym1_global(ProductArgs p) {
    __shared__ CtaScratch<THREADS> sc;
    uint32_t* bm = p.bitmaps + static_cast<int64_t>(blockIdx.x) * p.words;
    // nrows < 0: the rows are a fail list whose length is on the device
    const int nrows = p.nrows >= 0 ? p.nrows : *reinterpret_cast<volatile int32_t*>(p.fail_count);
    for (int rid = blockIdx.x; rid < nrows; rid += gridDim.x) {
        const int row = p.rows[rid];
        const int a0 = p.a_rpt[row];
        const int a1 = p.a_rpt[row + 1];
        const int2 win = cta_col_window<THREADS>(p.a_col, p.b_rpt, p.b_col, a0, a1, p.n_cols, sc);
        int lo = win.x;
        int hi = win.y;
        for (int pass = 0; pass < 2; pass++) {
            const int w0 = lo >> 5;
            const int nwords = hi >= lo ? (hi >> 5) - w0 + 1 : 0;
            for (int i = threadIdx.x; i < nwords; i += THREADS) bm[i] = 0u;
            __syncthreads();
            int cnt = 0;
            int miss = 0;
            cta_for_products<THREADS>(p.a_col, p.b_rpt, a0, a1, sc, [&](int qb, int) {
                const int32_t key = __ldg(p.b_col + qb);
                if (key < lo || key > hi) {
                    miss = 1;
                    return;
                }
                const uint32_t bit = 1u << (key & 31);
                const uint32_t old = atomicOr(bm + ((key >> 5) - w0), bit);
                cnt += (old & bit) ? 0 : 1;
            });
            if (!__syncthreads_or(miss)) {
                cnt = block_sum<THREADS>(cnt, sc.warp_tot);
                if (threadIdx.x == 0) p.c_rpt[row] = cnt;
                __syncthreads();
                break;
            }
            if (pass == 1) {  // a column index outside [0, B.n)
                if (threadIdx.x == 0) report(p.status, kStBadInput, row);
                break;
            }
            lo = 0;
            hi = p.n_cols - 1;
        }
    }
}

template<int G, int THREADS, int T>
cudaError_t launch_team(const ProductArgs& p, cudaStream_t s) {
    constexpr int R = THREADS / G;
    const int grid = (p.nrows + R - 1) / R;
    k_sym1_team<G, THREADS, T><<<grid, THREADS, sizeof(int32_t) * R * T, s>>>(p);
    return cudaGetLastError();
}

template<int THREADS, int T>
constexpr size_t cta_smem() {
    return sizeof(int32_t) * T + sizeof(CtaScratch<THREADS>);
}

template<int THREADS, int T>
cudaError_t launch_cta(const ProductArgs& p, cudaStream_t s) {
    k_sym1_cta<THREADS, T><<<p.nrows, THREADS, cta_smem<THREADS, T>(), s>>>(p);
    return cudaGetLastError();
}

template<int THREADS, int T>
cudaError_t launch_cluster(const ProductArgs& p, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(p.nrows * p.cluster));
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = cta_smem<THREADS, T>();
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(p.cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_sym1_cluster<THREADS, T>, p);
}

template<int THREADS>
cudaError_t launch_global(const ProductArgs& p, cudaStream_t s) {
    const int grid = (p.nrows >= 0 && p.nrows < p.nmaps) ? p.nrows : p.nmaps;
    k_sym1_global<THREADS><<<grid, THREADS, 0, s>>>(p);
    return cudaGetLastError();
}

// Team bins: (lanes per row, threads, table slots); limit = 80 % of slots.
// CTA bins: (threads, table slots).  The last CTA bin uses 216 KB of table.
constexpr int kT0 = 32, kT1 = 128, kT2 = 512, kT3 = 2048;
constexpr int kC4 = 8192, kC5 = 24576, kC6 = 55296;

constexpr int lim(int T) { return static_cast<int>(0.8 * T); }

const BinLauncher kLadder[] = {
    {BinKind::Team, lim(kT0), 256 / 4, 256, sizeof(int32_t) * (256 / 4) * kT0, "sym1_team4_t32",
     launch_team<4, 256, kT0>},
    {BinKind::Team, lim(kT1), 256 / 8, 256, sizeof(int32_t) * (256 / 8) * kT1, "sym1_team8_t128",
     launch_team<8, 256, kT1>},
    {BinKind::Team, lim(kT2), 256 / 16, 256, sizeof(int32_t) * (256 / 16) * kT2,
     "sym1_team16_t512", launch_team<16, 256, kT2>},
    {BinKind::Team, lim(kT3), 256 / 32, 256, sizeof(int32_t) * (256 / 32) * kT3,
     "sym1_team32_t2048", launch_team<32, 256, kT3>},
    {BinKind::Cta, lim(kC4), 1, 256, cta_smem<256, kC4>(), "sym1_cta256_t8192",
     launch_cta<256, kC4>},
    {BinKind::Cta, lim(kC5), 1, 512, cta_smem<512, kC5>(), "sym1_cta512_t24576",
     launch_cta<512, kC5>},
    {BinKind::Cta, lim(kC6), 1, 1024, cta_smem<1024, kC6>(), "sym1_cta1024_t55296",
     launch_cta<1024, kC6>},
    {BinKind::Cluster, INT32_MAX, 1, 1024, cta_smem<1024, kC6>(), "sym1_cluster_t55296",
     launch_cluster<1024, kC6>},
    {BinKind::Global, INT32_MAX, 1, 1024, 0, "sym1_global_bitmap", launch_global<1024>},
};

}  // namespace

int sym1_ladder(const BinLauncher** out) {
    *out = kLadder;
    return static_cast<int>(sizeof(kLadder) / sizeof(kLadder[0]));
}

cudaError_t sym1_prepare() {
    cudaError_t e = cudaSuccess;
#define B200_SMEM(kern, bytes)                                                            \
    if (e == cudaSuccess)                                                                 \
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                 static_cast<int>(bytes));
    B200_SMEM((k_sym1_team<4, 256, kT0>), kLadder[0].smem);
    B200_SMEM((k_sym1_team<8, 256, kT1>), kLadder[1].smem);
    B200_SMEM((k_sym1_team<16, 256, kT2>), kLadder[2].smem);
    B200_SMEM((k_sym1_team<32, 256, kT3>), kLadder[3].smem);
    B200_SMEM((k_sym1_cta<256, kC4>), kLadder[4].smem);
    B200_SMEM((k_sym1_cta<512, kC5>), kLadder[5].smem);
    B200_SMEM((k_sym1_cta<1024, kC6>), kLadder[6].smem);
    B200_SMEM((k_sym1_cluster<1024, kC6>), kLadder[7].smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sym1_cluster<1024, kC6>,
                                 cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
#undef B200_SMEM
    return e;
}

}  // namespace b200
