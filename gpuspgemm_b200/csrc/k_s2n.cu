// Symbolic phase 2 fused with the numeric phase, one kernel per row bin
// (key = nnz of the row, known exactly after the count phase and the scan).
//
// For every row the kernel
//   1. hashes the row's column keys into a shared-memory table
//      (sym2.cuh:84-101, 163-191),
//   2. sorts the keys and stores them as C.col[rpt[row] ...]
//      (sym2.cuh:104-120, 194-210),
//   3. accumulates c_ij += a_ik * b_kj with a binary search of the sorted keys
//      and a shared-memory atomic add (num.cuh:104-116, 162-182),
//   4. stores C.val.
// The reference runs 2 and 3 as separate phases with a second binning in
// between (proposal.cuh:59-73), re-reading C.col from global memory; here the
// sorted keys stay in shared memory.  The results are the same: the sorted
// key list is unique, and each value is the sum of the same rounded products.
#include <cooperative_groups.h>

#include "cta.cuh"
#include "kernels.hpp"
#include "sort.cuh"

namespace cg = cooperative_groups;

namespace b200 {

namespace {

template<typename V>
__device__ __forceinline__ V ldv(const void* base, int i) {
    return __ldg(static_cast<const V*>(base) + i);
}

// A row of C whose A row holds ONE entry (a_ik at column k) is a_ik times B's
// row k: its columns are B's (sorted, duplicate-free) and each value is one
// rounded product, as in Gustavson.  The one-pass fill bins copy such rows
// with `lanes` threads (lane `lane` of them) instead of staging, sorting and
// compressing them; in the 1M power-law product 61 % of the rows have one
// entry.  Writes the row's nnz to row_nnz.  Columns outside [0, B.n) are
// reported, as in the other fill paths.
template<typename V>
__device__ __forceinline__ void copy_scaled_b_row(const ProductArgs& p, int row, int a0, int c0,
                                                  int lane, int lanes) {
    const int k = __ldg(p.a_col + a0);
    const V a = ldv<V>(p.a_val, a0);
    const int bs = __ldg(p.b_rpt + k);
    const int n = __ldg(p.b_rpt + k + 1) - bs;
    int32_t* out_col = p.c_col + c0;
    V* out_val = static_cast<V*>(p.c_val) + c0;
    for (int i = lane; i < n; i += lanes) {
        const int32_t col = __ldg(p.b_col + bs + i);
        if (static_cast<uint32_t>(col) >= static_cast<uint32_t>(p.n_cols))
            report(p.status, kStBadInput, row, col);
        out_col[i] = col;
        out_val[i] = a * ldv<V>(p.b_val, bs + i);
    }
    if (lane == 0) p.row_nnz[row] = n;
}

// What a fill walk loads for one product: B's column and the rounded product
// a_ik * b_kj.  The walks keep kWalkU products per thread in flight.
template<typename V>
struct KeyProduct {
    int32_t key;
    V prod;
};
// Products in flight per thread, per walk of the expand-sort-compress and
// bitmap bins (measured on the 1M power-law product, serialised per-kernel
// times): the 256-thread bin 4 (0.285 -> 0.261 ms), the bitmap bin 2 (0.470
// -> 0.449 ms; 4 gave 0.456), the 16- and 32-lane teams 2 (0.140 -> 0.124 ms
// for 32 lanes), the 4- and 8-lane teams 1 (their rows hold few products; 2
// and 4 cost registers and took 0.097 -> 0.114 / 0.124 ms for 4 lanes).  The
// hash bins keep one product per thread: their walks end in a shared-memory
// CAS or a binary search, and wider walks made the stencil products slower
// (Galerkin A*P 1.49 -> 1.72 ms, R*AP 1.01 -> 1.12 ms).
constexpr int kWalkU = 4;
constexpr int kBitmapWalkU = 2;
template<int G>
constexpr int team_walk_u() {
    return G >= 16 ? 2 : 1;
}

// Values accumulate straight into the row's slice of C.val with global
// reductions (fire-and-forget FP64 adds in L2; the row's slice was zeroed by
// the same team or CTA before the barrier that precedes them).  That keeps no
// value array in shared memory -- only the key table -- so more rows are in
// flight per SM, and nothing is copied out at the end.

template<typename V, int G, int THREADS, int T>
__global__ __launch_bounds__(THREADS) void k_s2n_team(ProductArgs p) {
    constexpr int R = THREADS / G;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int32_t* s_keys = reinterpret_cast<int32_t*>(smem_raw);
    const int team = threadIdx.x / G;
    const int lane = team_lane<G>();
    const unsigned mask = team_mask<G>();
    const int rid = blockIdx.x * R + team;
    if (rid >= p.nrows) return;
    int32_t* keys = s_keys + team * T;
    const int row = p.rows[rid];
    const int c0 = p.c_rpt[row];
    // the row's exact nnz, or in one-pass mode its NIP (an upper bound)
    const int bound = p.c_rpt[row + 1] - c0;
    if (bound > T) {
        if (lane == 0) report(p.status, kStCapacity, row, bound);
        return;
    }
    for (int i = lane; i < T; i += G) keys[i] = kEmpty;
    team_sync<G>(mask);
    const int a0 = p.a_rpt[row];
    const int a1 = p.a_rpt[row + 1];
    team_for_products<G>(p.a_col, p.b_rpt, a0, a1, [&](int qb, int) {
        table_insert(keys, T, __ldg(p.b_col + qb), p.status, row);
    });
    team_sync<G>(mask);
    // sort only the row's keys: compact them to the front, then the register
    // sort leaves them in swizzled order (sort.cuh)
    const int cnt = team_compact<G>(keys, T, mask, lane);
    int nnz = bound;
    if (p.row_nnz != nullptr) {  // one-pass: the count is the row's nnz
        nnz = cnt;
        if (lane == 0) p.row_nnz[row] = cnt;
    } else if (cnt != nnz && lane == 0) {
        report(p.status, kStCapacity, row, cnt);
    }
    team_sort_swz<G, T / G>(keys, cnt, mask, lane);
    V* out = static_cast<V*>(p.c_val) + c0;
    for (int i = lane; i < nnz; i += G) {
        p.c_col[c0 + i] = keys[swz(i)];
        out[i] = V(0);
    }
    team_sync<G>(mask);
    team_for_products<G>(p.a_col, p.b_rpt, a0, a1, [&](int qb, int ai) {
        const int32_t key = __ldg(p.b_col + qb);
        const int pos = lower_bound_present_swz(keys, nnz, key);
        atomicAdd(out + pos, ldv<V>(p.a_val, ai) * ldv<V>(p.b_val, qb));
    });
}

// Expand-sort-compress fill of rows with at most NMAX products, for the
// one-pass mode (rows binned by NIP, each filling a NIP-sized slot).  One walk
// over the row's products stages every product in shared memory: its value
// c = a_ik * b_kj, and the key (column << SHIFT | q), q the product's place in
// the row.  The team's register sort orders the keys by column and, within a
// column, by q.  The first product of each column run then sums the run's
// values in that order and writes the column and the sum to the next slot.
// That needs no hash table, no second walk of the products, no binary search
// and no atomics, and sums each entry of C in the oracle's (Gustavson) order.
// The keys need B.n <= 2^(31 - SHIFT); the ladder that holds these kernels is
// used only for B.n <= kBitmapCols = 2^20 (SHIFT <= 10).
constexpr int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x >> 1); }

template<typename V, int G, int THREADS, int NMAX>
struct EscLayout {
    static constexpr int T = next_pow2(NMAX);  // sort capacity of a team
    static constexpr int SHIFT = ilog2(T);
    static constexpr size_t vals_bytes = sizeof(V) * NMAX * (THREADS / G);
    static constexpr size_t bytes = vals_bytes + sizeof(int32_t) * T * (THREADS / G);
    static_assert(SHIFT <= 10, "column keys of an ESC bin need 31 - SHIFT >= 21 bits");
};

template<typename V, int G, int THREADS, int NMAX>
__global__ __launch_bounds__(THREADS) void k_esc_team(ProductArgs p) {
    using L = EscLayout<V, G, THREADS, NMAX>;
    constexpr int R = THREADS / G;
    constexpr int T = L::T;
    constexpr int SHIFT = L::SHIFT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int team = threadIdx.x / G;
    const int lane = team_lane<G>();
    const unsigned mask = team_mask<G>();
    const int rid = blockIdx.x * R + team;
    if (rid >= p.nrows) return;
    V* vals = reinterpret_cast<V*>(smem_raw) + team * NMAX;
    int32_t* keys = reinterpret_cast<int32_t*>(smem_raw + L::vals_bytes) + team * T;
    const int row = p.rows[rid];
    const int c0 = p.c_rpt[row];
    const int nip = p.c_rpt[row + 1] - c0;  // the row's NIP-sized slot
    if (nip > NMAX || p.row_nnz == nullptr) {
        if (lane == 0) report(p.status, kStCapacity, row, nip);
        return;
    }
    if (p.a_rpt[row + 1] - p.a_rpt[row] == 1) {  // uniform over the team
        copy_scaled_b_row<V>(p, row, p.a_rpt[row], c0, lane, G);
        return;
    }
    team_for_products_mlp<G, team_walk_u<G>()>(
        p.a_col, p.b_rpt, p.a_rpt[row], p.a_rpt[row + 1],
        [&](int qb, int ai, int) {
            return KeyProduct<V>{__ldg(p.b_col + qb), ldv<V>(p.a_val, ai) * ldv<V>(p.b_val, qb)};
        },
        [&](const KeyProduct<V>& kp, int, int, int q) {
            if (q < NMAX) {
                int32_t col = kp.key;
                // a column outside [0, B.n) would corrupt the packed key:
                // report it, keep the key in range
                if (static_cast<uint32_t>(col) >= static_cast<uint32_t>(p.n_cols)) {
                    report(p.status, kStBadInput, row, col);
                    col = 0;
                }
                keys[q] = (col << SHIFT) | q;
                vals[q] = kp.prod;
            }
        });
    team_sync<G>(mask);
    team_sort_swz<G, T / G>(keys, nip, mask, lane);
    int32_t* out_col = p.c_col + c0;
    V* out_val = static_cast<V*>(p.c_val) + c0;
    const unsigned below = (1u << (threadIdx.x & 31u)) - 1u;
    int written = 0;
    int carry = -1;  // column of the element before the chunk
    for (int i0 = 0; i0 < nip; i0 += G) {
        const int i = i0 + lane;
        const int32_t key = i < nip ? keys[swz(i)] : kEmpty;
        const int col = key >> SHIFT;
        int prev = __shfl_up_sync(mask, col, 1, G);
        if (lane == 0) prev = carry;
        const bool head = i < nip && col != prev;
        const unsigned bits = __ballot_sync(mask, head) & mask;
        if (head) {
            V sum = vals[key & (T - 1)];
            for (int k = i + 1; k < nip; k++) {
                const int32_t next = keys[swz(k)];
                if ((next >> SHIFT) != col) break;
                sum += vals[next & (T - 1)];
            }
            const int r = written + __popc(bits & below);
            out_col[r] = col;
            out_val[r] = sum;
        }
        written += __popc(bits);
        carry = __shfl_sync(mask, col, G - 1, G);
    }
    if (lane == 0) p.row_nnz[row] = written;
}

// Expand-sort-compress of the small rows (the first three one-pass bins, up
// to 192 products) with whole warps over many rows.  A team of G lanes per row
// leaves most lanes idle there: the 1M power-law product has 826 k rows of
// 1-12 products, 2.9 on average (ncu: 9 of 32 lanes active per instruction
// with 4-lane teams).  A warp takes ROWS rows of the bin's list and packs
// them, in list order, into batches of at most 32 K products, K per lane.
// Per batch:
//   1. the batch's A entries, flattened over its rows, 32 at a time: each lane
//      finds its entry's row by a search over the rows' A-entry prefix (held
//      one per lane), loads the entry and its B row's extent, and a warp scan
//      of the B-row lengths places each entry's first product;
//   2. 32 products at a time, each lane finds its product's entry by a search
//      over that scan, loads B's column and value, and stages the key (row in
//      the batch << (20 + PB) | column << PB | product, PB = log2(32 K); the
//      three fit 32 bits) and the product a_ik * b_kj in shared memory;
//   3. a warp bitonic sort of the 32 K keys (element r * 32 + lane in
//      register r of the lane) orders them by row, column and product; the
//      first element of each (row, column) run sums the run in product order
//      (Gustavson's order, as the team kernels) and writes the column and sum
//      at its rank in the row; the last element of each row writes the row's
//      nnz.
// Single-entry rows take the same path.  Needs B.n <= 2^20 (the ladder that
// holds it) and the one-pass mode's NIP-sized slots; a row of more than 32 K
// products is reported.  Per bin (1M power-law product, serialised): rows of
// <= 12 products K = 1, 32 rows a warp (4-lane teams 0.092 -> 0.057 ms); <= 48
// K = 2, 8 rows (8-lane teams 0.067 -> 0.060; 4 or 16 rows no better); <= 192
// K = 8, 4 rows (16-lane teams 0.117 -> 0.104; 2 rows 0.103 but the product
// 1.108 -> 1.112 ms).
constexpr int kEscWarpThreads = 256;


template<typename V, int THREADS, int K, int ROWS>
__global__ __launch_bounds__(THREADS) void k_esc_warp(ProductArgs p) {
    static_assert(K == 1 || K == 2 || K == 4 || K == 8, "keys per lane");
    static_assert(ROWS >= 1 && ROWS <= kWarp, "rows per warp");
    constexpr int NW = THREADS / kWarp;
    constexpr int CAP = kWarp * K;  // products per batch
    constexpr int PB = ilog2(CAP);  // bits of a product's place in the batch
    constexpr int RS = 20 + PB;     // row-in-batch shift
    static_assert(RS + ilog2(2 * ROWS - 1) <= 32, "row, column and place fit 32 bits");
    constexpr unsigned kFull = 0xffffffffu;
    __shared__ uint32_t s_key[NW][CAP];
    __shared__ uint32_t s_sorted[NW][CAP];
    __shared__ V s_val[NW][CAP];
    const int lane = static_cast<int>(threadIdx.x & 31u);
    const int w = static_cast<int>(threadIdx.x >> 5);
    const int r0 = (blockIdx.x * NW + w) * ROWS;
    if (r0 >= p.nrows) return;  // uniform over the warp
    const int nr = min(ROWS, p.nrows - r0);
    // lane j < nr holds row j of the warp's rows
    int row = 0;
    int c0 = 0;
    int nip = 0;
    int a0 = 0;
    int deg = 0;
    if (lane < nr) {
        row = p.rows[r0 + lane];
        c0 = p.c_rpt[row];
        nip = p.c_rpt[row + 1] - c0;  // the row's NIP-sized slot
        a0 = p.a_rpt[row];
        deg = p.a_rpt[row + 1] - a0;
        if (nip > CAP || nip < 0 || p.row_nnz == nullptr) {
            report(p.status, kStCapacity, row, nip);
            nip = 0;  // left out; the status fails the product
            deg = 0;
        } else if (nip == 0) {
            p.row_nnz[row] = 0;
            deg = 0;  // entries whose B rows are all empty make no product
        }
    }
    const int pin = team_inclusive_scan<kWarp>(kFull, nip, lane);  // products through row lane
    const int din = team_inclusive_scan<kWarp>(kFull, deg, lane);  // A entries through row lane
    uint32_t* keys = s_key[w];
    uint32_t* sorted = s_sorted[w];
    V* vals = s_val[w];
    for (int j0 = 0; j0 < nr;) {  // uniform over the warp
        const int pbase = j0 > 0 ? __shfl_sync(kFull, pin, j0 - 1) : 0;
        const int dbase = j0 > 0 ? __shfl_sync(kFull, din, j0 - 1) : 0;
        // rows [j0, j1): the longest run from j0 whose products fit CAP (row
        // j0 always does; pin is non-decreasing, so the run is contiguous)
        const unsigned take = __ballot_sync(kFull, lane >= j0 && lane < nr && pin - pbase <= CAP);
        const int j1 = 32 - __clz(take);
        const int total = __shfl_sync(kFull, pin, j1 - 1) - pbase;
        const int dtotal = __shfl_sync(kFull, din, j1 - 1) - dbase;
        const int drel = din - dbase;  // A entries of rows [j0, lane] (row lanes)
        int done = 0;                  // products staged
        for (int f0 = 0; f0 < dtotal; f0 += kWarp) {  // uniform over the warp
            const int f = f0 + lane;
            // entry f's row: the first row lane with drel > f (the last with
            // drel <= f, plus one); for f < dtotal that lane is below j1 - 1
            int jr = j0 - 1;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const int c = jr + step;
                const int v = __shfl_sync(kFull, drel, c & 31);
                if (c < j1 && v <= f) jr = c;
            }
            jr += 1;
            const int src = jr & 31;
            const int a_first = __shfl_sync(kFull, a0, src);
            const int before = __shfl_sync(kFull, drel - deg, src);  // entries before row jr
            int len = 0;
            int bs = 0;
            V av = V(0);
            if (f < dtotal) {
                const int ai = a_first + (f - before);
                const int k = __ldg(p.a_col + ai);
                av = ldv<V>(p.a_val, ai);
                bs = __ldg(p.b_rpt + k);
                len = __ldg(p.b_rpt + k + 1) - bs;
            }
            const int lin = team_inclusive_scan<kWarp>(kFull, len, lane);
            const int chunk = __shfl_sync(kFull, lin, 31);  // <= CAP - done
#pragma unroll
            for (int t0 = 0; t0 < CAP; t0 += kWarp) {
                if (t0 >= chunk) break;  // uniform over the warp
                const int t = t0 + lane;
                // product t's entry: the first lane with lin > t
                int e = -1;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    const int c = e + step;
                    const int v = __shfl_sync(kFull, lin, c & 31);
                    if (v <= t) e = c;
                }
                e = (e + 1) & 31;
                const int e_bs = __shfl_sync(kFull, bs, e);
                const int e_first = __shfl_sync(kFull, lin - len, e);
                const V e_av = __shfl_sync(kFull, av, e);
                const int e_jr = __shfl_sync(kFull, jr, e);
                const int e_row = __shfl_sync(kFull, row, e_jr & 31);
                if (t < chunk) {
                    const int qb = e_bs + (t - e_first);
                    int32_t col = __ldg(p.b_col + qb);
                    const V prod = e_av * ldv<V>(p.b_val, qb);
                    // a column outside [0, B.n) would corrupt the packed key:
                    // report it, keep the key in range
                    if (static_cast<uint32_t>(col) >= static_cast<uint32_t>(p.n_cols)) {
                        report(p.status, kStBadInput, e_row, col);
                        col = 0;
                    }
                    const int pos = done + t;
                    keys[pos] = (static_cast<uint32_t>(e_jr - j0) << RS) |
                                (static_cast<uint32_t>(col) << PB) | static_cast<uint32_t>(pos);
                    vals[pos] = prod;
                }
            }
            done += chunk;
        }
        __syncwarp();
        uint32_t key[K];
#pragma unroll
        for (int r = 0; r < K; r++) {
            const int i = r * kWarp + lane;
            key[r] = i < total ? keys[i] : 0xffffffffu;
        }
        // bitonic sort of the warp's CAP keys, ascending; element i = r * 32 + lane
#pragma unroll
        for (int k = 2; k <= CAP; k <<= 1) {
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
                if (j >= kWarp) {  // partner in another register of this lane
                    const int jr = j / kWarp;
#pragma unroll
                    for (int r = 0; r < K; r++) {
                        if ((r & jr) == 0) {
                            const bool asc = ((r * kWarp + lane) & k) == 0;
                            const uint32_t x = key[r];
                            const uint32_t y = key[r + jr];
                            key[r] = asc ? min(x, y) : max(x, y);
                            key[r + jr] = asc ? max(x, y) : min(x, y);
                        }
                    }
                } else {
#pragma unroll
                    for (int r = 0; r < K; r++) {
                        const uint32_t other = __shfl_xor_sync(kFull, key[r], j);
                        const bool asc = ((r * kWarp + lane) & k) == 0;
                        const bool low = (lane & j) == 0;
                        key[r] = (low == asc) ? min(key[r], other) : max(key[r], other);
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < K; r++) sorted[r * kWarp + lane] = key[r];
        __syncwarp();
        // per register: run heads and row starts
        unsigned heads[K];
        unsigned starts[K];
#pragma unroll
        for (int r = 0; r < K; r++) {
            const int i = r * kWarp + lane;
            const bool valid = i < total;
            // element i - 1: this register of the lane below, or the last
            // lane's previous register
            const uint32_t up = __shfl_up_sync(kFull, key[r], 1);
            const uint32_t carry = __shfl_sync(kFull, key[r > 0 ? r - 1 : 0], 31);
            const uint32_t prev = lane > 0 ? up : (r > 0 ? carry : 0xffffffffu);
            heads[r] = __ballot_sync(kFull, valid && (i == 0 || (prev >> PB) != (key[r] >> PB)));
            starts[r] = __ballot_sync(kFull, valid && (i == 0 || (prev >> RS) != (key[r] >> RS)));
        }
        const unsigned upto = kFull >> (31 - lane);  // lanes <= this one
#pragma unroll
        for (int r = 0; r < K; r++) {
            const int i = r * kWarp + lane;
            const bool valid = i < total;
            const uint32_t kr = key[r];
            const uint32_t rr = kr >> RS;
            // the row's first element f: the last row start at or before i
            int f = 0;
#pragma unroll
            for (int q = 0; q <= r; q++) {
                const unsigned m = q < r ? starts[q] : (starts[q] & upto);
                if (m != 0u) f = q * kWarp + 31 - __clz(m);
            }
            // heads in [f, i]
            int rank = 0;
#pragma unroll
            for (int q = 0; q <= r; q++) {
                unsigned m = q < r ? heads[q] : (heads[q] & upto);
                const int fq = f - q * kWarp;  // f's lane in register q, if there
                if (fq >= kWarp) m = 0u;
                else if (fq > 0) m &= ~((1u << fq) - 1u);
                rank += __popc(m);
            }
            const int jrow = (j0 + static_cast<int>(rr)) & 31;
            const int out0 = __shfl_sync(kFull, c0, jrow);
            const int out_row = __shfl_sync(kFull, row, jrow);
            const bool head = valid && ((heads[r] >> lane) & 1u);
            if (head) {
                V sum = vals[kr & (CAP - 1)];
                for (int x = i + 1; x < total; x++) {
                    const uint32_t nk = sorted[x];
                    if ((nk >> PB) != (kr >> PB)) break;
                    sum += vals[nk & (CAP - 1)];
                }
                p.c_col[out0 + rank - 1] = static_cast<int32_t>((kr >> PB) & 0xfffffu);
                static_cast<V*>(p.c_val)[out0 + rank - 1] = sum;
            }
            const uint32_t down = __shfl_down_sync(kFull, kr, 1);
            const uint32_t wrap = __shfl_sync(kFull, key[r + 1 < K ? r + 1 : r], 0);
            const uint32_t next =
                i + 1 >= total ? 0xffffffffu : lane < 31 ? down : (r + 1 < K ? wrap : 0xffffffffu);
            const bool rend = valid && (i == total - 1 || (next >> RS) != rr);
            if (rend) p.row_nnz[out_row] = rank;
        }
        __syncwarp();
        j0 = j1;
    }
}

// Expand-sort-compress for rows of up to NMAX products with a whole CTA (the
// 256-thread bin's range).  As the team version, with an unsigned key
// (column << SHIFT | q), SHIFT = log2 of the sort capacity (B.n <= 2^(32 -
// SHIFT)).  The keys are staged in product order and sorted by a stable
// radix sort of their column bits only (sort.cuh cta_radix_sort: 3 passes
// for B.n <= 2^21), so a column's products stay in product order.
// Compression: each thread takes a contiguous run of sorted positions,
// counts the column heads in it, a block scan gives its first output slot,
// and each head sums its column's run (which may run into the next thread's
// positions) in product order.
template<typename V, int THREADS, int NMAX>
struct EscCtaLayout {
    static constexpr int P = next_pow2(NMAX);
    static constexpr int SHIFT = ilog2(P);
    static constexpr int RMAX = (NMAX + THREADS - 1) / THREADS;  // radix rounds per warp
    static constexpr size_t vals_bytes = sizeof(V) * NMAX;
    static constexpr size_t keys_bytes = sizeof(uint32_t) * NMAX;
    static constexpr size_t hist_bytes = sizeof(int32_t) * 128 * (THREADS / kWarp);
    static constexpr size_t bytes = vals_bytes + keys_bytes + hist_bytes + sizeof(CtaScratch<THREADS>);
    static_assert(bytes <= 232448, "an ESC CTA bin's shared memory exceeds 227 KB");
};

// SKIP_LE > 0: rows of at most SKIP_LE products are left to a smaller kernel
// of the same bin; SKIP_GT: rows of more than NMAX products are left to a
// larger one (instead of being reported).
template<typename V, int THREADS, int NMAX, int SKIP_LE = 0, bool SKIP_GT = false>
__global__ __launch_bounds__(THREADS) void k_esc_cta(ProductArgs p) {
    using L = EscCtaLayout<V, THREADS, NMAX>;
    constexpr int SHIFT = L::SHIFT;
    constexpr uint32_t QMASK = (1u << SHIFT) - 1u;
    constexpr int NW = THREADS / kWarp;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* vals = reinterpret_cast<V*>(smem_raw);
    uint32_t* keys = reinterpret_cast<uint32_t*>(smem_raw + L::vals_bytes);
    int32_t* hist = reinterpret_cast<int32_t*>(smem_raw + L::vals_bytes + L::keys_bytes);
    auto& sc = *reinterpret_cast<CtaScratch<THREADS>*>(smem_raw + L::vals_bytes + L::keys_bytes +
                                                        L::hist_bytes);
    const int tid = threadIdx.x;
    const int row = p.rows[blockIdx.x];
    const int c0 = p.c_rpt[row];
    const int nip = p.c_rpt[row + 1] - c0;  // the row's NIP-sized slot
    if (nip <= SKIP_LE || (SKIP_GT && nip > NMAX && p.row_nnz != nullptr)) return;
    if (nip > NMAX || p.row_nnz == nullptr) {
        if (tid == 0) report(p.status, kStCapacity, row, nip);
        return;
    }
    if (p.a_rpt[row + 1] - p.a_rpt[row] == 1) {  // uniform over the CTA
        copy_scaled_b_row<V>(p, row, p.a_rpt[row], c0, tid, THREADS);
        return;
    }
    cta_for_products_mlp<THREADS, kWalkU>(
        p.a_col, p.b_rpt, p.a_rpt[row], p.a_rpt[row + 1], sc,
        [&](int qb, int ai, int) {
            return KeyProduct<V>{__ldg(p.b_col + qb), ldv<V>(p.a_val, ai) * ldv<V>(p.b_val, qb)};
        },
        [&](const KeyProduct<V>& kp, int, int, int q) {
            if (q >= NMAX) return;
            int32_t col = kp.key;
            if (static_cast<uint32_t>(col) >= static_cast<uint32_t>(p.n_cols)) {
                report(p.status, kStBadInput, row, col);
                col = 0;
            }
            keys[q] = (static_cast<uint32_t>(col) << SHIFT) | static_cast<uint32_t>(q);
            vals[q] = kp.prod;
        });
    // the column bits of the keys: B.n - 1 needs this many
    const int colbits = 32 - __clz(p.n_cols > 1 ? p.n_cols - 1 : 1);
    cta_radix_sort<THREADS, L::RMAX>(keys, nip, SHIFT, colbits, hist, sc.warp_tot);
    const int per = (nip + THREADS - 1) / THREADS;
    const int i0 = min(tid * per, nip);
    const int i1 = min(i0 + per, nip);
    int heads = 0;
    {
        uint32_t prev = i0 > 0 ? (keys[i0 - 1] >> SHIFT) : 0xffffffffu;
        for (int i = i0; i < i1; i++) {
            const uint32_t c = keys[i] >> SHIFT;
            heads += c != prev;
            prev = c;
        }
    }
    const int inc = block_inclusive_scan<THREADS>(heads, sc.warp_tot);
    const int total = sc.warp_tot[NW - 1];
    int r = inc - heads;
    int32_t* out_col = p.c_col + c0;
    V* out_val = static_cast<V*>(p.c_val) + c0;
    uint32_t prev = i0 > 0 ? (keys[i0 - 1] >> SHIFT) : 0xffffffffu;
    for (int i = i0; i < i1; i++) {
        const uint32_t u = keys[i];
        const uint32_t c = u >> SHIFT;
        if (c != prev) {
            V sum = vals[u & QMASK];
            for (int k = i + 1; k < nip; k++) {
                const uint32_t w = keys[k];
                if ((w >> SHIFT) != c) break;
                sum += vals[w & QMASK];
            }
            out_col[r] = static_cast<int32_t>(c);
            out_val[r] = sum;
            r++;
        }
        prev = c;
    }
    if (tid == 0) p.row_nnz[row] = total;
}

// Compression of the team bins, sampled: `samples` rows spread evenly over
// A are counted exactly over their first kSampleProducts products (one warp
// per row, a 1024-slot shared hash set) when their NIP is at most the last
// team bin's limit, and those products and their distinct columns are summed
// per team bin (binned by NIP with the ladder's limits); the NIP of every
// sampled row, and of the longer ones apart, is summed too.  It needs A and B only, so it runs
// on a side stream beside the NIP pass; the host reads the sums with the NIP
// plan.  They choose one pass or two (rows above the team bins that repeat
// many columns fill small nnz-sized tables only in two passes) and let a
// team bin expand-sort-compress only when its rows repeat few columns: ESC
// sorts every product, the hash bins only the distinct columns.
constexpr int kSampleWarps = 8;
constexpr int kSampleSlots = 1024;
constexpr int kSampleProducts = 256;  // products counted per sampled row

__global__ __launch_bounds__(kSampleWarps * kWarp) void k_esc_sample(ProductArgs p, int32_t m,
                                                                      int32_t samples,
                                                                      EscLimits lim,
                                                                      EscSample* out) {
    __shared__ int32_t s_tab[kSampleWarps][kSampleSlots];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int w = blockIdx.x * kSampleWarps + wid;
    if (w >= samples) return;
    const int row = static_cast<int>(static_cast<int64_t>(w) * m / samples);
    const int a0 = p.a_rpt[row];
    const int a1 = p.a_rpt[row + 1];
    const int cap = lim.limit[kEscBins - 1];
    auto count_nip = [&](int64_t v, bool above) {
        if (lane == 0) {
            atomicAdd(reinterpret_cast<unsigned long long*>(&out->nip_seen),
                      static_cast<unsigned long long>(v));
            if (above)
                atomicAdd(reinterpret_cast<unsigned long long*>(&out->nip_above),
                          static_cast<unsigned long long>(v));
        }
    };
    if (a1 - a0 > cap) {  // more products than the team bins take (>= a1 - a0)
        count_nip(a1 - a0, true);
        return;
    }
    int nip = 0;
    for (int e = a0 + lane; e < a1; e += kWarp) {
        const int c = __ldg(p.a_col + e);
        nip += __ldg(p.b_rpt + c + 1) - __ldg(p.b_rpt + c);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nip += __shfl_xor_sync(0xffffffffu, nip, o);
    if (nip == 0) return;
    count_nip(nip, nip > cap);
    if (nip > cap || nip > 3 * kSampleSlots / 4) return;
    int b = 0;
    while (nip > lim.limit[b]) b++;
    // count the row's first kSampleProducts products only (the walk's latency
    // is the sample's cost): the A entries up to the one that reaches them
    int a_cut = a1;
    if (nip > kSampleProducts) {
        int run = 0;
        for (int base = a0; base < a1; base += kWarp) {
            const int e = base + lane;
            int len = 0;
            if (e < a1) {
                const int c = __ldg(p.a_col + e);
                len = __ldg(p.b_rpt + c + 1) - __ldg(p.b_rpt + c);
            }
            const int inc = team_inclusive_scan<kWarp>(0xffffffffu, len, lane);
            const unsigned hit = __ballot_sync(0xffffffffu, run + inc >= kSampleProducts);
            if (hit != 0u) {
                a_cut = base + __ffs(hit);
                break;
            }
            run += __shfl_sync(0xffffffffu, inc, kWarp - 1);
        }
    }
    int32_t* tab = s_tab[wid];
    for (int i = lane; i < kSampleSlots; i += kWarp) tab[i] = kEmpty;
    __syncwarp();
    team_for_products_at<kWarp>(p.a_col, p.b_rpt, a0, a_cut, [&](int qb, int, int q) {
        if (q < kSampleProducts)
            table_insert(tab, kSampleSlots, __ldg(p.b_col + qb), p.status, row);
    });
    __syncwarp();
    int cnt = 0;
    for (int i = lane; i < kSampleSlots; i += kWarp) cnt += tab[i] != kEmpty;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(&out->nip[b]),
                  static_cast<unsigned long long>(min(nip, kSampleProducts)));
        atomicAdd(reinterpret_cast<unsigned long long*>(&out->nnz[b]),
                  static_cast<unsigned long long>(cnt));
    }
}

template<int THREADS, int T, int CAP>
struct CtaLayout {
    static constexpr int P = next_pow2(CAP);
    static constexpr int K = T > P ? T : P;
    static constexpr size_t keys_bytes = sizeof(int32_t) * K;
    static constexpr size_t bytes = keys_bytes + sizeof(CtaScratch<THREADS>);
    static_assert(bytes <= 232448, "a CTA bin's shared memory exceeds 227 KB");
};

template<typename V, int THREADS, int T, int CAP>
__global__ __launch_bounds__(THREADS) void k_s2n_cta(ProductArgs p) {
    using L = CtaLayout<THREADS, T, CAP>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int32_t* keys = reinterpret_cast<int32_t*>(smem_raw);
    auto& sc = *reinterpret_cast<CtaScratch<THREADS>*>(smem_raw + L::keys_bytes);
    const int row = p.rows[blockIdx.x];
    const int c0 = p.c_rpt[row];
    // the row's exact nnz, or in one-pass mode its NIP (an upper bound)
    const int bound = p.c_rpt[row + 1] - c0;
    if (bound > CAP) {
        if (threadIdx.x == 0) report(p.status, kStCapacity, row, bound);
        return;
    }
    for (int i = threadIdx.x; i < T; i += THREADS) keys[i] = kEmpty;
    __syncthreads();
    const int a0 = p.a_rpt[row];
    const int a1 = p.a_rpt[row + 1];
    cta_for_products<THREADS>(p.a_col, p.b_rpt, a0, a1, sc, [&](int qb, int) {
        table_insert(keys, T, __ldg(p.b_col + qb), p.status, row);
    });
    const int cnt = cta_compact<THREADS>(keys, T, sc.warp_tot);
    int nnz = bound;
    if (p.row_nnz != nullptr) {  // one-pass: the count is the row's nnz
        nnz = cnt <= CAP ? cnt : CAP;
        if (threadIdx.x == 0) p.row_nnz[row] = nnz;
    } else if (cnt != nnz && threadIdx.x == 0) {
        report(p.status, kStCapacity, row, cnt);
    }
    // register sort of the row's keys; they come back in swizzled order
    static_assert(L::K >= THREADS * 16, "the register sort needs THREADS * 16 key slots");
    // (cnt > CAP only for an invalid operand, reported above; the clamp keeps
    // the sort inside the K key slots)
    cta_sort_swz<THREADS>(keys, cnt <= CAP ? cnt : CAP);
    V* out = static_cast<V*>(p.c_val) + c0;
    for (int i = threadIdx.x; i < nnz; i += THREADS) {
        p.c_col[c0 + i] = keys[swz(i)];
        out[i] = V(0);
    }
    __syncthreads();
    cta_for_products<THREADS>(p.a_col, p.b_rpt, a0, a1, sc, [&](int qb, int ai) {
        const int32_t key = __ldg(p.b_col + qb);
        const int pos = lower_bound_present_swz(keys, nnz, key);
        atomicAdd(out + pos, ldv<V>(p.a_val, ai) * ldv<V>(p.b_val, qb));
    });
}

// Bitmap bin (B.n <= kBitmapCols): the row's hash table is the identity hash
// over B's columns, one BIT per column, in shared memory (128 KB for 2^20
// columns).  atomicOr fills it; the set bits read in word order are the sorted
// column list, so no sort is needed.  A summary bitmap holds one bit per
// bitmap word that has any bit set (set by the product that set the word's
// first bit), so counting, extracting and clearing visit only the row's
// non-empty words: the cost of a row follows its products, not B.n.
//
// The kernel is persistent: one CTA per SM (the bitmap takes most of its
// shared memory) clears the bitmap once and then takes rows blockIdx.x,
// blockIdx.x + gridDim.x, ...  Thread t owns summary word t, i.e. bitmap
// words [32t, 32t + 32) = eight 4-word blocks.  Per row: fill; each thread
// counts the set bits of its non-empty words; a block scan gives every
// thread's first position, from which it writes its columns to C.col and
// records the rank of each of its blocks' first bit.  The bitmap stays
// intact, so a key's position in the row is its rank -- the block's rank plus
// the set bits before it in at most 4 words, all independent reads --
// instead of a binary search; values accumulate with global reductions into
// C.val.  Then each thread clears its non-empty words and summary word.
// (4-word blocks rather than 8: 0.289 -> 0.280 ms on the 1M power-law
// product, for 16 KB more shared memory.)  The cluster bin below keeps
// 8-word blocks in the same layout (its rank table uses half the space).
constexpr int kBitmapWords = kBitmapCols / 32;
constexpr int kSummaryWords = kBitmapWords / 32;

template<typename V, int THREADS, int CAP>
struct BitmapLayout {
    static constexpr size_t bm_bytes = sizeof(uint32_t) * kBitmapWords;
    static constexpr size_t summary_bytes = sizeof(uint32_t) * kSummaryWords;
    static constexpr size_t rank_bytes = sizeof(int32_t) * (kBitmapWords / 4);
    static constexpr size_t bytes =
        bm_bytes + summary_bytes + rank_bytes + sizeof(CtaScratch<THREADS>);
    static_assert(kSummaryWords == THREADS, "one summary word per thread");
};

template<typename V, int THREADS, int CAP>
__global__ __launch_bounds__(THREADS) void k_s2n_bitmap(ProductArgs p) {
    using L = BitmapLayout<V, THREADS, CAP>;
    constexpr int NW = THREADS / kWarp;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* bm = reinterpret_cast<uint32_t*>(smem_raw);
    uint32_t* summary = reinterpret_cast<uint32_t*>(smem_raw + L::bm_bytes);
    int32_t* block_rank = reinterpret_cast<int32_t*>(smem_raw + L::bm_bytes + L::summary_bytes);
    auto& sc = *reinterpret_cast<CtaScratch<THREADS>*>(smem_raw + L::bm_bytes +
                                                        L::summary_bytes + L::rank_bytes);
    const int tid = threadIdx.x;
    const int words = (p.n_cols + 31) >> 5;
    if (words > kBitmapWords) {
        if (tid == 0 && blockIdx.x < p.nrows) report(p.status, kStCapacity, p.rows[blockIdx.x], 0);
        return;
    }
    __shared__ int32_t s_rid;  // the row this CTA takes next
    for (int i = tid; i < words; i += THREADS) bm[i] = 0u;
    summary[tid] = 0u;
    const int w0 = tid * 32;  // this thread's bitmap words [w0, w0 + 32)
    for (int k = 0;; k++) {
        // rows are taken from the launch's counter as CTAs free up (the list
        // is ordered largest first), so the CTAs finish together
        __syncthreads();
        if (tid == 0) s_rid = p.work != nullptr ? atomicAdd(p.work, 1) : blockIdx.x + k * gridDim.x;
        __syncthreads();
        const int rid = s_rid;
        if (rid >= p.nrows) break;
        const int row = p.rows[rid];
        const int c0 = p.c_rpt[row];
        // the row's exact nnz, or in one-pass mode its NIP (an upper bound)
        const int bound = p.c_rpt[row + 1] - c0;
        if (bound > CAP) {  // uniform over the CTA
            if (tid == 0) report(p.status, kStCapacity, row, bound);
            continue;
        }
        const int a0 = p.a_rpt[row];
        const int a1 = p.a_rpt[row + 1];
        if (a1 - a0 == 1 && p.row_nnz != nullptr) {  // uniform over the CTA
            copy_scaled_b_row<V>(p, row, a0, c0, tid, THREADS);
            continue;
        }
        cta_for_products_mlp<THREADS, kBitmapWalkU>(
            p.a_col, p.b_rpt, a0, a1, sc, [&](int qb, int, int) { return __ldg(p.b_col + qb); },
            [&](int32_t key, int, int, int) {
                if (static_cast<uint32_t>(key) >= static_cast<uint32_t>(p.n_cols)) {
                    report(p.status, kStBadInput, row, key);  // outside the bitmap
                    return;
                }
                const int wi = key >> 5;
                if (atomicOr(bm + wi, 1u << (key & 31)) == 0u)
                    atomicOr(summary + (wi >> 5), 1u << (wi & 31));
            });
        const uint32_t sw = summary[tid];
        int cnt = 0;
        for (uint32_t m = sw; m != 0u; m &= m - 1u) cnt += __popc(bm[w0 + __ffs(m) - 1]);
        const int inc = block_inclusive_scan<THREADS>(cnt, sc.warp_tot);
        const int total = sc.warp_tot[NW - 1];
        int pos = inc - cnt;
        int32_t* cols = p.c_col + c0;
#pragma unroll
        for (int bb = 0; bb < 8; bb++) {
            block_rank[(w0 >> 2) + bb] = pos;
            for (uint32_t m = (sw >> (4 * bb)) & 0xfu; m != 0u; m &= m - 1u) {
                const int wi = w0 + 4 * bb + __ffs(m) - 1;
                for (uint32_t word = bm[wi]; word != 0u; word &= word - 1u) {
                    if (pos < bound) cols[pos] = wi * 32 + __ffs(word) - 1;
                    pos++;
                }
            }
        }
        int nnz = bound;
        if (p.row_nnz != nullptr) {  // one-pass: the count is the row's nnz
            nnz = total <= bound ? total : bound;
            if (tid == 0) p.row_nnz[row] = nnz;
        } else if (total != nnz && tid == 0) {
            report(p.status, kStCapacity, row, total);
        }
        V* out = static_cast<V*>(p.c_val) + c0;
        for (int i = tid; i < nnz; i += THREADS) out[i] = V(0);
        __syncthreads();
        cta_for_products_mlp<THREADS, kBitmapWalkU>(
            p.a_col, p.b_rpt, a0, a1, sc,
            [&](int qb, int ai, int) {
                return KeyProduct<V>{__ldg(p.b_col + qb), ldv<V>(p.a_val, ai) * ldv<V>(p.b_val, qb)};
            },
            [&](const KeyProduct<V>& kp, int, int, int) {
                const int32_t key = kp.key;
                if (static_cast<uint32_t>(key) >= static_cast<uint32_t>(p.n_cols)) return;
                const int wi = key >> 5;
                const int w4 = wi & ~3;
                int rank = block_rank[wi >> 2] + __popc(bm[wi] & ((1u << (key & 31)) - 1u));
#pragma unroll
                for (int t = 0; t < 3; t++)
                    if (w4 + t < wi) rank += __popc(bm[w4 + t]);
                if (rank < nnz) atomicAdd(out + rank, kp.prod);
            });
        for (uint32_t m = sw; m != 0u; m &= m - 1u) bm[w0 + __ffs(m) - 1] = 0u;
        summary[tid] = 0u;
        __syncthreads();
    }
}

// Cluster bitmap bin (wide B, 2^20 < B.n <= kClusterBitmapCols): the
// bitmap bin's bitmap, summary and block ranks spread over a thread-block
// cluster -- CTA c of the cluster holds columns [c 2^20, (c + 1) 2^20) in its
// shared memory and the other CTAs reach it through distributed shared memory
// (atom / ld.shared::cluster through map_shared_rank; no TMA) -- so the
// heaviest rows of a wide B stay on chip instead of falling to the global
// bitmap bin.  Persistent: every cluster takes rows cid, cid + nclusters, ...
// Per row:
//   1. the CTAs split the row's A entries in slices of THREADS (CTA c takes
//      slices c, c + csize, ...) and set each product's bit in the CTA that
//      owns its column (local or remote atomicOr), and that CTA's summary bit;
//   2. each CTA counts its slice's columns; the CTAs' counts, read across the
//      cluster, give every CTA its first output position, and each CTA writes
//      its sorted columns and block ranks (the bitmap bin's extraction);
//   3. the CTAs walk their slices again: a product's position is the owning
//      CTA's block rank plus the set bits before its own, read from the
//      owner's shared memory, and its value goes to C.val by a global
//      reduction;
//   4. each CTA clears its own non-empty words.
// Cluster barriers separate the steps (a remote bit set in step 1 is seen by
// the owner's count; nothing clears a bitmap another CTA may still read).
constexpr int kClusterBitmapMaxCtas = static_cast<int>(kClusterBitmapCols / kBitmapCols);

template<typename V, int THREADS>
__global__ __launch_bounds__(THREADS) void k_s2n_bitmap_cluster(ProductArgs p) {
    using L = BitmapLayout<V, THREADS, kBitmapCols>;
    constexpr int NW = THREADS / kWarp;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* bm = reinterpret_cast<uint32_t*>(smem_raw);
    uint32_t* summary = reinterpret_cast<uint32_t*>(smem_raw + L::bm_bytes);
    int32_t* block_rank = reinterpret_cast<int32_t*>(smem_raw + L::bm_bytes + L::summary_bytes);
    auto& sc = *reinterpret_cast<CtaScratch<THREADS>*>(smem_raw + L::bm_bytes +
                                                        L::summary_bytes + L::rank_bytes);
    __shared__ int32_t s_total;  // this CTA's column count of the current row
    cg::cluster_group cluster = cg::this_cluster();
    const int csize = static_cast<int>(cluster.num_blocks());
    const int crank = static_cast<int>(cluster.block_rank());
    const int nclusters = static_cast<int>(gridDim.x) / csize;
    const int cid = static_cast<int>(blockIdx.x) / csize;
    const int tid = threadIdx.x;
    const int slice_lo = crank * kBitmapCols;  // first column this CTA holds
    const int words = (min(kBitmapCols, max(0, p.n_cols - slice_lo)) + 31) >> 5;
    for (int i = tid; i < words; i += THREADS) bm[i] = 0u;
    summary[tid] = 0u;
    cluster.sync();
    const int w0 = tid * 32;  // this thread's bitmap words [w0, w0 + 32)
    for (int rid = cid; rid < p.nrows; rid += nclusters) {
        const int row = p.rows[rid];
        const int c0 = p.c_rpt[row];
        // the row's exact nnz, or in one-pass mode its NIP (an upper bound)
        const int bound = p.c_rpt[row + 1] - c0;
        const int a0 = p.a_rpt[row];
        const int a1 = p.a_rpt[row + 1];
        // 1. bits, each in the CTA that owns its column
        for (int base = a0 + crank * THREADS; base < a1; base += csize * THREADS) {
            cta_for_products_mlp<THREADS, kBitmapWalkU>(
                p.a_col, p.b_rpt, base, min(base + THREADS, a1), sc,
                [&](int qb, int, int) { return __ldg(p.b_col + qb); },
                [&](int32_t key, int, int, int) {
                    if (static_cast<uint32_t>(key) >= static_cast<uint32_t>(p.n_cols)) {
                        report(p.status, kStBadInput, row, key);  // outside every slice
                        return;
                    }
                    const int owner = key / kBitmapCols;
                    const int wi = (key % kBitmapCols) >> 5;
                    uint32_t* obm = owner == crank ? bm : cluster.map_shared_rank(bm, owner);
                    if (atomicOr(obm + wi, 1u << (key & 31)) == 0u) {
                        uint32_t* osum =
                            owner == crank ? summary : cluster.map_shared_rank(summary, owner);
                        atomicOr(osum + (wi >> 5), 1u << (wi & 31));
                    }
                });
        }
        cluster.sync();
        // 2. count, place and extract this CTA's columns
        const uint32_t sw = summary[tid];
        int cnt = 0;
        for (uint32_t m = sw; m != 0u; m &= m - 1u) cnt += __popc(bm[w0 + __ffs(m) - 1]);
        const int inc = block_inclusive_scan<THREADS>(cnt, sc.warp_tot);
        if (tid == 0) s_total = sc.warp_tot[NW - 1];
        cluster.sync();
        int before = 0;
        int total = 0;
        for (int r = 0; r < csize; r++) {
            const int t = *cluster.map_shared_rank(&s_total, r);
            total += t;
            before += r < crank ? t : 0;
        }
        int pos = before + inc - cnt;
        int32_t* cols = p.c_col + c0;
#pragma unroll
        for (int bb = 0; bb < 4; bb++) {
            block_rank[(w0 >> 3) + bb] = pos;
            for (uint32_t m = (sw >> (8 * bb)) & 0xffu; m != 0u; m &= m - 1u) {
                const int wi = w0 + 8 * bb + __ffs(m) - 1;
                for (uint32_t word = bm[wi]; word != 0u; word &= word - 1u) {
                    if (pos < bound) cols[pos] = slice_lo + wi * 32 + __ffs(word) - 1;
                    pos++;
                }
            }
        }
        int nnz = bound;
        if (p.row_nnz != nullptr) {  // one-pass: the count is the row's nnz
            nnz = total <= bound ? total : bound;
            if (crank == 0 && tid == 0) p.row_nnz[row] = nnz;
        } else if (total != nnz && crank == 0 && tid == 0) {
            report(p.status, kStCapacity, row, total);
        }
        V* out = static_cast<V*>(p.c_val) + c0;
        for (int i = crank * THREADS + tid; i < nnz; i += csize * THREADS) out[i] = V(0);
        cluster.sync();  // every CTA's block ranks and the zeroed values are in place
        // 3. values: positions from the owner's bitmap and block ranks
        for (int base = a0 + crank * THREADS; base < a1; base += csize * THREADS) {
            cta_for_products_mlp<THREADS, kBitmapWalkU>(
                p.a_col, p.b_rpt, base, min(base + THREADS, a1), sc,
                [&](int qb, int ai, int) {
                    return KeyProduct<V>{__ldg(p.b_col + qb),
                                         ldv<V>(p.a_val, ai) * ldv<V>(p.b_val, qb)};
                },
                [&](const KeyProduct<V>& kp, int, int, int) {
                    const int32_t key = kp.key;
                    if (static_cast<uint32_t>(key) >= static_cast<uint32_t>(p.n_cols)) return;
                    const int owner = key / kBitmapCols;
                    const int wi = (key % kBitmapCols) >> 5;
                    const int w8 = wi & ~7;
                    const uint32_t* obm =
                        owner == crank ? bm : cluster.map_shared_rank(bm, owner);
                    const int32_t* orank =
                        owner == crank ? block_rank : cluster.map_shared_rank(block_rank, owner);
                    int rank = orank[wi >> 3] + __popc(obm[wi] & ((1u << (key & 31)) - 1u));
#pragma unroll
                    for (int t = 0; t < 7; t++)
                        if (w8 + t < wi) rank += __popc(obm[w8 + t]);
                    if (rank < nnz) atomicAdd(out + rank, kp.prod);
                });
        }
        cluster.sync();  // no CTA reads another's bitmap any more
        // 4. clear this CTA's words for the next row
        for (uint32_t m = sw; m != 0u; m &= m - 1u) bm[w0 + __ffs(m) - 1] = 0u;
        summary[tid] = 0u;
        cluster.sync();  // cleared before any CTA sets the next row's bits
    }
}

// Global bin: a bitmap per row in flight (global scratch, B.n bits per CTA);
// only the row's column window [lo, hi] is cleared and read, and a key outside
// it (B rows not sorted) redoes the fill over [0, B.n).  The set bits, read in
// word order, ARE the sorted column list.  Values accumulate with global
// atomics after a binary search of the row's C.col in global memory
// (the reference's k_num_global, num.cuh:251-298).
template<typename V, int THREADS>
__global__ __launch_bounds__(THREADS) void k_s2n_global(ProductArgs p) {
    __shared__ CtaScratch<THREADS> sc;
    uint32_t* bm = p.bitmaps + static_cast<int64_t>(blockIdx.x) * p.words;
    for (int rid = blockIdx.x; rid < p.nrows; rid += gridDim.x) {
        const int row = p.rows[rid];
        const int c0 = p.c_rpt[row];
        // the row's exact nnz, or in one-pass mode its NIP (an upper bound)
        const int bound = p.c_rpt[row + 1] - c0;
        const int a0 = p.a_rpt[row];
        const int a1 = p.a_rpt[row + 1];
        const int2 win = cta_col_window<THREADS>(p.a_col, p.b_rpt, p.b_col, a0, a1, p.n_cols, sc);
        int lo = win.x;
        int hi = win.y;
        int w0 = 0;
        int nwords = 0;
        for (int pass = 0; pass < 2; pass++) {
            w0 = lo >> 5;
            nwords = hi >= lo ? (hi >> 5) - w0 + 1 : 0;
            for (int i = threadIdx.x; i < nwords; i += THREADS) bm[i] = 0u;
            __syncthreads();
            int miss = 0;
            cta_for_products<THREADS>(p.a_col, p.b_rpt, a0, a1, sc, [&](int qb, int) {
                const int32_t key = __ldg(p.b_col + qb);
                if (key < lo || key > hi) {
                    miss = 1;
                    return;
                }
                atomicOr(bm + ((key >> 5) - w0), 1u << (key & 31));
            });
            if (!__syncthreads_or(miss)) break;
            if (pass == 1) {  // a column index outside [0, B.n): keys skipped
                if (threadIdx.x == 0) report(p.status, kStBadInput, row);
                break;
            }
            lo = 0;
            hi = p.n_cols - 1;
        }
        int32_t* cols = p.c_col + c0;
        int base = 0;
        for (int c = 0; c < nwords; c += THREADS) {
            const int wi = c + threadIdx.x;
            uint32_t w = wi < nwords ? bm[wi] : 0u;
            const int cnt = __popc(w);
            const int inc = block_inclusive_scan<THREADS>(cnt, sc.warp_tot);
            int pos = base + inc - cnt;
            while (w != 0u) {
                const int b = __ffs(w) - 1;
                if (pos < bound) cols[pos] = (w0 + wi) * 32 + b;
                pos++;
                w &= w - 1u;
            }
            base += sc.warp_tot[THREADS / kWarp - 1];
            __syncthreads();
        }
        int nnz = bound;
        if (p.row_nnz != nullptr) {  // one-pass: the count is the row's nnz
            nnz = base <= bound ? base : bound;
            if (threadIdx.x == 0) p.row_nnz[row] = nnz;
        } else if (base != nnz && threadIdx.x == 0) {
            report(p.status, kStCapacity, row, base);
        }
        V* out = static_cast<V*>(p.c_val) + c0;
        for (int i = threadIdx.x; i < nnz; i += THREADS) out[i] = V(0);
        __syncthreads();
        if (nnz == 0) continue;  // only skipped (invalid) keys: nothing to add into
        cta_for_products<THREADS>(p.a_col, p.b_rpt, a0, a1, sc, [&](int qb, int ai) {
            const int32_t key = __ldg(p.b_col + qb);
            const int pos = lower_bound_present(cols, nnz, key);
            // a key that was skipped above (outside [0, B.n)) is not in the row
            if (cols[pos] == key) atomicAdd(out + pos, ldv<V>(p.a_val, ai) * ldv<V>(p.b_val, qb));
        });
    }
}

template<int G, int THREADS, int T>
constexpr size_t team_smem() {
    return sizeof(int32_t) * T * (THREADS / G);
}

template<typename V, int G, int THREADS, int T>
cudaError_t launch_team(const ProductArgs& p, cudaStream_t s) {
    constexpr int R = THREADS / G;
    const int grid = (p.nrows + R - 1) / R;
    k_s2n_team<V, G, THREADS, T><<<grid, THREADS, team_smem<G, THREADS, T>(), s>>>(p);
    return cudaGetLastError();
}

template<typename V, int G, int THREADS, int NMAX>
cudaError_t launch_esc(const ProductArgs& p, cudaStream_t s) {
    constexpr int R = THREADS / G;
    const int grid = (p.nrows + R - 1) / R;
    k_esc_team<V, G, THREADS, NMAX>
        <<<grid, THREADS, EscLayout<V, G, THREADS, NMAX>::bytes, s>>>(p);
    return cudaGetLastError();
}

template<typename V, int K, int ROWS>
cudaError_t launch_esc_warp(const ProductArgs& p, cudaStream_t s) {
    constexpr int R = kEscWarpThreads / kWarp * ROWS;  // rows per CTA
    const int grid = (p.nrows + R - 1) / R;
    k_esc_warp<V, kEscWarpThreads, K, ROWS><<<grid, kEscWarpThreads, 0, s>>>(p);
    return cudaGetLastError();
}

template<typename V, int THREADS, int NMAX>
cudaError_t launch_esc_cta(const ProductArgs& p, cudaStream_t s) {
    k_esc_cta<V, THREADS, NMAX><<<p.nrows, THREADS, EscCtaLayout<V, THREADS, NMAX>::bytes, s>>>(p);
    return cudaGetLastError();
}

// The 256-thread ESC bin split by row size: rows of more than kEscCtaSmall
// products with 256 threads, the others with 128 (half the fixed cost of each
// radix pass and scan, twice the CTAs per SM).  Both grids cover the whole
// row list; a CTA whose row belongs to the other kernel returns at once.
// (1M power-law product: the bin 0.233 -> 0.223 ms serialised.)
constexpr int kEscCtaSmall = 1024;

template<typename V>
cudaError_t launch_esc_cta_split(const ProductArgs& p, cudaStream_t s) {
    k_esc_cta<V, 256, 3072, kEscCtaSmall, false>
        <<<p.nrows, 256, EscCtaLayout<V, 256, 3072>::bytes, s>>>(p);
    if (cudaError_t e = cudaGetLastError(); e != cudaSuccess) return e;
    k_esc_cta<V, 128, kEscCtaSmall, 0, true>
        <<<p.nrows, 128, EscCtaLayout<V, 128, kEscCtaSmall>::bytes, s>>>(p);
    return cudaGetLastError();
}

template<typename V, int THREADS, int T, int CAP>
cudaError_t launch_cta(const ProductArgs& p, cudaStream_t s) {
    k_s2n_cta<V, THREADS, T, CAP>
        <<<p.nrows, THREADS, CtaLayout<THREADS, T, CAP>::bytes, s>>>(p);
    return cudaGetLastError();
}

// Order a bin's row list by slot size (the row's NIP in one-pass mode, its
// nnz in two), largest first: one CTA, a counting sort by size bucket (size /
// 32, capped), buckets in descending order, rows in a bucket in any order.
// With the persistent bins taking rows from a counter, the CTAs then finish
// together (largest first: each CTA's last row is a short one).  The kernel
// also zeroes the bin's row counter for the launch that follows.
constexpr int kSortRowsMax = 8192;
constexpr int kSortThreads = 1024;
constexpr int kSizeBuckets = 2048;

__global__ __launch_bounds__(kSortThreads) void k_rows_largest_first(int32_t* __restrict__ rows,
                                                                     int32_t n,
                                                                     const int32_t* __restrict__ c_rpt,
                                                                     int32_t* __restrict__ work) {
    constexpr int PER = kSizeBuckets / kSortThreads;
    __shared__ int32_t s_count[kSizeBuckets];  // per bucket: count, then first slot
    __shared__ int32_t s_out[kSortRowsMax];
    __shared__ int32_t s_warp[kSortThreads / kWarp];
    const int tid = threadIdx.x;
    if (tid == 0) *work = 0;
    for (int i = tid; i < kSizeBuckets; i += kSortThreads) s_count[i] = 0;
    __syncthreads();
    // descending: bucket 0 holds the largest rows
    auto bucket = [&](int r) {
        const int size = c_rpt[r + 1] - c_rpt[r];
        return kSizeBuckets - 1 - min(size >> 5, kSizeBuckets - 1);
    };
    for (int i = tid; i < n; i += kSortThreads) atomicAdd(&s_count[bucket(rows[i])], 1);
    __syncthreads();
    // exclusive scan of the bucket counts: PER consecutive buckets a thread
    int v[PER];
    int sum = 0;
#pragma unroll
    for (int c = 0; c < PER; c++) {
        v[c] = s_count[tid * PER + c];
        sum += v[c];
    }
    int run = block_inclusive_scan<kSortThreads>(sum, s_warp) - sum;
#pragma unroll
    for (int c = 0; c < PER; c++) {
        s_count[tid * PER + c] = run;
        run += v[c];
    }
    __syncthreads();
    for (int i = tid; i < n; i += kSortThreads) {
        const int r = rows[i];
        s_out[atomicAdd(&s_count[bucket(r)], 1)] = r;
    }
    __syncthreads();
    for (int i = tid; i < n; i += kSortThreads) rows[i] = s_out[i];
}

template<typename V, int THREADS, int CAP>
cudaError_t launch_bitmap(const ProductArgs& p, cudaStream_t s) {
    // persistent: one CTA per SM at most (the bitmap takes most of an SM's
    // shared memory)
    const int sms = p.sm_count > 0 ? p.sm_count : 148;
    const int grid = p.nrows < sms ? p.nrows : sms;
    if (p.work != nullptr) {
        // the bin's row list is the library's own (a binning pass wrote it);
        // the sort kernel also zeroes the row counter
        if (p.nrows > grid && p.nrows <= kSortRowsMax) {
            k_rows_largest_first<<<1, kSortThreads, 0, s>>>(const_cast<int32_t*>(p.rows),
                                                            p.nrows, p.c_rpt, p.work);
            if (cudaError_t e = cudaGetLastError(); e != cudaSuccess) return e;
        } else if (cudaError_t e = cudaMemsetAsync(p.work, 0, sizeof(int32_t), s);
                   e != cudaSuccess) {
            return e;
        }
    }
    k_s2n_bitmap<V, THREADS, CAP><<<grid, THREADS, BitmapLayout<V, THREADS, CAP>::bytes, s>>>(p);
    return cudaGetLastError();
}

template<typename V, int THREADS>
cudaError_t launch_global(const ProductArgs& p, cudaStream_t s) {
    const int grid = p.nrows < p.nmaps ? p.nrows : p.nmaps;
    k_s2n_global<V, THREADS><<<grid, THREADS, 0, s>>>(p);
    return cudaGetLastError();
}

// Cluster bitmap bin: a cluster of ceil(B.n / 2^20) CTAs (at most 8) per row
// in flight, as many clusters as fit on the device at once.  B.n beyond the
// cluster's reach, or no cluster of that size resident, runs the rows in the
// global bitmap bin instead.
template<typename V, int THREADS>
cudaError_t launch_bitmap_cluster(const ProductArgs& p, cudaStream_t s) {
    const int64_t need = (static_cast<int64_t>(p.n_cols) + kBitmapCols - 1) / kBitmapCols;
    if (need < 1 || need > kClusterBitmapMaxCtas) return launch_global<V, THREADS>(p, s);
    const int csize = static_cast<int>(need);
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = BitmapLayout<V, THREADS, kBitmapCols>::bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(csize);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int sms = p.sm_count > 0 ? p.sm_count : 148;
    cfg.gridDim = dim3(static_cast<unsigned>(csize * (sms / csize)));
    int resident = 0;
    if (cudaOccupancyMaxActiveClusters(&resident, k_s2n_bitmap_cluster<V, THREADS>, &cfg) !=
            cudaSuccess ||
        resident <= 0) {
        (void)cudaGetLastError();  // clear a failed query; the global bin takes the rows
        return launch_global<V, THREADS>(p, s);
    }
    const int nclusters = p.nrows < resident ? p.nrows : resident;
    cfg.gridDim = dim3(static_cast<unsigned>(csize * nclusters));
    return cudaLaunchKernelEx(&cfg, k_s2n_bitmap_cluster<V, THREADS>, p);
}

template<typename V>
struct S2nLadder {
    static const BinLauncher entries[];
    static const int count;
};

#define B200_S2N_LADDER(V)                                                                    \
    template<>                                                                                \
    const BinLauncher S2nLadder<V>::entries[] = {                                             \
        {BinKind::Team, 12, 64, 256, team_smem<4, 256, 16>(), "s2n_team4_t16",                \
         launch_team<V, 4, 256, 16>},                                                         \
        {BinKind::Team, 48, 32, 256, team_smem<8, 256, 64>(), "s2n_team8_t64",                \
         launch_team<V, 8, 256, 64>},                                                         \
        {BinKind::Team, 192, 16, 256, team_smem<16, 256, 256>(), "s2n_team16_t256",           \
         launch_team<V, 16, 256, 256>},                                                       \
        {BinKind::Team, 768, 8, 256, team_smem<32, 256, 1024>(), "s2n_team32_t1024",          \
         launch_team<V, 32, 256, 1024>},                                                      \
        {BinKind::Cta, 3072, 1, 256, CtaLayout<256, 4096, 3072>::bytes, "s2n_cta256_t4096",   \
         launch_cta<V, 256, 4096, 3072>},                                                     \
        {BinKind::Cta, 12288, 1, 512, CtaLayout<512, 16384, 12288>::bytes,                    \
         "s2n_cta512_t16384", launch_cta<V, 512, 16384, 12288>},                              \
        {BinKind::Cta, 32768, 1, 1024, CtaLayout<1024, 43008, 32768>::bytes,                  \
         "s2n_cta1024_t43008", launch_cta<V, 1024, 43008, 32768>},                            \
        {BinKind::Cluster, INT32_MAX, 1, 1024, BitmapLayout<V, 1024, kBitmapCols>::bytes,     \
         "s2n_bitmap_cluster", launch_bitmap_cluster<V, 1024>},                               \
        {BinKind::Global, INT32_MAX, 1, 1024, 0, "s2n_global_bitmap", launch_global<V, 1024>}, \
    };                                                                                        \
    template<>                                                                                \
    const int S2nLadder<V>::count = sizeof(S2nLadder<V>::entries) / sizeof(BinLauncher);

B200_S2N_LADDER(double)
B200_S2N_LADDER(float)
#undef B200_S2N_LADDER

// Ladder for B.n <= kBitmapCols: every row above the 256-thread bin uses the
// shared-memory bitmap bin (whose shared memory does not depend on the row);
// the global bin stays last for the per-bin test knob.
template<typename V>
struct S2nBitmapLadder {
    static const BinLauncher entries[];
    static const int count;
};

#define B200_S2N_BITMAP_LADDER(V)                                                             \
    template<>                                                                                \
    const BinLauncher S2nBitmapLadder<V>::entries[] = {                                       \
        S2nLadder<V>::entries[0], S2nLadder<V>::entries[1], S2nLadder<V>::entries[2],         \
        S2nLadder<V>::entries[3], S2nLadder<V>::entries[4],                                   \
        {BinKind::Cta, kBitmapCols, 1, 1024, BitmapLayout<V, 1024, kBitmapCols>::bytes,       \
         "s2n_bitmap1024", launch_bitmap<V, 1024, kBitmapCols>},                              \
        {BinKind::Global, INT32_MAX, 1, 1024, 0, "s2n_global_bitmap", launch_global<V, 1024>}, \
    };                                                                                        \
    template<>                                                                                \
    const int S2nBitmapLadder<V>::count =                                                     \
        sizeof(S2nBitmapLadder<V>::entries) / sizeof(BinLauncher);

B200_S2N_BITMAP_LADDER(double)
B200_S2N_BITMAP_LADDER(float)
#undef B200_S2N_BITMAP_LADDER

// One-pass ladder for B.n <= kBitmapCols: the smallest rows packed many to a
// warp (k_esc_warp), the team bins and the 256-thread bin expand, sort and
// compress (k_esc_team, k_esc_cta) with the hash bins' row limits; the bitmap
// and global bins are the bitmap ladder's.
template<typename V>
struct S2nEscLadder {
    static const BinLauncher entries[];
    static const int count;
};

#define B200_S2N_ESC_LADDER(V)                                                                \
    template<>                                                                                \
    const BinLauncher S2nEscLadder<V>::entries[] = {                                          \
        {BinKind::Team, 12, kEscWarpThreads, kEscWarpThreads, 0, "esc_warp_n12",              \
         launch_esc_warp<V, 1, 32>},                                                          \
        {BinKind::Team, 48, kEscWarpThreads / kWarp * 8, kEscWarpThreads, 0, "esc_warp2_n48",  \
         launch_esc_warp<V, 2, 8>},                                                           \
        {BinKind::Team, 192, kEscWarpThreads / kWarp * 4, kEscWarpThreads, 0,                  \
         "esc_warp8_n192", launch_esc_warp<V, 8, 4>},                                         \
        {BinKind::Team, 768, 8, 256, EscLayout<V, 32, 256, 768>::bytes, "esc_team32_n768",    \
         launch_esc<V, 32, 256, 768>},                                                        \
        {BinKind::Cta, 3072, 1, 256, EscCtaLayout<V, 256, 3072>::bytes, "esc_cta256_n3072",    \
         launch_esc_cta_split<V>},                                                            \
        S2nBitmapLadder<V>::entries[5], S2nBitmapLadder<V>::entries[6],                       \
    };                                                                                        \
    template<>                                                                                \
    const int S2nEscLadder<V>::count = sizeof(S2nEscLadder<V>::entries) / sizeof(BinLauncher);

B200_S2N_ESC_LADDER(double)
B200_S2N_ESC_LADDER(float)
#undef B200_S2N_ESC_LADDER

// The 32-lane expand-sort-compress bin for rows of at most kEscSplit products,
// launched when the device-side decision moved the 32-lane / 256-thread split
// to kEscSplit: half the shared memory of the 768-product kernel per team, so
// twice the CTAs per SM (ncu: the 768-product kernel ran 17 % warps active).
template<typename V>
struct EscSplitBin {
    static const BinLauncher entry;
};
template<typename V>
const BinLauncher EscSplitBin<V>::entry = {BinKind::Team, kEscSplit, 8, 256,
                                           EscLayout<V, 32, 256, kEscSplit>::bytes,
                                           "esc_team32_n512", launch_esc<V, 32, 256, kEscSplit>};

template<typename V>
cudaError_t prepare_one() {
    cudaError_t e = cudaSuccess;
#define B200_SMEM(kern, bytes)                                                            \
    if (e == cudaSuccess)                                                                 \
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,       \
                                 static_cast<int>(bytes));
    B200_SMEM((k_s2n_team<V, 4, 256, 16>), (team_smem<4, 256, 16>()));
    B200_SMEM((k_s2n_team<V, 8, 256, 64>), (team_smem<8, 256, 64>()));
    B200_SMEM((k_s2n_team<V, 16, 256, 256>), (team_smem<16, 256, 256>()));
    B200_SMEM((k_s2n_team<V, 32, 256, 1024>), (team_smem<32, 256, 1024>()));
    B200_SMEM((k_s2n_cta<V, 256, 4096, 3072>), (CtaLayout<256, 4096, 3072>::bytes));
    B200_SMEM((k_s2n_cta<V, 512, 16384, 12288>), (CtaLayout<512, 16384, 12288>::bytes));
    B200_SMEM((k_s2n_cta<V, 1024, 43008, 32768>), (CtaLayout<1024, 43008, 32768>::bytes));
    B200_SMEM((k_s2n_bitmap<V, 1024, kBitmapCols>), (BitmapLayout<V, 1024, kBitmapCols>::bytes));
    B200_SMEM((k_s2n_bitmap_cluster<V, 1024>), (BitmapLayout<V, 1024, kBitmapCols>::bytes));
    B200_SMEM((k_esc_team<V, 32, 256, 768>), (EscLayout<V, 32, 256, 768>::bytes));
    B200_SMEM((k_esc_team<V, 32, 256, kEscSplit>), (EscLayout<V, 32, 256, kEscSplit>::bytes));
    B200_SMEM((k_esc_cta<V, 256, 3072>), (EscCtaLayout<V, 256, 3072>::bytes));
    B200_SMEM((k_esc_cta<V, 256, 3072, kEscCtaSmall, false>), (EscCtaLayout<V, 256, 3072>::bytes));
    B200_SMEM((k_esc_cta<V, 128, kEscCtaSmall, 0, true>), (EscCtaLayout<V, 128, kEscCtaSmall>::bytes));
#undef B200_SMEM
    return e;
}

}  // namespace

int s2n_ladder_f64(const BinLauncher** out) {
    *out = S2nLadder<double>::entries;
    return S2nLadder<double>::count;
}

int s2n_ladder_f32(const BinLauncher** out) {
    *out = S2nLadder<float>::entries;
    return S2nLadder<float>::count;
}

int s2n_bitmap_ladder_f64(const BinLauncher** out) {
    *out = S2nBitmapLadder<double>::entries;
    return S2nBitmapLadder<double>::count;
}

int s2n_bitmap_ladder_f32(const BinLauncher** out) {
    *out = S2nBitmapLadder<float>::entries;
    return S2nBitmapLadder<float>::count;
}

int s2n_esc_ladder_f64(const BinLauncher** out) {
    *out = S2nEscLadder<double>::entries;
    return S2nEscLadder<double>::count;
}

int s2n_esc_ladder_f32(const BinLauncher** out) {
    *out = S2nEscLadder<float>::entries;
    return S2nEscLadder<float>::count;
}

const BinLauncher* s2n_esc_split_bin_f64() { return &EscSplitBin<double>::entry; }
const BinLauncher* s2n_esc_split_bin_f32() { return &EscSplitBin<float>::entry; }

cudaError_t launch_esc_sample(const ProductArgs& p, int32_t m, int32_t samples,
                              const EscLimits& lim, EscSample* out, cudaStream_t s) {
    if (samples <= 0) return cudaSuccess;
    k_esc_sample<<<(samples + kSampleWarps - 1) / kSampleWarps, kSampleWarps * kWarp, 0, s>>>(
        p, m, samples, lim, out);
    return cudaGetLastError();
}

__global__ void k_esc_decide(EscSample* sample, const __grid_constant__ Ladder base, int esc_mode,
                             Ladder* out) {
    constexpr int b = kEscBins - 1;
    const int64_t nip = sample->nip[b];
    const int64_t nnz = sample->nnz[b];
    const bool split = esc_mode == 1 ||
                       (esc_mode == 0 && nnz > 0 &&
                        static_cast<double>(nip) <= kEscMaxRatio[b] * static_cast<double>(nnz));
    Ladder l = base;
    if (split) l.limit[b] = kEscSplit;
    *out = l;
    sample->split = split ? 1 : 0;
}

cudaError_t launch_esc_decide(EscSample* sample, const Ladder& base, int esc_mode, Ladder* out,
                              cudaStream_t s) {
    k_esc_decide<<<1, 1, 0, s>>>(sample, base, esc_mode, out);
    return cudaGetLastError();
}

cudaError_t s2n_prepare() {
    cudaError_t e = prepare_one<double>();
    if (e == cudaSuccess) e = prepare_one<float>();
    return e;
}

}  // namespace b200
