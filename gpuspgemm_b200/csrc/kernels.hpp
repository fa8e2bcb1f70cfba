// Host-visible interface between the orchestration (spgemm.cu) and the kernel
// translation units.  Plain structs only; no torch types anywhere.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace b200 {

struct DevStatus;

constexpr int kMaxBins = 16;

// Row-bin ladder: row r (key k > 0) goes to the first bin b with k <= limit[b],
// and at least to bin min_bin.  Rows with key 0 have an empty C row and join no
// bin.  The reference's find_bin (binning.cuh:26-35) does the same linear walk
// over its RANGES tables (parameters.cuh:53-64, 85-95, 127-144).
struct Ladder {
    int32_t nb;
    int32_t min_bin;
    int32_t limit[kMaxBins];
};

// Results of a binning pass, mirrored to pinned host memory in one copy.
struct Plan {
    int64_t total_key;        // sum of keys (total NIP, or total nnz)
    int32_t max_key;          // max key over rows
    int32_t overflow;         // a sum left int32 range
    int32_t bin_size[kMaxBins];
    int32_t bin_off[kMaxBins];
};

// Everything a per-bin kernel needs.  Values are passed as void* and cast by
// the typed launcher.
struct ProductArgs {
    const int32_t* a_rpt;
    const int32_t* a_col;
    const void* a_val;
    const int32_t* b_rpt;
    const int32_t* b_col;
    const void* b_val;
    int32_t n_cols;         // B.n
    int32_t* c_rpt;         // NIP / nnz per row (symbolic) or row pointer (fill)
    int32_t* c_col;
    void* c_val;
    DevStatus* status;
    const int32_t* rows;    // this bin's rows
    int32_t nrows;
    // global-bin scratch: nmaps bitmaps of `words` 32-bit words each
    uint32_t* bitmaps;
    int64_t words;
    int32_t nmaps;
    // cluster bins
    int32_t cluster;        // CTAs per cluster
    int32_t* fail_rows;     // rows that spilled out of a cluster table
    int32_t* fail_count;
    // transpose: per entry of T, (row of A << 32 | position in A)
    uint64_t* keys;
    // one-pass fill: c_rpt gives each row a slot of its NIP entries (an upper
    // bound); the kernel writes the row's exact nnz here (nullptr: c_rpt is
    // C's exact row pointer)
    int32_t* row_nnz;
    // SMs of the device (persistent kernels size their grid by it; 0: 148)
    int32_t sm_count;
    // persistent bins: a device counter the CTAs take their next row from
    // (the launcher zeroes it; nullptr: rows dealt out by CTA index)
    int32_t* work;
};

enum class BinKind : int { Team = 0, Cta = 1, Cluster = 2, Global = 3 };

struct BinLauncher {
    BinKind kind;
    int32_t limit;          // largest key the kernel accepts
    int32_t rows_per_cta;   // 1 for CTA/cluster/global kinds
    int32_t threads;
    size_t smem;            // dynamic shared memory per CTA
    const char* name;
    cudaError_t (*launch)(const ProductArgs&, cudaStream_t);
};

// One-pass fill (no count phase) when its temporaries, NIP entries of column
// and value, fit this many bytes and the product has at least kOnePassMinNip
// intermediate products (below that its extra host synchronisation and
// launches cost more than the count phase it saves).
constexpr uint64_t kOnePassMaxBytes = uint64_t(4) << 30;
constexpr int64_t kOnePassMinNip = int64_t(1) << 21;
// Symbolic count ladder (key = NIP of the row).
int sym1_ladder(const BinLauncher** out);
// Fused fill + sort + numeric ladder (key = nnz of the row), per value type.
int s2n_ladder_f64(const BinLauncher** out);
int s2n_ladder_f32(const BinLauncher** out);
// The same for B.n <= kBitmapCols, whose large rows use a shared-memory bitmap.
constexpr int kBitmapCols = 1 << 20;
// The wide ladder's cluster bitmap bin holds up to this many columns (8 CTAs
// of kBitmapCols); past it its rows run in the global bitmap bin.
constexpr int64_t kClusterBitmapCols = int64_t(8) * kBitmapCols;
int s2n_bitmap_ladder_f64(const BinLauncher** out);
int s2n_bitmap_ladder_f32(const BinLauncher** out);
// One-pass ladder for B.n <= kBitmapCols (key = NIP of the row): the warp,
// team and 256-thread bins expand, sort and compress; then the bitmap ladder's
// bitmap and global bins.  Same bin count and limits as the bitmap ladder.
int s2n_esc_ladder_f64(const BinLauncher** out);
int s2n_esc_ladder_f32(const BinLauncher** out);
// The one-pass ladder's largest team bin when its split is kEscSplit
// (rows of at most kEscSplit products: a smaller kernel, more CTAs per SM).
const BinLauncher* s2n_esc_split_bin_f64();
const BinLauncher* s2n_esc_split_bin_f32();

// Sampled compression of the first kEscBins fill bins of a one-pass product:
// the NIP and exact nnz of up to `samples` rows spread evenly over A, summed
// per team bin (rows binned by NIP with `lim`; rows above the last limit are
// only counted in nip_above).  `p` needs A, B and the status word.
constexpr int kEscBins = 4;
constexpr int kEscSamples = 4096;
// A team bin expands, sorts and compresses when its sampled NIP / nnz is at
// most this (ESC sorts NIP keys where the hash bin sorts nnz; measured
// crossovers: none up to NIP/nnz 4 for rows of <= 48 products, ~1.45 at
// <= 192, ~1.1 at <= 768).
constexpr double kEscMaxRatio[kEscBins] = {8.0, 8.0, 1.4, 1.1};
// The one-pass ladder's bins that may expand-sort-compress: the team bins and
// the 256-thread bin, which follows the sample of the largest team bin.
constexpr int kEscLadderBins = kEscBins + 1;
// The sample runs for products with at least this many entries in A.
constexpr int64_t kSampleMinNnz = int64_t(1) << 16;
// Products with at least this many entries in A are expected to run one pass:
// they are binned for the fill right after the NIP pass, before the first
// synchronisation (the count binning follows only if they run two).
constexpr int64_t kEarlyOnePassNnz = int64_t(1) << 18;
// Auto mode keeps two passes when at least this share of the sampled NIP
// lies in rows above the team bins (one pass bins them by NIP into the CTA
// bins, two passes by nnz into small team tables) and the team bins' sampled
// NIP / nnz is at least kTwoPassMinRatio.
constexpr double kTwoPassMinShare = 0.5;
constexpr double kTwoPassMinRatio = 4.0;
struct EscLimits {
    int32_t limit[kEscBins];
};
struct EscSample {
    int64_t nip[kEscBins];
    int64_t nnz[kEscBins];
    int64_t nip_seen;   // NIP of every sampled row (A-row length for rows
    int64_t nip_above;  // longer than the last limit), and of those above it
    int32_t split;      // written by launch_esc_decide
    int32_t pad;
};
cudaError_t launch_esc_sample(const ProductArgs& p, int32_t m, int32_t samples,
                              const EscLimits& lim, EscSample* out, cudaStream_t s);
// The fill binning's limits, decided on the device from the sample: when the
// largest team bin expands, sorts and compresses (esc_mode 1, or 0 and its
// sampled NIP/nnz at most kEscMaxRatio), its rows above kEscSplit products
// go to the 256-thread bin (which then expands, sorts and compresses too):
// out = base with limit[kEscBins - 1] = kEscSplit, and sample->split = 1.
constexpr int32_t kEscSplit = 512;
cudaError_t launch_esc_decide(EscSample* sample, const Ladder& base, int esc_mode, Ladder* out,
                              cudaStream_t s);
// One-time per-device attribute setup (dynamic smem opt-in) for all kernels.
cudaError_t sym1_prepare();
cudaError_t s2n_prepare();

// ---- binning / scan kernels (k_bin.cu) ------------------------------------
constexpr int kBinThreads = 256;
constexpr int kBinRowsPerCta = 1024;

inline int bin_ctas(int32_t m) { return (m + kBinRowsPerCta - 1) / kBinRowsPerCta; }

// Pass 1 (key = NIP): writes nip[r] into c_rpt[r] (and nip_copy[r] when not
// nullptr), per-CTA bin histograms and the plan's total / max.  With `fill`
// given, also the per-CTA histograms by that ladder into hist_fill and the
// per-CTA NIP sums into cta_sum (the fill binning's first pass).
cudaError_t launch_nip_hist(const int32_t* a_rpt, const int32_t* a_col, const int32_t* b_rpt,
                            int32_t m, int32_t* c_rpt, int32_t* nip_copy, int32_t* hist,
                            Plan* plan, DevStatus* st, const Ladder& lad, cudaStream_t s,
                            int32_t* hist_fill = nullptr, int64_t* cta_sum = nullptr,
                            const Ladder* fill = nullptr);
// Pass 2 for histograms src_hist counted by a source ladder `src` whose
// limits include every limit of the final ladder (dlad when given, else lad):
// the outputs of launch_bin_offsets for the final ladder, all bins at once,
// except that hist (another array) receives offsets within each bin: the
// scatter that reads them is launched with bin_relative.  It also zeroes
// zero[0..nzero), words a later kernel needs cleared.
cudaError_t launch_bin_offsets_map(const int32_t* src_hist, int32_t* hist, int32_t nctas,
                                   const Ladder& src, int64_t* cta_sum, Plan* plan,
                                   const Ladder& lad, const Ladder* dlad, cudaStream_t s,
                                   unsigned long long* zero = nullptr, int32_t nzero = 0);
// Pass 1' (key = nnz already in c_rpt): per-CTA sums and bin histograms.
// dlad: limits chosen on the device (same bin count as lad), or nullptr.
cudaError_t launch_nnz_hist(const int32_t* c_rpt, int32_t m, int32_t* hist, int64_t* cta_sum,
                            Plan* plan, const Ladder& lad, cudaStream_t s,
                            const Ladder* dlad = nullptr);
// Pass 2: exclusive offsets of the per-CTA histograms (and of cta_sum when
// given), bin sizes/offsets into the plan.
cudaError_t launch_bin_offsets(int32_t* hist, int32_t nctas, int64_t* cta_sum, Plan* plan,
                               const Ladder& lad, cudaStream_t s);
// Pass 3: stable scatter of row ids into bins.  When `scan` is set, also
// rewrites c_rpt[0..m] as the exclusive scan of the nnz it holds.
cudaError_t launch_bin_scatter(int32_t* c_rpt, int32_t m, const int32_t* hist_off,
                               const int64_t* cta_off, int32_t* bins, const Plan* plan,
                               const Ladder& lad, bool scan, cudaStream_t s,
                               const Ladder* dlad = nullptr, bool bin_relative = false);
// One-pass row pointer: rewrite cnt[0..m) (each row's nnz) as its exclusive
// scan and cnt[m] as the total, in place, in one launch (tiles chained by
// decoupled look-back); the plan (zeroed by the caller) receives the total,
// the max and the int32 overflow flag.  state holds 1 + rpt_scan_tiles(m)
// zeroed words (a ticket counter, then one per tile); a look-back that waits
// too long reports kStWait in st.  Used for rpt_scan_tiles(m) <=
// kScanMaxTiles (the size of the state in the scratch).
constexpr int kScanTile = 4096;
constexpr int kScanMaxTiles = 2048;
inline int rpt_scan_tiles(int32_t m) { return (m + kScanTile - 1) / kScanTile; }
cudaError_t launch_rpt_scan1(int32_t* cnt, int32_t m, unsigned long long* state, Plan* plan,
                             DevStatus* st, cudaStream_t s);
// One-pass fill: copy each row's entries from its slot [off[r], ...) of the
// temporary arrays to [rpt[r], rpt[r+1]) of C (values of value_bytes 4 or 8);
// nothing at or past `cap`, C's capacity.
cudaError_t launch_compact_rows(const int32_t* off, const int32_t* rpt, int32_t m,
                                const int32_t* tmp_col, const void* tmp_val, int32_t* col,
                                void* val, int value_bytes, cudaStream_t s, int32_t cap);
// A one-pass C gets the product's NIP as its capacity before its nnz is known
// when the sampled rows' NIP / nnz is at most this; a C with more spare
// capacity than this factor is then copied to arrays of its size.
constexpr double kCapSlack = 1.1;
// Operand validation (checked mode).
cudaError_t launch_check_csr(const int32_t* rpt, const int32_t* col, int32_t m, int32_t n,
                             int32_t nnz, DevStatus* st, cudaStream_t s);
// Batched form (k_batch.cu): NIP per product; per-product split of a group's C.
cudaError_t launch_product_nip(const int32_t* a_rpt, const int32_t* a_col, const int32_t* b_rpt,
                               const int32_t* row_off, int32_t count, long long* nip,
                               cudaStream_t s);
cudaError_t launch_unpack(const int32_t* c_rpt, int32_t* c_col, const int32_t* row_off,
                          const int32_t* col_off, const int64_t* out_off, int32_t first,
                          int32_t count, int32_t* rpt_out, int32_t* pos_out, cudaStream_t s);
// CSR transpose (k_transpose.cu): row-sort ladder (key = length of a row of
// A^T), column counts, and the keyed scatter.
int transpose_ladder_f64(const BinLauncher** out);
int transpose_ladder_f32(const BinLauncher** out);
cudaError_t transpose_prepare();
cudaError_t launch_col_count(const int32_t* col, int32_t nnz, int32_t n, int32_t* cnt,
                             cudaStream_t s);
cudaError_t launch_tr_scatter(const int32_t* a_rpt, const int32_t* a_col, int32_t m, int32_t n,
                              const int32_t* t_rpt, int32_t* cursor, uint64_t* keys,
                              cudaStream_t s);
// NIP of many independent pairs in one launch (spgemm_get_nip_many).
struct NipPair {
    const int32_t* a_col;   // A_i's column indices (nnz entries)
    const int32_t* b_rpt;   // B_i's row pointer
    int32_t nnz;            // nnz(A_i)
    int32_t pad;
};
int32_t pairs_nip_ctas(int32_t nnz);  // CTAs the launch gives one pair
cudaError_t launch_pairs_nip(const NipPair* pairs, const int32_t* cta_off, int32_t count,
                             int32_t ctas, long long* nip, cudaStream_t s);
// Total NIP only (spgemm_get_nip).
cudaError_t launch_total_nip(const int32_t* a_rpt, const int32_t* a_col, const int32_t* b_rpt,
                             int32_t m, long long* out, cudaStream_t s);

}  // namespace b200
