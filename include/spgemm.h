/*
 * spgemm.h -- C ABI of the B200 (sm_100a) CSR SpGEMM library, libspgemm_b200.so.
 *
 * This is the drop-in boundary for the reference's hot path
 *     template<std::floating_point T>
 *     utils::DeviceCSR<T> proposal::proposal(const utils::DeviceCSR<T>& A,
 *                                            const utils::DeviceCSR<T>& B);
 * (geektrove/GPUSpGEMM src/libproposal/include/proposal/proposal.cuh:85-124),
 * which has no C ABI of its own.  Every entry point below names the reference
 * interface it replaces.  A header-only C++ shim with the reference's exact
 * signature sits in gpuspgemm_b200/csrc/b200_proposal.hpp.
 *
 * Conventions (same as the reference's utils::CSR, csr.cuh:22-31):
 *   - CSR with 0-based int32 indices: rpt[m+1], col[nnz], val[nnz];
 *   - columns of B sorted ascending and duplicate-free within each row
 *     (the binary-search numeric relies on it, num.cuh:104-116);
 *   - T is float or double (two entry points per operation).
 * Output C: m = A.m, n = B.n, sorted duplicate-free columns, every structural
 * product kept (an entry whose value cancels to 0.0 stays in C).
 *
 * Streams are passed as `void*` holding a cudaStream_t (NULL = legacy default
 * stream).  All device pointers are plain CUDA device addresses.
 */
#ifndef SPGEMM_B200_H
#define SPGEMM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPGEMM_ABI_VERSION 5

#if defined(__GNUC__)
#define SPGEMM_API __attribute__((visibility("default")))
#else
#define SPGEMM_API
#endif

/* Error codes.  The reference throws std::runtime_error from
 * utils::handle_cuda_error (src/libutils/include/utils/errors.cuh:11-22) and on
 * an unsupported device (proposal.cuh:123); the C ABI returns these instead and
 * spgemm_last_error_string() carries the message. */
typedef enum spgemm_status {
    SPGEMM_OK = 0,
    SPGEMM_ERR_INVALID_ARG = 1,        /* NULL pointer, negative size, A.n != B.m,
                                          unsorted/duplicate/out-of-range columns
                                          (checked mode) */
    SPGEMM_ERR_OOM = 2,                /* device or pinned-host allocation failed */
    SPGEMM_ERR_UNSUPPORTED_DEVICE = 3, /* not an sm_100 device */
    SPGEMM_ERR_OVERFLOW = 4,           /* nnz(C) does not fit int32 */
    SPGEMM_ERR_TIMEOUT = 5,            /* a bounded device wait ran out */
    SPGEMM_ERR_CUDA = 6,               /* a CUDA runtime call failed */
    SPGEMM_ERR_INTERNAL = 7            /* a kernel reported a bounded-probe or
                                          capacity failure through its status word */
} spgemm_status;

typedef struct spgemm_handle_s* spgemm_handle_t;

/* Read-only CSR operand.  Replaces const utils::DeviceCSR<T>& (csr.cuh:22-31). */
typedef struct spgemm_csr_view {
    int32_t m;
    int32_t n;
    int32_t nnz;
    const int32_t* rpt;
    const int32_t* col;
    const void* val; /* float* or double* to match the entry point */
} spgemm_csr_view;

/* CSR result.  Replaces the owning utils::DeviceCSR<T> that proposal() returns.
 * Device results are stream-ordered allocations on the call's stream, as in the
 * reference (cudaMallocAsync, setup.cuh:146, binning.cuh:236, sym2.cuh:396),
 * taken from the handle's memory pool (which keeps freed memory mapped), so
 * cudaFree() releases them as ~CSR does (csr.cuh:241-252);
 * spgemm_csr_free() does the same stream-ordered. */
typedef struct spgemm_csr_out {
    int32_t m;
    int32_t n;
    int32_t nnz;
    int32_t* rpt;
    int32_t* col;
    void* val;
} spgemm_csr_out;

/* Statistics of the most recent product on a handle. */
typedef struct spgemm_info {
    int64_t nip;             /* intermediate products = FLOP / 2 (nip.cuh:52-78) */
    int64_t nnz;             /* nnz(C) */
    int32_t max_row_nip;     /* max NIP over rows of C (setup.cuh:29-95) */
    int32_t max_row_nnz;     /* max nnz over rows of C (binning.cuh:213-217) */
    int32_t sym_bin_rows[16]; /* rows per symbolic-count bin */
    int32_t num_bin_rows[16]; /* rows per fill+numeric bin */
    int32_t sym_fail_rows;   /* rows whose cluster table overflowed -> global bin */
    int32_t n_sym_bins;
    int32_t n_num_bins;
    int32_t host_syncs;      /* host round-trips taken by the call */
    /* host-side microseconds since the call began, at: count binning queued,
     * host sync 1 done, count kernels queued, host sync 2 done, C allocated,
     * fill kernels queued, final sync done (unused entries 0) */
    float phase_us[8];
    int32_t one_pass;        /* 1: C's row sizes came from the one-pass fill */
    int32_t esc_mask;        /* bit b: one-pass fill bin b expanded, sorted and compressed */
} spgemm_info;

/* ---- lifecycle ------------------------------------------------------------ */

/* Create a handle bound to CUDA device `device` (-1 = current device).  The
 * handle owns scratch memory, side streams and pinned staging, reused across
 * calls (the reference creates MAX_N_BINS streams and its scratch per call,
 * setup.cuh:164-165, cleanup.cuh:15-31).  One handle per host thread. */
SPGEMM_API spgemm_status spgemm_create(spgemm_handle_t* handle, int device);
SPGEMM_API spgemm_status spgemm_destroy(spgemm_handle_t handle);

/* ---- the product ---------------------------------------------------------- */

/* C = A * B on the device.  Replaces proposal::proposal<double> / <float>
 * (proposal.cuh:85-124) and its phases setup / binning / sym1 / sym_binning2 /
 * sym2 / num / cleanup (setup.cuh:134-178, binning.cuh:146-243,
 * sym1.cuh:311-463, sym2.cuh:293-404, num.cuh:303-442, cleanup.cuh:15-31).
 * A, B: device arrays.  C: filled with library-allocated device arrays.
 * Synchronous on return, like the reference (cleanup.cuh:30). */
SPGEMM_API spgemm_status spgemm_csr_f64(spgemm_handle_t handle, const spgemm_csr_view* A,
                             const spgemm_csr_view* B, spgemm_csr_out* C, void* stream);
SPGEMM_API spgemm_status spgemm_csr_f32(spgemm_handle_t handle, const spgemm_csr_view* A,
                             const spgemm_csr_view* B, spgemm_csr_out* C, void* stream);

/* Release a device result (stream-ordered cudaFreeAsync); replaces ~CSR for
 * Location::Device (csr.cuh:114-117, runtime.cuh:59-66).  Zeroes *C. */
SPGEMM_API spgemm_status spgemm_csr_free(spgemm_csr_out* C, void* stream);

/* C = A * B with HOST operands and a HOST result: copies A and B to the device,
 * multiplies, copies C back.  Replaces the apps' convert/run pair
 * (src/apps/proposal.cu:15-26: HostCSR::to<Device>, proposal, to<Host>).
 * When A and B are the same host arrays (C = A * A), they are copied once.
 * C's three arrays live in one page-locked block from a process-wide pool
 * (so the device-to-host copy runs at full link speed); spgemm_host_csr_free
 * returns the block to the pool. */
SPGEMM_API spgemm_status spgemm_csr_host_f64(spgemm_handle_t handle, const spgemm_csr_view* A,
                                  const spgemm_csr_view* B, spgemm_csr_out* C,
                                  void* stream);
SPGEMM_API spgemm_status spgemm_csr_host_f32(spgemm_handle_t handle, const spgemm_csr_view* A,
                                  const spgemm_csr_view* B, spgemm_csr_out* C,
                                  void* stream);
SPGEMM_API spgemm_status spgemm_host_csr_free(spgemm_csr_out* C);

/* Total intermediate products of A*B (FLOP = 2 * nip).  Replaces
 * utils::get_nip (src/libutils/include/utils/nip.cuh:52-78). */
SPGEMM_API spgemm_status spgemm_get_nip(spgemm_handle_t handle, const spgemm_csr_view* A,
                             const spgemm_csr_view* B, int64_t* nip, void* stream);

/* NIP of `count` independent pairs (A[i], B[i]) in one launch and one host
 * synchronisation: nip[i] = sum over A[i]'s entries (r, k) of nnz(B[i](k,:)).
 * A, B and nip are HOST arrays of count entries; the views' arrays are on the
 * device.  For callers that size many products at once (the served form's
 * admission); the reference sizes one pair per call (utils::get_nip,
 * nip.cuh:52-78). */
SPGEMM_API spgemm_status spgemm_get_nip_many(spgemm_handle_t handle, int32_t count,
                                             const spgemm_csr_view* A, const spgemm_csr_view* B,
                                             int64_t* nip, void* stream);

/* Statistics of the last product run on `handle`. */
SPGEMM_API spgemm_status spgemm_last_info(spgemm_handle_t handle, spgemm_info* info);

/* ---- options -------------------------------------------------------------- */

typedef enum spgemm_option {
    /* Validate operands on the device before multiplying (sorted, duplicate-free,
     * in-range columns; monotone rpt).  0 = off (default), 1 = on. */
    SPGEMM_OPT_CHECKED = 1,
    /* Test knob: every non-empty row goes to at least this bin of the symbolic
     * count ladder (-1 = off).  Exercises each kernel variant on small inputs,
     * like the reference's per-bin parameter tables (parameters.cuh:29-153). */
    SPGEMM_OPT_MIN_SYM_BIN = 2,
    /* Test knob: same for the fill + numeric ladder (-1 = off). */
    SPGEMM_OPT_MIN_NUM_BIN = 3,
    /* Cluster size (CTAs) of the distributed-shared-memory bins: 2, 4 or 8. */
    SPGEMM_OPT_CLUSTER_SIZE = 4,
    /* Number of side streams the bins are spread over (1..8). */
    SPGEMM_OPT_STREAMS = 5,
    /* Record a CUDA event pair around every kernel launch of a product; read
     * the durations with spgemm_last_profile.  0 = off (default), 1 = on. */
    SPGEMM_OPT_PROFILE = 6,
    /* Test knob: every non-empty row of a transpose goes to at least this bin
     * of its row-sort ladder (-1 = off). */
    SPGEMM_OPT_MIN_TRANSPOSE_BIN = 7,
    /* How the row sizes of C are found.  0 (default): one pass when the
     * product has at least 2^21 intermediate products (NIP), its
     * temporaries -- NIP entries of column and value -- fit 4 GiB, and a
     * sample of 4,096 rows of A (products with A.nnz >= 2^16) does not show
     * most of the NIP in rows of more than 768 products whose columns repeat
     * on average 4 times or more (those fill far smaller tables in two
     * passes); else two.  1: always one pass; 2: always two passes.  Two
     * passes: the hash count kernels give each row's exact nnz, the fill
     * writes C in place.  One pass: rows are filled into NIP-sized slots
     * while their nnz is counted, then compacted into C -- no count kernels,
     * one more copy of C.  The one-pass temporaries belong to the handle and
     * are kept for its next products (freed with the handle). */
    SPGEMM_OPT_ONE_PASS = 8,
    /* One-pass products with B.n <= 2^20: whether the four team fill bins
     * (rows of up to 12, 48, 192 and 768 intermediate products) and the
     * 256-thread bin (up to 3,072) expand, sort and compress -- stage every
     * product, sort by column, sum each column's run in product order --
     * instead of hashing.  0 (default): per bin, when the NIP / nnz of the
     * bin's rows among 4,096 rows sampled from A is at most 8, 8, 1.4 and 1.1
     * (the 256-thread bin follows the last team bin's sample; products with
     * A.nnz >= 2^16 -- smaller ones hash); 1: always; 2: never.
     * spgemm_info.esc_mask says which bins did (bits 0-4). */
    SPGEMM_OPT_ESC = 9
} spgemm_option;

SPGEMM_API spgemm_status spgemm_set_option(spgemm_handle_t handle, spgemm_option option, int64_t value);
SPGEMM_API spgemm_status spgemm_get_option(spgemm_handle_t handle, spgemm_option option, int64_t* value);

/* Per-launch device time of the last product (SPGEMM_OPT_PROFILE on), timed
 * with CUDA events on the stream each kernel was launched on.  The reference
 * marks the same phases with NVTX ranges (proposal.cuh:30, setup.cuh:139,
 * sym1.cuh:316, sym2.cuh:298, num.cuh:308). */
typedef struct spgemm_kernel_time {
    char name[48];  /* kernel variant, e.g. "s2n_team8_t64" */
    int32_t phase;  /* 0 count binning, 1 count, 2 scan binning, 3 fill+numeric */
    int32_t bin;    /* ladder bin, -1 for binning kernels */
    int32_t rows;   /* rows the launch handled (-1 if only known on the device) */
    float ms;       /* event-timed duration */
    float start_ms; /* launch start after the call's first launch (a timeline when
                       launches run side by side on the handle's side streams) */
} spgemm_kernel_time;

SPGEMM_API spgemm_status spgemm_last_profile(spgemm_handle_t handle, spgemm_kernel_time* out,
                                             int32_t capacity, int32_t* count);

/* Number of bins of each ladder and the key limit of bin `bin` (rows whose
 * key -- NIP for the count ladder, nnz for the fill ladders -- is <= limit).
 * which: 0 count ladder; 1 fill ladder used when B.n > 2^20; 2 fill ladder
 * used when B.n <= 2^20 (its large rows use a shared-memory bitmap);
 * 3 row-sort ladder of spgemm_transpose_* (key = length of a row of A^T);
 * 4 one-pass fill ladder used when B.n <= 2^20 (key = NIP; its team bins
 * expand, sort and compress, see SPGEMM_OPT_ESC). */
SPGEMM_API spgemm_status spgemm_ladder_info(spgemm_handle_t handle, int which,
                                 int dtype_bytes, int* n_bins, int64_t* limits /*[16]*/);

/* ---- transpose and the Galerkin triple product ----------------------------- */

/* T = A^T (n x m) as a library-allocated CSR with sorted columns, freed with
 * spgemm_csr_free.  Values are moved, not computed, so T is exact.  No
 * counterpart in the reference: its Galerkin use (R = P^T for R*A*P) leaves the
 * transpose to the caller; here it stays on the device.  Synchronous on
 * return; one host synchronisation inside. */
SPGEMM_API spgemm_status spgemm_transpose_f64(spgemm_handle_t handle, const spgemm_csr_view* A,
                                              spgemm_csr_out* T, void* stream);
SPGEMM_API spgemm_status spgemm_transpose_f32(spgemm_handle_t handle, const spgemm_csr_view* A,
                                              spgemm_csr_out* T, void* stream);

/* C = R * (A * P): two chained products (each exactly as spgemm_csr_*), the
 * intermediate A*P freed before return.  R = NULL means R = P^T, transposed on
 * the device (then P.m must equal A.m).  Requires A.n == P.m and R.n == A.m.
 * spgemm_last_info then describes the second product, with `nip` and
 * `host_syncs` summed over the chain.  Replaces two proposal::proposal calls
 * (proposal.cuh:85-124) plus a caller-side transpose. */
SPGEMM_API spgemm_status spgemm_rap_f64(spgemm_handle_t handle, const spgemm_csr_view* R,
                                        const spgemm_csr_view* A, const spgemm_csr_view* P,
                                        spgemm_csr_out* C, void* stream);
SPGEMM_API spgemm_status spgemm_rap_f32(spgemm_handle_t handle, const spgemm_csr_view* R,
                                        const spgemm_csr_view* A, const spgemm_csr_view* P,
                                        spgemm_csr_out* C, void* stream);

/* ---- batched products ------------------------------------------------------ */

/* A batch of `count` independent products C_i = A_i * B_i, given as two packed
 * block-diagonal operands: A = blockdiag(A_0, A_1, ...), B = blockdiag(B_0, ...).
 * Product i owns
 *   rows    [a_row_off[i], a_row_off[i+1]) of A (and of C),
 *   columns [b_row_off[i], b_row_off[i+1]) of A = rows of B,
 *   columns [c_col_off[i], c_col_off[i+1]) of B (and of C);
 * A_i's and B_i's column indices are global (already shifted by those offsets),
 * so the packed operands are ordinary CSR matrices.  All three offset arrays
 * are HOST arrays of count + 1 entries.  No counterpart in the reference, which
 * multiplies one pair per call. */
typedef struct spgemm_batch_desc {
    int32_t count;
    const int32_t* a_row_off;
    const int32_t* b_row_off;
    const int32_t* c_col_off;
} spgemm_batch_desc;

/* Result of a batch: one CSR per product, with LOCAL indices (row pointer from
 * 0, columns in [0, n_i)), as views into a few device allocations.  `products`
 * is a host array of `count` entries; `blocks` lists the device allocations. */
typedef struct spgemm_batch_out {
    int32_t count;
    spgemm_csr_out* products;
    int32_t n_blocks;
    void** blocks;
    int32_t n_groups;  /* block-diagonal sub-products the batch was run as */
} spgemm_batch_out;

/* Run the batch as one binned product of the block-diagonal operands (split
 * into as few groups as int32 nnz allows: each group's intermediate products
 * stay below 2^31), so rows of every product share bins, kernels and streams
 * instead of one launch sequence per product.  Synchronous on return. */
SPGEMM_API spgemm_status spgemm_batch_f64(spgemm_handle_t handle, const spgemm_batch_desc* desc,
                                          const spgemm_csr_view* A, const spgemm_csr_view* B,
                                          spgemm_batch_out* out, void* stream);
SPGEMM_API spgemm_status spgemm_batch_f32(spgemm_handle_t handle, const spgemm_batch_desc* desc,
                                          const spgemm_csr_view* A, const spgemm_csr_view* B,
                                          spgemm_batch_out* out, void* stream);
SPGEMM_API spgemm_status spgemm_batch_free(spgemm_batch_out* out, void* stream);

/* ---- plans: symbolic once, numeric many ------------------------------------ */

/* A plan fixes C's structure and the fill phase's bins for operands whose
 * STRUCTURE stays the same while their VALUES change (same device arrays,
 * updated in place): iterative solvers, AMG setup with new coefficients, a
 * batch of the same products every step.  Creating it runs the whole product
 * once (C is returned as from spgemm_csr_* / spgemm_batch_*) and captures the
 * fill kernels -- every bin of every group, side-stream branches included --
 * as ONE CUDA graph.  spgemm_plan_execute replays it: C's values (and, again,
 * its sorted columns) are recomputed from A's and B's current values with one
 * graph launch and no host synchronisation.
 *
 * tune = 1 runs an autotuner first: it builds the plan for every candidate of
 * a small grid -- the team fill bins' routing limits scaled by 1, 0.75 or 0.5
 * (rows above a scaled limit go to the next, wider bin) times 4 or 8 side
 * streams (parallel branches of the graph) -- times three replays of each and
 * keeps the fastest (spgemm_plan_get_info reports all of them).  tune = 0
 * keeps the default ladder.
 *
 * A, B, C (and a batch's blocks) must stay allocated while the plan lives;
 * destroy the plan after its last execution has completed.  No counterpart in
 * the reference, which recomputes the structure on every call. */
typedef struct spgemm_plan_s* spgemm_plan_t;

#define SPGEMM_PLAN_MAX_CANDIDATES 16

typedef struct spgemm_plan_info {
    int32_t candidates;   /* configurations built (1 without tuning) */
    int32_t chosen;       /* index of the one the plan keeps */
    float team_scale[SPGEMM_PLAN_MAX_CANDIDATES]; /* routing limits of the team fill bins x this
                                                     (the hash table and lanes a row gets) */
    float cta_scale[SPGEMM_PLAN_MAX_CANDIDATES];  /* the same for the CTA fill bins (the table
                                                     and block size a row gets) */
    int32_t streams[SPGEMM_PLAN_MAX_CANDIDATES];  /* side streams = parallel graph branches */
    float ms[SPGEMM_PLAN_MAX_CANDIDATES];         /* median replay time of each */
} spgemm_plan_info;

SPGEMM_API spgemm_status spgemm_plan_csr_f64(spgemm_handle_t handle, const spgemm_csr_view* A,
                                             const spgemm_csr_view* B, int32_t tune,
                                             spgemm_csr_out* C, spgemm_plan_t* plan,
                                             void* stream);
SPGEMM_API spgemm_status spgemm_plan_csr_f32(spgemm_handle_t handle, const spgemm_csr_view* A,
                                             const spgemm_csr_view* B, int32_t tune,
                                             spgemm_csr_out* C, spgemm_plan_t* plan,
                                             void* stream);
SPGEMM_API spgemm_status spgemm_plan_batch_f64(spgemm_handle_t handle,
                                               const spgemm_batch_desc* desc,
                                               const spgemm_csr_view* A, const spgemm_csr_view* B,
                                               int32_t tune, spgemm_batch_out* out,
                                               spgemm_plan_t* plan, void* stream);
SPGEMM_API spgemm_status spgemm_plan_batch_f32(spgemm_handle_t handle,
                                               const spgemm_batch_desc* desc,
                                               const spgemm_csr_view* A, const spgemm_csr_view* B,
                                               int32_t tune, spgemm_batch_out* out,
                                               spgemm_plan_t* plan, void* stream);
/* Replay: asynchronous on `stream` (one graph launch). */
SPGEMM_API spgemm_status spgemm_plan_execute(spgemm_plan_t plan, void* stream);
/* Synchronise `stream` and report device-side errors of the executions since
 * the last check (capacity or probe-bound flags, as for a product). */
SPGEMM_API spgemm_status spgemm_plan_check(spgemm_plan_t plan, void* stream);
SPGEMM_API spgemm_status spgemm_plan_get_info(spgemm_plan_t plan, spgemm_plan_info* info);
SPGEMM_API spgemm_status spgemm_plan_destroy(spgemm_plan_t plan);

/* ---- allocation-free row sizes --------------------------------------------- */

/* Largest B.n that spgemm_row_nnz_noalloc accepts. */
#define SPGEMM_NOALLOC_MAX_COLS (1 << 20)

/* Exact number of nonzeros of every row of C = A * B, written to the caller's
 * device array c_row_nnz[A.m], WITHOUT allocating anything: no cudaMalloc,
 * cudaMallocAsync, cudaFree or allocating library call, and no handle (a
 * handle owns allocated scratch).  No counterpart in the reference: it is for
 * callers that cannot allocate at the point where they size a product, for
 * example because all device memory is already owned by their own pool, or
 * because an allocation there would synchronise the device.  The caller can
 * scan the counts into a row pointer and allocate C from its own memory.
 *
 * Only the index arrays of A and B are read (val may be NULL).  B's columns
 * must lie in [0, B.n) with B.n <= SPGEMM_NOALLOC_MAX_COLS; larger B.n is
 * rejected with SPGEMM_ERR_INVALID_ARG.  A column of B outside [0, B.n) is
 * skipped, and every row of C that reaches it gets the count -1 (the call
 * itself does not synchronise, so the check is reported in the output).
 * Runs on the current device and returns without synchronising
 * (stream-ordered on `stream`).  At most 32 CTAs run (one per scratch slot),
 * so large products take longer here than in spgemm_csr_*.
 *
 * Scratch: a fixed 4 MiB bitmap area compiled into the library's device image
 * (every GPU that loads the library holds it until the process exits).  The
 * first call on a device looks up that area's device address
 * (cudaGetSymbolAddress), so make the first call on each device outside any
 * stream capture.  Every call uses the same area and clears it first, so calls
 * that overlap on the GPU (other streams, other host threads) race: serialise
 * them. */
SPGEMM_API spgemm_status spgemm_row_nnz_noalloc(const spgemm_csr_view* A,
                                                const spgemm_csr_view* B, int32_t* c_row_nnz,
                                                void* stream);

/* ---- errors / version ----------------------------------------------------- */

/* Message of the last error raised on the calling thread ("" if none). */
SPGEMM_API const char* spgemm_last_error_string(void);
SPGEMM_API const char* spgemm_status_string(spgemm_status status);
SPGEMM_API int spgemm_abi_version(void);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* SPGEMM_B200_H */
