// Host orchestration of the B200 CSR SpGEMM and its C ABI (include/spgemm.h).
//
// One product (reference: proposal_inner, proposal.cuh:26-80):
//   count pass      NIP per row -> per-CTA histograms -> offsets -> stable
//                   scatter of rows into count bins            [host sync 1]
//   sym1            one kernel per non-empty count bin, heavy bins first,
//                   spread over side streams; cluster-bin spills go to the
//                   global bin in stream order (no host round-trip)
//   scan pass       nnz histograms -> offsets -> scatter + exclusive scan of
//                   C.rpt                                         [host sync 2]
//   fill+numeric    allocate C.col / C.val, one fused kernel per non-empty bin
//                   [final sync]
// The reference synchronises with the host after every binning step and
// creates/destroys its streams and scratch in every call (setup.cuh:164-165,
// cleanup.cuh:15-31); here streams, events and scratch live in the handle.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/spgemm.h"
#include "common.cuh"
#include "kernels.hpp"

namespace b200 {
namespace {

thread_local std::string g_last_error;

spgemm_status fail(spgemm_status st, const std::string& msg) {
    g_last_error = msg;
    return st;
}

spgemm_status cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? SPGEMM_ERR_OOM : SPGEMM_ERR_CUDA;
}

#define B200_TRY(expr)                                                \
    do {                                                              \
        cudaError_t e_ = (expr);                                      \
        if (e_ != cudaSuccess) return cuda_fail(e_, #expr);           \
    } while (0)

constexpr int kMaxSide = 8;
// Bytes of the scratch front (status, plans, fail counter, sample, ladder)
// that one synchronisation copies back.
constexpr size_t kFrontBytes = 4096;
// Bitmap pool budget of the global bins (bytes).
constexpr int64_t kBitmapBudget = int64_t(1) << 30;

struct Scratch {
    DevStatus* status;
    Plan* plan1;
    // the one-pass row pointer's look-back: a ticket counter and one state per
    // tile (behind the mirrored front)
    unsigned long long* scan_state;
    Plan* plan2;
    int32_t* hist1;
    int32_t* hist2;
    int32_t* hist3;  // the NIP pass's fill-ladder counts (early one-pass products)
    int64_t* cta_sum;
    int32_t* bins1;
    int32_t* bins2;
    int32_t* fail_rows;
    int32_t* fail_count;
    EscSample* sample;
    Ladder* dladder;  // the one-pass fill binning's limits, decided on the device
    int32_t* work;    // one row counter per fill bin (persistent bins)
};

struct ProfRec {
    const char* name;
    int32_t phase;
    int32_t bin;
    int32_t rows;
    cudaEvent_t a;
    cudaEvent_t b;
};

// Pinned host mirror of the device-side plan words, copied in one transfer.
struct HostMirror {
    Plan plan;
    Plan plan_b;  // a second plan, when one synchronisation reads two
    DevStatus status;
    int32_t fail_count;
    int32_t pad[3];
    EscSample sample;
};

}  // namespace
}  // namespace b200

struct spgemm_handle_s {
    int device = 0;
    int sm_count = 148;
    cudaStream_t side[b200::kMaxSide] = {};
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_sample = nullptr;  // the compression sample's side stream is done
    cudaEvent_t ev_mirror = nullptr;  // the scratch front's copy to the host is done
    cudaEvent_t ev_front = nullptr;   // the scratch front is final (the copy may start)
    cudaEvent_t ev_join[b200::kMaxSide] = {};
    int nside = 4;
    // scratch (grown, never shrunk)
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    uint32_t* bitmaps = nullptr;
    size_t bitmap_bytes = 0;
    // one-pass temporaries (NIP slots, their columns and values): grown,
    // never shrunk, like the scratch.  Taking them from the pool per call
    // cost ~2.7 ms of host time whenever live results had fragmented it
    // (products of different shapes in turn, as in R * (A * P)).
    void* onepass = nullptr;
    size_t onepass_bytes = 0;
    void* slots = nullptr;  // one-pass NIP slot starts (m + 1), grown like the rest
    size_t slots_bytes = 0;
    b200::HostMirror* mirror = nullptr;  // pinned
    char* front_host = nullptr;          // pinned copy of the scratch front
    // host-operand staging on the device
    void* in_buf = nullptr;
    size_t in_bytes = 0;
    // options
    int checked = 0;
    int min_sym_bin = -1;
    int min_num_bin = -1;
    int cluster = 4;
    int profile = 0;
    int min_tr_bin = -1;
    int one_pass = 0;  // 0 chosen by temporary size, 1 always, 2 never (two-pass)
    int esc = 0;  // one-pass team bins: 0 ESC where sampled compression is low, 1 always, 2 never
    // C's arrays come from the device's shared stream-ordered pool (see
    // device_pool); it keeps freed memory mapped so repeated products do not
    // re-map hundreds of MB per call.  cudaFree / cudaFreeAsync release them.
    cudaMemPool_t pool = nullptr;
    spgemm_info info = {};
    // profiling: an event pair per launch, resolved after the final sync
    std::vector<b200::ProfRec> prof;
    std::vector<cudaEvent_t> prof_events;
    std::vector<spgemm_kernel_time> prof_done;
};

// A plan: the fill phase of one product (or of every group of a batch)
// captured as a CUDA graph over buffers the plan owns, replayed by
// spgemm_plan_execute to recompute C from A's and B's current values.
struct spgemm_plan_s {
    int device = 0;
    cudaMemPool_t pool = nullptr;
    cudaStream_t capture = nullptr;       // private stream the graphs were captured on
    cudaGraph_t graph = nullptr;          // the whole plan (a parent graph for batches)
    std::vector<cudaGraph_t> children;    // per-group graphs of a batch plan
    cudaGraphExec_t exec = nullptr;
    b200::DevStatus* status = nullptr;    // written by the captured kernels
    b200::DevStatus* status_host = nullptr;  // pinned
    std::vector<void*> owned;             // device buffers the graph reads
    spgemm_plan_info info = {};
};

namespace b200 {
namespace {

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Handle buffers grow stream-ordered from the device pool: no device-wide
// synchronisation, so a handle growing its scratch never stalls work that
// other handles have in flight.
spgemm_status regrow(spgemm_handle_s* h, void** buf, size_t* have, size_t need,
                     cudaStream_t stream) {
    if (need <= *have) return SPGEMM_OK;
    if (*buf != nullptr) {
        B200_TRY(cudaFreeAsync(*buf, stream));
        *buf = nullptr;
        *have = 0;
    }
    B200_TRY(cudaMallocFromPoolAsync(buf, need, h->pool, stream));
    *have = need;
    return SPGEMM_OK;
}

spgemm_status ensure_scratch(spgemm_handle_s* h, int32_t m, Scratch* s, cudaStream_t stream) {
    const size_t nctas = static_cast<size_t>(bin_ctas(m > 0 ? m : 1));
    const size_t mm = static_cast<size_t>(m > 0 ? m : 1);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    const size_t o_status = take(sizeof(DevStatus));
    const size_t o_plan1 = take(sizeof(Plan));
    const size_t o_plan2 = take(sizeof(Plan));
    const size_t o_fail_count = take(sizeof(int32_t));
    const size_t o_sample = take(sizeof(EscSample));
    const size_t o_dladder = take(sizeof(Ladder));
    const size_t o_hist1 = take(sizeof(int32_t) * kMaxBins * nctas);
    const size_t o_hist2 = take(sizeof(int32_t) * kMaxBins * nctas);
    const size_t o_hist3 = take(sizeof(int32_t) * kMaxBins * nctas);
    const size_t o_sum = take(sizeof(int64_t) * nctas);
    const size_t o_bins1 = take(sizeof(int32_t) * mm);
    const size_t o_bins2 = take(sizeof(int32_t) * mm);
    const size_t o_fail = take(sizeof(int32_t) * mm);
    const size_t o_work = take(sizeof(int32_t) * kMaxBins);
    const size_t o_scan = take(sizeof(unsigned long long) * (1 + kScanMaxTiles));
    if (spgemm_status st = regrow(h, &h->scratch, &h->scratch_bytes, off + off / 4, stream);
        st != SPGEMM_OK)
        return st;
    char* b = static_cast<char*>(h->scratch);
    s->status = reinterpret_cast<DevStatus*>(b + o_status);
    s->plan1 = reinterpret_cast<Plan*>(b + o_plan1);
    s->plan2 = reinterpret_cast<Plan*>(b + o_plan2);
    s->fail_count = reinterpret_cast<int32_t*>(b + o_fail_count);
    s->sample = reinterpret_cast<EscSample*>(b + o_sample);
    s->dladder = reinterpret_cast<Ladder*>(b + o_dladder);
    s->hist1 = reinterpret_cast<int32_t*>(b + o_hist1);
    s->hist2 = reinterpret_cast<int32_t*>(b + o_hist2);
    s->hist3 = reinterpret_cast<int32_t*>(b + o_hist3);
    s->cta_sum = reinterpret_cast<int64_t*>(b + o_sum);
    s->bins1 = reinterpret_cast<int32_t*>(b + o_bins1);
    s->bins2 = reinterpret_cast<int32_t*>(b + o_bins2);
    s->fail_rows = reinterpret_cast<int32_t*>(b + o_fail);
    s->work = reinterpret_cast<int32_t*>(b + o_work);
    s->scan_state = reinterpret_cast<unsigned long long*>(b + o_scan);
    return SPGEMM_OK;
}

spgemm_status ensure_bitmaps(spgemm_handle_s* h, int64_t words, int32_t rows, int32_t* nmaps,
                            cudaStream_t stream) {
    const int64_t per_map = words * 4;
    int64_t n = std::min<int64_t>(rows, h->sm_count);
    n = std::min<int64_t>(n, std::max<int64_t>(1, kBitmapBudget / std::max<int64_t>(per_map, 1)));
    n = std::max<int64_t>(n, 1);
    const size_t need = static_cast<size_t>(n * per_map);
    if (spgemm_status st = regrow(h, reinterpret_cast<void**>(&h->bitmaps), &h->bitmap_bytes,
                                  need, stream);
        st != SPGEMM_OK)
        return st;
    *nmaps = static_cast<int32_t>(n);
    return SPGEMM_OK;
}

// Rows of a fill plan that may need the global bins' bitmaps: the global
// bin's, and the cluster bitmap bin's when B.n is past the columns a cluster
// holds (that bin then hands its rows to the global kernel).
int32_t global_bitmap_rows(const BinLauncher* bins, int nb, const Plan& plan, int32_t n) {
    int32_t rows = plan.bin_size[nb - 1];
    if (nb >= 2 && bins[nb - 2].kind == BinKind::Cluster &&
        static_cast<int64_t>(n) > kClusterBitmapCols)
        rows = std::max(rows, plan.bin_size[nb - 2]);
    return rows;
}

Ladder make_ladder(const BinLauncher* bins, int nb, int min_bin) {
    Ladder l = {};
    l.nb = nb;
    l.min_bin = min_bin < 0 ? 0 : std::min(min_bin, nb - 1);
    for (int i = 0; i < nb; i++) l.limit[i] = bins[i].limit;
    return l;
}

spgemm_status fork_streams(spgemm_handle_s* h, cudaStream_t main) {
    B200_TRY(cudaEventRecord(h->ev_fork, main));
    for (int i = 0; i < h->nside; i++) B200_TRY(cudaStreamWaitEvent(h->side[i], h->ev_fork, 0));
    return SPGEMM_OK;
}

spgemm_status join_streams(spgemm_handle_s* h, cudaStream_t main) {
    for (int i = 0; i < h->nside; i++) {
        B200_TRY(cudaEventRecord(h->ev_join[i], h->side[i]));
        B200_TRY(cudaStreamWaitEvent(main, h->ev_join[i], 0));
    }
    return SPGEMM_OK;
}

spgemm_status check_view(const spgemm_csr_view* v, const char* name) {
    if (v == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, std::string(name) + " is NULL");
    if (v->m < 0 || v->n < 0 || v->nnz < 0)
        return fail(SPGEMM_ERR_INVALID_ARG, std::string(name) + " has a negative dimension");
    if (v->rpt == nullptr)
        return fail(SPGEMM_ERR_INVALID_ARG, std::string(name) + ".rpt is NULL");
    if (v->nnz > 0 && (v->col == nullptr || v->val == nullptr))
        return fail(SPGEMM_ERR_INVALID_ARG, std::string(name) + ".col/.val is NULL");
    return SPGEMM_OK;
}

spgemm_status status_to_error(const DevStatus& st) {
    if (st.flags == 0u) return SPGEMM_OK;
    char buf[256];
    if (st.flags & kStBadInput) {
        std::snprintf(buf, sizeof buf,
                      "invalid operand: unsorted, duplicate or out-of-range column, or bad row "
                      "pointer (row %d, check %d)",
                      st.row, st.detail);
        return fail(SPGEMM_ERR_INVALID_ARG, buf);
    }
    if (st.flags & kStWait) {
        std::snprintf(buf, sizeof buf,
                      "a bounded device wait ran out (the row pointer's look-back: tile %d "
                      "waiting on tile %d or one of the 31 before it)",
                      st.row, st.detail);
        return fail(SPGEMM_ERR_TIMEOUT, buf);
    }
    std::snprintf(buf, sizeof buf, "device status 0x%x at row %d (detail %d)", st.flags, st.row,
                  st.detail);
    return fail(SPGEMM_ERR_INTERNAL, buf);
}

// The status word, both plans, the fail counter and the sample sit at the
// front of the handle's scratch (ensure_scratch): one copy brings them all
// back, and the host picks the words it asked for out of it.
// The host's copy of the scratch front (plans, sample sums, status words)
// in two halves: mirror_start queues the copy and an event behind the work
// that wrote them, so later work can be queued before the host waits;
// mirror_finish waits for that event only and unpacks the copy.  The copy
// runs on the last side stream (behind an event on `stream`), so the work
// queued on `stream` after it does not wait for it; that work must not write
// the front.
spgemm_status mirror_start(spgemm_handle_s* h, cudaStream_t stream, const Scratch& s) {
    const char* dev0 = static_cast<const char*>(h->scratch);
    const size_t front = static_cast<size_t>(reinterpret_cast<const char*>(s.hist1) - dev0);
    if (front > kFrontBytes) return fail(SPGEMM_ERR_INTERNAL, "scratch front exceeds its mirror");
    cudaStream_t copy = h->side[kMaxSide - 1];
    B200_TRY(cudaEventRecord(h->ev_front, stream));
    B200_TRY(cudaStreamWaitEvent(copy, h->ev_front, 0));
    B200_TRY(cudaMemcpyAsync(h->front_host, h->scratch, front, cudaMemcpyDeviceToHost, copy));
    B200_TRY(cudaEventRecord(h->ev_mirror, copy));
    return SPGEMM_OK;
}

spgemm_status mirror_finish(spgemm_handle_s* h, const Plan* plan, const Scratch& s,
                            bool with_sample = false, const Plan* plan_b = nullptr) {
    const char* dev0 = static_cast<const char*>(h->scratch);
    B200_TRY(cudaEventSynchronize(h->ev_mirror));
    h->info.host_syncs++;
    auto at = [&](const void* dev) {
        return h->front_host + (static_cast<const char*>(dev) - dev0);
    };
    std::memcpy(&h->mirror->plan, at(plan), sizeof(Plan));
    if (plan_b != nullptr) std::memcpy(&h->mirror->plan_b, at(plan_b), sizeof(Plan));
    if (with_sample) std::memcpy(&h->mirror->sample, at(s.sample), sizeof(EscSample));
    std::memcpy(&h->mirror->status, at(s.status), sizeof(DevStatus));
    std::memcpy(&h->mirror->fail_count, at(s.fail_count), sizeof(int32_t));
    return SPGEMM_OK;
}

spgemm_status sync_mirror(spgemm_handle_s* h, cudaStream_t stream, const Plan* plan,
                          const Scratch& s, bool with_sample = false,
                          const Plan* plan_b = nullptr) {
    const char* dev0 = static_cast<const char*>(h->scratch);
    const size_t front = static_cast<size_t>(reinterpret_cast<const char*>(s.hist1) - dev0);
    if (front > kFrontBytes) return fail(SPGEMM_ERR_INTERNAL, "scratch front exceeds its mirror");
    B200_TRY(cudaMemcpyAsync(h->front_host, h->scratch, front, cudaMemcpyDeviceToHost, stream));
    B200_TRY(cudaStreamSynchronize(stream));
    h->info.host_syncs++;
    auto at = [&](const void* dev) {
        return h->front_host + (static_cast<const char*>(dev) - dev0);
    };
    std::memcpy(&h->mirror->plan, at(plan), sizeof(Plan));
    if (plan_b != nullptr) std::memcpy(&h->mirror->plan_b, at(plan_b), sizeof(Plan));
    if (with_sample) std::memcpy(&h->mirror->sample, at(s.sample), sizeof(EscSample));
    std::memcpy(&h->mirror->status, at(s.status), sizeof(DevStatus));
    std::memcpy(&h->mirror->fail_count, at(s.fail_count), sizeof(int32_t));
    return SPGEMM_OK;
}

cudaError_t prof_event(spgemm_handle_s* h, cudaEvent_t* ev) {
    const size_t used = h->prof.size() * 2;
    while (h->prof_events.size() < used + 2) {
        cudaEvent_t e;
        cudaError_t err = cudaEventCreate(&e);
        if (err != cudaSuccess) return err;
        h->prof_events.push_back(e);
    }
    ev[0] = h->prof_events[used];
    ev[1] = h->prof_events[used + 1];
    return cudaSuccess;
}

// Launch through `fn` on `stream`; with profiling on, bracket it by an event
// pair recorded on the same stream.
template<typename F>
spgemm_status timed(spgemm_handle_s* h, const char* name, int phase, int bin, int rows,
                    cudaStream_t stream, F&& fn) {
    cudaEvent_t ev[2] = {nullptr, nullptr};
    if (h->profile) {
        B200_TRY(prof_event(h, ev));
        B200_TRY(cudaEventRecord(ev[0], stream));
    }
    cudaError_t e = fn(stream);
    if (e != cudaSuccess) return cuda_fail(e, name);
    if (h->profile) {
        B200_TRY(cudaEventRecord(ev[1], stream));
        h->prof.push_back(ProfRec{name, phase, bin, rows, ev[0], ev[1]});
    }
    return SPGEMM_OK;
}

// After the stream is synchronised: turn the recorded pairs into durations.
void resolve_profile(spgemm_handle_s* h) {
    h->prof_done.clear();
    // start offsets from the call's first launch event
    const cudaEvent_t t0 = h->prof.empty() ? nullptr : h->prof.front().a;
    for (const ProfRec& r : h->prof) {
        spgemm_kernel_time k = {};
        std::snprintf(k.name, sizeof k.name, "%s", r.name);
        k.phase = r.phase;
        k.bin = r.bin;
        k.rows = r.rows;
        float ms = -1.0f;
        if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) ms = -1.0f;
        k.ms = ms;
        float start = -1.0f;
        if (cudaEventElapsedTime(&start, t0, r.a) != cudaSuccess) start = -1.0f;
        k.start_ms = start;
        h->prof_done.push_back(k);
    }
    h->prof.clear();
}

// One kernel per non-empty bin, heavy bins first, round-robin over the side
// streams (forked from and joined back into `main`).
spgemm_status launch_bins(spgemm_handle_s* h, const BinLauncher* bins, int nb, int phase,
                          const Plan& plan, const int32_t* row_lists, const ProductArgs& base,
                          cudaStream_t main) {
    if (spgemm_status st = fork_streams(h, main); st != SPGEMM_OK) return st;
    // the heaviest non-empty bin (the first launched) has side stream 0 --
    // the high-priority one -- to itself: it is the phase's longest kernel,
    // and nothing queues behind it; the others share the remaining streams
    int next = 0;
    for (int b = nb - 1; b >= 0; b--) {
        const int rows = plan.bin_size[b];
        if (rows <= 0) continue;
        ProductArgs a = base;
        a.rows = row_lists + plan.bin_off[b];
        a.nrows = rows;
        a.work = base.work != nullptr ? base.work + b : nullptr;
        cudaStream_t s = h->side[next == 0 || h->nside == 1 ? 0 : 1 + (next - 1) % (h->nside - 1)];
        next++;
        const BinLauncher& L = bins[b];
        if (spgemm_status st = timed(h, L.name, phase, b, rows, s,
                                     [&](cudaStream_t ss) { return L.launch(a, ss); });
            st != SPGEMM_OK)
            return st;
    }
    return join_streams(h, main);
}

// Plan capture request for product(): the team fill bins' routing limits are
// scaled by team_scale (rows above the scaled limit go to the next, wider
// bin; a tuning knob), and with `plan` set the fill launches are captured as
// a graph over plan-owned copies of the bin lists, bitmaps and status word.
// launch_now: instantiate the graph into plan->exec and run it (single
// products); otherwise hand it back in `graph` (batch groups).
struct CaptureReq {
    double team_scale = 1.0;
    double cta_scale = 1.0;  // the same for the CTA bins (block size and table of a row)
    spgemm_plan_s* plan = nullptr;
    bool launch_now = true;
    cudaGraph_t graph = nullptr;
};

Ladder scaled_ladder(const BinLauncher* bins, int nb, int min_bin, double team_scale,
                     double cta_scale = 1.0) {
    Ladder l = make_ladder(bins, nb, min_bin);
    if (team_scale >= 1.0 && cta_scale >= 1.0) return l;
    int prev = 0;
    for (int i = 0; i < nb; i++) {
        // the team bins' limits by team_scale, the CTA bins' by cta_scale
        // (the bitmap bin, whose limit is the column count, keeps it)
        const double sc = bins[i].kind == BinKind::Team ? team_scale
                          : (bins[i].kind == BinKind::Cta && bins[i].limit < kBitmapCols)
                              ? cta_scale
                              : 1.0;
        if (sc < 1.0) {
            const int lim = static_cast<int>(bins[i].limit * sc);
            l.limit[i] = lim > prev ? lim : prev + 1;  // limits stay increasing
        }
        prev = l.limit[i];
    }
    return l;
}

spgemm_status plan_alloc(spgemm_plan_s* plan, void** p, size_t bytes, cudaStream_t stream) {
    B200_TRY(cudaMallocFromPoolAsync(p, bytes, plan->pool, stream));
    plan->owned.push_back(*p);
    return SPGEMM_OK;
}

template<typename V>
spgemm_status product(spgemm_handle_s* h, const spgemm_csr_view* A, const spgemm_csr_view* B,
                      spgemm_csr_out* C, cudaStream_t stream, CaptureReq* cr = nullptr) {
    if (h == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "handle is NULL");
    if (C == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "C is NULL");
    if (spgemm_status st = check_view(A, "A"); st != SPGEMM_OK) return st;
    if (spgemm_status st = check_view(B, "B"); st != SPGEMM_OK) return st;
    if (A->n != B->m)
        return fail(SPGEMM_ERR_INVALID_ARG, "A.n (" + std::to_string(A->n) +
                                                ") must equal B.m (" + std::to_string(B->m) + ")");
    std::memset(C, 0, sizeof(*C));
    h->info = spgemm_info{};
    h->prof.clear();
    h->prof_done.clear();
    B200_TRY(cudaSetDevice(h->device));

    const int32_t m = A->m;
    const int32_t n = B->n;
    C->m = m;
    C->n = n;

    const BinLauncher* sym = nullptr;
    const int nsym = sym1_ladder(&sym);
    const BinLauncher* fil = nullptr;
    const bool narrow = n <= kBitmapCols;
    const int nfil = sizeof(V) == 8 ? (narrow ? s2n_bitmap_ladder_f64(&fil) : s2n_ladder_f64(&fil))
                                    : (narrow ? s2n_bitmap_ladder_f32(&fil) : s2n_ladder_f32(&fil));
    h->info.n_sym_bins = nsym;
    h->info.n_num_bins = nfil;

    int32_t* c_rpt = nullptr;
    const auto t_start = std::chrono::steady_clock::now();
    auto mark = [&](int i) {
        h->info.phase_us[i] = static_cast<float>(
            std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t_start)
                .count());
    };
    B200_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&c_rpt),
                                     sizeof(int32_t) * (size_t(m) + 1), h->pool, stream));
    C->rpt = c_rpt;
    auto bail = [&](spgemm_status st) {
        const std::string msg = g_last_error;
        cudaStreamSynchronize(h->side[0]);  // a compression sample may still read A and B
        cudaStreamSynchronize(stream);
        spgemm_csr_free(C, stream);
        cudaStreamSynchronize(stream);
        h->prof.clear();
        g_last_error = msg;
        return st;
    };
#define B200_STEP(expr)                                                  \
    do {                                                                 \
        spgemm_status st_ = (expr);                                      \
        if (st_ != SPGEMM_OK) return bail(st_);                          \
    } while (0)
#define B200_STEP_R(expr)                                                \
    do {                                                                 \
        spgemm_status st_ = (expr);                                      \
        if (st_ != SPGEMM_OK) return st_;                                \
    } while (0)

    Scratch s;
    B200_STEP(ensure_scratch(h, m, &s, stream));
    // status, plans and fail counter are contiguous at the front of the scratch
    if (cudaError_t e = cudaMemsetAsync(
            h->scratch, 0, reinterpret_cast<char*>(s.hist1) - static_cast<char*>(h->scratch),
            stream);
        e != cudaSuccess)
        return bail(cuda_fail(e, "memset scratch"));
    if (h->checked) {
        B200_STEP(timed(h, "check_csr_A", 0, -1, A->m, stream, [&](cudaStream_t ss) {
            return launch_check_csr(A->rpt, A->col, A->m, A->n, A->nnz, s.status, ss);
        }));
        B200_STEP(timed(h, "check_csr_B", 0, -1, B->m, stream, [&](cudaStream_t ss) {
            return launch_check_csr(B->rpt, B->col, B->m, B->n, B->nnz, s.status, ss);
        }));
        // no kernel indexes through an operand that failed validation
        B200_STEP(sync_mirror(h, stream, s.plan1, s));
        B200_STEP(status_to_error(h->mirror->status));
    }
    if (m == 0 || A->nnz == 0 || B->nnz == 0) {
        if (cudaError_t e = cudaMemsetAsync(c_rpt, 0, sizeof(int32_t) * (size_t(m) + 1), stream);
            e != cudaSuccess)
            return bail(cuda_fail(e, "memset C.rpt"));
        B200_STEP(sync_mirror(h, stream, s.plan1, s));
        B200_STEP(status_to_error(h->mirror->status));
        resolve_profile(h);
        return SPGEMM_OK;
    }

    // ---- count pass: NIP per row and bins ---------------------------------
    const int nctas = bin_ctas(m);
    const Ladder lad1 = make_ladder(sym, nsym, h->min_sym_bin);
    // Compression sample (products that may run one pass): it reads A and B
    // only, so it runs on a side stream beside the NIP pass (forked before
    // it), then decides the one-pass fill binning's limits on the device.
    // Its sums come back with the fill binning's plan: they choose one pass
    // or two and, per fill bin, expand-sort-compress or hashing.
    const Ladder ladf = make_ladder(fil, nfil, h->min_num_bin);
    const int esc_mode = (narrow && h->esc != 2) ? h->esc : 2;
    const bool sampled = cr == nullptr && h->one_pass != 2 && A->nnz >= kSampleMinNnz &&
                         (h->one_pass == 0 || esc_mode == 0);
    if (sampled) {
        EscLimits el{};
        for (int b = 0; b < kEscBins; b++) el.limit[b] = fil[b].limit;
        const int32_t samples = std::min<int32_t>(m, kEscSamples);
        cudaStream_t side = h->side[0];
        ProductArgs ps = {};
        ps.a_rpt = A->rpt;
        ps.a_col = A->col;
        ps.b_rpt = B->rpt;
        ps.b_col = B->col;
        ps.status = s.status;
        // (the sample's sums were zeroed with the scratch front above)
        if (cudaError_t e = cudaEventRecord(h->ev_fork, stream); e != cudaSuccess)
            return bail(cuda_fail(e, "fork the sample stream"));
        if (cudaError_t e = cudaStreamWaitEvent(side, h->ev_fork, 0); e != cudaSuccess)
            return bail(cuda_fail(e, "fork the sample stream"));
        B200_STEP(timed(h, "esc_sample", 0, -1, samples, side, [&](cudaStream_t ss) {
            return launch_esc_sample(ps, m, samples, el, s.sample, ss);
        }));
        B200_STEP(timed(h, "esc_decide", 0, -1, 1, side, [&](cudaStream_t ss) {
            return launch_esc_decide(s.sample, ladf, esc_mode, s.dladder, ss);
        }));
        if (cudaError_t e = cudaEventRecord(h->ev_sample, side); e != cudaSuccess)
            return bail(cuda_fail(e, "join the sample stream"));
    }
    // A product likely to run one pass is binned for the fill right away and
    // decided at the one synchronisation that follows; the count binning then
    // runs only if it turns out two-pass.  Its fill binning scans a copy of
    // the NIP per row, which the NIP pass writes beside C.rpt.
    const bool early = cr == nullptr && h->one_pass != 2 &&
                       (h->one_pass == 1 || A->nnz >= kEarlyOnePassNnz);
    int32_t* off = nullptr;  // the one-pass NIP slots: a scan of the NIP per row
    bool off_written = false;
    if (early) {
        B200_STEP(regrow(h, &h->slots, &h->slots_bytes, sizeof(int32_t) * (size_t(m) + 1),
                         stream));
        off = static_cast<int32_t*>(h->slots);
        off_written = true;
    }
    // The fill binning by NIP (the one-pass path's), with limits decided on
    // the device when the sample ran: off = the scan of the NIP per row.
    Ladder ladh = ladf;
    if (esc_mode == 1) ladh.limit[kEscBins - 1] = kEscSplit;
    const Ladder* dlad = sampled ? s.dladder : nullptr;
    // Early products: the NIP pass also counts the rows by the fill ladder's
    // limits plus the split the device may choose (the sample runs beside
    // it), and the fill binning maps those counts onto the chosen ladder.
    Ladder ladx = ladh;
    ladx.min_bin = 0;  // the mapping applies the chosen ladder's
    bool ladx_ok = true;
    if (sampled) {
        int pos = 0;
        while (pos < ladx.nb && ladx.limit[pos] < kEscSplit) pos++;
        if (pos == ladx.nb || ladx.limit[pos] != kEscSplit) {
            if (ladx.nb < kMaxBins) {
                for (int i = ladx.nb; i > pos; i--) ladx.limit[i] = ladx.limit[i - 1];
                ladx.limit[pos] = kEscSplit;
                ladx.nb++;
            } else {
                ladx_ok = false;  // no room: the fill binning counts the rows itself
            }
        }
    }
    const bool nip_counts_fill = early && ladx_ok;
    bool mirror_pending = false;  // mirror_start ran: the first wait is on its event
    // the row pointer's look-back scan needs its ticket and tile states zeroed
    const bool scan1 = rpt_scan_tiles(m) <= kScanMaxTiles;
    const size_t scan_bytes = sizeof(unsigned long long) * (1 + size_t(rpt_scan_tiles(m)));
    bool scan_zeroed = false;
    B200_STEP(timed(h, "nip_hist", 0, -1, m, stream, [&](cudaStream_t ss) {
        return launch_nip_hist(A->rpt, A->col, B->rpt, m, c_rpt, off, s.hist1, s.plan1, s.status,
                               lad1, ss, s.hist3, s.cta_sum, nip_counts_fill ? &ladx : nullptr);
    }));
    auto fill_binning = [&]() -> spgemm_status {
        if (nip_counts_fill) {
            // the NIP pass counted the rows by ladx: offsets for the chosen
            // ladder, then the scatter
            if (sampled) B200_TRY(cudaStreamWaitEvent(stream, h->ev_sample, 0));
            // (the row pointer's look-back state is zeroed by the same launch)
            B200_STEP_R(timed(h, "nip_fill_offsets", 2, -1, m, stream, [&](cudaStream_t ss) {
                return launch_bin_offsets_map(s.hist3, s.hist2, nctas, ladx, s.cta_sum, s.plan2,
                                              ladh, dlad, ss, scan1 ? s.scan_state : nullptr,
                                              scan1 ? static_cast<int32_t>(scan_bytes / 8) : 0);
            }));
            scan_zeroed = scan1;
            // everything the host decides on is final here (the NIP pass's
            // plan, the fill plan, the sample, the status): its copy goes
            // ahead of the scatter, which then overlaps the host's wait
            B200_STEP_R(mirror_start(h, stream, s));
            mirror_pending = true;
            B200_STEP_R(timed(h, "nip_fill_scatter", 2, -1, m, stream, [&](cudaStream_t ss) {
                return launch_bin_scatter(off, m, s.hist2, s.cta_sum, s.bins2, s.plan2, ladh, true,
                                          ss, dlad, true);
            }));
            return SPGEMM_OK;
        }
        if (!off_written) {
            B200_STEP_R(regrow(h, &h->slots, &h->slots_bytes, sizeof(int32_t) * (size_t(m) + 1),
                               stream));
            off = static_cast<int32_t*>(h->slots);
            B200_TRY(cudaMemcpyAsync(off, c_rpt, sizeof(int32_t) * size_t(m),
                                     cudaMemcpyDeviceToDevice, stream));
            off_written = true;
        }
        if (sampled) B200_TRY(cudaStreamWaitEvent(stream, h->ev_sample, 0));
        B200_STEP_R(timed(h, "nip_fill_hist", 2, -1, m, stream, [&](cudaStream_t ss) {
            return launch_nnz_hist(off, m, s.hist2, s.cta_sum, s.plan2, ladh, ss, dlad);
        }));
        B200_STEP_R(timed(h, "nip_fill_offsets", 2, -1, m, stream, [&](cudaStream_t ss) {
            return launch_bin_offsets(s.hist2, nctas, s.cta_sum, s.plan2, ladh, ss);
        }));
        B200_STEP_R(timed(h, "nip_fill_scatter", 2, -1, m, stream, [&](cudaStream_t ss) {
            return launch_bin_scatter(off, m, s.hist2, s.cta_sum, s.bins2, s.plan2, ladh, true, ss,
                                      dlad);
        }));
        return SPGEMM_OK;
    };
    // The count binning by NIP (the two-pass path's).
    auto count_binning = [&]() -> spgemm_status {
        B200_STEP_R(timed(h, "bin_offsets", 0, -1, m, stream, [&](cudaStream_t ss) {
            return launch_bin_offsets(s.hist1, nctas, nullptr, s.plan1, lad1, ss);
        }));
        B200_STEP_R(timed(h, "bin_scatter", 0, -1, m, stream, [&](cudaStream_t ss) {
            return launch_bin_scatter(c_rpt, m, s.hist1, nullptr, s.bins1, s.plan1, lad1, false,
                                      ss);
        }));
        return SPGEMM_OK;
    };
    if (early) {
        B200_STEP(fill_binning());
    } else {
        B200_STEP(count_binning());
    }
    mark(0);
    if (mirror_pending) {
        B200_STEP(mirror_finish(h, s.plan1, s, early && sampled, early ? s.plan2 : nullptr));
    } else {
        B200_STEP(sync_mirror(h, stream, s.plan1, s, early && sampled, early ? s.plan2 : nullptr));
    }
    mark(1);
    B200_STEP(status_to_error(h->mirror->status));
    Plan p1 = h->mirror->plan;  // bin sizes valid once the count binning ran
    h->info.nip = p1.total_key;
    h->info.max_row_nip = p1.max_key;
    bool counted = !early;
    if (counted)
        for (int b = 0; b < nsym && b < 16; b++) h->info.sym_bin_rows[b] = p1.bin_size[b];

    ProductArgs pa = {};
    pa.a_rpt = A->rpt;
    pa.a_col = A->col;
    pa.a_val = A->val;
    pa.b_rpt = B->rpt;
    pa.b_col = B->col;
    pa.b_val = B->val;
    pa.n_cols = n;
    pa.c_rpt = c_rpt;
    pa.status = s.status;
    pa.cluster = h->cluster;
    pa.fail_rows = s.fail_rows;
    pa.fail_count = s.fail_count;
    pa.words = (static_cast<int64_t>(n) + 31) / 32;
    pa.sm_count = h->sm_count;
    pa.work = s.work;

    // ---- one-pass fill: no count phase ------------------------------------
    // Rows are binned by NIP (an upper bound of their nnz) on the fill ladder
    // and filled into NIP-sized slots of temporary arrays; each fill kernel
    // records its row's exact nnz in C.rpt, which a scan turns into the row
    // pointer, and the rows are then compacted into C.  That replaces the count
    // kernels, the scan binning and their second pass over every product with
    // one copy of C, at the price of temporaries of NIP entries.  Plans keep
    // the two-pass path (their graph replays the fill alone).
    //
    // In auto mode a compression sample taken beside the fill binning can
    // still send the product to two passes (rows above the team bins that
    // repeat many columns); the binning by NIP is then the only work lost.
    const int64_t nip_total = p1.total_key;
    const bool one_pass =
        cr == nullptr && h->one_pass != 2 && nip_total <= INT32_MAX &&
        (h->one_pass == 1 ||
         (nip_total >= kOnePassMinNip &&
          static_cast<uint64_t>(nip_total) * (4 + sizeof(V)) <= kOnePassMaxBytes));
    h->info.one_pass = one_pass ? 1 : 0;
    if (one_pass) {
        int32_t* tmp_col = nullptr;
        void* tmp_val = nullptr;
        auto release = [&]() {};
#define B200_ONE(expr)                                                   \
    do {                                                                 \
        spgemm_status st_ = (expr);                                      \
        if (st_ != SPGEMM_OK) {                                          \
            release();                                                   \
            return bail(st_);                                            \
        }                                                                \
    } while (0)
#define B200_ONE_CUDA(expr, what)                                        \
    do {                                                                 \
        cudaError_t e_ = (expr);                                         \
        if (e_ != cudaSuccess) {                                         \
            release();                                                   \
            return bail(cuda_fail(e_, what));                            \
        }                                                                \
    } while (0)
        // B.n <= 2^20: fill bins may expand, sort and compress instead of
        // hashing (same limits, so the binning does not depend on it)
        BinLauncher one_fil[16];
        for (int b = 0; b < nfil && b < 16; b++) one_fil[b] = fil[b];
        const bool esc_ok = esc_mode != 2;
        const bool esc_sampled = esc_mode == 0;  // by the sample, if it ran
        if (!early) {
            B200_ONE(fill_binning());
            mark(2);
            B200_ONE(sync_mirror(h, stream, s.plan2, s, sampled, s.plan2));
        }
        mark(3);
        B200_ONE(status_to_error(h->mirror->status));
        const Plan pf = h->mirror->plan_b;
        const EscSample es = h->mirror->sample;
        // sampled: the NIP of rows above the team bins, the team bins' NIP/nnz
        int64_t team_nip = 0;
        int64_t team_nnz = 0;
        for (int b = 0; b < kEscBins; b++) {
            team_nip += es.nip[b];
            team_nnz += es.nnz[b];
        }
        const bool wide_rows_compress =
            sampled && es.nip_seen > 0 && team_nnz > 0 &&
            static_cast<double>(es.nip_above) >=
                kTwoPassMinShare * static_cast<double>(es.nip_seen) &&
            static_cast<double>(team_nip) >= kTwoPassMinRatio * static_cast<double>(team_nnz);
        if (h->one_pass == 0 && wide_rows_compress) {
            // two passes after all: C.rpt still holds the NIP per row
            h->info.one_pass = 0;
        } else {
        // NIP-sized temporaries: tmp_col (NIP + 4 columns: a row's tail never
        // leaves the buffer) and tmp_val (NIP values), 256-byte aligned
        {
            const size_t o_val = align_up(sizeof(int32_t) * size_t(nip_total) + 16, 256);
            const size_t need = o_val + sizeof(V) * size_t(nip_total);
            B200_ONE(regrow(h, &h->onepass, &h->onepass_bytes, need, stream));
            char* base = static_cast<char*>(h->onepass);
            tmp_col = reinterpret_cast<int32_t*>(base);
            tmp_val = base + o_val;
        }
        // C.rpt receives each row's exact nnz from the fill kernel of its bin;
        // a row without products keeps the NIP of 0 the NIP pass wrote there
        // (and the scan writes C.rpt[m])
        if (esc_ok) {
            const BinLauncher* esc = nullptr;
            const int nesc = sizeof(V) == 8 ? s2n_esc_ladder_f64(&esc) : s2n_esc_ladder_f32(&esc);
            // the largest team bin and the 256-thread bin follow the device's
            // decision (which also moved the split of their limits)
            const bool split = esc_mode == 1 || (sampled && es.split != 0);
            for (int b = 0; b < kEscLadderBins && b < nesc && b < nfil; b++) {
                const bool use =
                    b >= kEscBins - 1
                        ? split
                        : (!esc_sampled || (sampled && es.nnz[b] > 0 &&
                                            static_cast<double>(es.nip[b]) <=
                                                kEscMaxRatio[b] * static_cast<double>(es.nnz[b])));
                if (use) {
                    one_fil[b] = esc[b];
                    // split: the largest team bin holds rows of <= kEscSplit products
                    if (b == kEscBins - 1 && split)
                        one_fil[b] = sizeof(V) == 8 ? *s2n_esc_split_bin_f64()
                                                    : *s2n_esc_split_bin_f32();
                    h->info.esc_mask |= 1 << b;
                }
            }
        }
        for (int b = 0; b < nfil && b < 16; b++) h->info.num_bin_rows[b] = pf.bin_size[b];
        pa.c_rpt = off;
        pa.c_col = tmp_col;
        pa.c_val = tmp_val;
        pa.row_nnz = c_rpt;
        if (const int32_t gr = global_bitmap_rows(fil, nfil, pf, n); gr > 0) {
            int32_t nmaps = 0;
            B200_ONE(ensure_bitmaps(h, pa.words, gr, &nmaps, stream));
            pa.bitmaps = h->bitmaps;
            pa.nmaps = nmaps;
        }
        mark(4);
        B200_ONE(launch_bins(h, one_fil, nfil, 3, pf, s.bins2, pa, stream));
        // row pointer from the counts, into the count binning's plan (reset:
        // its max and overflow only ever grow): one look-back scan -- or, past
        // its tile limit, a one-bin pass of the binning kernels
        B200_ONE_CUDA(cudaMemsetAsync(s.plan1, 0, sizeof(Plan), stream), "reset a plan");
        if (scan1 && !scan_zeroed)
            B200_ONE_CUDA(cudaMemsetAsync(s.scan_state, 0, scan_bytes, stream), "reset the scan");
        if (scan1) {
            B200_ONE(timed(h, "count_scan_rows", 2, -1, m, stream, [&](cudaStream_t ss) {
                return launch_rpt_scan1(c_rpt, m, s.scan_state, s.plan1, s.status, ss);
            }));
        } else {
            Ladder one = {};
            one.nb = 1;
            one.limit[0] = INT32_MAX;
            B200_ONE(timed(h, "count_scan_hist", 2, -1, m, stream, [&](cudaStream_t ss) {
                return launch_nnz_hist(c_rpt, m, s.hist1, s.cta_sum, s.plan1, one, ss);
            }));
            B200_ONE(timed(h, "count_scan_offsets", 2, -1, m, stream, [&](cudaStream_t ss) {
                return launch_bin_offsets(s.hist1, nctas, s.cta_sum, s.plan1, one, ss);
            }));
            B200_ONE(timed(h, "count_scan_scatter", 2, -1, m, stream, [&](cudaStream_t ss) {
                return launch_bin_scatter(c_rpt, m, s.hist1, s.cta_sum, s.bins1, s.plan1, one,
                                          true, ss);
            }));
        }
        mark(5);
        // Products whose sampled rows repeat few columns give C the NIP as
        // its capacity right away, so the compaction follows the scan with
        // no host round trip; a C that turns out more than kCapSlack
        // smaller is copied to arrays of its size after the last
        // synchronisation.  Others size C exactly, from the scan.
        const bool c_by_nip = sampled && team_nnz > 0 &&
                              static_cast<double>(team_nip) <=
                                  kCapSlack * static_cast<double>(team_nnz);
        if (c_by_nip) {
            B200_ONE_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&C->col),
                                                  sizeof(int32_t) * size_t(nip_total) + 16,
                                                  h->pool, stream),
                          "allocate C.col");
            B200_ONE_CUDA(cudaMallocFromPoolAsync(&C->val, sizeof(V) * size_t(nip_total),
                                                  h->pool, stream),
                          "allocate C.val");
            B200_ONE(timed(h, "compact_rows", 3, -1, m, stream, [&](cudaStream_t ss) {
                return launch_compact_rows(off, c_rpt, m, tmp_col, tmp_val, C->col, C->val,
                                           static_cast<int>(sizeof(V)), ss,
                                           static_cast<int32_t>(nip_total));
            }));
            release();
            auto drop_c = [&]() {
                (void)cudaFreeAsync(C->col, stream);
                (void)cudaFreeAsync(C->val, stream);
                C->col = nullptr;
                C->val = nullptr;
            };
            if (spgemm_status st = sync_mirror(h, stream, s.plan1, s); st != SPGEMM_OK)
                return drop_c(), bail(st);
            if (spgemm_status st = status_to_error(h->mirror->status); st != SPGEMM_OK)
                return drop_c(), bail(st);
            const Plan pc = h->mirror->plan;
            if (pc.overflow || pc.total_key > nip_total)
                return drop_c(),
                       bail(fail(SPGEMM_ERR_INTERNAL, "one-pass row counts out of range"));
            const int32_t nnz = static_cast<int32_t>(pc.total_key);
            h->info.nnz = nnz;
            h->info.max_row_nnz = pc.max_key;
            C->nnz = nnz;
            bool resized = false;
            if (nnz == 0) {
                drop_c();
            } else if (static_cast<double>(nnz) * kCapSlack < static_cast<double>(nip_total)) {
                resized = true;
                // more spare capacity than the slack: arrays of C's size
                int32_t* col = nullptr;
                void* val = nullptr;
                cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&col),
                                                        sizeof(int32_t) * size_t(nnz) + 16,
                                                        h->pool, stream);
                if (e == cudaSuccess)
                    e = cudaMallocFromPoolAsync(&val, sizeof(V) * size_t(nnz), h->pool, stream);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(col, C->col, sizeof(int32_t) * size_t(nnz),
                                        cudaMemcpyDeviceToDevice, stream);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(val, C->val, sizeof(V) * size_t(nnz),
                                        cudaMemcpyDeviceToDevice, stream);
                drop_c();
                C->col = col;
                C->val = val;
                if (e != cudaSuccess) {
                    drop_c();
                    return bail(cuda_fail(e, "size C"));
                }
            }
            if (resized) {
                if (cudaError_t e = cudaStreamSynchronize(stream); e != cudaSuccess)
                    return bail(cuda_fail(e, "final synchronize"));
                h->info.host_syncs++;
            }
            mark(6);
            resolve_profile(h);
            return SPGEMM_OK;
        }
        B200_ONE(sync_mirror(h, stream, s.plan1, s));
        B200_ONE(status_to_error(h->mirror->status));
        const Plan pc = h->mirror->plan;
        if (pc.overflow || pc.total_key > nip_total)
            return release(), bail(fail(SPGEMM_ERR_INTERNAL, "one-pass row counts out of range"));
        const int32_t nnz = static_cast<int32_t>(pc.total_key);
        h->info.nnz = nnz;
        h->info.max_row_nnz = pc.max_key;
        C->nnz = nnz;
        if (nnz > 0) {
            B200_ONE_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&C->col),
                                                  sizeof(int32_t) * size_t(nnz) + 16, h->pool,
                                                  stream),
                          "allocate C.col");
            B200_ONE_CUDA(cudaMallocFromPoolAsync(&C->val, sizeof(V) * size_t(nnz), h->pool,
                                                  stream),
                          "allocate C.val");
            B200_ONE(timed(h, "compact_rows", 3, -1, m, stream, [&](cudaStream_t ss) {
                return launch_compact_rows(off, c_rpt, m, tmp_col, tmp_val, C->col, C->val,
                                           static_cast<int>(sizeof(V)), ss, nnz);
            }));
        }
        release();
        if (cudaError_t e = cudaStreamSynchronize(stream); e != cudaSuccess)
            return bail(cuda_fail(e, "final synchronize"));
        mark(6);
        h->info.host_syncs++;
        resolve_profile(h);
        return SPGEMM_OK;
        }
#undef B200_ONE_CUDA
#undef B200_ONE
    }
    if (sampled && h->info.one_pass == 0) {
        // two passes: the sample's work is not needed, but it still reads A
        // and B; the final synchronisation must cover it
        if (cudaError_t e = cudaStreamWaitEvent(stream, h->ev_sample, 0); e != cudaSuccess)
            return bail(cuda_fail(e, "join the sample stream"));
    }
    if (early || one_pass) {
        // the fill binning by NIP ran: its plan is reused by the scan pass
        if (cudaError_t e = cudaMemsetAsync(s.plan2, 0, sizeof(Plan), stream); e != cudaSuccess)
            return bail(cuda_fail(e, "reset a plan"));
    }
    if (!counted) {
        // a product binned early for one pass runs two: its count binning now
        B200_STEP(count_binning());
        B200_STEP(sync_mirror(h, stream, s.plan1, s));
        B200_STEP(status_to_error(h->mirror->status));
        p1 = h->mirror->plan;
        for (int b = 0; b < nsym && b < 16; b++) h->info.sym_bin_rows[b] = p1.bin_size[b];
    }

    // ---- sym1: exact nnz per row --------------------------------------------
    const int glob1 = nsym - 1;  // global bin (cluster spills, or the test knob)
    const int clus1 = nsym - 2;  // cluster bin
    const int32_t cluster_rows = p1.bin_size[clus1];
    const int32_t global_rows = p1.bin_size[glob1];
    if (cluster_rows > 0 || global_rows > 0) {
        int32_t nmaps = 0;
        B200_STEP(ensure_bitmaps(h, pa.words, std::max(cluster_rows, global_rows), &nmaps, stream));
        pa.bitmaps = h->bitmaps;
        pa.nmaps = nmaps;
    }
    // cluster bin, then its spills, then knob-forced global rows: one chain on
    // the first side stream; the other bins round-robin on the rest
    B200_STEP(fork_streams(h, stream));
    {
        cudaStream_t chain = h->side[0];
        if (cluster_rows > 0) {
            ProductArgs a = pa;
            a.rows = s.bins1 + p1.bin_off[clus1];
            a.nrows = cluster_rows;
            B200_STEP(timed(h, sym[clus1].name, 1, clus1, cluster_rows, chain,
                            [&](cudaStream_t ss) { return sym[clus1].launch(a, ss); }));
            // rows that spilled out of the cluster table: their count is only
            // known on the device, so the global kernel runs on a grid of
            // bitmap slots and reads its row count from the device
            ProductArgs f = pa;
            f.rows = s.fail_rows;
            f.nrows = -1;
            B200_STEP(timed(h, "sym1_global_spills", 1, glob1, -1, chain,
                            [&](cudaStream_t ss) { return sym[glob1].launch(f, ss); }));
        }
        if (global_rows > 0) {
            ProductArgs a = pa;
            a.rows = s.bins1 + p1.bin_off[glob1];
            a.nrows = global_rows;
            B200_STEP(timed(h, sym[glob1].name, 1, glob1, global_rows, chain,
                            [&](cudaStream_t ss) { return sym[glob1].launch(a, ss); }));
        }
        const bool chain_used = cluster_rows > 0 || global_rows > 0;
        const int first = chain_used && h->nside > 1 ? 1 : 0;
        int next = first;
        for (int b = clus1 - 1; b >= 0; b--) {
            const int rows = p1.bin_size[b];
            if (rows <= 0) continue;
            ProductArgs a = pa;
            a.rows = s.bins1 + p1.bin_off[b];
            a.nrows = rows;
            B200_STEP(timed(h, sym[b].name, 1, b, rows, h->side[next],
                            [&](cudaStream_t ss) { return sym[b].launch(a, ss); }));
            next = next + 1 < h->nside ? next + 1 : first;
        }
    }
    B200_STEP(join_streams(h, stream));

    // ---- scan pass: row pointer and fill bins -------------------------------
    const Ladder lad2 = scaled_ladder(fil, nfil, h->min_num_bin, cr ? cr->team_scale : 1.0,
                                      cr ? cr->cta_scale : 1.0);
    B200_STEP(timed(h, "nnz_hist", 2, -1, m, stream, [&](cudaStream_t ss) {
        return launch_nnz_hist(c_rpt, m, s.hist2, s.cta_sum, s.plan2, lad2, ss);
    }));
    B200_STEP(timed(h, "scan_offsets", 2, -1, m, stream, [&](cudaStream_t ss) {
        return launch_bin_offsets(s.hist2, nctas, s.cta_sum, s.plan2, lad2, ss);
    }));
    B200_STEP(timed(h, "scan_scatter", 2, -1, m, stream, [&](cudaStream_t ss) {
        return launch_bin_scatter(c_rpt, m, s.hist2, s.cta_sum, s.bins2, s.plan2, lad2, true,
                                  ss);
    }));
    mark(2);
    B200_STEP(sync_mirror(h, stream, s.plan2, s));
    mark(3);
    B200_STEP(status_to_error(h->mirror->status));
    const Plan p2 = h->mirror->plan;
    h->info.sym_fail_rows = h->mirror->fail_count;
    if (p2.overflow)
        return bail(fail(SPGEMM_ERR_OVERFLOW,
                         "nnz(C) = " + std::to_string(p2.total_key) + " exceeds int32"));
    const int32_t nnz = static_cast<int32_t>(p2.total_key);
    h->info.nnz = nnz;
    h->info.max_row_nnz = p2.max_key;
    for (int b = 0; b < nfil && b < 16; b++) h->info.num_bin_rows[b] = p2.bin_size[b];
    C->nnz = nnz;
    if (nnz == 0) {
        resolve_profile(h);
        return SPGEMM_OK;
    }

    // ---- fill + sort + numeric ----------------------------------------------
    // C.col gets 16 bytes of tail padding so 16-byte-granular staging of a
    // row's tail never leaves the allocation
    if (cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&C->col),
                                                sizeof(int32_t) * size_t(nnz) + 16, h->pool,
                                                stream);
        e != cudaSuccess)
        return bail(cuda_fail(e, "allocate C.col"));
    if (cudaError_t e = cudaMallocFromPoolAsync(&C->val, sizeof(V) * size_t(nnz), h->pool, stream);
        e != cudaSuccess)
        return bail(cuda_fail(e, "allocate C.val"));
    pa.c_col = C->col;
    pa.c_val = C->val;
    if (const int32_t gr = global_bitmap_rows(fil, nfil, p2, n); gr > 0) {
        int32_t nmaps = 0;
        B200_STEP(ensure_bitmaps(h, pa.words, gr, &nmaps, stream));
        pa.bitmaps = h->bitmaps;
        pa.nmaps = nmaps;
    }
    mark(4);
    DevStatus* fill_status = s.status;
    if (cr != nullptr && cr->plan != nullptr) {
        // the graph reads copies the plan owns: later products reuse the
        // handle's scratch and bitmaps
        spgemm_plan_s* plan = cr->plan;
        int32_t* bins = nullptr;
        B200_STEP(plan_alloc(plan, reinterpret_cast<void**>(&bins), sizeof(int32_t) * size_t(m),
                             stream));
        if (cudaError_t e = cudaMemcpyAsync(bins, s.bins2, sizeof(int32_t) * size_t(m),
                                            cudaMemcpyDeviceToDevice, stream);
            e != cudaSuccess)
            return bail(cuda_fail(e, "copy fill bins"));
        if (pa.bitmaps != nullptr) {
            void* bm = nullptr;
            B200_STEP(plan_alloc(plan, &bm, sizeof(uint32_t) * size_t(pa.words) * size_t(pa.nmaps),
                                 stream));
            pa.bitmaps = static_cast<uint32_t*>(bm);
        }
        int32_t* work = nullptr;  // the persistent bins' row counters
        B200_STEP(plan_alloc(plan, reinterpret_cast<void**>(&work), sizeof(int32_t) * kMaxBins,
                             stream));
        pa.work = work;
        pa.status = plan->status;
        fill_status = plan->status;
        const int saved_profile = h->profile;
        h->profile = 0;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(plan->capture, cudaStreamCaptureModeThreadLocal);
        spgemm_status st = e == cudaSuccess
                               ? launch_bins(h, fil, nfil, 3, p2, bins, pa, plan->capture)
                               : cuda_fail(e, "begin capture");
        const cudaError_t ee = cudaStreamEndCapture(plan->capture, &g);
        h->profile = saved_profile;
        if (st != SPGEMM_OK) {
            if (g) cudaGraphDestroy(g);
            return bail(st);
        }
        if (ee != cudaSuccess) return bail(cuda_fail(ee, "end capture"));
        if (cr->launch_now) {
            plan->graph = g;
            if (cudaError_t e2 = cudaGraphInstantiate(&plan->exec, g, 0); e2 != cudaSuccess)
                return bail(cuda_fail(e2, "instantiate the fill graph"));
            if (cudaError_t e2 = cudaGraphLaunch(plan->exec, stream); e2 != cudaSuccess)
                return bail(cuda_fail(e2, "launch the fill graph"));
        } else {
            cr->graph = g;
        }
    } else {
        B200_STEP(launch_bins(h, fil, nfil, 3, p2, s.bins2, pa, stream));
    }
    mark(5);
    if (cudaError_t e = cudaMemcpyAsync(&h->mirror->status, fill_status, sizeof(DevStatus),
                                        cudaMemcpyDeviceToHost, stream);
        e != cudaSuccess)
        return bail(cuda_fail(e, "read status"));
    if (cudaError_t e = cudaStreamSynchronize(stream); e != cudaSuccess)
        return bail(cuda_fail(e, "final synchronize"));
    mark(6);
    h->info.host_syncs++;
    B200_STEP(status_to_error(h->mirror->status));
    resolve_profile(h);
#undef B200_STEP
    return SPGEMM_OK;
}

// ---- batched products -------------------------------------------------------
// C_i = A_i * B_i for every product of a block-diagonal batch: the products
// are grouped so that each group's intermediate products (an upper bound of its
// nnz) stay below 2^31, and each group runs as ONE product of the row range of
// the packed operands -- its rows share bins, kernels and side streams.  A
// split kernel then gives every product its own row pointer (from 0) and local
// column indices, as views into the group's arrays.
template<typename V>
spgemm_status batch(spgemm_handle_s* h, const spgemm_batch_desc* d, const spgemm_csr_view* A,
                    const spgemm_csr_view* B, spgemm_batch_out* out, cudaStream_t stream,
                    spgemm_plan_s* plan = nullptr, double team_scale = 1.0,
                    double cta_scale = 1.0) {
    if (h == nullptr || d == nullptr || out == nullptr)
        return fail(SPGEMM_ERR_INVALID_ARG, "NULL argument");
    std::memset(out, 0, sizeof(*out));
    if (spgemm_status st = check_view(A, "A"); st != SPGEMM_OK) return st;
    if (spgemm_status st = check_view(B, "B"); st != SPGEMM_OK) return st;
    const int32_t count = d->count;
    if (count < 0) return fail(SPGEMM_ERR_INVALID_ARG, "negative batch count");
    if (count == 0) return SPGEMM_OK;
    if (d->a_row_off == nullptr || d->b_row_off == nullptr || d->c_col_off == nullptr)
        return fail(SPGEMM_ERR_INVALID_ARG, "NULL batch offset array");
    if (A->n != B->m) return fail(SPGEMM_ERR_INVALID_ARG, "A.n must equal B.m");
    if (d->a_row_off[0] != 0 || d->b_row_off[0] != 0 || d->c_col_off[0] != 0 ||
        d->a_row_off[count] != A->m || d->b_row_off[count] != B->m ||
        d->c_col_off[count] != B->n)
        return fail(SPGEMM_ERR_INVALID_ARG,
                    "batch offsets must start at 0 and end at A.m, B.m and B.n");
    for (int i = 0; i < count; i++)
        if (d->a_row_off[i + 1] < d->a_row_off[i] || d->b_row_off[i + 1] < d->b_row_off[i] ||
            d->c_col_off[i + 1] < d->c_col_off[i])
            return fail(SPGEMM_ERR_INVALID_ARG, "batch offsets must be non-decreasing");
    B200_TRY(cudaSetDevice(h->device));

    // per-product output row-pointer offsets: product i starts at a_row_off[i] + i
    std::vector<int64_t> out_off(count + 1);
    for (int i = 0; i <= count; i++) out_off[i] = int64_t(d->a_row_off[i]) + i;

    // device copies of the offsets, the per-product NIP, and the split results
    const size_t nb_row = sizeof(int32_t) * (size_t(count) + 1);
    const size_t nb_off = sizeof(int64_t) * (size_t(count) + 1);
    const size_t nb_nip = sizeof(long long) * size_t(count);
    const size_t nb_pos = sizeof(int32_t) * 2 * size_t(count);
    const size_t o_row = 0;
    const size_t o_col = align_up(o_row + nb_row, 256);
    const size_t o_off = align_up(o_col + nb_row, 256);
    const size_t o_nip = align_up(o_off + nb_off, 256);
    const size_t o_pos = align_up(o_nip + nb_nip, 256);
    const size_t total = align_up(o_pos + nb_pos, 256);
    char* dbuf = nullptr;
    B200_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&dbuf), total, h->pool, stream));
    // a plan's graph reads the offsets and writes the positions at every run
    auto release = [&]() {
        if (plan == nullptr) cudaFreeAsync(dbuf, stream);
    };
    if (plan != nullptr) plan->owned.push_back(dbuf);
    int32_t* d_row = reinterpret_cast<int32_t*>(dbuf + o_row);
    int32_t* d_col = reinterpret_cast<int32_t*>(dbuf + o_col);
    int64_t* d_off = reinterpret_cast<int64_t*>(dbuf + o_off);
    long long* d_nip = reinterpret_cast<long long*>(dbuf + o_nip);
    int32_t* d_pos = reinterpret_cast<int32_t*>(dbuf + o_pos);
    std::vector<long long> nip(count);
    cudaError_t e = cudaMemcpyAsync(d_row, d->a_row_off, nb_row, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_col, d->c_col_off, nb_row, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_off, out_off.data(), nb_off, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = launch_product_nip(A->rpt, A->col, B->rpt, d_row, count, d_nip, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(nip.data(), d_nip, nb_nip, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "batch planning");
    }

    // the per-product row pointers of all products share one allocation
    int32_t* rpt_out = nullptr;
    e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&rpt_out),
                                sizeof(int32_t) * size_t(out_off[count]), h->pool, stream);
    if (e != cudaSuccess) {
        release();
        return cuda_fail(e, "allocate batch row pointers");
    }
    std::vector<void*> blocks{rpt_out};
    std::vector<spgemm_csr_out> prods(count);
    auto unwind = [&](spgemm_status st) {
        const std::string msg = g_last_error;
        for (void* b : blocks) cudaFreeAsync(b, stream);
        release();
        cudaStreamSynchronize(stream);
        g_last_error = msg;
        return st;
    };

    const int saved_checked = h->checked;
    h->checked = 0;  // group views start mid-matrix; the packed operands are checked once
    if (saved_checked) {
        Scratch sc;
        if (spgemm_status st = ensure_scratch(h, std::max(A->m, B->m), &sc, stream); st != SPGEMM_OK) {
            h->checked = saved_checked;
            return unwind(st);
        }
        cudaMemsetAsync(sc.status, 0, sizeof(DevStatus), stream);
        e = launch_check_csr(A->rpt, A->col, A->m, A->n, A->nnz, sc.status, stream);
        if (e == cudaSuccess) e = launch_check_csr(B->rpt, B->col, B->m, B->n, B->nnz, sc.status, stream);
        spgemm_status st = e == cudaSuccess ? sync_mirror(h, stream, sc.plan1, sc) : cuda_fail(e, "check");
        if (st == SPGEMM_OK) st = status_to_error(h->mirror->status);
        if (st != SPGEMM_OK) {
            h->checked = saved_checked;
            return unwind(st);
        }
    }

    constexpr long long kGroupLimit = INT32_MAX;
    int32_t groups = 0;
    std::vector<std::pair<cudaGraph_t, cudaGraph_t>> group_graphs;  // plan: (fill, split)
    spgemm_info acc = {};
    for (int p0 = 0; p0 < count;) {
        long long sum = 0;
        int p1 = p0;
        while (p1 < count && (p1 == p0 || sum + nip[p1] <= kGroupLimit)) sum += nip[p1++];
        const int32_t r0 = d->a_row_off[p0];
        const int32_t r1 = d->a_row_off[p1];
        spgemm_csr_view Ag = *A;
        Ag.m = r1 - r0;
        Ag.rpt = A->rpt + r0;
        spgemm_csr_out Cg;
        CaptureReq cr;
        cr.team_scale = team_scale;
        cr.cta_scale = cta_scale;
        cr.plan = plan;
        cr.launch_now = false;
        // every group runs the two-pass path (a plan captures its fill; a plain
        // batch measured no faster through the one-pass path, 4,096 products
        // 472 vs 474 ms, and the served loop's batches slower)
        spgemm_status st = product<V>(h, &Ag, B, &Cg, stream, &cr);
        if (st != SPGEMM_OK) {
            h->checked = saved_checked;
            return unwind(st);
        }
        groups++;
        acc.nip += h->info.nip;
        acc.nnz += h->info.nnz;
        acc.host_syncs += h->info.host_syncs;
        acc.max_row_nip = std::max(acc.max_row_nip, h->info.max_row_nip);
        acc.max_row_nnz = std::max(acc.max_row_nnz, h->info.max_row_nnz);
        for (int b = 0; b < 16; b++) {
            acc.sym_bin_rows[b] += h->info.sym_bin_rows[b];
            acc.num_bin_rows[b] += h->info.num_bin_rows[b];
        }
        if (Cg.col) blocks.push_back(Cg.col);
        if (Cg.val) blocks.push_back(Cg.val);
        if (plan == nullptr) {
            e = launch_unpack(Cg.rpt, Cg.col, d_row, d_col, d_off, p0, p1 - p0, rpt_out, d_pos,
                              stream);
            if (e == cudaSuccess) e = cudaFreeAsync(Cg.rpt, stream);  // split copies what it needs
        } else {
            // the group's fill graph, then its split, as two nodes of the plan
            plan->owned.push_back(Cg.rpt);  // the split reads it at every run
            cudaGraph_t split = nullptr;
            e = cudaStreamBeginCapture(plan->capture, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess)
                e = launch_unpack(Cg.rpt, Cg.col, d_row, d_col, d_off, p0, p1 - p0, rpt_out,
                                  d_pos, plan->capture);
            const cudaError_t ee = cudaStreamEndCapture(plan->capture, &split);
            if (e == cudaSuccess) e = ee;
            if (e == cudaSuccess) {
                group_graphs.emplace_back(cr.graph, split);  // no fill graph when nnz = 0
                if (cr.graph) plan->children.push_back(cr.graph);
                plan->children.push_back(split);
            } else {
                if (cr.graph) cudaGraphDestroy(cr.graph);
                if (split) cudaGraphDestroy(split);
            }
        }
        if (e != cudaSuccess) {
            h->checked = saved_checked;
            return unwind(cuda_fail(e, "batch split"));
        }
        for (int i = p0; i < p1; i++) {
            prods[i].m = d->a_row_off[i + 1] - d->a_row_off[i];
            prods[i].n = d->c_col_off[i + 1] - d->c_col_off[i];
            prods[i].rpt = rpt_out + out_off[i];
            prods[i].col = Cg.col;  // offset added once the positions are back
            prods[i].val = Cg.val;
        }
        p0 = p1;
    }
    h->checked = saved_checked;
    if (plan != nullptr) {
        // one parent graph: per group, fill then split; groups are independent
        e = cudaGraphCreate(&plan->graph, 0);
        for (size_t i = 0; e == cudaSuccess && i < group_graphs.size(); i++) {
            cudaGraphNode_t fill = nullptr;
            cudaGraphNode_t split = nullptr;
            if (group_graphs[i].first != nullptr)
                e = cudaGraphAddChildGraphNode(&fill, plan->graph, nullptr, 0,
                                               group_graphs[i].first);
            if (e == cudaSuccess)
                e = cudaGraphAddChildGraphNode(&split, plan->graph, fill ? &fill : nullptr,
                                               fill ? 1 : 0, group_graphs[i].second);
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&plan->exec, plan->graph, 0);
        if (e == cudaSuccess) e = cudaGraphLaunch(plan->exec, stream);
        if (e != cudaSuccess) return unwind(cuda_fail(e, "batch plan graph"));
    }
    std::vector<int32_t> pos(2 * size_t(count));
    e = cudaMemcpyAsync(pos.data(), d_pos, nb_pos, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return unwind(cuda_fail(e, "batch positions"));
    for (int i = 0; i < count; i++) {
        prods[i].nnz = pos[2 * i + 1];
        if (prods[i].col) {
            prods[i].col += pos[2 * i];
            prods[i].val = static_cast<V*>(prods[i].val) + pos[2 * i];
        }
        if (prods[i].nnz == 0) {
            prods[i].col = nullptr;
            prods[i].val = nullptr;
        }
    }
    release();
    acc.n_sym_bins = h->info.n_sym_bins;
    acc.n_num_bins = h->info.n_num_bins;
    h->info = acc;
    out->count = count;
    out->products = static_cast<spgemm_csr_out*>(std::malloc(sizeof(spgemm_csr_out) * count));
    out->blocks = static_cast<void**>(std::malloc(sizeof(void*) * blocks.size()));
    if (out->products == nullptr || out->blocks == nullptr) {
        std::free(out->products);
        std::free(out->blocks);
        std::memset(out, 0, sizeof(*out));
        return unwind(fail(SPGEMM_ERR_OOM, "host allocation of the batch result"));
    }
    std::memcpy(out->products, prods.data(), sizeof(spgemm_csr_out) * count);
    std::memcpy(out->blocks, blocks.data(), sizeof(void*) * blocks.size());
    out->n_blocks = static_cast<int32_t>(blocks.size());
    out->n_groups = groups;
    return SPGEMM_OK;
}

// Page-locked host blocks for host results, reused across calls (process
// wide, so spgemm_host_csr_free needs no handle).  A result's three arrays
// share one block; freeing the result returns the block to the pool.
struct PinnedBlock {
    void* p;
    size_t bytes;
    bool used;
};
std::mutex g_pin_mu;
std::vector<PinnedBlock> g_pin;

void* pinned_take(size_t bytes) {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    PinnedBlock* best = nullptr;
    for (PinnedBlock& b : g_pin)
        if (!b.used && b.bytes >= bytes && (best == nullptr || b.bytes < best->bytes)) best = &b;
    if (best != nullptr) {
        best->used = true;
        return best->p;
    }
    const size_t rounded = align_up(bytes + bytes / 8, size_t(2) << 20);
    void* p = nullptr;
    if (cudaMallocHost(&p, rounded) != cudaSuccess) return nullptr;
    g_pin.push_back(PinnedBlock{p, rounded, true});
    return p;
}

bool pinned_give_back(void* p) {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    for (PinnedBlock& b : g_pin) {
        if (b.p == p) {
            b.used = false;
            return true;
        }
    }
    return false;
}

template<typename V>
spgemm_status product_host(spgemm_handle_s* h, const spgemm_csr_view* A,
                           const spgemm_csr_view* B, spgemm_csr_out* C, cudaStream_t stream) {
    if (h == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "handle is NULL");
    if (C == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "C is NULL");
    if (spgemm_status st = check_view(A, "A"); st != SPGEMM_OK) return st;
    if (spgemm_status st = check_view(B, "B"); st != SPGEMM_OK) return st;
    B200_TRY(cudaSetDevice(h->device));
    auto bytes_of = [](const spgemm_csr_view* v) {
        return align_up(sizeof(int32_t) * (size_t(v->m) + 1), 256) +
               align_up(sizeof(int32_t) * size_t(v->nnz), 256) +
               align_up(sizeof(V) * size_t(v->nnz), 256);
    };
    // C = A * A with one host matrix (the same arrays passed twice): copy it
    // to the device once
    const bool same = A->m == B->m && A->n == B->n && A->nnz == B->nnz && A->rpt == B->rpt &&
                      A->col == B->col && A->val == B->val;
    const size_t need = bytes_of(A) + (same ? 0 : bytes_of(B));
    if (spgemm_status st = regrow(h, &h->in_buf, &h->in_bytes, need, stream); st != SPGEMM_OK)
        return st;
    char* p = static_cast<char*>(h->in_buf);
    auto upload = [&](const spgemm_csr_view* v, spgemm_csr_view* d) -> cudaError_t {
        *d = *v;
        int32_t* rpt = reinterpret_cast<int32_t*>(p);
        p += align_up(sizeof(int32_t) * (size_t(v->m) + 1), 256);
        int32_t* col = reinterpret_cast<int32_t*>(p);
        p += align_up(sizeof(int32_t) * size_t(v->nnz), 256);
        V* val = reinterpret_cast<V*>(p);
        p += align_up(sizeof(V) * size_t(v->nnz), 256);
        cudaError_t e = cudaMemcpyAsync(rpt, v->rpt, sizeof(int32_t) * (size_t(v->m) + 1),
                                        cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess && v->nnz > 0)
            e = cudaMemcpyAsync(col, v->col, sizeof(int32_t) * size_t(v->nnz),
                                cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess && v->nnz > 0)
            e = cudaMemcpyAsync(val, v->val, sizeof(V) * size_t(v->nnz), cudaMemcpyHostToDevice,
                                stream);
        d->rpt = rpt;
        d->col = col;
        d->val = val;
        return e;
    };
    spgemm_csr_view dA, dB;
    B200_TRY(upload(A, &dA));
    if (same)
        dB = dA;
    else
        B200_TRY(upload(B, &dB));
    spgemm_csr_out dC;
    if (spgemm_status st = product<V>(h, &dA, &dB, &dC, stream); st != SPGEMM_OK) return st;
    std::memset(C, 0, sizeof(*C));
    C->m = dC.m;
    C->n = dC.n;
    C->nnz = dC.nnz;
    const size_t rpt_b = align_up(sizeof(int32_t) * (size_t(dC.m) + 1), 256);
    const size_t col_b = align_up(sizeof(int32_t) * std::max<size_t>(dC.nnz, 1), 256);
    const size_t val_b = align_up(sizeof(V) * std::max<size_t>(dC.nnz, 1), 256);
    char* blk = static_cast<char*>(pinned_take(rpt_b + col_b + val_b));
    if (blk == nullptr) {
        std::memset(C, 0, sizeof(*C));
        spgemm_csr_free(&dC, stream);
        return fail(SPGEMM_ERR_OOM, "page-locked host allocation of C failed");
    }
    C->rpt = reinterpret_cast<int32_t*>(blk);
    C->col = reinterpret_cast<int32_t*>(blk + rpt_b);
    C->val = blk + rpt_b + col_b;
    cudaError_t e = cudaMemcpyAsync(C->rpt, dC.rpt, sizeof(int32_t) * (size_t(dC.m) + 1),
                                    cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && dC.nnz > 0)
        e = cudaMemcpyAsync(C->col, dC.col, sizeof(int32_t) * size_t(dC.nnz),
                            cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && dC.nnz > 0)
        e = cudaMemcpyAsync(C->val, dC.val, sizeof(V) * size_t(dC.nnz), cudaMemcpyDeviceToHost,
                            stream);
    spgemm_csr_free(&dC, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        spgemm_host_csr_free(C);
        return cuda_fail(e, "copy C to host");
    }
    return SPGEMM_OK;
}

// ---- CSR transpose -----------------------------------------------------------
// T = A^T with sorted columns (k_transpose.cu): column counts, the binning pass
// with the scan (T.rpt and length bins of T's rows), a keyed scatter, then one
// sort kernel per non-empty length bin.  One host synchronisation (the bin
// sizes), like each binning pass of a product.
template<typename V>
spgemm_status transpose(spgemm_handle_s* h, const spgemm_csr_view* A, spgemm_csr_out* T,
                        cudaStream_t stream) {
    if (h == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "handle is NULL");
    if (T == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "T is NULL");
    if (spgemm_status st = check_view(A, "A"); st != SPGEMM_OK) return st;
    std::memset(T, 0, sizeof(*T));
    h->info = spgemm_info{};
    h->prof.clear();
    h->prof_done.clear();
    B200_TRY(cudaSetDevice(h->device));
    const int32_t m = A->m;
    const int32_t n = A->n;
    const int32_t nnz = A->nnz;
    T->m = n;
    T->n = m;
    const BinLauncher* tl = nullptr;
    const int ntl = sizeof(V) == 8 ? transpose_ladder_f64(&tl) : transpose_ladder_f32(&tl);
    h->info.n_num_bins = ntl;
    B200_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&T->rpt),
                                     sizeof(int32_t) * (size_t(n) + 1), h->pool, stream));
    uint64_t* keys = nullptr;
    int32_t* cursor = nullptr;
    auto bail = [&](spgemm_status st) {
        const std::string msg = g_last_error;
        cudaStreamSynchronize(stream);
        if (keys) cudaFreeAsync(keys, stream);
        if (cursor) cudaFreeAsync(cursor, stream);
        spgemm_csr_free(T, stream);
        cudaStreamSynchronize(stream);
        h->prof.clear();
        g_last_error = msg;
        return st;
    };
#define B200_STEP(expr)                                                  \
    do {                                                                 \
        spgemm_status st_ = (expr);                                      \
        if (st_ != SPGEMM_OK) return bail(st_);                          \
    } while (0)
#define B200_CUDA(expr, what)                                            \
    do {                                                                 \
        cudaError_t e_ = (expr);                                         \
        if (e_ != cudaSuccess) return bail(cuda_fail(e_, what));         \
    } while (0)
    Scratch s;
    B200_STEP(ensure_scratch(h, n, &s, stream));
    B200_CUDA(cudaMemsetAsync(h->scratch, 0,
                              reinterpret_cast<char*>(s.hist1) - static_cast<char*>(h->scratch),
                              stream),
              "memset scratch");
    if (h->checked) {
        B200_STEP(timed(h, "check_csr_A", 0, -1, m, stream, [&](cudaStream_t ss) {
            return launch_check_csr(A->rpt, A->col, m, n, nnz, s.status, ss);
        }));
        B200_STEP(sync_mirror(h, stream, s.plan1, s));
        B200_STEP(status_to_error(h->mirror->status));
    }
    B200_CUDA(cudaMemsetAsync(T->rpt, 0, sizeof(int32_t) * (size_t(n) + 1), stream),
              "memset T.rpt");
    if (nnz == 0 || n == 0) {
        B200_CUDA(cudaStreamSynchronize(stream), "synchronize");
        return SPGEMM_OK;
    }
    B200_STEP(timed(h, "col_count", 1, -1, nnz, stream, [&](cudaStream_t ss) {
        return launch_col_count(A->col, nnz, n, T->rpt, ss);
    }));
    const Ladder lad = make_ladder(tl, ntl, h->min_tr_bin);
    const int nctas = bin_ctas(n);
    B200_STEP(timed(h, "tr_hist", 2, -1, n, stream, [&](cudaStream_t ss) {
        return launch_nnz_hist(T->rpt, n, s.hist2, s.cta_sum, s.plan2, lad, ss);
    }));
    B200_STEP(timed(h, "tr_offsets", 2, -1, n, stream, [&](cudaStream_t ss) {
        return launch_bin_offsets(s.hist2, nctas, s.cta_sum, s.plan2, lad, ss);
    }));
    B200_STEP(timed(h, "tr_scan_scatter", 2, -1, n, stream, [&](cudaStream_t ss) {
        return launch_bin_scatter(T->rpt, n, s.hist2, s.cta_sum, s.bins2, s.plan2, lad, true,
                                  ss);
    }));
    B200_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&keys),
                                      sizeof(uint64_t) * size_t(nnz), h->pool, stream),
              "allocate transpose keys");
    B200_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&cursor),
                                      sizeof(int32_t) * size_t(n), h->pool, stream),
              "allocate transpose cursors");
    B200_CUDA(cudaMemsetAsync(cursor, 0, sizeof(int32_t) * size_t(n), stream), "memset cursors");
    B200_STEP(timed(h, "tr_scatter", 3, -1, m, stream, [&](cudaStream_t ss) {
        return launch_tr_scatter(A->rpt, A->col, m, n, T->rpt, cursor, keys, ss);
    }));
    B200_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&T->col),
                                      sizeof(int32_t) * size_t(nnz) + 16, h->pool, stream),
              "allocate T.col");
    B200_CUDA(cudaMallocFromPoolAsync(&T->val, sizeof(V) * size_t(nnz), h->pool, stream),
              "allocate T.val");
    T->nnz = nnz;
    B200_STEP(sync_mirror(h, stream, s.plan2, s));
    B200_STEP(status_to_error(h->mirror->status));
    const Plan plan = h->mirror->plan;
    if (plan.total_key != nnz)
        return bail(fail(SPGEMM_ERR_INVALID_ARG, "A.col holds a column index outside [0, A.n)"));
    h->info.nnz = nnz;
    h->info.max_row_nnz = plan.max_key;
    for (int b = 0; b < ntl && b < 16; b++) h->info.num_bin_rows[b] = plan.bin_size[b];
    ProductArgs pa = {};
    pa.a_val = A->val;
    pa.c_rpt = T->rpt;
    pa.c_col = T->col;
    pa.c_val = T->val;
    pa.status = s.status;
    pa.keys = keys;
    B200_STEP(launch_bins(h, tl, ntl, 4, plan, s.bins2, pa, stream));
    B200_CUDA(cudaFreeAsync(keys, stream), "free transpose keys");
    keys = nullptr;
    B200_CUDA(cudaFreeAsync(cursor, stream), "free transpose cursors");
    cursor = nullptr;
    B200_CUDA(cudaMemcpyAsync(&h->mirror->status, s.status, sizeof(DevStatus),
                              cudaMemcpyDeviceToHost, stream),
              "read status");
    B200_CUDA(cudaStreamSynchronize(stream), "final synchronize");
    h->info.host_syncs++;
    B200_STEP(status_to_error(h->mirror->status));
    resolve_profile(h);
#undef B200_CUDA
#undef B200_STEP
    return SPGEMM_OK;
}

spgemm_csr_view view_of(const spgemm_csr_out& c) {
    spgemm_csr_view v;
    v.m = c.m;
    v.n = c.n;
    v.nnz = c.nnz;
    v.rpt = c.rpt;
    v.col = c.col;
    v.val = c.val;
    return v;
}

// ---- Galerkin triple product C = R * (A * P) -----------------------------------
// Two chained products on the handle's scratch and pool; with R = NULL the
// restriction is P^T, transposed on the device.  The intermediate A*P (and
// P^T) are freed stream-ordered before return.
template<typename V>
spgemm_status rap(spgemm_handle_s* h, const spgemm_csr_view* R, const spgemm_csr_view* A,
                  const spgemm_csr_view* P, spgemm_csr_out* C, cudaStream_t stream) {
    if (h == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "handle is NULL");
    if (C == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "C is NULL");
    if (spgemm_status st = check_view(A, "A"); st != SPGEMM_OK) return st;
    if (spgemm_status st = check_view(P, "P"); st != SPGEMM_OK) return st;
    if (R != nullptr) {
        if (spgemm_status st = check_view(R, "R"); st != SPGEMM_OK) return st;
        if (R->n != A->m)
            return fail(SPGEMM_ERR_INVALID_ARG, "R.n (" + std::to_string(R->n) +
                                                    ") must equal A.m (" + std::to_string(A->m) +
                                                    ")");
    } else if (P->m != A->m) {
        return fail(SPGEMM_ERR_INVALID_ARG, "with R = P^T, P.m (" + std::to_string(P->m) +
                                                ") must equal A.m (" + std::to_string(A->m) + ")");
    }
    if (A->n != P->m)
        return fail(SPGEMM_ERR_INVALID_ARG, "A.n (" + std::to_string(A->n) +
                                                ") must equal P.m (" + std::to_string(P->m) + ")");
    std::memset(C, 0, sizeof(*C));
    spgemm_csr_out AP, PT;
    std::memset(&PT, 0, sizeof(PT));
    if (spgemm_status st = product<V>(h, A, P, &AP, stream); st != SPGEMM_OK) return st;
    const spgemm_info info_ap = h->info;
    spgemm_csr_view rv;
    if (R == nullptr) {
        if (spgemm_status st = transpose<V>(h, P, &PT, stream); st != SPGEMM_OK) {
            spgemm_csr_free(&AP, stream);
            return st;
        }
        rv = view_of(PT);
    } else {
        rv = *R;
    }
    const spgemm_csr_view apv = view_of(AP);
    const spgemm_status st = product<V>(h, &rv, &apv, C, stream);
    spgemm_csr_free(&AP, stream);
    if (R == nullptr) spgemm_csr_free(&PT, stream);
    if (st != SPGEMM_OK) return st;
    // info describes the second product; NIP and host syncs cover the chain
    h->info.nip += info_ap.nip;
    h->info.host_syncs += info_ap.host_syncs;
    return SPGEMM_OK;
}

// ---- plans: the fill phase as a replayable CUDA graph -------------------------

spgemm_status plan_new(spgemm_handle_s* h, spgemm_plan_s** out, cudaStream_t stream) {
    auto* p = new spgemm_plan_s();
    p->device = h->device;
    p->pool = h->pool;
    *out = p;
    B200_TRY(cudaStreamCreateWithFlags(&p->capture, cudaStreamNonBlocking));
    B200_TRY(cudaMallocHost(reinterpret_cast<void**>(&p->status_host), sizeof(DevStatus)));
    B200_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p->status), sizeof(DevStatus),
                                     p->pool, stream));
    p->owned.push_back(p->status);
    B200_TRY(cudaMemsetAsync(p->status, 0, sizeof(DevStatus), stream));
    return SPGEMM_OK;
}

// The caller has synchronised every stream the plan ran on.
void plan_free(spgemm_plan_s* p) {
    if (p == nullptr) return;
    cudaSetDevice(p->device);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    for (cudaGraph_t g : p->children)
        if (g) cudaGraphDestroy(g);
    for (void* b : p->owned) cudaFreeAsync(b, p->capture);
    if (p->capture) {
        cudaStreamSynchronize(p->capture);
        cudaStreamDestroy(p->capture);
    }
    if (p->status_host) cudaFreeHost(p->status_host);
    delete p;
}

// Median of three timed replays (after one warm replay) on `stream`.
spgemm_status plan_time(spgemm_plan_s* p, cudaStream_t stream, float* ms) {
    *ms = 0.0f;
    if (p->exec == nullptr) return SPGEMM_OK;  // nothing to fill (nnz(C) = 0)
    cudaEvent_t a, b;
    B200_TRY(cudaEventCreate(&a));
    B200_TRY(cudaEventCreate(&b));
    float t[3] = {};
    cudaError_t e = cudaGraphLaunch(p->exec, stream);
    for (int i = 0; e == cudaSuccess && i < 3; i++) {
        e = cudaEventRecord(a, stream);
        if (e == cudaSuccess) e = cudaGraphLaunch(p->exec, stream);
        if (e == cudaSuccess) e = cudaEventRecord(b, stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t[i], a, b);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) return cuda_fail(e, "time a plan");
    std::sort(t, t + 3);
    *ms = t[1];
    return SPGEMM_OK;
}

// Build a plan with `make(plan, team_scale, cta_scale)` -- a product or a
// batch in plan mode, which also fills the caller's output -- once with the
// default configuration, or, when tuning, once per candidate, keeping the
// fastest replay.  The candidates: the team bins' routing limits scaled by
// 1, 0.75 or 0.5 (a row then runs with a larger hash table and more lanes),
// the CTA bins' by 1 or 0.5 (a larger table and block: 256 -> 512 -> 1,024
// threads), and 4 or 8 side streams (parallel branches of the graph).  `drop`
// frees the output of a candidate that loses.
template<typename Make, typename Drop>
spgemm_status plan_build(spgemm_handle_s* h, int tune, cudaStream_t stream, Make&& make,
                         Drop&& drop, spgemm_plan_s** out) {
    static constexpr double kScales[] = {1.0, 0.75, 0.5};
    static constexpr double kCtaScales[] = {1.0, 0.5};
    static constexpr int kStreams[] = {4, 8};
    struct Cand {
        double scale;
        double cta;
        int streams;
    };
    std::vector<Cand> cands;
    if (tune) {
        for (double sc : kScales)
            for (double cs : kCtaScales)
                for (int ns : kStreams) cands.push_back({sc, cs, ns});
    } else {
        cands.push_back({1.0, 1.0, h->nside});
    }
    static_assert(sizeof(kScales) / sizeof(double) * sizeof(kCtaScales) / sizeof(double) *
                          sizeof(kStreams) / sizeof(int) <=
                      SPGEMM_PLAN_MAX_CANDIDATES,
                  "plan info holds every candidate");
    const int saved_nside = h->nside;
    spgemm_plan_s* best = nullptr;
    int best_i = -1;
    spgemm_plan_info info = {};
    info.candidates = static_cast<int32_t>(cands.size());
    spgemm_status st = SPGEMM_OK;
    for (size_t i = 0; i < cands.size() && st == SPGEMM_OK; i++) {
        h->nside = cands[i].streams;
        spgemm_plan_s* p = nullptr;
        st = plan_new(h, &p, stream);
        if (st == SPGEMM_OK) st = make(p, cands[i].scale, cands[i].cta);
        float ms = 0.0f;
        if (st == SPGEMM_OK) st = plan_time(p, stream, &ms);
        if (st != SPGEMM_OK) {
            cudaStreamSynchronize(stream);
            plan_free(p);
            break;
        }
        info.team_scale[i] = static_cast<float>(cands[i].scale);
        info.cta_scale[i] = static_cast<float>(cands[i].cta);
        info.streams[i] = cands[i].streams;
        info.ms[i] = ms;
        if (best == nullptr || ms < info.ms[best_i]) {
            if (best != nullptr) {
                drop(true);  // the previous best's output
                plan_free(best);
            }
            best = p;
            best_i = static_cast<int>(i);
        } else {
            drop(false);  // this candidate's output
            plan_free(p);
        }
    }
    h->nside = saved_nside;
    if (st != SPGEMM_OK) {
        if (best != nullptr) {
            drop(true);
            plan_free(best);
        }
        return st;
    }
    info.chosen = best_i;
    best->info = info;
    *out = best;
    return SPGEMM_OK;
}

// One stream-ordered memory pool per device for every handle's results,
// created on first use and never destroyed: results may outlive the handle
// that made them, and a pool must not go away under live allocations.  Its
// release threshold is the maximum, so freed memory stays mapped for the next
// product.  It is trimmed only when the last handle on its device goes away:
// trimming under other live handles would make their next products re-map
// their memory.
std::mutex g_pool_mu;
cudaMemPool_t g_pools[64] = {};
int g_pool_users[64] = {};

void release_pool(int dev) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (dev < 0 || dev >= 64 || g_pools[dev] == nullptr) return;
    if (--g_pool_users[dev] == 0) cudaMemPoolTrimTo(g_pools[dev], 0);
}

spgemm_status device_pool(int dev, cudaMemPool_t* out) {
    if (dev < 0 || dev >= 64) return fail(SPGEMM_ERR_INVALID_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (g_pools[dev] == nullptr) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        B200_TRY(cudaMemPoolCreate(&p, &props));
        uint64_t keep = UINT64_MAX;
        B200_TRY(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep));
        g_pools[dev] = p;
    }
    g_pool_users[dev]++;
    *out = g_pools[dev];
    return SPGEMM_OK;
}

template<typename V>
spgemm_status plan_csr(spgemm_handle_t h, const spgemm_csr_view* A, const spgemm_csr_view* B,
                       int32_t tune, spgemm_csr_out* C, spgemm_plan_t* plan, void* stream) {
    if (h == nullptr || C == nullptr || plan == nullptr)
        return fail(SPGEMM_ERR_INVALID_ARG, "NULL argument");
    *plan = nullptr;
    std::memset(C, 0, sizeof(*C));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    B200_TRY(cudaSetDevice(h->device));
    // the kept plan's output is in *C; a losing candidate's output is freed
    spgemm_csr_out cur = {};
    auto make = [&](spgemm_plan_s* p, double scale, double cta) {
        CaptureReq cr;
        cr.team_scale = scale;
        cr.cta_scale = cta;
        cr.plan = p;
        cr.launch_now = true;
        return product<V>(h, A, B, &cur, s, &cr);
    };
    auto drop = [&](bool previous_best) {
        if (previous_best) {
            spgemm_csr_free(C, s);
            *C = cur;
        } else {
            spgemm_csr_free(&cur, s);
        }
    };
    spgemm_plan_s* p = nullptr;
    // plan_build calls make() then drop(); the first candidate becomes the best
    // without a drop, so move its output into *C right after
    auto make_first = [&](spgemm_plan_s* pl, double scale, double cta) {
        const spgemm_status st = make(pl, scale, cta);
        if (st == SPGEMM_OK && C->rpt == nullptr) *C = cur;
        return st;
    };
    const spgemm_status st = plan_build(h, tune, s, make_first, drop, &p);
    if (st != SPGEMM_OK) return st;
    *plan = p;
    return SPGEMM_OK;
}

template<typename V>
spgemm_status plan_batch(spgemm_handle_t h, const spgemm_batch_desc* d, const spgemm_csr_view* A,
                         const spgemm_csr_view* B, int32_t tune, spgemm_batch_out* out,
                         spgemm_plan_t* plan, void* stream) {
    if (h == nullptr || out == nullptr || plan == nullptr)
        return fail(SPGEMM_ERR_INVALID_ARG, "NULL argument");
    *plan = nullptr;
    std::memset(out, 0, sizeof(*out));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    B200_TRY(cudaSetDevice(h->device));
    spgemm_batch_out cur = {};
    auto make = [&](spgemm_plan_s* p, double scale, double cta) {
        const spgemm_status st = batch<V>(h, d, A, B, &cur, s, p, scale, cta);
        if (st == SPGEMM_OK && out->products == nullptr) *out = cur;
        return st;
    };
    auto drop = [&](bool previous_best) {
        if (previous_best) {
            spgemm_batch_free(out, s);
            *out = cur;
        } else {
            spgemm_batch_free(&cur, s);
        }
    };
    spgemm_plan_s* p = nullptr;
    const spgemm_status st = plan_build(h, tune, s, make, drop, &p);
    if (st != SPGEMM_OK) return st;
    *plan = p;
    return SPGEMM_OK;
}

}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }

}  // namespace b200

using namespace b200;

extern "C" {

int spgemm_abi_version(void) { return SPGEMM_ABI_VERSION; }

const char* spgemm_last_error_string(void) { return g_last_error.c_str(); }

const char* spgemm_status_string(spgemm_status st) {
    switch (st) {
        case SPGEMM_OK: return "SPGEMM_OK";
        case SPGEMM_ERR_INVALID_ARG: return "SPGEMM_ERR_INVALID_ARG";
        case SPGEMM_ERR_OOM: return "SPGEMM_ERR_OOM";
        case SPGEMM_ERR_UNSUPPORTED_DEVICE: return "SPGEMM_ERR_UNSUPPORTED_DEVICE";
        case SPGEMM_ERR_OVERFLOW: return "SPGEMM_ERR_OVERFLOW";
        case SPGEMM_ERR_TIMEOUT: return "SPGEMM_ERR_TIMEOUT";
        case SPGEMM_ERR_CUDA: return "SPGEMM_ERR_CUDA";
        case SPGEMM_ERR_INTERNAL: return "SPGEMM_ERR_INTERNAL";
    }
    return "SPGEMM_ERR_UNKNOWN";
}

spgemm_status spgemm_create(spgemm_handle_t* handle, int device) {
    if (handle == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "handle is NULL");
    *handle = nullptr;
    int dev = device;
    if (dev < 0) B200_TRY(cudaGetDevice(&dev));
    int major = 0;
    int minor = 0;
    B200_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    B200_TRY(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev));
    if (major != 10 || minor != 0)
        return fail(SPGEMM_ERR_UNSUPPORTED_DEVICE,
                    "compute capability " + std::to_string(major) + "." + std::to_string(minor) +
                        " is not sm_100 (this library is built for sm_100a only)");
    B200_TRY(cudaSetDevice(dev));
    auto* h = new spgemm_handle_s();
    h->device = dev;
    B200_TRY(cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, dev));
    B200_TRY(sym1_prepare());
    B200_TRY(s2n_prepare());
    B200_TRY(transpose_prepare());
    for (int i = 0; i < kMaxSide; i++) {
        // side stream 0 runs each phase's heaviest bin: the highest priority,
        // so its CTAs take free SMs ahead of the lighter bins'
        int lo_prio = 0;
        int hi_prio = 0;
        B200_TRY(cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio));
        B200_TRY(cudaStreamCreateWithPriority(&h->side[i], cudaStreamNonBlocking,
                                              i == 0 ? hi_prio : lo_prio));
        B200_TRY(cudaEventCreateWithFlags(&h->ev_join[i], cudaEventDisableTiming));
    }
    B200_TRY(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    B200_TRY(cudaEventCreateWithFlags(&h->ev_sample, cudaEventDisableTiming));
    B200_TRY(cudaEventCreateWithFlags(&h->ev_mirror, cudaEventDisableTiming));
    B200_TRY(cudaEventCreateWithFlags(&h->ev_front, cudaEventDisableTiming));
    B200_TRY(cudaMallocHost(reinterpret_cast<void**>(&h->mirror), sizeof(HostMirror)));
    B200_TRY(cudaMallocHost(reinterpret_cast<void**>(&h->front_host), kFrontBytes));
    if (spgemm_status st = device_pool(dev, &h->pool); st != SPGEMM_OK) return st;
    *handle = h;
    return SPGEMM_OK;
}

spgemm_status spgemm_destroy(spgemm_handle_t h) {
    if (h == nullptr) return SPGEMM_OK;
    cudaSetDevice(h->device);
    cudaDeviceSynchronize();
    for (int i = 0; i < kMaxSide; i++) {
        if (h->side[i]) cudaStreamDestroy(h->side[i]);
        if (h->ev_join[i]) cudaEventDestroy(h->ev_join[i]);
    }
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_sample) cudaEventDestroy(h->ev_sample);
    if (h->ev_mirror) cudaEventDestroy(h->ev_mirror);
    if (h->ev_front) cudaEventDestroy(h->ev_front);
    if (h->scratch) cudaFree(h->scratch);
    if (h->bitmaps) cudaFree(h->bitmaps);
    if (h->onepass) cudaFree(h->onepass);
    if (h->slots) cudaFree(h->slots);
    if (h->in_buf) cudaFree(h->in_buf);
    if (h->mirror) cudaFreeHost(h->mirror);
    if (h->front_host) cudaFreeHost(h->front_host);
    for (cudaEvent_t e : h->prof_events) cudaEventDestroy(e);
    // the pool is shared and outlives handles (results may outlive them too);
    // the last handle on the device gives its unused cached memory back
    if (h->pool) release_pool(h->device);
    delete h;
    return SPGEMM_OK;
}

spgemm_status spgemm_csr_f64(spgemm_handle_t h, const spgemm_csr_view* A,
                             const spgemm_csr_view* B, spgemm_csr_out* C, void* stream) {
    return product<double>(h, A, B, C, static_cast<cudaStream_t>(stream));
}

spgemm_status spgemm_csr_f32(spgemm_handle_t h, const spgemm_csr_view* A,
                             const spgemm_csr_view* B, spgemm_csr_out* C, void* stream) {
    return product<float>(h, A, B, C, static_cast<cudaStream_t>(stream));
}

spgemm_status spgemm_csr_host_f64(spgemm_handle_t h, const spgemm_csr_view* A,
                                  const spgemm_csr_view* B, spgemm_csr_out* C, void* stream) {
    return product_host<double>(h, A, B, C, static_cast<cudaStream_t>(stream));
}

spgemm_status spgemm_csr_host_f32(spgemm_handle_t h, const spgemm_csr_view* A,
                                  const spgemm_csr_view* B, spgemm_csr_out* C, void* stream) {
    return product_host<float>(h, A, B, C, static_cast<cudaStream_t>(stream));
}

spgemm_status spgemm_transpose_f64(spgemm_handle_t h, const spgemm_csr_view* A,
                                   spgemm_csr_out* T, void* stream) {
    return transpose<double>(h, A, T, static_cast<cudaStream_t>(stream));
}

spgemm_status spgemm_transpose_f32(spgemm_handle_t h, const spgemm_csr_view* A,
                                   spgemm_csr_out* T, void* stream) {
    return transpose<float>(h, A, T, static_cast<cudaStream_t>(stream));
}

spgemm_status spgemm_rap_f64(spgemm_handle_t h, const spgemm_csr_view* R,
                             const spgemm_csr_view* A, const spgemm_csr_view* P,
                             spgemm_csr_out* C, void* stream) {
    return rap<double>(h, R, A, P, C, static_cast<cudaStream_t>(stream));
}

spgemm_status spgemm_rap_f32(spgemm_handle_t h, const spgemm_csr_view* R,
                             const spgemm_csr_view* A, const spgemm_csr_view* P,
                             spgemm_csr_out* C, void* stream) {
    return rap<float>(h, R, A, P, C, static_cast<cudaStream_t>(stream));
}

spgemm_status spgemm_plan_csr_f64(spgemm_handle_t h, const spgemm_csr_view* A,
                                  const spgemm_csr_view* B, int32_t tune, spgemm_csr_out* C,
                                  spgemm_plan_t* plan, void* stream) {
    return plan_csr<double>(h, A, B, tune, C, plan, stream);
}

spgemm_status spgemm_plan_csr_f32(spgemm_handle_t h, const spgemm_csr_view* A,
                                  const spgemm_csr_view* B, int32_t tune, spgemm_csr_out* C,
                                  spgemm_plan_t* plan, void* stream) {
    return plan_csr<float>(h, A, B, tune, C, plan, stream);
}

spgemm_status spgemm_plan_batch_f64(spgemm_handle_t h, const spgemm_batch_desc* d,
                                    const spgemm_csr_view* A, const spgemm_csr_view* B,
                                    int32_t tune, spgemm_batch_out* out, spgemm_plan_t* plan,
                                    void* stream) {
    return plan_batch<double>(h, d, A, B, tune, out, plan, stream);
}

spgemm_status spgemm_plan_batch_f32(spgemm_handle_t h, const spgemm_batch_desc* d,
                                    const spgemm_csr_view* A, const spgemm_csr_view* B,
                                    int32_t tune, spgemm_batch_out* out, spgemm_plan_t* plan,
                                    void* stream) {
    return plan_batch<float>(h, d, A, B, tune, out, plan, stream);
}

spgemm_status spgemm_plan_execute(spgemm_plan_t plan, void* stream) {
    if (plan == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "plan is NULL");
    if (plan->exec == nullptr) return SPGEMM_OK;  // C has no entries to recompute
    B200_TRY(cudaSetDevice(plan->device));
    B200_TRY(cudaGraphLaunch(plan->exec, static_cast<cudaStream_t>(stream)));
    return SPGEMM_OK;
}

spgemm_status spgemm_plan_check(spgemm_plan_t plan, void* stream) {
    if (plan == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "plan is NULL");
    B200_TRY(cudaSetDevice(plan->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    B200_TRY(cudaMemcpyAsync(plan->status_host, plan->status, sizeof(DevStatus),
                             cudaMemcpyDeviceToHost, s));
    B200_TRY(cudaMemsetAsync(plan->status, 0, sizeof(DevStatus), s));
    B200_TRY(cudaStreamSynchronize(s));
    return status_to_error(*plan->status_host);
}

spgemm_status spgemm_plan_get_info(spgemm_plan_t plan, spgemm_plan_info* info) {
    if (plan == nullptr || info == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "NULL argument");
    *info = plan->info;
    return SPGEMM_OK;
}

spgemm_status spgemm_plan_destroy(spgemm_plan_t plan) {
    plan_free(plan);
    return SPGEMM_OK;
}

spgemm_status spgemm_batch_f64(spgemm_handle_t h, const spgemm_batch_desc* d,
                               const spgemm_csr_view* A, const spgemm_csr_view* B,
                               spgemm_batch_out* out, void* stream) {
    return batch<double>(h, d, A, B, out, static_cast<cudaStream_t>(stream));
}

spgemm_status spgemm_batch_f32(spgemm_handle_t h, const spgemm_batch_desc* d,
                               const spgemm_csr_view* A, const spgemm_csr_view* B,
                               spgemm_batch_out* out, void* stream) {
    return batch<float>(h, d, A, B, out, static_cast<cudaStream_t>(stream));
}

spgemm_status spgemm_batch_free(spgemm_batch_out* out, void* stream) {
    if (out == nullptr) return SPGEMM_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSuccess;
    for (int32_t i = 0; i < out->n_blocks; i++) {
        const cudaError_t ei = cudaFreeAsync(out->blocks[i], s);
        if (e == cudaSuccess) e = ei;
    }
    std::free(out->blocks);
    std::free(out->products);
    std::memset(out, 0, sizeof(*out));
    if (e != cudaSuccess) return cuda_fail(e, "cudaFreeAsync");
    return SPGEMM_OK;
}

spgemm_status spgemm_csr_free(spgemm_csr_out* C, void* stream) {
    if (C == nullptr) return SPGEMM_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSuccess;
    if (C->rpt) e = cudaFreeAsync(C->rpt, s);
    if (C->col && e == cudaSuccess) e = cudaFreeAsync(C->col, s);
    if (C->val && e == cudaSuccess) e = cudaFreeAsync(C->val, s);
    std::memset(C, 0, sizeof(*C));
    if (e != cudaSuccess) return cuda_fail(e, "cudaFreeAsync");
    return SPGEMM_OK;
}

spgemm_status spgemm_host_csr_free(spgemm_csr_out* C) {
    if (C == nullptr) return SPGEMM_OK;
    if (C->rpt != nullptr && !pinned_give_back(C->rpt)) {
        std::free(C->rpt);
        std::free(C->col);
        std::free(C->val);
    }
    std::memset(C, 0, sizeof(*C));
    return SPGEMM_OK;
}

spgemm_status spgemm_get_nip(spgemm_handle_t h, const spgemm_csr_view* A,
                             const spgemm_csr_view* B, int64_t* nip, void* stream) {
    if (h == nullptr || nip == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "NULL argument");
    if (spgemm_status st = check_view(A, "A"); st != SPGEMM_OK) return st;
    if (spgemm_status st = check_view(B, "B"); st != SPGEMM_OK) return st;
    if (A->n != B->m) return fail(SPGEMM_ERR_INVALID_ARG, "A.n must equal B.m");
    B200_TRY(cudaSetDevice(h->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch sc;
    if (spgemm_status st = ensure_scratch(h, A->m, &sc, s); st != SPGEMM_OK) return st;
    long long* d = reinterpret_cast<long long*>(sc.cta_sum);
    B200_TRY(cudaMemsetAsync(d, 0, sizeof(long long), s));
    B200_TRY(launch_total_nip(A->rpt, A->col, B->rpt, A->m, d, s));
    long long v = 0;
    B200_TRY(cudaMemcpyAsync(&h->mirror->plan.total_key, d, sizeof(long long),
                             cudaMemcpyDeviceToHost, s));
    B200_TRY(cudaStreamSynchronize(s));
    v = h->mirror->plan.total_key;
    *nip = v;
    return SPGEMM_OK;
}

spgemm_status spgemm_get_nip_many(spgemm_handle_t h, int32_t count, const spgemm_csr_view* A,
                                  const spgemm_csr_view* B, int64_t* nip, void* stream) {
    if (h == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "handle is NULL");
    if (count < 0) return fail(SPGEMM_ERR_INVALID_ARG, "negative count");
    if (count == 0) return SPGEMM_OK;
    if (A == nullptr || B == nullptr || nip == nullptr)
        return fail(SPGEMM_ERR_INVALID_ARG, "NULL argument");
    std::vector<NipPair> pairs(count);
    std::vector<int32_t> cta_off(size_t(count) + 1);
    int64_t ctas = 0;
    for (int32_t i = 0; i < count; i++) {
        if (spgemm_status st = check_view(A + i, "A[i]"); st != SPGEMM_OK) return st;
        if (spgemm_status st = check_view(B + i, "B[i]"); st != SPGEMM_OK) return st;
        if (A[i].n != B[i].m)
            return fail(SPGEMM_ERR_INVALID_ARG,
                        "A[" + std::to_string(i) + "].n must equal B[" + std::to_string(i) + "].m");
        pairs[i] = NipPair{A[i].col, B[i].rpt, A[i].nnz, 0};
        cta_off[i] = static_cast<int32_t>(ctas);
        ctas += pairs_nip_ctas(A[i].nnz);
        if (ctas > INT32_MAX) return fail(SPGEMM_ERR_OVERFLOW, "too many entries in one call");
    }
    cta_off[count] = static_cast<int32_t>(ctas);
    B200_TRY(cudaSetDevice(h->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t o_pairs = 0;
    const size_t o_off = align_up(o_pairs + sizeof(NipPair) * size_t(count), 256);
    const size_t o_nip = align_up(o_off + sizeof(int32_t) * (size_t(count) + 1), 256);
    const size_t bytes = o_nip + sizeof(long long) * size_t(count);
    char* d = nullptr;
    B200_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d), bytes, h->pool, s));
    cudaError_t e = cudaMemcpyAsync(d + o_pairs, pairs.data(), sizeof(NipPair) * size_t(count),
                                    cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d + o_off, cta_off.data(), sizeof(int32_t) * (size_t(count) + 1),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d + o_nip, 0, sizeof(long long) * size_t(count), s);
    if (e == cudaSuccess)
        e = launch_pairs_nip(reinterpret_cast<const NipPair*>(d + o_pairs),
                             reinterpret_cast<const int32_t*>(d + o_off), count,
                             static_cast<int32_t>(ctas), reinterpret_cast<long long*>(d + o_nip), s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(nip, d + o_nip, sizeof(long long) * size_t(count),
                            cudaMemcpyDeviceToHost, s);
    const cudaError_t ef = cudaFreeAsync(d, s);
    if (e == cudaSuccess) e = ef;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "get_nip_many");
    return SPGEMM_OK;
}

spgemm_status spgemm_last_profile(spgemm_handle_t h, spgemm_kernel_time* out, int32_t capacity,
                                  int32_t* count) {
    if (h == nullptr || count == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "NULL argument");
    const int32_t n = static_cast<int32_t>(h->prof_done.size());
    *count = n;
    if (out != nullptr)
        for (int32_t i = 0; i < n && i < capacity; i++) out[i] = h->prof_done[i];
    return SPGEMM_OK;
}

spgemm_status spgemm_last_info(spgemm_handle_t h, spgemm_info* info) {
    if (h == nullptr || info == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "NULL argument");
    *info = h->info;
    return SPGEMM_OK;
}

spgemm_status spgemm_set_option(spgemm_handle_t h, spgemm_option opt, int64_t value) {
    if (h == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "handle is NULL");
    switch (opt) {
        case SPGEMM_OPT_CHECKED: h->checked = value != 0; return SPGEMM_OK;
        case SPGEMM_OPT_MIN_SYM_BIN: h->min_sym_bin = static_cast<int>(value); return SPGEMM_OK;
        case SPGEMM_OPT_MIN_NUM_BIN: h->min_num_bin = static_cast<int>(value); return SPGEMM_OK;
        case SPGEMM_OPT_CLUSTER_SIZE:
            if (value != 2 && value != 4 && value != 8)
                return fail(SPGEMM_ERR_INVALID_ARG, "cluster size must be 2, 4 or 8");
            h->cluster = static_cast<int>(value);
            return SPGEMM_OK;
        case SPGEMM_OPT_STREAMS:
            if (value < 1 || value > kMaxSide)
                return fail(SPGEMM_ERR_INVALID_ARG, "streams must be in 1..8");
            h->nside = static_cast<int>(value);
            return SPGEMM_OK;
        case SPGEMM_OPT_PROFILE: h->profile = value != 0; return SPGEMM_OK;
        case SPGEMM_OPT_MIN_TRANSPOSE_BIN: h->min_tr_bin = static_cast<int>(value); return SPGEMM_OK;
        case SPGEMM_OPT_ONE_PASS:
            if (value < 0 || value > 2)
                return fail(SPGEMM_ERR_INVALID_ARG, "one-pass must be 0, 1 or 2");
            h->one_pass = static_cast<int>(value);
            return SPGEMM_OK;
        case SPGEMM_OPT_ESC:
            if (value < 0 || value > 2) return fail(SPGEMM_ERR_INVALID_ARG, "ESC must be 0, 1 or 2");
            h->esc = static_cast<int>(value);
            return SPGEMM_OK;
    }
    return fail(SPGEMM_ERR_INVALID_ARG, "unknown option");
}

spgemm_status spgemm_get_option(spgemm_handle_t h, spgemm_option opt, int64_t* value) {
    if (h == nullptr || value == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "NULL argument");
    switch (opt) {
        case SPGEMM_OPT_CHECKED: *value = h->checked; return SPGEMM_OK;
        case SPGEMM_OPT_MIN_SYM_BIN: *value = h->min_sym_bin; return SPGEMM_OK;
        case SPGEMM_OPT_MIN_NUM_BIN: *value = h->min_num_bin; return SPGEMM_OK;
        case SPGEMM_OPT_CLUSTER_SIZE: *value = h->cluster; return SPGEMM_OK;
        case SPGEMM_OPT_STREAMS: *value = h->nside; return SPGEMM_OK;
        case SPGEMM_OPT_PROFILE: *value = h->profile; return SPGEMM_OK;
        case SPGEMM_OPT_MIN_TRANSPOSE_BIN: *value = h->min_tr_bin; return SPGEMM_OK;
        case SPGEMM_OPT_ONE_PASS: *value = h->one_pass; return SPGEMM_OK;
        case SPGEMM_OPT_ESC: *value = h->esc; return SPGEMM_OK;
    }
    return fail(SPGEMM_ERR_INVALID_ARG, "unknown option");
}

spgemm_status spgemm_ladder_info(spgemm_handle_t h, int which, int dtype_bytes, int* n_bins,
                                 int64_t* limits) {
    (void)h;
    if (n_bins == nullptr || limits == nullptr) return fail(SPGEMM_ERR_INVALID_ARG, "NULL");
    const BinLauncher* l = nullptr;
    int nb = 0;
    if (which == 0) {
        nb = sym1_ladder(&l);
    } else if (which == 1) {
        nb = dtype_bytes == 8 ? s2n_ladder_f64(&l) : s2n_ladder_f32(&l);
    } else if (which == 2) {
        nb = dtype_bytes == 8 ? s2n_bitmap_ladder_f64(&l) : s2n_bitmap_ladder_f32(&l);
    } else if (which == 3) {
        nb = dtype_bytes == 8 ? transpose_ladder_f64(&l) : transpose_ladder_f32(&l);
    } else if (which == 4) {
        nb = dtype_bytes == 8 ? s2n_esc_ladder_f64(&l) : s2n_esc_ladder_f32(&l);
    } else {
        return fail(SPGEMM_ERR_INVALID_ARG, "ladder id must be 0..4");
    }
    *n_bins = nb;
    for (int i = 0; i < 16; i++) limits[i] = i < nb ? l[i].limit : 0;
    return SPGEMM_OK;
}

}  // extern "C"
