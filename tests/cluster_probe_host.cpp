// Host restatement of the cluster count bin's insert loop, driven by
// tests/test_cluster_probe.py.  It includes the kernel's own insert step
// (gpuspgemm_b200/csrc/cluster_insert.cuh) and runs it over a plain array in
// place of the cluster's distributed shared memory: `csize` CTAs of `T` slots,
// the row's products dealt to the CTAs as k_sym1_cluster deals them (slices
// of `threads` A entries, CTA c taking slices c, c + csize, ...), one key per
// CTA in turn to stand for the CTAs running side by side.
//
// Usage: cluster_probe_host CASE T csize threads
//   CASE  overflow   one slice whose distinct keys exceed the whole table
//         fits       distinct keys well under the load limit, over all CTAs
//         repeats    many products over few distinct keys
//         chain      keys that all hash to one slot (the probe cap)
// Prints one JSON object: spilled, count, distinct, max_probes, occupied,
// slots, limit, probes_after_spill, keys_after_spill.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <set>
#include <string>
#include <vector>

#include "../gpuspgemm_b200/csrc/cluster_insert.cuh"

namespace {

constexpr int32_t kEmptyKey = 0x7fffffff;

struct HostTable {
    std::vector<int32_t> slot;
    std::vector<int32_t> count;  // per CTA
    std::vector<int32_t> spill_flag;  // per CTA copy
    int32_t total = 0;
    int32_t load_limit = 0;
    int32_t ncta = 0;
    int cta = 0;  // the CTA whose thread runs the current insert
};

struct HostOps {
    HostTable* t;
    uint32_t slots() const { return static_cast<uint32_t>(t->slot.size()); }
    int32_t empty() const { return kEmptyKey; }
    int32_t limit() const { return t->load_limit; }
    int32_t csize() const { return t->ncta; }
    int32_t cas(uint32_t h, int32_t key) {
        const int32_t old = t->slot[h];
        if (old == kEmptyKey) t->slot[h] = key;
        return old;
    }
    bool spilled() { return t->spill_flag[t->cta] != 0; }
    void spill() {
        for (auto& f : t->spill_flag) f = 1;
    }
    int32_t count_local() { return t->count[t->cta]++; }
    int32_t publish(int32_t add) { return t->total += add; }
};

}  // namespace

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s CASE T csize threads\n", argv[0]);
        return 2;
    }
    const std::string which = argv[1];
    const int T = std::atoi(argv[2]);
    const int csize = std::atoi(argv[3]);
    const int threads = std::atoi(argv[4]);
    const uint32_t slots = static_cast<uint32_t>(T) * static_cast<uint32_t>(csize);

    // the row: A entries, each with its B row of keys
    std::vector<std::vector<int32_t>> brows;
    std::mt19937 rng(20261203);
    if (which == "overflow") {
        // one slice (fewer A entries than a CTA's slice): every key goes
        // through CTA 0, and the row's distinct keys exceed the table
        const int n_a = threads / 2;
        const int per = static_cast<int>(slots / static_cast<uint32_t>(n_a)) * 3 / 2 + 1;
        int32_t next = 0;
        for (int a = 0; a < n_a; a++) {
            std::vector<int32_t> r(per);
            for (auto& k : r) k = next++;
            brows.push_back(std::move(r));
        }
    } else if (which == "fits") {
        const int n_a = threads * csize * 2;
        const int per = static_cast<int>(slots / 2 / static_cast<uint32_t>(n_a));
        int32_t next = 0;
        for (int a = 0; a < n_a; a++) {
            std::vector<int32_t> r(per);
            for (auto& k : r) k = next++;
            brows.push_back(std::move(r));
        }
    } else if (which == "repeats") {
        const int n_a = threads * csize * 3;
        const int distinct = static_cast<int>(slots / 4);
        std::uniform_int_distribution<int32_t> d(0, distinct - 1);
        for (int a = 0; a < n_a; a++) {
            std::set<int32_t> s;
            while (s.size() < 40) s.insert(d(rng));
            brows.emplace_back(s.begin(), s.end());
        }
    } else if (which == "chain") {
        // keys that share one home slot: each new key probes one slot more
        const uint32_t home = b200::cluster_hash(0, slots);
        std::vector<int32_t> same;
        for (int32_t k = 0; same.size() < 2 * b200::kClusterMaxProbes; k++)
            if (b200::cluster_hash(k, slots) == home) same.push_back(k);
        brows.push_back(same);
    } else {
        std::fprintf(stderr, "unknown case %s\n", which.c_str());
        return 2;
    }

    // products per CTA in the kernel's order
    std::vector<std::vector<int32_t>> work(csize);
    const int n_a = static_cast<int>(brows.size());
    for (int base = 0, slice = 0; base < n_a; base += threads, slice++) {
        const int c = slice % csize;
        for (int a = base; a < std::min(base + threads, n_a); a++)
            work[c].insert(work[c].end(), brows[a].begin(), brows[a].end());
    }
    std::set<int32_t> distinct;
    for (const auto& r : brows) distinct.insert(r.begin(), r.end());

    HostTable t;
    t.slot.assign(slots, kEmptyKey);
    t.count.assign(csize, 0);
    t.spill_flag.assign(csize, 0);
    t.load_limit = static_cast<int32_t>(0.8 * static_cast<double>(slots));
    t.ncta = csize;
    HostOps ops{&t};

    uint32_t max_probes = 0;
    long long probes_after_spill = 0;
    long long keys_after_spill = 0;
    std::vector<size_t> pos(csize, 0);
    bool any = true;
    while (any) {
        any = false;
        for (int c = 0; c < csize; c++) {
            if (pos[c] >= work[c].size()) continue;
            any = true;
            t.cta = c;
            const bool was = t.spill_flag[c] != 0;
            uint32_t probes = 0;
            if (!was) b200::cluster_insert(ops, work[c][pos[c]], &probes);
            if (was) {
                probes_after_spill += probes;
                keys_after_spill++;
            }
            max_probes = std::max(max_probes, probes);
            pos[c]++;
        }
    }
    long long occupied = 0;
    for (int32_t k : t.slot) occupied += k != kEmptyKey;
    long long count = 0;
    for (int32_t c : t.count) count += c;
    std::printf(
        "{\"spilled\": %d, \"count\": %lld, \"distinct\": %zu, \"max_probes\": %u, "
        "\"occupied\": %lld, \"slots\": %u, \"limit\": %d, \"probes_after_spill\": %lld, "
        "\"keys_after_spill\": %lld, \"max_probes_allowed\": %u}\n",
        t.spill_flag[0], count, distinct.size(), max_probes, occupied, slots, t.load_limit,
        probes_after_spill, keys_after_spill, b200::kClusterMaxProbes);
    return 0;
}
