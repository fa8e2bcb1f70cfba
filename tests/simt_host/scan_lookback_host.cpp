// Host run of the one-pass row pointer's look-back scan (k_rpt_scan1 in
// gpuspgemm_b200/csrc/k_bin.cu), through the host SIMT emulation.  The
// kernel's source is included as generated by tests/test_scan_lookback.py
// (k_bin_host.cpp: shared arrays mapped onto the emulated CTA's memory, two
// test knobs: emu_withhold_prefix and emu_lookback_spins).
//
//   scan_lookback_host scan <withhold>   exact scans of several row counts
//   scan_lookback_host wait              a predecessor that never publishes
//
// Prints one JSON object per case.
#include "k_bin_host.cpp"

#include <random>
#include <string>

using namespace b200;

static int run_scan(bool withhold) {
    emu_withhold_prefix = withhold;
    std::mt19937 rng(7);
    int bad = 0;
    for (int m : {1, 100, 4095, 4096, 4097, 12288, 140000, 300001}) {
        std::vector<int32_t> cnt(m + 1, 0), want(m + 1, 0);
        int mx = 0;
        for (int i = 0; i < m; i++) {
            int v = rng() % 8 == 0 ? static_cast<int>(rng() % 3000) : static_cast<int>(rng() % 40);
            if (rng() % 50 == 0) v = 0;
            cnt[i] = v;
            mx = std::max(mx, v);
        }
        long long run = 0;
        for (int i = 0; i < m; i++) {
            want[i] = static_cast<int32_t>(run);
            run += cnt[i];
        }
        want[m] = static_cast<int32_t>(run);
        const int tiles = rpt_scan_tiles(m);
        std::vector<unsigned long long> state(1 + tiles, 0ull);
        Plan plan{};
        DevStatus st{};
        for (int b = 0; b < tiles; b++)
            emu_run_cta(b, kScanThreads, 0,
                        [&] { k_rpt_scan1(cnt.data(), m, tiles, state.data(), &plan, &st); });
        long wrong = 0;
        for (int i = 0; i <= m; i++) wrong += cnt[i] != want[i];
        const bool ok = wrong == 0 && plan.total_key == run && plan.max_key == mx &&
                        plan.overflow == 0 && st.flags == 0 &&
                        state[0] == static_cast<unsigned long long>(tiles);
        std::printf("{\"m\": %d, \"tiles\": %d, \"wrong\": %ld, \"total\": %lld, \"want_total\": %lld, "
                    "\"max\": %d, \"want_max\": %d, \"status\": %u, \"ok\": %s}\n",
                    m, tiles, wrong, static_cast<long long>(plan.total_key), run, plan.max_key, mx,
                    st.flags, ok ? "true" : "false");
        bad += !ok;
    }
    return bad;
}

static int run_wait() {
    // tile 0's ticket is taken but its CTA never runs: tile 1's look-back
    // must give up after emu_lookback_spins rounds and report kStWait
    emu_lookback_spins = 1 << 10;
    const int m = 3 * kScanTile;
    std::vector<int32_t> cnt(m + 1, 1);
    std::vector<unsigned long long> state(4, 0ull);
    state[0] = 1;
    Plan plan{};
    DevStatus st{};
    emu_run_cta(0, kScanThreads, 0, [&] { k_rpt_scan1(cnt.data(), m, 3, state.data(), &plan, &st); });
    std::printf("{\"status\": %u, \"row\": %d, \"detail\": %d, \"wait_flag\": %u}\n", st.flags, st.row,
                st.detail, static_cast<unsigned>(kStWait));
    return 0;
}

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "scan";
    if (mode == "wait") return run_wait();
    return run_scan(argc > 2 && std::string(argv[2]) == "1") != 0 ? 1 : 0;
}
