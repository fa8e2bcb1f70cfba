// Insert step of the cluster count bin (k_sym1_cluster): one column key into a
// linear-probing table spread over the shared memory of a thread-block
// cluster's CTAs, with the row's load limit tested on every new key and a cap
// on the probes of any one key.
//
// The logic is written once for the device and for the host: the kernel
// instantiates it with distributed-shared-memory operations, and the CPU test
// (tests/cluster_probe_host.cpp) with a plain array, so the bounds it checks
// are the kernel's own.
//
// Bounds (the reference's k_sym1_smem_max tests its load limit on every
// insert, sym1.cuh:219-222):
//   * a key probes at most kClusterMaxProbes slots; a key that finds neither
//     an empty slot nor itself within them spills the row (its count goes to
//     the global bin) instead of scanning the rest of the table;
//   * every CTA counts its new keys in its own shared memory and adds them to
//     the cluster-wide total in steps of kClusterCountStep; when that total
//     passes limit - csize * kClusterCountStep the row spills.  The keys not
//     yet added are fewer than csize * kClusterCountStep, so the table holds
//     at most limit + (keys in flight when the flag is raised) keys;
//   * once the row spills, every later probe loop stops at its next check
//     of the CTA's own copy of the spill flag.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define B200_HD __host__ __device__ __forceinline__
#else
#define B200_HD inline
#endif

namespace b200 {

constexpr uint32_t kClusterMaxProbes = 512;   // probes of one key before the row spills
constexpr int32_t kClusterCountStep = 256;    // new keys a CTA counts before it publishes them
constexpr uint32_t kClusterAbortEvery = 16;   // probes between two reads of the spill flag

// The count kernels' hash (common.cuh hash_slot), written without device
// intrinsics: the high half of (key * 0x9E3779B1 mod 2^32) * T.
B200_HD uint32_t cluster_hash(int32_t key, uint32_t T) {
    const uint32_t x = static_cast<uint32_t>(key) * 0x9E3779B1u;
    return static_cast<uint32_t>((static_cast<uint64_t>(x) * T) >> 32);
}

enum ClusterInsert : int { kInsNew = 0, kInsPresent = 1, kInsSpill = 2 };

// Ops provides
//   uint32_t slots() const              table slots over the whole cluster
//   int32_t  cas(uint32_t h, int32_t k) compare-and-swap slot h from empty to
//                                       k; returns the slot's previous key
//   int32_t  empty() const              the empty-slot key
//   bool     spilled()                  this CTA's copy of the spill flag
//   void     spill()                    raise the flag in every CTA
//   int32_t  count_local()              ++ this CTA's new-key count; old value
//   int32_t  publish(int32_t add)       add to the cluster total; new value
//   int32_t  limit() const              the row's load limit (keys)
//   int32_t  csize() const              CTAs in the cluster
// `probes` (optional) receives the number of slots this key probed.
template<class Ops>
B200_HD int cluster_insert(Ops& ops, int32_t key, uint32_t* probes = nullptr) {
    const uint32_t T = ops.slots();
    uint32_t h = cluster_hash(key, T);
    for (uint32_t probe = 0; probe < kClusterMaxProbes; probe++) {
        if (probe % kClusterAbortEvery == 0 && ops.spilled()) {
            if (probes) *probes = probe;
            return kInsSpill;
        }
        const int32_t old = ops.cas(h, key);
        if (old == ops.empty()) {
            if (probes) *probes = probe + 1;
            const int32_t before = ops.count_local();
            if ((before + 1) % kClusterCountStep == 0) {
                const int32_t total = ops.publish(kClusterCountStep);
                if (total > ops.limit() - ops.csize() * kClusterCountStep) ops.spill();
            }
            return kInsNew;
        }
        if (old == key) {
            if (probes) *probes = probe + 1;
            return kInsPresent;
        }
        h = (h + 1 == T) ? 0u : h + 1;
    }
    if (probes) *probes = kClusterMaxProbes;
    ops.spill();
    return kInsSpill;
}

}  // namespace b200
