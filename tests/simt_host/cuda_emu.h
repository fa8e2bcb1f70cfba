// Host SIMT emulation, test infrastructure: runs a kernel's own source on the
// CPU with one OS thread per CUDA thread, real barriers for
// __syncthreads/__syncwarp and exchange slots for warp collectives.  CTAs run
// one after another (emu_run_cta).  Collective masks must be aligned
// power-of-two lane groups.  Only the intrinsics the tested kernels use are
// here.
#pragma once
#include <algorithm>
#include <atomic>
#include <barrier>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <thread>
#include <vector>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __launch_bounds__(...)
#define __align__(x) alignas(x)
#define __grid_constant__
#define __restrict__

struct EmuDim { unsigned x = 0, y = 0, z = 0; };
inline thread_local EmuDim threadIdx;
inline EmuDim blockIdx, blockDim, gridDim;

struct EmuWarp {
    uint64_t slot[32];
    std::unique_ptr<std::barrier<>> bar[6][32];
};
struct EmuCta {
    std::unique_ptr<std::barrier<>> bar;
    std::vector<EmuWarp> warps;
    unsigned char* dyn = nullptr;
    unsigned char* stat = nullptr;
};
inline EmuCta* emu_cta = nullptr;
inline unsigned char* emu_smem() { return emu_cta->dyn; }
template<class T> inline T* emu_static() { return reinterpret_cast<T*>(emu_cta->stat); }

inline std::barrier<>& emu_group_bar(unsigned mask) {
    EmuWarp& w = emu_cta->warps[threadIdx.x >> 5];
    const int g = __builtin_popcount(mask);
    const int lg = __builtin_ctz(g);
    const int lane = threadIdx.x & 31;
    if (g != (1 << lg) || ((mask >> lane) & 1u) == 0 || (__builtin_ctz(mask) % g) != 0) {
        std::fprintf(stderr, "emu: bad mask %08x at lane %d\n", mask, lane);
        std::abort();
    }
    return *w.bar[lg][__builtin_ctz(mask) / g];
}
inline void __syncwarp(unsigned mask = 0xffffffffu) { emu_group_bar(mask).arrive_and_wait(); }
inline void __syncthreads() { emu_cta->bar->arrive_and_wait(); }
inline int emu_or_flag = 0;
inline int __syncthreads_or(int pr) {
    if (threadIdx.x == 0) emu_or_flag = 0;
    emu_cta->bar->arrive_and_wait();
    if (pr) std::atomic_ref<int>(emu_or_flag).fetch_or(1);
    emu_cta->bar->arrive_and_wait();
    const int r = emu_or_flag;
    emu_cta->bar->arrive_and_wait();
    return r;
}
inline void __threadfence() {}
inline void __threadfence_block() {}

template<class T> inline T emu_exchange(unsigned mask, T v, int src_lane) {
    static_assert(sizeof(T) <= 8, "slot");
    EmuWarp& w = emu_cta->warps[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    uint64_t bits = 0;
    std::memcpy(&bits, &v, sizeof(T));
    w.slot[lane] = bits;
    emu_group_bar(mask).arrive_and_wait();
    T out;
    std::memcpy(&out, &w.slot[src_lane & 31], sizeof(T));
    emu_group_bar(mask).arrive_and_wait();
    return out;
}
inline int emu_group_base(unsigned mask) { return __builtin_ctz(mask); }
template<class T> inline T __shfl_sync(unsigned mask, T v, int src, int width = 32) {
    const int lane = threadIdx.x & 31;
    const int base = lane & ~(width - 1);
    return emu_exchange(mask, v, base + (src & (width - 1)));
}
template<class T> inline T __shfl_up_sync(unsigned mask, T v, unsigned d, int width = 32) {
    const int lane = threadIdx.x & 31;
    const int base = lane & ~(width - 1);
    const int s = (lane - base) >= static_cast<int>(d) ? lane - static_cast<int>(d) : lane;
    (void)base;
    return emu_exchange(mask, v, s);
}
template<class T> inline T __shfl_down_sync(unsigned mask, T v, unsigned d, int width = 32) {
    const int lane = threadIdx.x & 31;
    const int base = lane & ~(width - 1);
    const int s = (lane - base) + static_cast<int>(d) < width ? lane + static_cast<int>(d) : lane;
    return emu_exchange(mask, v, s);
}
template<class T> inline T __shfl_xor_sync(unsigned mask, T v, int lm, int width = 32) {
    const int lane = threadIdx.x & 31;
    const int base = lane & ~(width - 1);
    const int s = base + (((lane - base) ^ lm) & (width - 1));
    return emu_exchange(mask, v, s);
}
inline unsigned __ballot_sync(unsigned mask, int pred) {
    EmuWarp& w = emu_cta->warps[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    w.slot[lane] = pred ? 1 : 0;
    emu_group_bar(mask).arrive_and_wait();
    unsigned r = 0;
    for (int i = 0; i < 32; i++)
        if (((mask >> i) & 1u) && w.slot[i]) r |= 1u << i;
    emu_group_bar(mask).arrive_and_wait();
    return r;
}
inline int __any_sync(unsigned mask, int p) { return __ballot_sync(mask, p) != 0; }
inline int __all_sync(unsigned mask, int p) { return __ballot_sync(mask, p) == mask; }
template<class T> inline unsigned __match_any_sync(unsigned mask, T v) {
    EmuWarp& w = emu_cta->warps[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    uint64_t bits = 0;
    std::memcpy(&bits, &v, sizeof(T));
    w.slot[lane] = bits;
    emu_group_bar(mask).arrive_and_wait();
    unsigned r = 0;
    for (int i = 0; i < 32; i++)
        if (((mask >> i) & 1u) && w.slot[i] == bits) r |= 1u << i;
    emu_group_bar(mask).arrive_and_wait();
    return r;
}
inline int __reduce_max_sync(unsigned mask, int v) {
    int m = v;
    for (int o = 16; o > 0; o >>= 1) m = std::max(m, __shfl_xor_sync(mask, m, o));
    return m;
}
inline int __reduce_min_sync(unsigned mask, int v) {
    int m = v;
    for (int o = 16; o > 0; o >>= 1) m = std::min(m, __shfl_xor_sync(mask, m, o));
    return m;
}
inline int atomicAdd(int* p, int v) { return std::atomic_ref<int>(*p).fetch_add(v); }
inline unsigned atomicAdd(unsigned* p, unsigned v) { return std::atomic_ref<unsigned>(*p).fetch_add(v); }
inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) {
    return std::atomic_ref<unsigned long long>(*p).fetch_add(v);
}
inline double atomicAdd(double* p, double v) { return std::atomic_ref<double>(*p).fetch_add(v); }
inline float atomicAdd(float* p, float v) { return std::atomic_ref<float>(*p).fetch_add(v); }
inline int atomicCAS(int* p, int cmp, int v) {
    std::atomic_ref<int>(*p).compare_exchange_strong(cmp, v);
    return cmp;
}
inline unsigned atomicOr(unsigned* p, unsigned v) { return std::atomic_ref<unsigned>(*p).fetch_or(v); }
inline unsigned long long atomicExch(unsigned long long* p, unsigned long long v) {
    return std::atomic_ref<unsigned long long>(*p).exchange(v);
}
inline void __nanosleep(unsigned) {}
template<class T> inline T __ldcs(const T* p) { return *p; }
template<class T> inline void __stcs(T* p, T v) { *p = v; }
template<class T> inline T emu_atomic_max(T* p, T v) {
    std::atomic_ref<T> a(*p);
    T cur = a.load();
    while (cur < v && !a.compare_exchange_weak(cur, v)) {}
    return cur;
}
inline int atomicMax(int* p, int v) { return emu_atomic_max(p, v); }
inline long long atomicMax(long long* p, long long v) { return emu_atomic_max(p, v); }
template<class T> inline T __ldg(const T* p) { return *p; }
inline int __popc(unsigned x) { return __builtin_popcount(x); }
inline int __ffs(int x) { return __builtin_ffs(x); }
inline int __ffs(unsigned x) { return __builtin_ffs(static_cast<int>(x)); }
inline int __clz(int x) { return x == 0 ? 32 : __builtin_clz(static_cast<unsigned>(x)); }
inline int __clz(unsigned x) { return x == 0 ? 32 : __builtin_clz(x); }
inline unsigned __umulhi(unsigned a, unsigned b) { return static_cast<unsigned>((static_cast<uint64_t>(a) * b) >> 32); }
template<class A, class B> inline auto min(A a, B b) { return a < b ? a : b; }
template<class A, class B> inline auto max(A a, B b) { return a < b ? b : a; }

inline void emu_run_cta(int block, int nthreads, size_t dyn, const std::function<void()>& body) {
    EmuCta cta;
    blockDim.x = nthreads;
    blockIdx.x = block;
    cta.bar = std::make_unique<std::barrier<>>(nthreads);
    cta.warps.resize((nthreads + 31) / 32);
    for (auto& w : cta.warps)
        for (int lg = 0; lg < 6; lg++)
            for (int gi = 0; gi < (32 >> lg); gi++) w.bar[lg][gi] = std::make_unique<std::barrier<>>(1 << lg);
    cta.dyn = static_cast<unsigned char*>(std::aligned_alloc(16, ((dyn ? dyn : 16) + 15) / 16 * 16));
    std::memset(cta.dyn, 0xCD, dyn);
    cta.stat = static_cast<unsigned char*>(std::aligned_alloc(16, 262144));
    std::memset(cta.stat, 0xCD, 262144);
    emu_cta = &cta;
    std::vector<std::thread> ts;
    ts.reserve(nthreads);
    for (int t = 0; t < nthreads; t++)
        ts.emplace_back([&, t] {
            threadIdx.x = t;
            body();
            cta.bar->arrive_and_drop();
        });
    for (auto& th : ts) th.join();
    std::free(cta.dyn);
    std::free(cta.stat);
}
