// emu_shim.h — runs the CUDA kernel sources of ems_b200/csrc on the CPU.
//
// TEST INFRASTRUCTURE. Each CUDA thread of a block becomes a std::thread,
// __syncthreads a std::barrier; the TMA bulk copies complete at once and an
// mbarrier is a phase counter. The arithmetic intrinsics are the plain IEEE
// operations (build with -ffp-contract=off), so the emulated kernel computes
// what the device computes, and its indexing can be checked against the
// buffers before the kernel ever runs on a GPU.
#pragma once

#include <atomic>
#include <barrier>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
#define __launch_bounds__(...)
#define __align__(n) alignas(n)
#define __grid_constant__

struct uint2 {
    uint32_t x, y;
};
struct alignas(16) float4 {
    float x, y, z, w;
};
inline float4 make_float4(float x, float y, float z, float w) { return float4{x, y, z, w}; }
struct alignas(16) uint4 {
    uint32_t x, y, z, w;
};
inline uint4 make_uint4(uint32_t x, uint32_t y, uint32_t z, uint32_t w) { return uint4{x, y, z, w}; }
inline uint2 make_uint2(uint32_t x, uint32_t y) { return uint2{x, y}; }

struct EmuDim {
    unsigned x = 0, y = 0, z = 0;
};
inline uint2 make_uint2(uint32_t x, uint32_t y);
extern thread_local EmuDim threadIdx;
extern EmuDim blockIdx, blockDim, gridDim;

inline float __fmul_rn(float a, float b) { return a * b; }
inline float __fadd_rn(float a, float b) { return a + b; }
inline float __fsub_rn(float a, float b) { return a - b; }
inline double __dmul_rn(double a, double b) { return a * b; }
inline double __dadd_rn(double a, double b) { return a + b; }
inline double __dsub_rn(double a, double b) { return a - b; }
inline double __ddiv_rn(double a, double b) { return a / b; }
inline uint32_t min(uint32_t a, uint32_t b) { return a < b ? a : b; }
inline int __ffs(uint32_t x) { return __builtin_ffs((int)x); }
template <class T>
inline T __ldg(const T* p) { return *p; }
inline double __fma_rn(double a, double b, double c) { return std::fma(a, b, c); }
// Host stand-in (the emulated kernels here do not use it for parity).
inline void sincospi(double x, double* s, double* c) {
    *s = std::sin(3.14159265358979323846 * x);
    *c = std::cos(3.14159265358979323846 * x);
}

inline unsigned atomicAdd(uint32_t* p, uint32_t v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
inline int atomicExch(int* p, int v) { return __atomic_exchange_n(p, v, __ATOMIC_SEQ_CST); }

namespace emu {
struct Block {
    std::barrier<>* bar = nullptr;
    unsigned char* smem = nullptr;
    size_t smem_bytes = 0;
    std::vector<double> sums;
    std::atomic<int> errors{0};
    char msg[256] = {0};
};
extern Block* cur;

void fail(const char* what);

inline unsigned char* dynamic_smem() { return cur->smem; }

// Barrier word: low 32 bits completed phases, high 32 bits bytes pending.
inline void expect_tx(uint64_t* bar, uint32_t bytes) {
    uint64_t v = __atomic_load_n(bar, __ATOMIC_SEQ_CST);
    if ((v >> 32) != 0) fail("expect_tx on a barrier with bytes pending");
    __atomic_store_n(bar, (v & 0xffffffffull) | ((uint64_t)bytes << 32), __ATOMIC_SEQ_CST);
}

inline void bulk(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    unsigned char* d = (unsigned char*)dst;
    if (d < cur->smem || d + bytes > cur->smem + cur->smem_bytes) fail("bulk copy outside shared memory");
    if (((uintptr_t)dst & 15) || ((uintptr_t)src & 15) || (bytes & 15)) fail("bulk copy not 16-byte aligned");
    std::memcpy(dst, src, bytes);
    uint64_t v = __atomic_load_n(bar, __ATOMIC_SEQ_CST);
    uint64_t pend = v >> 32;
    if (pend < bytes) fail("bulk copy beyond the expected bytes");
    pend -= bytes;
    uint64_t phase = v & 0xffffffffull;
    if (pend == 0) phase++;
    __atomic_store_n(bar, phase | (pend << 32), __ATOMIC_SEQ_CST);
}

inline bool wait(uint64_t* bar, uint32_t parity) {
    for (long it = 0; it < 200000000L; ++it) {
        uint64_t v = __atomic_load_n(bar, __ATOMIC_SEQ_CST);
        if (((v & 0xffffffffull) & 1u) != parity) return true;
        std::this_thread::yield();
    }
    fail("mbarrier wait never satisfied");
    return false;
}

inline double block_sum(double v) {
    const unsigned t = threadIdx.x + blockDim.x * threadIdx.y;
    cur->sums[t] = v;
    cur->bar->arrive_and_wait();
    double s = 0.0;
    if (t == 0)
        for (unsigned q = 0; q < blockDim.x * blockDim.y; ++q) s += cur->sums[q];
    cur->bar->arrive_and_wait();
    return s;
}
}  // namespace emu

inline void __syncthreads() { emu::cur->bar->arrive_and_wait(); }
