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
#include <chrono>
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

// The host stand-in of a TMA tensor map (what cuTensorMapEncodeTiled is
// given for the engine's f32 field maps): base, extents (innermost first),
// the strides of dimensions 1 and 2 in elements, the box.
struct CUtensorMap {
    const float* base;
    uint64_t dim[3];
    uint64_t stride[2];
    uint32_t box[3];
};

namespace emu {
struct Block {
    std::barrier<>* bar = nullptr;
    unsigned char* smem = nullptr;
    size_t smem_bytes = 0;
    std::vector<double> sums;
    std::atomic<int> errors{0};
    std::atomic<int> orflag{0};
    std::barrier<>* wbar[32] = {};  // per warp of 32 threads (__syncwarp), where a kernel needs it
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

// A tiled 3-D tensor copy global → shared: the box at coordinates (x, y, z),
// entries outside the tensor zero-filled, completing the box's bytes on
// `bar`. Checks what the hardware requires: a destination inside shared
// memory on a 128-byte boundary, and x × 4 bytes a multiple of 16.
inline void tensor3d(void* dst, const CUtensorMap* m, int x, int y, int z, uint64_t* bar) {
    const size_t n = (size_t)m->box[0] * m->box[1] * m->box[2];
    unsigned char* d = (unsigned char*)dst;
    if (d < cur->smem || d + n * 4 > cur->smem + cur->smem_bytes) fail("tensor copy outside shared memory");
    if ((uintptr_t)(d - cur->smem) & 127) fail("tensor copy destination not 128-byte aligned");
    if (((long)x * 4) % 16 != 0) fail("tensor copy x coordinate not 16-byte aligned");
    float* o = (float*)dst;
    for (uint32_t c = 0; c < m->box[2]; ++c)
        for (uint32_t b = 0; b < m->box[1]; ++b)
            for (uint32_t a = 0; a < m->box[0]; ++a) {
                const long xx = (long)x + a, yy = (long)y + b, zz = (long)z + c;
                const bool in = xx >= 0 && yy >= 0 && zz >= 0 && (uint64_t)xx < m->dim[0] &&
                                (uint64_t)yy < m->dim[1] && (uint64_t)zz < m->dim[2];
                *o++ = in ? m->base[(uint64_t)zz * m->stride[1] + (uint64_t)yy * m->stride[0] + (uint64_t)xx] : 0.0f;
            }
    const uint32_t bytes = (uint32_t)(n * 4);
    uint64_t v = __atomic_load_n(bar, __ATOMIC_SEQ_CST);
    uint64_t pend = v >> 32;
    if (pend < bytes) fail("tensor copy beyond the expected bytes");
    pend -= bytes;
    uint64_t phase = v & 0xffffffffull;
    if (pend == 0) phase++;
    __atomic_store_n(bar, phase | (pend << 32), __ATOMIC_SEQ_CST);
}

// __syncthreads_or: a barrier that returns whether any thread passed true.
inline bool sync_or(bool v);
inline void syncwarp();

// A bounded wait: false after `limit_ns` of wall time (or 200 M polls)
// without the phase completing, as the device code's waits give up.
inline bool wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = 2000000000ull) {
    const auto t0 = std::chrono::steady_clock::now();
    for (long it = 0; it < 200000000L; ++it) {
        uint64_t v = __atomic_load_n(bar, __ATOMIC_SEQ_CST);
        if (((v & 0xffffffffull) & 1u) != parity) return true;
        if ((it & 255) == 255 &&
            (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count() >
                limit_ns)
            return false;
        std::this_thread::yield();
    }
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

// __syncwarp: the 32 threads of the caller's warp meet.
inline void emu::syncwarp() {
    std::barrier<>* b = cur->wbar[threadIdx.x / 32];
    if (!b) {
        fail("__syncwarp without warp barriers");
        return;
    }
    b->arrive_and_wait();
}

inline bool emu::sync_or(bool v) {
    cur->bar->arrive_and_wait();
    if (v) cur->orflag.store(1);
    cur->bar->arrive_and_wait();
    const bool r = cur->orflag.load() != 0;
    cur->bar->arrive_and_wait();
    if (threadIdx.x == 0 && threadIdx.y == 0) cur->orflag.store(0);
    return r;
}
