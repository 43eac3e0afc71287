// arith.cuh — the engine's element arithmetic (sm_100a device code).
//
// Every field update uses explicitly rounded IEEE operations (__fmul_rn,
// __fadd_rn, __fsub_rn and their f64 forms), so no multiply-add is ever
// contracted and each value is the reference's expression bit for bit.
#pragma once

#include <cfloat>
#include <cstdint>

namespace emsk {

// Rounds subnormal results to zero (src/engine/kernel.rs:30-33).
__device__ __forceinline__ float flush(float x) { return fabsf(x) < FLT_MIN ? 0.0f : x; }

// openEMS's f32 leapfrog of one Lorentz/Drude pole (OpenEmsPole,
// src/engine/dispersive.rs:846-899, 1414-1425): V <- A·V + B·(u^n − W),
// W <- W + K·V, returns u − V, every operation flushed. The state (V, W)
// is held as f64 copies of f32 values.
__device__ __forceinline__ float oe_pole_step(double A, double K, double B, double& j, double& q, float prev, float u) {
    const float a = (float)A, k = (float)K, b = (float)B, v0 = (float)j, w0 = (float)q;
    const float v = flush(__fadd_rn(flush(__fmul_rn(a, v0)), flush(__fmul_rn(b, flush(__fsub_rn(prev, w0))))));
    j = (double)v;
    q = (double)flush(__fadd_rn(w0, flush(__fmul_rn(k, v))));
    return flush(__fsub_rn(u, v));
}

// openEMS's f32 Debye update of an edge whose np poles are all Debye poles
// (openems_debye_step, src/engine/dispersive.rs:930-960): constants F, 1 − g,
// b of pole q at A[q·st], G[q·st], B[q·st]; polarisations Q in j[q].
__device__ __forceinline__ float oe_debye_edge(const double* A, const double* G, const double* B, uint32_t st,
                                               double* j, uint32_t np, float prev, float u_star) {
    const float F = (float)A[0];
    float sum = 0.0f;
    for (uint32_t q = 0; q < np; ++q) {
        const float om = (float)G[q * st], b = (float)B[q * st], Q = (float)j[q];
        const float P = flush(__fadd_rn(flush(__fmul_rn(om, Q)), flush(__fmul_rn(b, prev))));
        sum = flush(__fadd_rn(sum, flush(__fsub_rn(P, Q))));
        j[q] = (double)P;
    }
    const float un = flush(__fmul_rn(F, flush(__fsub_rn(u_star, sum))));
    for (uint32_t q = 0; q < np; ++q) {
        const float b = (float)B[q * st];
        j[q] = (double)flush(__fadd_rn((float)j[q], flush(__fmul_rn(b, un))));
    }
    return flush(__fsub_rn(u_star, flush(__fsub_rn(u_star, un))));
}

// flush(ca·u + cb·((a − b) − (c − d))) (src/engine/kernel.rs:252-273).
__device__ __forceinline__ float e_upd(float ca, float u, float cb, float a, float b, float c, float d) {
    return flush(__fadd_rn(__fmul_rn(ca, u), __fmul_rn(cb, __fsub_rn(__fsub_rn(a, b), __fsub_rn(c, d)))));
}

// flush(da·h − db·((a − b) − (c − d))) (src/engine/kernel.rs:58-79).
__device__ __forceinline__ float h_upd(float da, float h, float db, float a, float b, float c, float d) {
    return flush(__fsub_rn(__fmul_rn(da, h), __fmul_rn(db, __fsub_rn(__fsub_rn(a, b), __fsub_rn(c, d)))));
}

// openEMS's summation order with every operation flushed (CurlOrder::OpenEms,
// src/engine/kernel.rs:35-50): h = da·h − db·(((a − b) + d) − c) and
// u = ca·u + cb·(((a − b) − c) + d).
__device__ __forceinline__ float h_upd_oe(float da, float h, float db, float a, float b, float c, float d) {
    const float curl = flush(__fsub_rn(flush(__fadd_rn(flush(__fsub_rn(a, b)), d)), c));
    return flush(__fsub_rn(flush(__fmul_rn(da, h)), flush(__fmul_rn(db, curl))));
}
__device__ __forceinline__ float e_upd_oe(float ca, float u, float cb, float a, float b, float c, float d) {
    const float curl = flush(__fadd_rn(flush(__fsub_rn(flush(__fsub_rn(a, b)), c)), d));
    return flush(__fadd_rn(flush(__fmul_rn(ca, u)), flush(__fmul_rn(cb, curl))));
}

// The update in the summation order OE selects (false: the reference's).
template <bool OE>
__device__ __forceinline__ float h_upd_t(float da, float h, float db, float a, float b, float c, float d) {
    return OE ? h_upd_oe(da, h, db, a, b, c, d) : h_upd(da, h, db, a, b, c, d);
}
template <bool OE>
__device__ __forceinline__ float e_upd_t(float ca, float u, float cb, float a, float b, float c, float d) {
    return OE ? e_upd_oe(ca, u, cb, a, b, c, d) : e_upd(ca, u, cb, a, b, c, d);
}

// (1 + a)·p/b, 0 where b = 0 (src/engine/kernel.rs:116-120).
__device__ __forceinline__ double weight(float a, double p, float b) {
    return b != 0.0f ? __ddiv_rn(__dmul_rn(__dadd_rn(1.0, (double)a), p), (double)b) : 0.0;
}

// Block-wide f64 sum in a fixed order (blockDim.x·blockDim.y a multiple of
// 32, at most THREADS); result valid in thread (0, 0).
#ifdef EMS_HOST_EMULATION
template <unsigned THREADS>
__device__ __forceinline__ double block_sum(double v) { return emu::block_sum(v); }
#else
template <unsigned THREADS>
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sh[THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_down_sync(0xffffffffu, v, o));
    // Linear thread index (blocks may be 2-D); warps of 32 consecutive ids.
    const unsigned t = threadIdx.x + blockDim.x * threadIdx.y;
    const unsigned n = blockDim.x * blockDim.y;
    if (t % 32 == 0) sh[t / 32] = v;
    __syncthreads();
    double s = 0.0;
    if (t == 0)
        for (unsigned q = 0; q < n / 32; ++q) s = __dadd_rn(s, sh[q]);
    return s;
}
#endif

}  // namespace emsk
