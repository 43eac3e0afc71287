// separate.cuh — the two-kernel step of the B200 FDTD engine (sm_100a).
//
// One kernel updates every H dual edge and applies, in registration order,
// the CPML correction of the H edges and the magnetic-pole ADE; the serial
// post_h hooks run; a second kernel updates every E edge with the CPML
// correction of the E edges and the electric-pole ADE. Both work in place:
// the H kernel reads only voltages and its own currents, the E kernel only
// currents and its own voltages. The tables are those of the fused kernel
// (pooled coefficient rows, CPML slab bitmasks, poles as runs along z); the
// expressions are the reference's, so the results equal it bit for bit.
//
// A thread updates four consecutive z-nodes with 16-byte loads and stores
// (rows start 128-byte aligned); the z-neighbour beyond its four comes from
// one extra 4-byte load. A block is 32 threads (128 z-nodes) × 4 y-rows of
// one x-plane. Entries a reference update never writes (padding) keep their
// value: a vector store writes back what it read there.
#pragma once

#include "fused.cuh"

namespace emsk {

constexpr unsigned kSepK = 32, kSepJ = 4, kVec = 4;

// Row of coefficient lane l for the (x, y) row `row` (pooled or dense).
__device__ __forceinline__ const float* lane_row(const FusedParams& P, int l, uint32_t row) {
    const Lane& L = P.lane[l];
    return L.dense ? L.dense + (size_t)row * P.g.pitch : L.rows + (size_t)L.rid[row] * P.g.pitch;
}

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float el(const float4& v, int e) { return e == 0 ? v.x : (e == 1 ? v.y : (e == 2 ? v.z : v.w)); }
__device__ __forceinline__ void set_el(float4& v, int e, float x) {
    if (e == 0) v.x = x;
    else if (e == 1) v.y = x;
    else if (e == 2) v.z = x;
    else v.w = x;
}

// The slab hooks of one edge in registration order: CPML then poles, or
// poles then CPML. rr: the edge row's pole runs (count 0: none).
template <bool H, int C>
__device__ __forceinline__ float hooks(const FusedParams& P, uint32_t cbits, const uint4& rr, uint32_t i, uint32_t j,
                                       uint32_t k, float t, float coef, float A, float B, float prev) {
    constexpr int side = H ? 0 : 1;
    const bool in_runs = k >= rr.z && k < rr.w;
    // The pole correction's coefficient is the edge's cb (E) or db (H).
    const float pc = H ? -coef : coef;
    // Electric poles start from u^n (the voltage this thread read before
    // updating it); magnetic poles from the current saved after the last
    // E update (zero before the first), as the reference does.
    if (P.poles_first && in_runs)
        t = H ? poles_run(P.runs_h, P.sets_h, P.pj_h, P.pq_h, P.dt, rr, k, t, prev, pc, P.prev_h)
              : poles_run(P.runs, P.sets, P.pj, P.pq, P.dt, rr, k, t, prev, pc, nullptr);
    if (cbits) t = cpml_apply<true, side, C>(P, cbits, i, j, k, t, coef, A, __fmul_rn(-1.0f, B));
    if (!P.poles_first && in_runs)
        t = H ? poles_run(P.runs_h, P.sets_h, P.pj_h, P.pq_h, P.dt, rr, k, t, prev, pc, P.prev_h)
              : poles_run(P.runs, P.sets, P.pj, P.pq, P.dt, rr, k, t, prev, pc, nullptr);
    return t;
}

__device__ __forceinline__ uint4 row_runs(const uint4* rr, bool has, uint32_t i, int c, uint32_t ny, uint32_t j) {
    return has ? rr[((size_t)i * 3 + c) * ny + j] : make_uint4(0, 0, 0, 0);
}

// H update with the post_h slab hooks; with ENERGY each block writes its
// share of the energy invariant in units of dt/4.
template <bool ENERGY>
__global__ void __launch_bounds__(kSepK* kSepJ) k_step_h(const __grid_constant__ FusedParams P) {
    const Grid& g = P.g;
    const uint32_t k0 = (blockIdx.x * kSepK + threadIdx.x) * kVec;
    const uint32_t j = blockIdx.y * kSepJ + threadIdx.y, i = blockIdx.z;
    double w = 0.0;
    if (k0 < g.nz && j < g.ny) {
        const uint32_t si = g.ny * g.pitch;
        const uint32_t idx = i * si + j * g.pitch + k0;
        const uint32_t row = i * g.ny + j;
        const bool jn = j + 1 < g.ny, in_ = i + 1 < g.nx;
        const bool k4 = k0 + kVec < g.nz;  // the z-neighbour of the last node exists
        const float4 ux = ld4(P.un[0] + idx), uy = ld4(P.un[1] + idx), uz = ld4(P.un[2] + idx);
        const float uxk4 = k4 ? P.un[0][idx + kVec] : 0.0f, uyk4 = k4 ? P.un[1][idx + kVec] : 0.0f;
        const uint32_t cm01 = P.cmask[0][i] | P.cmask[1][j];
        if (ENERGY) {
            const float4 ca0 = ld4(lane_row(P, 0, row) + k0), cb0 = ld4(lane_row(P, 3, row) + k0);
            const float4 ca1 = ld4(lane_row(P, 1, row) + k0), cb1 = ld4(lane_row(P, 4, row) + k0);
            const float4 ca2 = ld4(lane_row(P, 2, row) + k0), cb2 = ld4(lane_row(P, 5, row) + k0);
#pragma unroll
            for (int e = 0; e < (int)kVec; ++e) {
                if (k0 + e >= g.nz) break;
                const double x = el(ux, e), y = el(uy, e), z = el(uz, e);
                w = __dadd_rn(w, weight(el(ca0, e), __dmul_rn(x, x), el(cb0, e)));
                w = __dadd_rn(w, weight(el(ca1, e), __dmul_rn(y, y), el(cb1, e)));
                w = __dadd_rn(w, weight(el(ca2, e), __dmul_rn(z, z), el(cb2, e)));
            }
        }
        // x: (uz[j+1] − uz[j]) − (uy[k+1] − uy[k])
        if (jn) {
            const float4 da = ld4(lane_row(P, 6, row) + k0), db = ld4(lane_row(P, 9, row) + k0);
            const float4 uzj = ld4(P.un[2] + idx + g.pitch);
            const float4 old = ld4(P.in[0] + idx);
            const uint4 rr = row_runs(P.row_runs_h, P.has_poles_h, i, 0, g.ny, j);
            float4 out = old;
#pragma unroll
            for (int e = 0; e < (int)kVec; ++e) {
                const uint32_t k = k0 + e;
                if (k + 1 >= g.nz) break;
                const float uy1 = e + 1 < (int)kVec ? el(uy, e + 1) : uyk4;
                const float A = __fsub_rn(el(uzj, e), el(uz, e)), B = __fsub_rn(uy1, el(uy, e));
                const float o = el(old, e), a = el(da, e), b = el(db, e);
                const float nw = flush(__fsub_rn(__fmul_rn(a, o), __fmul_rn(b, __fsub_rn(A, B))));
                if (ENERGY) w = __dadd_rn(w, weight(a, __dmul_rn((double)o, (double)nw), b));
                set_el(out, e, hooks<true, 0>(P, cm01 | P.cmask[2][k], rr, i, j, k, nw, -b, A, B, o));
            }
            st4(P.in[0] + idx, out);
        }
        // y: (ux[k+1] − ux[k]) − (uz[i+1] − uz[i])
        if (in_) {
            const float4 da = ld4(lane_row(P, 7, row) + k0), db = ld4(lane_row(P, 10, row) + k0);
            const float4 uzi = ld4(P.un[2] + idx + si);
            const float4 old = ld4(P.in[1] + idx);
            const uint4 rr = row_runs(P.row_runs_h, P.has_poles_h, i, 1, g.ny, j);
            float4 out = old;
#pragma unroll
            for (int e = 0; e < (int)kVec; ++e) {
                const uint32_t k = k0 + e;
                if (k + 1 >= g.nz) break;
                const float ux1 = e + 1 < (int)kVec ? el(ux, e + 1) : uxk4;
                const float A = __fsub_rn(ux1, el(ux, e)), B = __fsub_rn(el(uzi, e), el(uz, e));
                const float o = el(old, e), a = el(da, e), b = el(db, e);
                const float nw = flush(__fsub_rn(__fmul_rn(a, o), __fmul_rn(b, __fsub_rn(A, B))));
                if (ENERGY) w = __dadd_rn(w, weight(a, __dmul_rn((double)o, (double)nw), b));
                set_el(out, e, hooks<true, 1>(P, cm01 | P.cmask[2][k], rr, i, j, k, nw, -b, A, B, o));
            }
            st4(P.in[1] + idx, out);
        }
        // z: (uy[i+1] − uy[i]) − (ux[j+1] − ux[j])
        if (in_ && jn) {
            const float4 da = ld4(lane_row(P, 8, row) + k0), db = ld4(lane_row(P, 11, row) + k0);
            const float4 uyi = ld4(P.un[1] + idx + si), uxj = ld4(P.un[0] + idx + g.pitch);
            const float4 old = ld4(P.in[2] + idx);
            const uint4 rr = row_runs(P.row_runs_h, P.has_poles_h, i, 2, g.ny, j);
            float4 out = old;
#pragma unroll
            for (int e = 0; e < (int)kVec; ++e) {
                const uint32_t k = k0 + e;
                if (k >= g.nz) break;
                const float A = __fsub_rn(el(uyi, e), el(uy, e)), B = __fsub_rn(el(uxj, e), el(ux, e));
                const float o = el(old, e), a = el(da, e), b = el(db, e);
                const float nw = flush(__fsub_rn(__fmul_rn(a, o), __fmul_rn(b, __fsub_rn(A, B))));
                if (ENERGY) w = __dadd_rn(w, weight(a, __dmul_rn((double)o, (double)nw), b));
                set_el(out, e, hooks<true, 2>(P, cm01 | P.cmask[2][k], rr, i, j, k, nw, -b, A, B, o));
            }
            st4(P.in[2] + idx, out);
        }
    }
    if (ENERGY) {
        const double s = block_sum<kSepK * kSepJ>(w);
        if (threadIdx.x == 0 && threadIdx.y == 0)
            P.partials[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
    }
}

// E update with the post_e slab hooks.
__global__ void __launch_bounds__(kSepK* kSepJ) k_step_e(const __grid_constant__ FusedParams P) {
    const Grid& g = P.g;
    const uint32_t k0 = (blockIdx.x * kSepK + threadIdx.x) * kVec;
    const uint32_t j = blockIdx.y * kSepJ + threadIdx.y, i = blockIdx.z;
    if (k0 >= g.nz || j >= g.ny) return;
    const uint32_t si = g.ny * g.pitch;
    const uint32_t idx = i * si + j * g.pitch + k0;
    const uint32_t row = i * g.ny + j;
    const float4 ix = ld4(P.in[0] + idx), iy = ld4(P.in[1] + idx), iz = ld4(P.in[2] + idx);
    // The z-neighbour below the first node (zero outside the domain).
    const float ixk = k0 > 0 ? P.in[0][idx - 1] : 0.0f, iyk = k0 > 0 ? P.in[1][idx - 1] : 0.0f;
    const uint32_t cm01 = P.cmask[0][i] | P.cmask[1][j];
    const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    // x: (iz[j] − iz[j−1]) − (iy[k] − iy[k−1])
    if (i + 1 < g.nx) {
        const float4 ca = ld4(lane_row(P, 0, row) + k0), cb = ld4(lane_row(P, 3, row) + k0);
        const float4 izj = j > 0 ? ld4(P.in[2] + idx - g.pitch) : zero4;
        const float4 old = ld4(P.un[0] + idx);
        const uint4 rr = row_runs(P.row_runs, P.has_poles, i, 0, g.ny, j);
        float4 out = old;
#pragma unroll
        for (int e = 0; e < (int)kVec; ++e) {
            const uint32_t k = k0 + e;
            if (k >= g.nz) break;
            const float iy0 = e > 0 ? el(iy, e - 1) : iyk;
            const float A = __fsub_rn(el(iz, e), el(izj, e)), B = __fsub_rn(el(iy, e), iy0);
            const float o = el(old, e), a = el(ca, e), b = el(cb, e);
            const float t = flush(__fadd_rn(__fmul_rn(a, o), __fmul_rn(b, __fsub_rn(A, B))));
            set_el(out, e, hooks<false, 0>(P, cm01 | P.cmask[2][k], rr, i, j, k, t, b, A, B, o));
        }
        st4(P.un[0] + idx, out);
    }
    // y: (ix[k] − ix[k−1]) − (iz[i] − iz[i−1])
    if (j + 1 < g.ny) {
        const float4 ca = ld4(lane_row(P, 1, row) + k0), cb = ld4(lane_row(P, 4, row) + k0);
        const float4 izi = i > 0 ? ld4(P.in[2] + idx - si) : zero4;
        const float4 old = ld4(P.un[1] + idx);
        const uint4 rr = row_runs(P.row_runs, P.has_poles, i, 1, g.ny, j);
        float4 out = old;
#pragma unroll
        for (int e = 0; e < (int)kVec; ++e) {
            const uint32_t k = k0 + e;
            if (k >= g.nz) break;
            const float ix0 = e > 0 ? el(ix, e - 1) : ixk;
            const float A = __fsub_rn(el(ix, e), ix0), B = __fsub_rn(el(iz, e), el(izi, e));
            const float o = el(old, e), a = el(ca, e), b = el(cb, e);
            const float t = flush(__fadd_rn(__fmul_rn(a, o), __fmul_rn(b, __fsub_rn(A, B))));
            set_el(out, e, hooks<false, 1>(P, cm01 | P.cmask[2][k], rr, i, j, k, t, b, A, B, o));
        }
        st4(P.un[1] + idx, out);
    }
    // z: (iy[i] − iy[i−1]) − (ix[j] − ix[j−1])
    {
        const float4 ca = ld4(lane_row(P, 2, row) + k0), cb = ld4(lane_row(P, 5, row) + k0);
        const float4 iyi = i > 0 ? ld4(P.in[1] + idx - si) : zero4;
        const float4 ixj = j > 0 ? ld4(P.in[0] + idx - g.pitch) : zero4;
        const float4 old = ld4(P.un[2] + idx);
        const uint4 rr = row_runs(P.row_runs, P.has_poles, i, 2, g.ny, j);
        float4 out = old;
#pragma unroll
        for (int e = 0; e < (int)kVec; ++e) {
            const uint32_t k = k0 + e;
            if (k + 1 >= g.nz) break;
            const float A = __fsub_rn(el(iy, e), el(iyi, e)), B = __fsub_rn(el(ix, e), el(ixj, e));
            const float o = el(old, e), a = el(ca, e), b = el(cb, e);
            const float t = flush(__fadd_rn(__fmul_rn(a, o), __fmul_rn(b, __fsub_rn(A, B))));
            set_el(out, e, hooks<false, 2>(P, cm01 | P.cmask[2][k], rr, i, j, k, t, b, A, B, o));
        }
        st4(P.un[2] + idx, out);
    }
}

}  // namespace emsk
