// separate.cuh — the two-kernel step of the B200 FDTD engine (sm_100a).
//
// One kernel updates every H dual edge and applies, in registration order,
// the CPML correction of the H edges and the magnetic-pole ADE; the serial
// post_h hooks run; a second kernel updates every E edge with the CPML
// correction of the E edges and the electric-pole ADE. Both work in place:
// the H kernel reads only voltages and its own currents, the E kernel only
// currents and its own voltages. The tables are those of the fused kernel
// (pooled coefficient rows, CPML slabs per component, poles as runs along
// z); the expressions are the reference's, so the results equal it bit for
// bit. A block is 32 z-nodes × 4 y-rows of one x-plane.
#pragma once

#include "fused.cuh"

namespace emsk {

constexpr unsigned kSepK = 32, kSepJ = 4;

// Row of coefficient lane l for the (x, y) row `row` (pooled or dense).
__device__ __forceinline__ const float* lane_row(const FusedParams& P, int l, size_t row) {
    const Lane& L = P.lane[l];
    return L.dense ? L.dense + row * P.g.pitch : L.rows + (size_t)L.rid[row] * P.g.pitch;
}

// The slab hooks of one edge in registration order: CPML then poles, or
// poles then CPML.
template <bool H>
__device__ __forceinline__ float hooks(const FusedParams& P, uint32_t cbits, int c, uint32_t i, uint32_t j, uint32_t k,
                                       float t, float coef, float A, float B, float prev) {
    constexpr int side = H ? 0 : 1;
    const uint4 rr = H ? (P.has_poles_h ? P.row_runs_h[((size_t)i * 3 + c) * P.g.ny + j] : make_uint4(0, 0, 0, 0))
                       : (P.has_poles ? P.row_runs[((size_t)i * 3 + c) * P.g.ny + j] : make_uint4(0, 0, 0, 0));
    const bool in_runs = k >= rr.z && k < rr.w;
    // The pole correction's coefficient is the edge's cb (E) or db (H).
    const float pc = H ? -coef : coef;
    // Electric poles start from u^n (the voltage this thread read before
    // updating it); magnetic poles from the current saved after the last
    // E update (zero before the first), as the reference does.
    if (P.poles_first && in_runs)
        t = H ? poles_run(P.runs_h, P.sets_h, P.pj_h, P.pq_h, P.dt, rr, k, t, prev, pc, P.prev_h)
              : poles_run(P.runs, P.sets, P.pj, P.pq, P.dt, rr, k, t, prev, pc, nullptr);
    if (cbits)
        t = c == 0 ? cpml_apply<true, side, 0>(P, cbits, i, j, k, t, coef, A, __fmul_rn(-1.0f, B))
                   : (c == 1 ? cpml_apply<true, side, 1>(P, cbits, i, j, k, t, coef, A, __fmul_rn(-1.0f, B))
                             : cpml_apply<true, side, 2>(P, cbits, i, j, k, t, coef, A, __fmul_rn(-1.0f, B)));
    if (!P.poles_first && in_runs)
        t = H ? poles_run(P.runs_h, P.sets_h, P.pj_h, P.pq_h, P.dt, rr, k, t, prev, pc, P.prev_h)
              : poles_run(P.runs, P.sets, P.pj, P.pq, P.dt, rr, k, t, prev, pc, nullptr);
    return t;
}

// H update with the post_h slab hooks; with ENERGY each block writes its
// share of the energy invariant in units of dt/4.
template <bool ENERGY>
__global__ void __launch_bounds__(kSepK* kSepJ) k_step_h(const __grid_constant__ FusedParams P) {
    const Grid& g = P.g;
    const uint32_t k = blockIdx.x * kSepK + threadIdx.x, j = blockIdx.y * kSepJ + threadIdx.y, i = blockIdx.z;
    double w = 0.0;
    if (k < g.nz && j < g.ny) {
        const uint32_t si = g.ny * g.pitch;
        const uint32_t idx = i * si + j * g.pitch + k;
        const size_t row = (size_t)i * g.ny + j;
        const float ux = P.un[0][idx], uy = P.un[1][idx], uz = P.un[2][idx];
        const uint32_t cbits = cpml_bits(P, i, j, k);
        if (ENERGY) {
            w = __dadd_rn(w, weight(lane_row(P, 0, row)[k], __dmul_rn((double)ux, (double)ux), lane_row(P, 3, row)[k]));
            w = __dadd_rn(w, weight(lane_row(P, 1, row)[k], __dmul_rn((double)uy, (double)uy), lane_row(P, 4, row)[k]));
            w = __dadd_rn(w, weight(lane_row(P, 2, row)[k], __dmul_rn((double)uz, (double)uz), lane_row(P, 5, row)[k]));
        }
        // x: (uz[j+1] − uz[j]) − (uy[k+1] − uy[k])
        if (j + 1 < g.ny && k + 1 < g.nz) {
            const float da = lane_row(P, 6, row)[k], db = lane_row(P, 9, row)[k];
            const float A = __fsub_rn(P.un[2][idx + g.pitch], uz), B = __fsub_rn(P.un[1][idx + 1], uy);
            const float old = P.in[0][idx];
            const float nw = flush(__fsub_rn(__fmul_rn(da, old), __fmul_rn(db, __fsub_rn(A, B))));
            if (ENERGY) w = __dadd_rn(w, weight(da, __dmul_rn((double)old, (double)nw), db));
            P.in[0][idx] = hooks<true>(P, cbits, 0, i, j, k, nw, -db, A, B, old);
        }
        // y: (ux[k+1] − ux[k]) − (uz[i+1] − uz[i])
        if (i + 1 < g.nx && k + 1 < g.nz) {
            const float da = lane_row(P, 7, row)[k], db = lane_row(P, 10, row)[k];
            const float A = __fsub_rn(P.un[0][idx + 1], ux), B = __fsub_rn(P.un[2][idx + si], uz);
            const float old = P.in[1][idx];
            const float nw = flush(__fsub_rn(__fmul_rn(da, old), __fmul_rn(db, __fsub_rn(A, B))));
            if (ENERGY) w = __dadd_rn(w, weight(da, __dmul_rn((double)old, (double)nw), db));
            P.in[1][idx] = hooks<true>(P, cbits, 1, i, j, k, nw, -db, A, B, old);
        }
        // z: (uy[i+1] − uy[i]) − (ux[j+1] − ux[j])
        if (i + 1 < g.nx && j + 1 < g.ny) {
            const float da = lane_row(P, 8, row)[k], db = lane_row(P, 11, row)[k];
            const float A = __fsub_rn(P.un[1][idx + si], uy), B = __fsub_rn(P.un[0][idx + g.pitch], ux);
            const float old = P.in[2][idx];
            const float nw = flush(__fsub_rn(__fmul_rn(da, old), __fmul_rn(db, __fsub_rn(A, B))));
            if (ENERGY) w = __dadd_rn(w, weight(da, __dmul_rn((double)old, (double)nw), db));
            P.in[2][idx] = hooks<true>(P, cbits, 2, i, j, k, nw, -db, A, B, old);
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
    const uint32_t k = blockIdx.x * kSepK + threadIdx.x, j = blockIdx.y * kSepJ + threadIdx.y, i = blockIdx.z;
    if (k >= g.nz || j >= g.ny) return;
    const uint32_t si = g.ny * g.pitch;
    const uint32_t idx = i * si + j * g.pitch + k;
    const size_t row = (size_t)i * g.ny + j;
    const float ix = P.in[0][idx], iy = P.in[1][idx], iz = P.in[2][idx];
    const uint32_t cbits = cpml_bits(P, i, j, k);
    // x: (iz[j] − iz[j−1]) − (iy[k] − iy[k−1])
    if (i + 1 < g.nx) {
        const float ca = lane_row(P, 0, row)[k], cb = lane_row(P, 3, row)[k];
        const float A = __fsub_rn(iz, j > 0 ? P.in[2][idx - g.pitch] : 0.0f);
        const float B = __fsub_rn(iy, k > 0 ? P.in[1][idx - 1] : 0.0f);
        const float old = P.un[0][idx];
        const float t = flush(__fadd_rn(__fmul_rn(ca, old), __fmul_rn(cb, __fsub_rn(A, B))));
        P.un[0][idx] = hooks<false>(P, cbits, 0, i, j, k, t, cb, A, B, old);
    }
    // y: (ix[k] − ix[k−1]) − (iz[i] − iz[i−1])
    if (j + 1 < g.ny) {
        const float ca = lane_row(P, 1, row)[k], cb = lane_row(P, 4, row)[k];
        const float A = __fsub_rn(ix, k > 0 ? P.in[0][idx - 1] : 0.0f);
        const float B = __fsub_rn(iz, i > 0 ? P.in[2][idx - si] : 0.0f);
        const float old = P.un[1][idx];
        const float t = flush(__fadd_rn(__fmul_rn(ca, old), __fmul_rn(cb, __fsub_rn(A, B))));
        P.un[1][idx] = hooks<false>(P, cbits, 1, i, j, k, t, cb, A, B, old);
    }
    // z: (iy[i] − iy[i−1]) − (ix[j] − ix[j−1])
    if (k + 1 < g.nz) {
        const float ca = lane_row(P, 2, row)[k], cb = lane_row(P, 5, row)[k];
        const float A = __fsub_rn(iy, i > 0 ? P.in[1][idx - si] : 0.0f);
        const float B = __fsub_rn(ix, j > 0 ? P.in[0][idx - g.pitch] : 0.0f);
        const float old = P.un[2][idx];
        const float t = flush(__fadd_rn(__fmul_rn(ca, old), __fmul_rn(cb, __fsub_rn(A, B))));
        P.un[2][idx] = hooks<false>(P, cbits, 2, i, j, k, t, cb, A, B, old);
    }
}

}  // namespace emsk
