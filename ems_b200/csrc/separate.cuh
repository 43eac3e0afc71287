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
// A thread updates eight consecutive z-nodes of one row with two 16-byte
// loads and stores per array (rows start 128-byte aligned); the z-neighbour
// beyond its eight comes from one extra 4-byte load. The 32 lanes of a warp
// take 32 consecutive y-rows, so a warp's loads fill whole 32-byte sectors
// and everything that varies along z (z-normal CPML layers, a dispersive
// slab normal to z) branches alike in all lanes. A block is 32 rows × 4
// segments (32 z-nodes) of one x-plane. Entries a reference update never
// writes (padding) keep their value: a vector store writes back what it read.
#pragma once

#include "fused.cuh"

namespace emsk {

// Block: kSepK lanes along y × kSepJ z-segments of kSeg nodes.
constexpr unsigned kSepK = 32, kSepJ = 4, kSeg = 8;

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

// A thread's z-segment: kSeg consecutive nodes of one row, loaded as two
// 16-byte vectors (one 32-byte sector).
struct Seg {
    float4 a, b;
    __device__ __forceinline__ float operator[](int e) const { return e < 4 ? el(a, e) : el(b, e - 4); }
    __device__ __forceinline__ void set(int e, float x) {
        if (e < 4) set_el(a, e, x);
        else set_el(b, e - 4, x);
    }
};

__device__ __forceinline__ Seg lds(const float* p) { return Seg{ld4(p), ld4(p + 4)}; }
__device__ __forceinline__ void sts(float* p, const Seg& v) {
    st4(p, v.a);
    st4(p + 4, v.b);
}
__device__ __forceinline__ Seg zseg() {
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return Seg{z, z};
}

// H update with the post_h slab hooks; with ENERGY each block writes its
// share of the energy invariant in units of dt/4. Lane ↔ y-row, thread ↔ a
// z-segment of kSeg nodes: features along z (z layers, a slab normal to z)
// take the same branch in every lane.
template <bool ENERGY>
__global__ void __launch_bounds__(kSepK* kSepJ) k_step_h(const __grid_constant__ FusedParams P) {
    const Grid& g = P.g;
    const uint32_t j = blockIdx.y * kSepK + threadIdx.x;
    const uint32_t k0 = (blockIdx.x * kSepJ + threadIdx.y) * kSeg, i = blockIdx.z;
    double w = 0.0;
    if (k0 < g.nz && j < g.ny) {
        const uint32_t si = g.ny * g.pitch;
        const uint32_t idx = i * si + j * g.pitch + k0;
        const uint32_t row = i * g.ny + j;
        const bool jn = j + 1 < g.ny, in_ = i + 1 < g.nx;
        const bool kn = k0 + kSeg < g.nz;  // the z-neighbour of the last node exists
        const Seg ux = lds(P.un[0] + idx), uy = lds(P.un[1] + idx), uz = lds(P.un[2] + idx);
        const uint32_t cm01 = P.cmask[0][i] | P.cmask[1][j];
        if (ENERGY) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const Seg ca = lds(lane_row(P, c, row) + k0), cb = lds(lane_row(P, 3 + c, row) + k0);
                const Seg& u = c == 0 ? ux : (c == 1 ? uy : uz);
#pragma unroll
                for (int e = 0; e < (int)kSeg; ++e) {
                    if (k0 + e >= g.nz) break;
                    const double x = u[e];
                    w = __dadd_rn(w, weight(ca[e], __dmul_rn(x, x), cb[e]));
                }
            }
        }
        // x: (uz[j+1] − uz[j]) − (uy[k+1] − uy[k])
        if (jn) {
            const Seg da = lds(lane_row(P, 6, row) + k0), db = lds(lane_row(P, 9, row) + k0);
            const Seg uzj = lds(P.un[2] + idx + g.pitch);
            const float uyk = kn ? P.un[1][idx + kSeg] : 0.0f;
            const Seg old = lds(P.in[0] + idx);
            const uint4 rr = row_runs(P.row_runs_h, P.has_poles_h, i, 0, g.ny, j);
            Seg out = old;
#pragma unroll
            for (int e = 0; e < (int)kSeg; ++e) {
                const uint32_t k = k0 + e;
                if (k + 1 >= g.nz) break;
                const float uy1 = e + 1 < (int)kSeg ? uy[e + 1] : uyk;
                const float A = __fsub_rn(uzj[e], uz[e]), B = __fsub_rn(uy1, uy[e]);
                const float o = old[e], a = da[e], b = db[e];
                const float nw = flush(__fsub_rn(__fmul_rn(a, o), __fmul_rn(b, __fsub_rn(A, B))));
                if (ENERGY) w = __dadd_rn(w, weight(a, __dmul_rn((double)o, (double)nw), b));
                out.set(e, hooks<true, 0>(P, cm01 | P.cmask[2][k], rr, i, j, k, nw, -b, A, B, o));
            }
            sts(P.in[0] + idx, out);
        }
        // y: (ux[k+1] − ux[k]) − (uz[i+1] − uz[i])
        if (in_) {
            const Seg da = lds(lane_row(P, 7, row) + k0), db = lds(lane_row(P, 10, row) + k0);
            const Seg uzi = lds(P.un[2] + idx + si);
            const float uxk = kn ? P.un[0][idx + kSeg] : 0.0f;
            const Seg old = lds(P.in[1] + idx);
            const uint4 rr = row_runs(P.row_runs_h, P.has_poles_h, i, 1, g.ny, j);
            Seg out = old;
#pragma unroll
            for (int e = 0; e < (int)kSeg; ++e) {
                const uint32_t k = k0 + e;
                if (k + 1 >= g.nz) break;
                const float ux1 = e + 1 < (int)kSeg ? ux[e + 1] : uxk;
                const float A = __fsub_rn(ux1, ux[e]), B = __fsub_rn(uzi[e], uz[e]);
                const float o = old[e], a = da[e], b = db[e];
                const float nw = flush(__fsub_rn(__fmul_rn(a, o), __fmul_rn(b, __fsub_rn(A, B))));
                if (ENERGY) w = __dadd_rn(w, weight(a, __dmul_rn((double)o, (double)nw), b));
                out.set(e, hooks<true, 1>(P, cm01 | P.cmask[2][k], rr, i, j, k, nw, -b, A, B, o));
            }
            sts(P.in[1] + idx, out);
        }
        // z: (uy[i+1] − uy[i]) − (ux[j+1] − ux[j])
        if (in_ && jn) {
            const Seg da = lds(lane_row(P, 8, row) + k0), db = lds(lane_row(P, 11, row) + k0);
            const Seg uyi = lds(P.un[1] + idx + si), uxj = lds(P.un[0] + idx + g.pitch);
            const Seg old = lds(P.in[2] + idx);
            const uint4 rr = row_runs(P.row_runs_h, P.has_poles_h, i, 2, g.ny, j);
            Seg out = old;
#pragma unroll
            for (int e = 0; e < (int)kSeg; ++e) {
                const uint32_t k = k0 + e;
                if (k >= g.nz) break;
                const float A = __fsub_rn(uyi[e], uy[e]), B = __fsub_rn(uxj[e], ux[e]);
                const float o = old[e], a = da[e], b = db[e];
                const float nw = flush(__fsub_rn(__fmul_rn(a, o), __fmul_rn(b, __fsub_rn(A, B))));
                if (ENERGY) w = __dadd_rn(w, weight(a, __dmul_rn((double)o, (double)nw), b));
                out.set(e, hooks<true, 2>(P, cm01 | P.cmask[2][k], rr, i, j, k, nw, -b, A, B, o));
            }
            sts(P.in[2] + idx, out);
        }
    }
    if (ENERGY) {
        const double s = block_sum<kSepK * kSepJ>(w);
        if (threadIdx.x == 0 && threadIdx.y == 0)
            P.partials[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
    }
}

// E update with the post_e slab hooks (same mapping as k_step_h).
__global__ void __launch_bounds__(kSepK* kSepJ) k_step_e(const __grid_constant__ FusedParams P) {
    const Grid& g = P.g;
    const uint32_t j = blockIdx.y * kSepK + threadIdx.x;
    const uint32_t k0 = (blockIdx.x * kSepJ + threadIdx.y) * kSeg, i = blockIdx.z;
    if (k0 >= g.nz || j >= g.ny) return;
    const uint32_t si = g.ny * g.pitch;
    const uint32_t idx = i * si + j * g.pitch + k0;
    const uint32_t row = i * g.ny + j;
    const uint32_t cm01 = P.cmask[0][i] | P.cmask[1][j];
    // x: (iz[j] − iz[j−1]) − (iy[k] − iy[k−1])
    if (i + 1 < g.nx) {
        const Seg ca = lds(lane_row(P, 0, row) + k0), cb = lds(lane_row(P, 3, row) + k0);
        const Seg iz = lds(P.in[2] + idx), iy = lds(P.in[1] + idx);
        const Seg izj = j > 0 ? lds(P.in[2] + idx - g.pitch) : zseg();
        const float iyk = k0 > 0 ? P.in[1][idx - 1] : 0.0f;
        const Seg old = lds(P.un[0] + idx);
        const uint4 rr = row_runs(P.row_runs, P.has_poles, i, 0, g.ny, j);
        Seg out = old;
#pragma unroll
        for (int e = 0; e < (int)kSeg; ++e) {
            const uint32_t k = k0 + e;
            if (k >= g.nz) break;
            const float iy0 = e > 0 ? iy[e - 1] : iyk;
            const float A = __fsub_rn(iz[e], izj[e]), B = __fsub_rn(iy[e], iy0);
            const float o = old[e], a = ca[e], b = cb[e];
            const float t = flush(__fadd_rn(__fmul_rn(a, o), __fmul_rn(b, __fsub_rn(A, B))));
            out.set(e, hooks<false, 0>(P, cm01 | P.cmask[2][k], rr, i, j, k, t, b, A, B, o));
        }
        sts(P.un[0] + idx, out);
    }
    // y: (ix[k] − ix[k−1]) − (iz[i] − iz[i−1])
    if (j + 1 < g.ny) {
        const Seg ca = lds(lane_row(P, 1, row) + k0), cb = lds(lane_row(P, 4, row) + k0);
        const Seg ix = lds(P.in[0] + idx), iz = lds(P.in[2] + idx);
        const Seg izi = i > 0 ? lds(P.in[2] + idx - si) : zseg();
        const float ixk = k0 > 0 ? P.in[0][idx - 1] : 0.0f;
        const Seg old = lds(P.un[1] + idx);
        const uint4 rr = row_runs(P.row_runs, P.has_poles, i, 1, g.ny, j);
        Seg out = old;
#pragma unroll
        for (int e = 0; e < (int)kSeg; ++e) {
            const uint32_t k = k0 + e;
            if (k >= g.nz) break;
            const float ix0 = e > 0 ? ix[e - 1] : ixk;
            const float A = __fsub_rn(ix[e], ix0), B = __fsub_rn(iz[e], izi[e]);
            const float o = old[e], a = ca[e], b = cb[e];
            const float t = flush(__fadd_rn(__fmul_rn(a, o), __fmul_rn(b, __fsub_rn(A, B))));
            out.set(e, hooks<false, 1>(P, cm01 | P.cmask[2][k], rr, i, j, k, t, b, A, B, o));
        }
        sts(P.un[1] + idx, out);
    }
    // z: (iy[i] − iy[i−1]) − (ix[j] − ix[j−1])
    {
        const Seg ca = lds(lane_row(P, 2, row) + k0), cb = lds(lane_row(P, 5, row) + k0);
        const Seg iy = lds(P.in[1] + idx), ix = lds(P.in[0] + idx);
        const Seg iyi = i > 0 ? lds(P.in[1] + idx - si) : zseg();
        const Seg ixj = j > 0 ? lds(P.in[0] + idx - g.pitch) : zseg();
        const Seg old = lds(P.un[2] + idx);
        const uint4 rr = row_runs(P.row_runs, P.has_poles, i, 2, g.ny, j);
        Seg out = old;
#pragma unroll
        for (int e = 0; e < (int)kSeg; ++e) {
            const uint32_t k = k0 + e;
            if (k + 1 >= g.nz) break;
            const float A = __fsub_rn(iy[e], iyi[e]), B = __fsub_rn(ix[e], ixj[e]);
            const float o = old[e], a = ca[e], b = cb[e];
            const float t = flush(__fadd_rn(__fmul_rn(a, o), __fmul_rn(b, __fsub_rn(A, B))));
            out.set(e, hooks<false, 2>(P, cm01 | P.cmask[2][k], rr, i, j, k, t, b, A, B, o));
        }
        sts(P.un[2] + idx, out);
    }
}

}  // namespace emsk
