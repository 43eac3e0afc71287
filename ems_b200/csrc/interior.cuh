// interior.cuh — one pass of the H and E updates over the interior box
// (sm_100a device code).
//
// The split schedule moves 72 bytes per node and step: the H update reads u
// and reads and writes i (36 B), the E update reads i again and reads and
// writes u (36 B). Over the box of nodes that no slab hook touches between
// the two updates (inside every CPML layer; no magnetic hooks in the model)
// this kernel does both updates in one pass at 48 B per node: the step reads
// the old fields from one buffer and writes the new ones into the other (the
// engine swaps them after the step), so a block can march along x without
// waiting for its neighbours. The nodes outside the box run the split
// kernels first (H update and its CPML correction; they read the same old
// buffer) and after it (E update and CPML); a node's H value is the same
// wherever it is computed, so a block recomputes the few H values its E
// update needs from the neighbouring blocks' nodes (one row below, one quad
// of z-nodes below) instead of reading them, and reads those outside the box
// from what the split kernel wrote. All arithmetic is the split kernels'.
#pragma once

#include "../../include/ems_gpu.h"
#include "split.cuh"
#include <algorithm>
#include <string>

namespace emsk {

constexpr unsigned kInRows = 7;     // rows a block updates (warp 0 computes the row below them)
constexpr unsigned kInWarps = kInRows + 1;
constexpr unsigned kInQuads = 31;   // quads of z-nodes a warp updates (lane 0 computes the quad below them)
constexpr unsigned kInPlanes = 32;  // default planes a block marches through
constexpr unsigned kInPrefetch = 2; // planes ahead whose old fields are prefetched into L2

__device__ __forceinline__ void l2_prefetch(const float* p) {
#ifndef EMS_HOST_EMULATION
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
#else
    (void)p;
#endif
}

// H of the quad (i, j, k0..k0+3) from the old fields (uo, io) and the old u
// of the quad, for a quad whose nodes all have their H and E edges (interior
// of the domain): the arithmetic of split_h_quad.
template <bool OE>
__device__ __forceinline__ void interior_h(const FusedParams& P, uint32_t i, uint32_t j, uint32_t k0, Q4& ux, Q4& uy,
                                           Q4& uz, Q4& hx_n, Q4& hy_n, Q4& hz_n) {
    const Grid& g = P.g;
    const uint32_t sj = g.pitch, si = g.ny * g.pitch;
    const uint32_t idx = i * si + j * sj + k0;
    const uint32_t row = i * g.ny + j;
    ux = ldq(P.uo[0] + idx);
    uy = ldq(P.uo[1] + idx);
    uz = ldq(P.uo[2] + idx);
    const Q4 uzj = ldq(P.uo[2] + idx + sj), uxj = ldq(P.uo[0] + idx + sj);
    const Q4 uzi = ldq(P.uo[2] + idx + si), uyi = ldq(P.uo[1] + idx + si);
    const float uy4 = __ldg(P.uo[1] + idx + 4), ux4 = __ldg(P.uo[0] + idx + 4);
    const Q4 hx = ldq(P.io[0] + idx), hy = ldq(P.io[1] + idx), hz = ldq(P.io[2] + idx);
    const Q4 dax = ldq(lane_row(P, 6, row) + k0), dbx = ldq(lane_row(P, 9, row) + k0);
    const Q4 day = ldq(lane_row(P, 7, row) + k0), dby = ldq(lane_row(P, 10, row) + k0);
    const Q4 daz = ldq(lane_row(P, 8, row) + k0), dbz = ldq(lane_row(P, 11, row) + k0);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float uy1 = e < 3 ? uy.v[e + 1] : uy4, ux1 = e < 3 ? ux.v[e + 1] : ux4;
        hx_n.v[e] = h_upd_t<OE>(dax.v[e], hx.v[e], dbx.v[e], uzj.v[e], uz.v[e], uy1, uy.v[e]);
        hy_n.v[e] = h_upd_t<OE>(day.v[e], hy.v[e], dby.v[e], ux1, ux.v[e], uzi.v[e], uz.v[e]);
        hz_n.v[e] = h_upd_t<OE>(daz.v[e], hz.v[e], dbz.v[e], uyi.v[e], uy.v[e], uxj.v[e], ux.v[e]);
    }
}

// Grid: (z tiles of kInQuads quads, y tiles of kInRows rows, x chunks of
// `planes` planes) over the box; a chunk starts by computing the H values of
// the plane before it again (or reads them outside the box). Thread (warp w, lane l): row
// lo[1] + tile·kInRows + w − 1, quad lo[2] + 4·(tile·kInQuads + l − 1); warp 0
// and lane 0 only provide H values to the others.
template <bool OE>
__global__ void __launch_bounds__(32 * kInWarps, 3) k_interior(const __grid_constant__ FusedParams P,
                                                            const InteriorBox B, uint32_t planes) {
    EMS_SHARED float4 sh[2][3][kInWarps][32];  // H(i) of every thread's quad, by plane parity
    const Grid& g = P.g;
    const uint32_t sj = g.pitch, si = g.ny * g.pitch;
    const uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31u;
    const uint32_t j = B.lo[1] + blockIdx.y * kInRows + w - 1u;
    const uint32_t k0 = B.lo[2] + 4u * (blockIdx.x * kInQuads + l) - 4u;
    const uint32_t xs = B.lo[0] + blockIdx.z * planes;
    const uint32_t xe = xs + planes < B.hi[0] ? xs + planes : B.hi[0];
    const bool in_box = j < B.hi[1] && k0 + 4u <= B.hi[2];
    const bool feeder = w == 0 || l == 0;
    const bool owner = !feeder && in_box;
    // A feeder quad outside the box (the row or quad just below it) was
    // written by the split H update before this kernel; one inside is
    // computed again here. The corner feeder (w = 0, l = 0) feeds nobody.
    const bool provide = feeder && in_box && !(w == 0 && l == 0);
    const bool outside = j < B.lo[1] || k0 < B.lo[2];
    Q4 hy_p = zq(), hz_p = zq();  // H(i − 1), y and z, of an owner's quad
    if (owner && xs > B.lo[0]) {
        Q4 ax, ay, az, hx_n;
        interior_h<OE>(P, xs - 1u, j, k0, ax, ay, az, hx_n, hy_p, hz_p);
    } else if (owner) {
        const uint32_t idx = (xs - 1u) * si + j * sj + k0;
        hy_p = ldq(P.in[1] + idx);
        hz_p = ldq(P.in[2] + idx);
    }
    for (uint32_t i = xs; i < xe; ++i) {
        const uint32_t par = (i - xs) & 1u;
        const uint32_t idx = i * si + j * sj + k0;
        // The old fields of the plane kInPrefetch ahead into L2, so that the
        // loads of the next planes (and this plane's reads of plane i + 1)
        // wait for L2 rather than for DRAM.
        if ((owner || provide) && i + kInPrefetch < g.nx) {
            const uint32_t pf = idx + kInPrefetch * si;
            l2_prefetch(P.uo[0] + pf);
            l2_prefetch(P.uo[1] + pf);
            l2_prefetch(P.uo[2] + pf);
            l2_prefetch(P.io[0] + pf);
            l2_prefetch(P.io[1] + pf);
            l2_prefetch(P.io[2] + pf);
        }
        Q4 ux, uy, uz, hx, hy, hz;
        if (owner || (provide && !outside)) {
            interior_h<OE>(P, i, j, k0, ux, uy, uz, hx, hy, hz);
        } else if (provide) {
            hx = ldq(P.in[0] + idx);
            hy = ldq(P.in[1] + idx);
            hz = ldq(P.in[2] + idx);
        }
        if (owner) {
            stq(P.in[0] + idx, hx);
            stq(P.in[1] + idx, hy);
            stq(P.in[2] + idx, hz);
        }
        if (owner || provide) {
            sh[par][0][w][l] = make_float4(hx.v[0], hx.v[1], hx.v[2], hx.v[3]);
            sh[par][1][w][l] = make_float4(hy.v[0], hy.v[1], hy.v[2], hy.v[3]);
            sh[par][2][w][l] = make_float4(hz.v[0], hz.v[1], hz.v[2], hz.v[3]);
        }
        __syncthreads();
        if (owner) {
            // E update (split_e_quad): H(i) of the quad, of the row below
            // (z, x), of the node below the quad (y, x) and H(i − 1) (z, y).
            const float4 xj = sh[par][0][w - 1u][l], zj = sh[par][2][w - 1u][l];
            const float iym = sh[par][1][w][l - 1u].w, ixm = sh[par][0][w][l - 1u].w;
            const Q4 ixj{{xj.x, xj.y, xj.z, xj.w}}, izj{{zj.x, zj.y, zj.z, zj.w}};
            const uint32_t row = i * g.ny + j;
            const Q4 cax = ldq(lane_row(P, 0, row) + k0), cbx = ldq(lane_row(P, 3, row) + k0);
            const Q4 cay = ldq(lane_row(P, 1, row) + k0), cby = ldq(lane_row(P, 4, row) + k0);
            const Q4 caz = ldq(lane_row(P, 2, row) + k0), cbz = ldq(lane_row(P, 5, row) + k0);
            Q4 nx_, ny_, nz_;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float iy0 = e > 0 ? hy.v[e - 1] : iym, ix0 = e > 0 ? hx.v[e - 1] : ixm;
                nx_.v[e] = e_upd_t<OE>(cax.v[e], ux.v[e], cbx.v[e], hz.v[e], izj.v[e], hy.v[e], iy0);
                ny_.v[e] = e_upd_t<OE>(cay.v[e], uy.v[e], cby.v[e], hx.v[e], ix0, hz.v[e], hz_p.v[e]);
                nz_.v[e] = e_upd_t<OE>(caz.v[e], uz.v[e], cbz.v[e], hy.v[e], hy_p.v[e], hx.v[e], ixj.v[e]);
            }
            stq(P.un[0] + idx, nx_);
            stq(P.un[1] + idx, ny_);
            stq(P.un[2] + idx, nz_);
            hy_p = hy;
            hz_p = hz;
        }
        // The next plane writes the other parity; the one after it waits at
        // the next barrier, which every thread reaches only after reading
        // this plane's values.
    }
}

// The interior box of a model: every node inside all CPML layers (both
// sides), away from the domain faces; "" or why the model cannot run the
// interior schedule (hooks between the two updates other than the CPML
// correction: magnetic poles and sources; operators whose hooks read or
// write fields around the E update: lumped elements, Mur faces, openEMS PML
// layers).
inline std::string interior_box(const ems_engine_desc* d, const Grid& g, InteriorBox& B) {
    B = InteriorBox{};
    const uint32_t n[3] = {g.nx, g.ny, g.nz};
    uint32_t lo[3] = {1u, 1u, 4u};
    uint32_t hi[3] = {g.nx - 1u, g.ny - 1u, (g.nz - 1u) & ~3u};
    for (size_t k = 0; k < d->n_ops; ++k) {
        const ems_op& op = d->ops[k];
        if (op.kind == EMS_OP_CPML) {
            const auto* c = (const ems_cpml*)op.table;
            for (size_t q = 0; q < c->n_slabs; ++q) {
                const ems_cpml_slab& sl = c->slabs[q];
                const int a = sl.normal;
                if (sl.lo[a] + sl.hi[a] <= n[a]) lo[a] = std::max(lo[a], (uint32_t)sl.hi[a]);  // a low-face layer
                else hi[a] = std::min(hi[a], (uint32_t)sl.lo[a]);
            }
        } else if (op.kind == EMS_OP_POLES) {
            if (((const ems_poles*)op.table)->magnetic.n_edges) return "magnetic poles";
        } else if (op.kind == EMS_OP_SOURCE) {
            const int kind = ((const ems_source*)op.table)->kind;
            if (kind == EMS_SOFT_H || kind == EMS_HARD_H) return "magnetic sources";
        } else if (op.kind != EMS_OP_PROBE) {
            return "lumped elements, Mur faces, openEMS PML layers or conducting sheets";
        }
    }
    lo[2] = (lo[2] + 3u) & ~3u;
    hi[2] &= ~3u;
    if (hi[0] < lo[0] + 4u || hi[1] < lo[1] + 2u || hi[2] < lo[2] + 8u) return "no interior box";
    for (int a = 0; a < 3; ++a) {
        B.lo[a] = lo[a];
        B.hi[a] = hi[a];
    }
    return "";
}

// Blocks of k_interior over box B along z, y and x (chunks of `planes`).
inline void interior_blocks(const InteriorBox& B, uint32_t planes, uint32_t n[3]) {
    const uint32_t quads = (B.hi[2] - B.lo[2]) / 4u;
    n[0] = (quads + kInQuads - 1u) / kInQuads;
    n[1] = (B.hi[1] - B.lo[1] + kInRows - 1u) / kInRows;
    n[2] = (B.hi[0] - B.lo[0] + planes - 1u) / planes;
}

}  // namespace emsk
