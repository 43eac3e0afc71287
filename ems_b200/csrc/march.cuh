// march.cuh — the marching step of the B200 FDTD engine (sm_100a device code).
//
// One kernel advances the H and the E fields of the whole grid by one step,
// with the CPML corrections of both sides in line: 48 bytes of field
// traffic per node (the old u and i read once, the new ones written once)
// plus the ψ of the layer nodes, against 72 bytes for the split step. The
// old fields are read from one buffer and the new ones written into the
// other (the engine swaps them after the step), so no block ever waits for
// another.
//
// A block owns a tile of R rows × 128 z-nodes (a warp per row, four z-nodes
// per lane) and marches along x through a chunk of planes. Each plane's
// window of the old fields (u: the tile with one row below and one above and
// four z-nodes either side; i: the tile with the row below) is brought into
// shared memory by six TMA tensor copies (cp.async.bulk.tensor, out-of-grid
// entries zero-filled) into an S-stage ring, S − 1 planes ahead of the
// plane being updated. An extra warp recomputes the H values of the row
// below the tile, which the tile's E update needs (the same arithmetic gives
// the same bits), and the H values of the z-node below the tile; the H
// values of the plane before a chunk are computed again from that plane.
// Every expression is the split kernels' (split.cuh) and the CPML chain is
// the shell kernel's, so the result equals theirs and the reference's bit
// for bit. The electric poles of an edge are applied right after its E
// update and CPML correction, in the order the operators were registered,
// from the old value of the edge (u^n); the serial hooks run after this
// kernel on the new fields. Models with hooks between the two updates
// (magnetic poles and sources) or around the E update (lumped elements, Mur
// faces, openEMS PML layers) do not use it.
#pragma once

#include "../../include/ems_gpu.h"
#include "split.cuh"
#include <string>

#ifndef EMS_HOST_EMULATION
#include <cuda.h>
#endif

namespace emsk {

constexpr uint32_t kMzQuads = 32;             // quads of z-nodes of a tile row (one per lane)
constexpr uint32_t kMzNodes = 4 * kMzQuads;   // z-nodes of a tile row
constexpr uint32_t kMuW = kMzNodes + 8;       // u window row: z-nodes k0 − 4 … k0 + 131
constexpr uint32_t kMiW = kMzNodes + 4;       // i window and H tile row: z-nodes k0 − 4 … k0 + 127
constexpr uint32_t kMarchPlanes = 32;         // default planes a block marches through

// The six tensor maps of one field buffer pair's old fields: u_x, u_y, u_z
// with boxes of kMuW × (R + 2) × 1 and i_x, i_y, i_z with kMiW × (R + 1) × 1
// (z, y, x; the z extent is the padded row, so padding reads as stored).
struct MarchMaps {
    CUtensorMap u[3];
    CUtensorMap i[3];
};

__host__ __device__ constexpr uint32_t march_round128(uint32_t b) { return (b + 127u) & ~127u; }

// Shared memory of a block: S mbarriers, S stages of (u box × 3, i box × 3),
// the H tile (3 components × (R + 1) rows × kMiW).
template <uint32_t R>
struct MarchLayout {
    static constexpr uint32_t ubox = march_round128((R + 2) * kMuW * 4);
    static constexpr uint32_t ibox = march_round128((R + 1) * kMiW * 4);
    static constexpr uint32_t ubytes = (R + 2) * kMuW * 4;  // bytes a u copy delivers
    static constexpr uint32_t ibytes = (R + 1) * kMiW * 4;
    static constexpr uint32_t stage = 3 * ubox + 3 * ibox;
    static constexpr uint32_t htile = march_round128(3 * (R + 1) * kMiW * 4);
    static constexpr uint32_t bars = 128;
    static constexpr uint32_t bytes(uint32_t S) { return bars + S * stage + htile; }
};

#ifndef EMS_HOST_EMULATION
// One 3-D tensor copy global → shared, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool march_any(bool v) { return __syncthreads_or(v ? 1 : 0) != 0; }
#else
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    emu::tensor3d(dst, map, x, y, z, bar);
}
__device__ __forceinline__ bool march_any(bool v) { return emu::sync_or(v); }
#endif

__device__ __forceinline__ Q4 lds4(const float* p) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    return Q4{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ void sts4(float* p, const Q4& q) {
    *reinterpret_cast<float4*>(p) = make_float4(q.v[0], q.v[1], q.v[2], q.v[3]);
}

// The H update of the quad (p, j, k..k+3) from the staged windows, with
// the CPML correction of every existing edge: split_h_quad's and
// shell_node's arithmetic. `uo` points at the quad in the u_x window of
// plane p (the u_y and u_z windows follow at US floats, the row above at
// kMuW), `u1` at it in the u_x window of plane p + 1, `io` in the i_x
// window (i_y, i_z at IS floats). Entries that are not edges keep their old
// value. PSI: write the new ψ (the owner of the node; a recomputation for a
// neighbour does not).
template <bool OE, bool PSI, uint32_t US, uint32_t IS>
__device__ __forceinline__ void march_h(const FusedParams& P, uint32_t p, uint32_t j, uint32_t k, const float* uo,
                                        const float* u1, const float* io, Q4& ux, Q4& uy, Q4& uz, Q4& nx_, Q4& ny_,
                                        Q4& nz_) {
    const Grid& g = P.g;
    ux = lds4(uo);
    uy = lds4(uo + US);
    uz = lds4(uo + 2 * US);
    const Q4 uzj = lds4(uo + 2 * US + kMuW), uxj = lds4(uo + kMuW);
    const float uy4 = uo[US + 4], ux4 = uo[4];
    const Q4 uzi = lds4(u1 + 2 * US), uyi = lds4(u1 + US);
    const Q4 hx = lds4(io), hy = lds4(io + IS), hz = lds4(io + 2 * IS);
    const uint32_t row = p * g.ny + j;
    const Q4 dax = ldq(lane_row(P, 6, row) + k), dbx = ldq(lane_row(P, 9, row) + k);
    const Q4 day = ldq(lane_row(P, 7, row) + k), dby = ldq(lane_row(P, 10, row) + k);
    const Q4 daz = ldq(lane_row(P, 8, row) + k), dbz = ldq(lane_row(P, 11, row) + k);
    const bool jn = j + 1 < g.ny, in_ = p + 1 < g.nx;
    const uint32_t cm = P.cmask[0][p] | P.cmask[1][j];
    nx_ = hx;
    ny_ = hy;
    nz_ = hz;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const uint32_t kk = k + e;
        if (kk >= g.nz) break;
        const bool kn = kk + 1 < g.nz;
        const uint32_t bits = cm | P.cmask[2][kk];
        const float uy1 = e < 3 ? uy.v[e + 1] : uy4, ux1 = e < 3 ? ux.v[e + 1] : ux4;
        if (jn && kn) {
            float t = h_upd_t<OE>(dax.v[e], hx.v[e], dbx.v[e], uzj.v[e], uz.v[e], uy1, uy.v[e]);
            if (bits & 0xfu)
                t = cpml_apply<PSI, 0, 0>(P, bits, p, j, kk, t, -dbx.v[e], __fsub_rn(uzj.v[e], uz.v[e]),
                                          __fmul_rn(-1.0f, __fsub_rn(uy1, uy.v[e])));
            nx_.v[e] = t;
        }
        if (in_ && kn) {
            float t = h_upd_t<OE>(day.v[e], hy.v[e], dby.v[e], ux1, ux.v[e], uzi.v[e], uz.v[e]);
            if (bits & 0xf0u)
                t = cpml_apply<PSI, 0, 1>(P, bits, p, j, kk, t, -dby.v[e], __fsub_rn(ux1, ux.v[e]),
                                          __fmul_rn(-1.0f, __fsub_rn(uzi.v[e], uz.v[e])));
            ny_.v[e] = t;
        }
        if (in_ && jn) {
            float t = h_upd_t<OE>(daz.v[e], hz.v[e], dbz.v[e], uyi.v[e], uy.v[e], uxj.v[e], ux.v[e]);
            if (bits & 0xf00u)
                t = cpml_apply<PSI, 0, 2>(P, bits, p, j, kk, t, -dbz.v[e], __fsub_rn(uyi.v[e], uy.v[e]),
                                          __fmul_rn(-1.0f, __fsub_rn(uxj.v[e], ux.v[e])));
            nz_.v[e] = t;
        }
    }
}

// The x and y H values of the single node (p, j, k) (k ≥ 0), which the E
// update of the node above it reads: the arithmetic of march_h without
// writing ψ. `uo` points at the node in the u_x window of plane p.
template <bool OE, uint32_t US, uint32_t IS>
__device__ __forceinline__ void march_h_node(const FusedParams& P, uint32_t p, uint32_t j, uint32_t k,
                                             const float* uo, const float* u1, const float* io, float& hx_n,
                                             float& hy_n) {
    const Grid& g = P.g;
    const uint32_t row = p * g.ny + j;
    const float ux = uo[0], uy = uo[US], uz = uo[2 * US];
    const float uzj = uo[2 * US + kMuW], uy1 = uo[US + 1], ux1 = uo[1], uzi = u1[2 * US];
    const bool jn = j + 1 < g.ny, in_ = p + 1 < g.nx, kn = k + 1 < g.nz;
    const uint32_t bits = P.cmask[0][p] | P.cmask[1][j] | P.cmask[2][k];
    hx_n = io[0];
    hy_n = io[IS];
    if (jn && kn) {
        const float db = lane_row(P, 9, row)[k];
        float t = h_upd_t<OE>(lane_row(P, 6, row)[k], hx_n, db, uzj, uz, uy1, uy);
        if (bits & 0xfu)
            t = cpml_apply<false, 0, 0>(P, bits, p, j, k, t, -db, __fsub_rn(uzj, uz), __fmul_rn(-1.0f, __fsub_rn(uy1, uy)));
        hx_n = t;
    }
    if (in_ && kn) {
        const float db = lane_row(P, 10, row)[k];
        float t = h_upd_t<OE>(lane_row(P, 7, row)[k], hy_n, db, ux1, ux, uzi, uz);
        if (bits & 0xf0u)
            t = cpml_apply<false, 0, 1>(P, bits, p, j, k, t, -db, __fsub_rn(ux1, ux), __fmul_rn(-1.0f, __fsub_rn(uzi, uz)));
        hy_n = t;
    }
}

// The slab hooks of the E edge of component C at (p, j, k) after its
// update t, in registration order (the two-kernel schedule's hooks): the
// CPML correction with the curl differences A and B, and the electric poles
// of the edge's run starting from u^n = `prev`.
template <int C>
__device__ __forceinline__ float march_e_hooks(const FusedParams& P, uint32_t bits, const uint4& rr, uint32_t p,
                                               uint32_t j, uint32_t k, float t, float cb, float A, float B,
                                               float prev) {
    const bool in_runs = k >= rr.z && k < rr.w;
    if (P.poles_first && in_runs) t = poles_run(P.runs, P.sets, P.pj, P.pq, P.dt, rr, k, t, prev, cb, nullptr);
    if (bits & (0xfu << (12 + 4 * C))) t = cpml_apply<true, 1, C>(P, bits, p, j, k, t, cb, A, __fmul_rn(-1.0f, B));
    if (!P.poles_first && in_runs) t = poles_run(P.runs, P.sets, P.pj, P.pq, P.dt, rr, k, t, prev, cb, nullptr);
    return t;
}

// Grid: (z tiles of kMzNodes over the padded row, y tiles of R rows, x
// chunks of `planes`); block: R + 1 warps. Warp 0 recomputes the H row below
// the tile (and lanes 0..R−1 of it the node below the tile of rows
// 0..R−1); warp w ≥ 1 owns row j0 + w − 1. A bounded wait that runs out
// sets P.status and the block returns.
template <uint32_t R, uint32_t S, bool OE>
__global__ void __launch_bounds__(32 * (R + 1), 2) k_march(const __grid_constant__ FusedParams P,
                                                           const __grid_constant__ MarchMaps M, uint32_t planes) {
    using L = MarchLayout<R>;
    constexpr uint32_t US = L::ubox / 4, IS = L::ibox / 4, HS = (R + 1) * kMiW;
    EMS_DYNAMIC_SMEM(smem);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    float* ring = reinterpret_cast<float*>(smem + L::bars);
    float* ht = reinterpret_cast<float*>(smem + L::bars + S * L::stage);
    const Grid& g = P.g;
    const uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31u;
    const uint32_t j0 = blockIdx.y * R, k0 = blockIdx.x * kMzNodes;
    const int jr = (int)j0 + (int)w - 1;  // this warp's row (warp 0: the row below the tile)
    const uint32_t k = k0 + 4u * l;
    const uint32_t xs = blockIdx.z * planes;
    const uint32_t xe = min(xs + planes, g.nx);
    const uint32_t q0 = xs ? xs - 1u : 0u;  // the first plane loaded
    const uint32_t last = xe;               // the last plane loaded (u of the plane after the chunk)
    const bool row_ok = jr >= 0 && jr < (int)g.ny;
    const bool quad_ok = k < g.pitch;
    const bool owner = w > 0 && row_ok && quad_ok;
    // Lanes 0..R−1 of warp 0: the node k0 − 1 of row j0 + l.
    const int jz = (int)j0 + (int)l;
    const bool zfeed = w == 0 && l < R && k0 > 0 && jz < (int)g.ny;
    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < S; ++s) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto stage_of = [&](uint32_t q) { return (q - q0) % S; };
    // Test hook: the first block arms its first barrier with more bytes than
    // its copies deliver (every copy lands; the phase never completes).
    const uint32_t extra = blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 ? P.test_extra_tx : 0u;
    const uint64_t limit = P.wait_ns ? P.wait_ns : kWaitNs;
    auto issue = [&](uint32_t q) {
        uint64_t* b = &bar[stage_of(q)];
        float* st = ring + stage_of(q) * (L::stage / 4);
        mbar_expect_tx(b, 3 * L::ubytes + 3 * L::ibytes + (q == q0 ? extra : 0u));
        for (int c = 0; c < 3; ++c)
            tma_load_3d(st + c * US, &M.u[c], (int)k0 - 4, (int)j0 - 1, (int)q, b);
        for (int c = 0; c < 3; ++c)
            tma_load_3d(st + 3 * US + c * IS, &M.i[c], (int)k0 - 4, (int)j0 - 1, (int)q, b);
    };
    auto parity = [&](uint32_t q) { return ((q - q0) / S) & 1u; };
    static_assert(S >= 3, "the ring must hold planes p and p + 1 while p + 2 loads");
    uint32_t issued = q0;  // thread 0: planes below this one are issued
    if (threadIdx.x == 0)
        for (; issued <= last && issued < q0 + S - 1; ++issued) issue(issued);
    // H of the plane before, y and z components, of the owned quad.
    Q4 hy_p = zq(), hz_p = zq();
    const uint32_t sj = g.pitch, si = g.ny * g.pitch;
    for (uint32_t p = q0; p < xe; ++p) {
        bool ok = true;
        if (threadIdx.x == 0)
            ok = mbar_wait(&bar[stage_of(p)], parity(p), limit) && mbar_wait(&bar[stage_of(p + 1)], parity(p + 1), limit);
        if (march_any(!ok)) {
            if (threadIdx.x == 0) {
                atomicExch(P.status, 1);
                // Let the copies still in flight land (each wait bounded)
                // before the block's shared memory is given up.
                for (uint32_t q = p; q < issued; ++q) mbar_wait(&bar[stage_of(q)], parity(q), limit);
            }
            return;
        }
        // Stage p − 1 is free: every thread has left the iteration that read it.
        if (threadIdx.x == 0 && p + S - 1 <= last) issue(issued++);
        const float* st0 = ring + stage_of(p) * (L::stage / 4);
        const float* st1 = ring + stage_of(p + 1) * (L::stage / 4);
        const bool warm = p < xs;  // the plane before the chunk: H values only
        Q4 ux = zq(), uy = zq(), uz = zq(), hx = zq(), hy = zq(), hz = zq();
        const uint32_t zoff = 4u + 4u * l;
        if (row_ok && quad_ok) {
            const float* uo = st0 + w * kMuW + zoff;
            const float* u1 = st1 + w * kMuW + zoff;
            const float* io = st0 + 3 * US + w * kMiW + zoff;
            if (owner && !warm)
                march_h<OE, true, US, IS>(P, p, (uint32_t)jr, k, uo, u1, io, ux, uy, uz, hx, hy, hz);
            else
                march_h<OE, false, US, IS>(P, p, (uint32_t)jr, k, uo, u1, io, ux, uy, uz, hx, hy, hz);
        }
        if (warm) {
            hy_p = hy;
            hz_p = hz;
            continue;  // the next iteration's barrier orders the ring
        }
        float* hrow = ht + w * kMiW + zoff;
        sts4(hrow, hx);
        sts4(hrow + HS, hy);
        sts4(hrow + 2 * HS, hz);
        float zx = 0.0f, zy = 0.0f;
        if (zfeed) {
            // Node k0 − 1 of row jz: window row jz − j0 + 1, z offset 3.
            const uint32_t tr = (uint32_t)(jz - (int)j0) + 1u;
            march_h_node<OE, US, IS>(P, p, (uint32_t)jz, k0 - 1u, st0 + tr * kMuW + 3u, st1 + tr * kMuW + 3u,
                                     st0 + 3 * US + tr * kMiW + 3u, zx, zy);
        }
        if (w == 0 && l < R) {
            ht[(l + 1) * kMiW + 3] = zx;  // zero where the tile starts at k = 0
            ht[HS + (l + 1) * kMiW + 3] = zy;
        }
        if (owner) {
            const uint32_t idx = p * si + (uint32_t)jr * sj + k;
            stq(P.in[0] + idx, hx);
            stq(P.in[1] + idx, hy);
            stq(P.in[2] + idx, hz);
        }
        __syncthreads();
        if (owner) {
            // E update (split_e_quad), its CPML correction and its electric
            // poles in registration order: H of the quad, of the row below
            // (z, x), of the node below the quad (y, x) and of the plane
            // before (z, y); the poles start from u^n, the old value.
            const uint32_t j = (uint32_t)jr;
            const Q4 izj = lds4(hrow - kMiW + 2 * HS), ixj = lds4(hrow - kMiW);
            const float iym = hrow[HS - 1], ixm = hrow[-1];
            const uint32_t row = p * g.ny + j;
            const Q4 cax = ldq(lane_row(P, 0, row) + k), cbx = ldq(lane_row(P, 3, row) + k);
            const Q4 cay = ldq(lane_row(P, 1, row) + k), cby = ldq(lane_row(P, 4, row) + k);
            const Q4 caz = ldq(lane_row(P, 2, row) + k), cbz = ldq(lane_row(P, 5, row) + k);
            const uint4 rrx = row_runs(P.row_runs, P.has_poles, p, 0, g.ny, j);
            const uint4 rry = row_runs(P.row_runs, P.has_poles, p, 1, g.ny, j);
            const uint4 rrz = row_runs(P.row_runs, P.has_poles, p, 2, g.ny, j);
            const bool xi = p + 1 < g.nx, yj = j + 1 < g.ny;
            const uint32_t cm = P.cmask[0][p] | P.cmask[1][j];
            Q4 nx_ = ux, ny_ = uy, nz_ = uz;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const uint32_t kk = k + e;
                if (kk >= g.nz) break;
                const uint32_t bits = cm | P.cmask[2][kk];
                const float iy0 = e > 0 ? hy.v[e - 1] : iym, ix0 = e > 0 ? hx.v[e - 1] : ixm;
                if (xi)
                    nx_.v[e] = march_e_hooks<0>(P, bits, rrx, p, j, kk,
                                                e_upd_t<OE>(cax.v[e], ux.v[e], cbx.v[e], hz.v[e], izj.v[e], hy.v[e], iy0),
                                                cbx.v[e], __fsub_rn(hz.v[e], izj.v[e]), __fsub_rn(hy.v[e], iy0), ux.v[e]);
                if (yj)
                    ny_.v[e] = march_e_hooks<1>(P, bits, rry, p, j, kk,
                                                e_upd_t<OE>(cay.v[e], uy.v[e], cby.v[e], hx.v[e], ix0, hz.v[e], hz_p.v[e]),
                                                cby.v[e], __fsub_rn(hx.v[e], ix0), __fsub_rn(hz.v[e], hz_p.v[e]), uy.v[e]);
                if (kk + 1 < g.nz)
                    nz_.v[e] = march_e_hooks<2>(P, bits, rrz, p, j, kk,
                                                e_upd_t<OE>(caz.v[e], uz.v[e], cbz.v[e], hy.v[e], hy_p.v[e], hx.v[e], ixj.v[e]),
                                                cbz.v[e], __fsub_rn(hy.v[e], hy_p.v[e]), __fsub_rn(hx.v[e], ixj.v[e]), uz.v[e]);
            }
            const uint32_t idx = p * si + j * sj + k;
            stq(P.un[0] + idx, nx_);
            stq(P.un[1] + idx, ny_);
            stq(P.un[2] + idx, nz_);
            // A non-finite value makes x·0 NaN: one flag for the host's next check.
            float z = 0.0f;
#pragma unroll
            for (int e = 0; e < 4; ++e)
                z = __fadd_rn(z, __fadd_rn(__fmul_rn(nx_.v[e], 0.0f), __fadd_rn(__fmul_rn(ny_.v[e], 0.0f),
                                                                                   __fmul_rn(nz_.v[e], 0.0f))));
            if (z != z && P.diverged) atomicExch(P.diverged, 1);
        }
        hy_p = hy;
        hz_p = hz;
    }
}

// Why a model cannot run the marching step ("" if it can): the hooks
// between the two updates (magnetic poles and sources), or operators whose
// hooks read or write fields around the E update (lumped elements, Mur
// faces, openEMS PML layers).
inline std::string march_why(const ems_engine_desc* d) {
    for (size_t k = 0; k < d->n_ops; ++k) {
        const ems_op& op = d->ops[k];
        if (op.kind == EMS_OP_CPML) {
        } else if (op.kind == EMS_OP_POLES) {
            if (((const ems_poles*)op.table)->magnetic.n_edges) return "magnetic poles";
        } else if (op.kind == EMS_OP_SOURCE) {
            const int kind = ((const ems_source*)op.table)->kind;
            if (kind == EMS_SOFT_H || kind == EMS_HARD_H) return "magnetic sources";
        } else if (op.kind != EMS_OP_PROBE) {
            return "lumped elements, Mur faces or openEMS PML layers";
        }
    }
    if (d->nodes[0] < 2 || d->nodes[1] < 2 || d->nodes[2] < 2) return "grid too small";
    return "";
}

// Blocks of k_march along z, y and x (chunks of `planes`).
inline void march_blocks(const Grid& g, uint32_t R, uint32_t planes, uint32_t n[3]) {
    n[0] = (g.pitch + kMzNodes - 1) / kMzNodes;
    n[1] = (g.ny + R - 1) / R;
    n[2] = (g.nx + planes - 1) / planes;
}

}  // namespace emsk
