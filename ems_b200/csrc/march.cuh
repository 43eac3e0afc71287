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
// window of the old fields (u: the tile with one row below and one above,
// i: the tile with the row below; four z-nodes either side) is brought into
// shared memory by six TMA tensor copies (cp.async.bulk.tensor, out-of-grid
// entries zero-filled) into an S-stage ring, S − 2 planes ahead of the ones
// being read. An extra warp recomputes the H values of the row below the
// tile, which the tile's E update needs (the same arithmetic gives the same
// bits), and the H values of the z-node below the tile; the H values of the
// plane before a chunk are computed again from that plane.
//
// The updates run for every node without any hook; then each warp applies
// the CPML chains of its row (after the H update, and after the E update)
// to exactly the nodes in a layer, one (node, component) per lane, the
// operands read back from shared memory: the H values of the plane (and of
// the plane before, in a second tile) and the new E values (in the i window
// of the plane, free by then). So the layers at the ends of every row cost
// a few lanes of one pass, not a divergent copy of the whole update. The
// electric poles run after this kernel, on the new fields, as the pole
// kernel of the split schedule with u^n from the old buffer. Every
// expression is the split kernels' (split.cuh) and the CPML chain the shell
// kernel's, so the result equals theirs and the reference's bit for bit. The electric poles of an edge are applied right after its E
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

constexpr uint32_t kMzQuads = 32;            // quads of z-nodes of a tile row (one per lane)
constexpr uint32_t kMzNodes = 4 * kMzQuads;  // z-nodes of a tile row
constexpr uint32_t kMW = kMzNodes + 8;       // window and tile rows: z-nodes k0 − 4 … k0 + 131
constexpr uint32_t kMarchPlanes = 32;        // default planes a block marches through

// The six tensor maps of one field buffer's old fields: u_x, u_y, u_z with
// boxes of kMW × (R + 2) × 1 and i_x, i_y, i_z with kMW × (R + 1) × 1 (z, y,
// x; the z extent is the padded row, so padding reads as stored).
struct MarchMaps {
    CUtensorMap u[3];
    CUtensorMap i[3];
};

__host__ __device__ constexpr uint32_t march_round128(uint32_t b) { return (b + 127u) & ~127u; }

// Shared memory of a block: S mbarriers, S stages of (u box × 3, i box × 3),
// the H tile of the plane (3 components × (R + 1) rows × kMW), the y and z
// H values of the plane before (2 × (R + 1) rows × kMW), the block's z
// window of each coefficient lane's background row (12 × kMW) and of the
// z-layer masks (kMW).
template <uint32_t R>
struct MarchLayout {
    static constexpr uint32_t ubytes = (R + 2) * kMW * 4;  // bytes a u copy delivers
    static constexpr uint32_t ibytes = (R + 1) * kMW * 4;
    static constexpr uint32_t ubox = march_round128(ubytes);
    static constexpr uint32_t ibox = march_round128(ibytes);
    static constexpr uint32_t stage = 3 * ubox + 3 * ibox;
    static constexpr uint32_t htile = march_round128(3 * (R + 1) * kMW * 4);
    static constexpr uint32_t hptile = march_round128(2 * (R + 1) * kMW * 4);
    static constexpr uint32_t bgtile = march_round128(12 * kMW * 4);
    static constexpr uint32_t cztile = march_round128(kMW * 4);
    static constexpr uint32_t bars = 128;
    static constexpr uint32_t bytes(uint32_t S) { return bars + S * stage + htile + hptile + bgtile + cztile; }
    // Blocks of S stages that fit one SM's 228 KiB of shared memory (1 KiB
    // of it reserved per block): the occupancy the launch bounds ask for.
    static constexpr uint32_t blocks(uint32_t S) { return 233472u / (bytes(S) + 1024u); }
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
__device__ __forceinline__ void march_syncwarp() { __syncwarp(); }
#else
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    emu::tensor3d(dst, map, x, y, z, bar);
}
__device__ __forceinline__ bool march_any(bool v) { return emu::sync_or(v); }
__device__ __forceinline__ void march_syncwarp() { emu::syncwarp(); }
#endif

__device__ __forceinline__ Q4 lds4(const float* p) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    return Q4{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ void sts4(float* p, const Q4& q) {
    *reinterpret_cast<float4*>(p) = make_float4(q.v[0], q.v[1], q.v[2], q.v[3]);
}

// The CPML chain of component C on side SIDE by the slabs whose bits are set
// in `bits`, in application order (cpml_apply, inline).
template <bool WRITE, int SIDE, int C>
__device__ __forceinline__ float march_cpml(const FusedParams& P, uint32_t bits, uint32_t i, uint32_t j, uint32_t k,
                                            float t, float coef, float sA, float sB) {
    uint32_t m = (bits >> (SIDE * 12 + C * 4)) & 15u;
    while (m) {
        const int q = __ffs(m) - 1;
        m &= m - 1;
        t = cpml_body_inl<WRITE>(&P.slab[SIDE][C][q], 1, i, j, k, C, t, coef, sA, sB);
    }
    return t;
}

// The row ids of the twelve coefficient lanes for the (x, y) row `row`
// (0 for a dense lane), loaded one plane ahead of their use.
__device__ __forceinline__ void march_rids(const FusedParams& P, uint32_t row, uint32_t (&r)[12]) {
#pragma unroll
    for (int ln = 0; ln < 12; ++ln) r[ln] = P.lane[ln].dense ? 0u : __ldg(P.lane[ln].rid + row);
}

// The coefficient quad of lane `ln` at (row, k..k+3): the block's copy of
// the lane's background row (`bgq`: that tile at the quad) when the row uses
// it, else the pooled row or the dense array in global memory.
__device__ __forceinline__ Q4 march_coef4(const FusedParams& P, int ln, uint32_t rid, uint32_t row, uint32_t k,
                                          const float* bgq) {
    const Lane& L = P.lane[ln];
    if (L.dense) return ldq(L.dense + (size_t)row * P.g.pitch + k);
    if (rid == L.bg) return lds4(bgq + ln * kMW);
    return ldq(L.rows + (size_t)rid * P.g.pitch + k);
}
__device__ __forceinline__ float march_coef1(const FusedParams& P, int ln, uint32_t rid, uint32_t row, uint32_t k,
                                             const float* bgz) {
    const Lane& L = P.lane[ln];
    if (L.dense) return L.dense[(size_t)row * P.g.pitch + k];
    if (rid == L.bg) return bgz[ln * kMW];
    return L.rows[(size_t)rid * P.g.pitch + k];
}

// Window and tile addressing: component c's plane of a u window, an i
// window or an H tile starts at c × (its box / 4) floats; row r (r = 0: the
// row below the tile) at r × kMW; z-node k0 − 4 + z at z.

// The update of component C of the H quad (p, j, k..k+3), no hooks:
// split_h_quad's arithmetic, operands from the staged windows (`uo` the
// quad's entry in plane p's u_x window, `u1` in plane p + 1's, `io` in the
// i_x window), the new values (old ones where an entry is not an edge) to
// `hout`, the quad's entry in the H_x tile.
template <int C, bool OE, uint32_t US, uint32_t IS, uint32_t HS>
__device__ __forceinline__ void march_h_upd(const FusedParams& P, uint32_t p, uint32_t j, uint32_t k, bool all,
                                            const uint32_t (&rid)[12], const float* bgq, const float* uo,
                                            const float* u1, const float* io, float* hout) {
    const Grid& g = P.g;
    // (a − b) − (c − d): a, b along next(C), c, d along prev(C).
    const float* ap = C == 0 ? uo + 2 * US + kMW : (C == 1 ? uo : u1 + US);
    const float* bp = C == 0 ? uo + 2 * US : (C == 1 ? uo : uo + US);
    const float* cp = C == 0 ? uo + US : (C == 1 ? u1 + 2 * US : uo + kMW);
    const float* dp = C == 0 ? uo + US : (C == 1 ? uo + 2 * US : uo);
    const Q4 a = lds4(ap), b = lds4(bp), c = lds4(cp), d = lds4(dp);
    const float a4 = C == 1 ? ap[4] : 0.0f, c4 = C == 0 ? cp[4] : 0.0f;  // the node after the quad
    const Q4 h = lds4(io + C * IS);
    const uint32_t row = p * g.ny + j;
    const Q4 da = march_coef4(P, 6 + C, rid[6 + C], row, k, bgq), db = march_coef4(P, 9 + C, rid[9 + C], row, k, bgq);
    const bool exists_pj = C == 0 ? j + 1 < g.ny : (C == 1 ? p + 1 < g.nx : (p + 1 < g.nx && j + 1 < g.ny));
    Q4 out = h;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float av = C == 1 ? (e < 3 ? a.v[e + 1] : a4) : a.v[e];
        const float cv = C == 0 ? (e < 3 ? c.v[e + 1] : c4) : c.v[e];
        const float t = h_upd_t<OE>(da.v[e], h.v[e], db.v[e], av, b.v[e], cv, d.v[e]);
        // all: every edge of the quad exists (the common case).
        if (all || (exists_pj && (C == 2 ? k + e < g.nz : k + e + 1 < g.nz))) out.v[e] = t;
    }
    sts4(hout + C * HS, out);
}

// The update of component C of the E quad (p, j, k..k+3), no hooks:
// split_e_quad's arithmetic, the H operands from the H tile of this plane
// (`hq` the quad's entry in the H_x tile; the row below at −kMW, the node
// below at −1) and of the plane before (`hp`), the old u from `uq` (the
// quad's entry in plane p's u_x window); the new values to `eout` (the
// quad's entry in the E_x tile).
template <int C, bool OE, uint32_t US, uint32_t HS, uint32_t PS>
__device__ __forceinline__ void march_e_upd(const FusedParams& P, uint32_t p, uint32_t j, uint32_t k, bool all,
                                            const uint32_t (&rid)[12], const float* bgq, const float* uq,
                                            const float* hq, const float* hp, float* eout) {
    const Grid& g = P.g;
    // x: (hz − hz(j−1)) − (hy − hy(k−1)); y: (hx − hx(k−1)) − (hz − hz(i−1));
    // z: (hy − hy(i−1)) − (hx − hx(j−1)).
    const float* ap = C == 0 ? hq + 2 * HS : (C == 1 ? hq : hq + HS);
    const float* cp = C == 0 ? hq + HS : (C == 1 ? hq + 2 * HS : hq);
    const Q4 a = lds4(ap), c = lds4(cp);
    // hp: the y and z H values of the plane before (H_y, H_z at PS floats apart).
    const Q4 b = C == 0 ? lds4(ap - kMW) : (C == 1 ? zq() : lds4(hp));
    const Q4 d = C == 0 ? zq() : (C == 1 ? lds4(hp + PS) : lds4(cp - kMW));
    const float bm = C == 1 ? ap[-1] : 0.0f, dm = C == 0 ? cp[-1] : 0.0f;  // the node below the quad
    const Q4 u = lds4(uq + C * US);
    const uint32_t row = p * g.ny + j;
    const Q4 ca = march_coef4(P, C, rid[C], row, k, bgq), cb = march_coef4(P, 3 + C, rid[3 + C], row, k, bgq);
    const bool exists_pj = C == 0 ? p + 1 < g.nx : (C == 1 ? j + 1 < g.ny : true);
    Q4 out = u;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const float bv = C == 1 ? (e > 0 ? a.v[e - 1] : bm) : b.v[e];
        const float dv = C == 0 ? (e > 0 ? c.v[e - 1] : dm) : d.v[e];
        const float t = e_upd_t<OE>(ca.v[e], u.v[e], cb.v[e], a.v[e], bv, c.v[e], dv);
        if (all || (exists_pj && (C == 2 ? k + e + 1 < g.nz : k + e < g.nz))) out.v[e] = t;
    }
    sts4(eout + C * HS, out);
}

// Disjoint intervals of z-node offsets (within a tile) whose nodes a warp
// visits after an update; counts in nodes. At most six: the two z layers
// of a side, and one run span per component, unmerged at worst.
struct MarchSpans {
    uint32_t lo[6], hi[6];
    uint32_t n;  // intervals
    uint32_t nodes;
    // Adds [a, b), merging every interval it overlaps or touches, so that no
    // node is listed twice.
    __device__ __forceinline__ void add(uint32_t a, uint32_t b) {
        if (a >= b) return;
        uint32_t q = 0;
        while (q < n) {
            if (a <= hi[q] && b >= lo[q]) {
                a = min(a, lo[q]);
                b = b > hi[q] ? b : hi[q];
                nodes -= hi[q] - lo[q];
                --n;
                lo[q] = lo[n];
                hi[q] = hi[n];
                q = 0;  // the wider interval may meet one already passed
            } else {
                ++q;
            }
        }
        lo[n] = a;
        hi[n] = b;
        nodes += b - a;
        ++n;
    }
    // The offset of the v-th node of the intervals.
    __device__ __forceinline__ uint32_t at(uint32_t v) const {
        uint32_t q = 0;
        while (q + 1 < n && v >= hi[q] - lo[q]) {
            v -= hi[q] - lo[q];
            ++q;
        }
        return lo[q] + v;
    }
};

// The z offsets [k0, k0 + nodes) of a tile that the CPML slabs normal to z
// of side SIDE hold (slabs span the grid on their other axes).
template <int SIDE>
__device__ __forceinline__ void march_z_layers(const FusedParams& P, uint32_t k0, uint32_t nodes, MarchSpans& S) {
    for (int c = 0; c < 3; ++c)
        for (int q = 0; q < P.nslab[SIDE][c]; ++q) {
            const FSlab& s = P.slab[SIDE][c][q];
            if (s.normal != 2) continue;
            const uint32_t a = s.lo[2] > k0 ? s.lo[2] - k0 : 0u;
            const uint32_t b = s.hi[2] > k0 ? min(s.hi[2] - k0, nodes) : 0u;
            S.add(a, b);
        }
}

// The H-side CPML chain of (node k0 + z, component c) of the warp's row j,
// if the node's edge exists and lies in a layer, on the value in the H
// tile (`ht` the H_x tile at the warp's row, z-node k0 − 4 at 0), the
// curl differences from the u windows (`uw`, `u1` at the warp's row).
template <bool OE, uint32_t US, uint32_t HS>
__device__ __forceinline__ void march_h_fix(const FusedParams& P, bool psi, uint32_t p, uint32_t j, uint32_t kk,
                                            uint32_t z, int c, uint32_t cm, const uint32_t* czs,
                                            const uint32_t (&rid)[12], const float* bgs, const float* uw,
                                            const float* u1, float* ht) {
    const Grid& g = P.g;
    const uint32_t bits = cm | czs[z + 4u];
    if (!((bits >> (4 * c)) & 15u)) return;
    const bool jn = j + 1 < g.ny, in_ = p + 1 < g.nx, kn = kk + 1 < g.nz;
    const uint32_t w = z + 4u;  // window column
    const uint32_t row = p * g.ny + j;
    float* t = ht + c * HS + w;
    if (c == 0 && jn && kn) {
        const float A = __fsub_rn(uw[2 * US + kMW + w], uw[2 * US + w]), B = __fsub_rn(uw[US + w + 1], uw[US + w]);
        const float db = march_coef1(P, 9, rid[9], row, kk, bgs + w);
        *t = psi ? march_cpml<true, 0, 0>(P, bits, p, j, kk, *t, -db, A, __fmul_rn(-1.0f, B))
                 : march_cpml<false, 0, 0>(P, bits, p, j, kk, *t, -db, A, __fmul_rn(-1.0f, B));
    } else if (c == 1 && in_ && kn) {
        const float A = __fsub_rn(uw[w + 1], uw[w]), B = __fsub_rn(u1[2 * US + w], uw[2 * US + w]);
        const float db = march_coef1(P, 10, rid[10], row, kk, bgs + w);
        *t = psi ? march_cpml<true, 0, 1>(P, bits, p, j, kk, *t, -db, A, __fmul_rn(-1.0f, B))
                 : march_cpml<false, 0, 1>(P, bits, p, j, kk, *t, -db, A, __fmul_rn(-1.0f, B));
    } else if (c == 2 && in_ && jn) {
        const float A = __fsub_rn(u1[US + w], uw[US + w]), B = __fsub_rn(uw[kMW + w], uw[w]);
        const float db = march_coef1(P, 11, rid[11], row, kk, bgs + w);
        *t = psi ? march_cpml<true, 0, 2>(P, bits, p, j, kk, *t, -db, A, __fmul_rn(-1.0f, B))
                 : march_cpml<false, 0, 2>(P, bits, p, j, kk, *t, -db, A, __fmul_rn(-1.0f, B));
    }
}

// The E-side CPML chain of (node k0 + z, component c) of the warp's row j,
// if the node's edge exists and lies in a layer, with the curl differences
// from the H tiles (`ht` this plane's, `hp` the plane before's, at the
// warp's row), on the new value in the E tile (`et`).
template <bool OE, uint32_t US, uint32_t HS, uint32_t PS>
__device__ __forceinline__ void march_e_fix(const FusedParams& P, uint32_t p, uint32_t j, uint32_t kk, uint32_t z,
                                            int c, uint32_t cm, const uint32_t* czs, const uint32_t (&rid)[12],
                                            const float* bgs, const float* ht, const float* hp, float* et) {
    const Grid& g = P.g;
    const bool exists = c == 0 ? p + 1 < g.nx : (c == 1 ? j + 1 < g.ny : kk + 1 < g.nz);
    if (!exists) return;
    const uint32_t bits = cm | czs[z + 4u];
    if (!((bits >> (12 + 4 * c)) & 15u)) return;
    const uint32_t w = z + 4u;
    const uint32_t row = p * g.ny + j;
    const float cb = march_coef1(P, 3 + c, c == 0 ? rid[3] : (c == 1 ? rid[4] : rid[5]), row, kk, bgs + w);
    const float* hb = ht - kMW;  // the row below
    float A, B;
    if (c == 0) {
        A = __fsub_rn(ht[2 * HS + w], hb[2 * HS + w]);
        B = __fsub_rn(ht[HS + w], ht[HS + w - 1]);
    } else if (c == 1) {
        A = __fsub_rn(ht[w], ht[w - 1]);
        B = __fsub_rn(ht[2 * HS + w], hp[PS + w]);
    } else {
        A = __fsub_rn(ht[HS + w], hp[w]);
        B = __fsub_rn(ht[w], hb[w]);
    }
    float t = et[c * HS + w];
    const float sB = __fmul_rn(-1.0f, B);
    t = c == 0 ? march_cpml<true, 1, 0>(P, bits, p, j, kk, t, cb, A, sB)
               : (c == 1 ? march_cpml<true, 1, 1>(P, bits, p, j, kk, t, cb, A, sB)
                         : march_cpml<true, 1, 2>(P, bits, p, j, kk, t, cb, A, sB));
    et[c * HS + w] = t;
}

// The x and y H values of the single node (p, j, k), k ≥ 0, which the E
// update of the node above it reads: the update and its CPML chain without
// writing ψ. `uo` points at the node in plane p's u_x window.
template <bool OE, uint32_t US, uint32_t IS>
__device__ __forceinline__ void march_h_node(const FusedParams& P, uint32_t p, uint32_t j, uint32_t k,
                                             const uint32_t (&zr)[4], const float* uo, const float* u1,
                                             const float* io, float& hx_n, float& hy_n) {
    const Grid& g = P.g;
    const uint32_t row = p * g.ny + j;
    // zr: the row ids of lanes 6, 7, 9, 10 (da_x, da_y, db_x, db_y) for this row.
    const Lane *l6 = &P.lane[6], *l7 = &P.lane[7], *l9 = &P.lane[9], *l10 = &P.lane[10];
    auto at = [&](const Lane* L, uint32_t r) {
        return L->dense ? L->dense[(size_t)row * g.pitch + k] : L->rows[(size_t)r * g.pitch + k];
    };
    const float ux = uo[0], uy = uo[US], uz = uo[2 * US];
    const float uzj = uo[2 * US + kMW], uy1 = uo[US + 1], ux1 = uo[1], uzi = u1[2 * US];
    const bool jn = j + 1 < g.ny, in_ = p + 1 < g.nx, kn = k + 1 < g.nz;
    const uint32_t bits = P.cmask[0][p] | P.cmask[1][j] | P.cmask[2][k];
    hx_n = io[0];
    hy_n = io[IS];
    if (jn && kn) {
        const float db = at(l9, zr[2]);
        float t = h_upd_t<OE>(at(l6, zr[0]), hx_n, db, uzj, uz, uy1, uy);
        if (bits & 0xfu)
            t = march_cpml<false, 0, 0>(P, bits, p, j, k, t, -db, __fsub_rn(uzj, uz), __fmul_rn(-1.0f, __fsub_rn(uy1, uy)));
        hx_n = t;
    }
    if (in_ && kn) {
        const float db = at(l10, zr[3]);
        float t = h_upd_t<OE>(at(l7, zr[1]), hy_n, db, ux1, ux, uzi, uz);
        if (bits & 0xf0u)
            t = march_cpml<false, 0, 1>(P, bits, p, j, k, t, -db, __fsub_rn(ux1, ux), __fmul_rn(-1.0f, __fsub_rn(uzi, uz)));
        hy_n = t;
    }
}

// Sets the divergence flag when a value of the three quads is not finite
// (x·0 is NaN exactly for a NaN or an infinite x).
__device__ __forceinline__ void march_check_finite(const FusedParams& P, const Q4& x, const Q4& y, const Q4& z) {
    float s = 0.0f;
#pragma unroll
    for (int e = 0; e < 4; ++e) s = __fadd_rn(s, __fadd_rn(__fadd_rn(x.v[e], y.v[e]), z.v[e]));
    s = __fmul_rn(s, 0.0f);
    if (s != s && P.diverged) atomicExch(P.diverged, 1);
}

// Thread 0 of a block: the six tensor copies of plane q (u_x, u_y, u_z
// windows, then the i windows) into stage (q − q0) mod S, completing on its
// barrier, which expects their bytes (plus `extra`, the test hook).
template <uint32_t R, uint32_t S>
__device__ __forceinline__ void march_issue(const MarchMaps& M, uint64_t* bar, float* ring, uint32_t q, uint32_t q0,
                                            uint32_t k0, uint32_t j0, uint32_t extra) {
    using L = MarchLayout<R>;
    uint64_t* b = &bar[(q - q0) % S];
    float* st = ring + ((q - q0) % S) * (L::stage / 4);
    mbar_expect_tx(b, 3 * L::ubytes + 3 * L::ibytes + extra);
    for (int c = 0; c < 3; ++c) tma_load_3d(st + c * (L::ubox / 4), &M.u[c], (int)k0 - 4, (int)j0 - 1, (int)q, b);
    for (int c = 0; c < 3; ++c)
        tma_load_3d(st + 3 * (L::ubox / 4) + c * (L::ibox / 4), &M.i[c], (int)k0 - 4, (int)j0 - 1, (int)q, b);
}

// Grid: (z tiles of kMzNodes over the padded row, y tiles of R rows, x
// chunks of `planes`); block: R + 1 warps. Warp 0 recomputes the H row below
// the tile (and lanes 0..R−1 of it the node below the tile of rows
// 0..R−1); warp w ≥ 1 owns row j0 + w − 1. A bounded wait that runs out
// sets P.status and the block returns.
template <uint32_t R, uint32_t S, bool OE>
__global__ void __launch_bounds__(32 * (R + 1), MarchLayout<R>::blocks(S))
    k_march(const __grid_constant__ FusedParams P, const __grid_constant__ MarchMaps M, uint32_t planes) {
    using L = MarchLayout<R>;
    constexpr uint32_t US = L::ubox / 4, IS = L::ibox / 4, HS = (R + 1) * kMW, PS = (R + 1) * kMW;
    static_assert(S >= 3, "the ring must hold planes p and p + 1 while p + 2 loads");
    static_assert(HS <= IS, "the E tile lives in the i window of its plane");
    EMS_DYNAMIC_SMEM(smem);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
    float* ring = reinterpret_cast<float*>(smem + L::bars);
    float* ht = reinterpret_cast<float*>(smem + L::bars + S * L::stage);              // H of the plane
    float* hpt = reinterpret_cast<float*>(smem + L::bars + S * L::stage + L::htile);  // H_y, H_z of the plane before
    float* bgs = reinterpret_cast<float*>(smem + L::bars + S * L::stage + L::htile + L::hptile);
    uint32_t* czs = reinterpret_cast<uint32_t*>(smem + L::bars + S * L::stage + L::htile + L::hptile + L::bgtile);
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
    const bool owner = w > 0 && row_ok;
    const uint32_t j = row_ok ? (uint32_t)jr : 0u;
    const uint32_t tnodes = g.nz > k0 ? min(g.nz - k0, kMzNodes) : 0u;  // nodes of the tile
    // Lanes 0..R−1 of warp 0: the node k0 − 1 of row j0 + l.
    const int jz = (int)j0 + (int)l;
    const bool zfeed = w == 0 && l < R && k0 > 0 && jz < (int)g.ny;
    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < S; ++s) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    // The H values of the plane before the first: zero (no plane −1). The
    // background coefficient rows and the z-layer masks of the z window.
    for (uint32_t t = threadIdx.x; t < L::hptile / 4; t += blockDim.x) hpt[t] = 0.0f;
    for (uint32_t t = threadIdx.x; t < 12 * kMW; t += blockDim.x) {
        const uint32_t ln = t / kMW, zz = k0 + t % kMW;  // z-node k0 − 4 + (t mod kMW) + 4
        const Lane& LL = P.lane[ln];
        const int kk = (int)zz - 4;
        bgs[t] = (!LL.dense && kk >= 0 && (uint32_t)kk < g.pitch) ? LL.rows[(size_t)LL.bg * g.pitch + kk] : 0.0f;
    }
    for (uint32_t t = threadIdx.x; t < kMW; t += blockDim.x) {
        const int kk = (int)(k0 + t) - 4;
        czs[t] = (kk >= 0 && (uint32_t)kk < g.nz) ? P.cmask[2][kk] : 0u;
    }
    __syncthreads();
    // The tile's z-layer nodes of each side (rows in no layer visit only these).
    MarchSpans zl_h{}, zl_e{};
    march_z_layers<0>(P, k0, tnodes, zl_h);
    march_z_layers<1>(P, k0, tnodes, zl_e);
    // Test hook: the first block arms its first barrier with more bytes than
    // its copies deliver (every copy lands; the phase never completes).
    const uint32_t extra = blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 ? P.test_extra_tx : 0u;
    const uint64_t limit = P.wait_ns ? P.wait_ns : kWaitNs;
    uint32_t issued = q0;  // thread 0: planes below this one are issued
    if (threadIdx.x == 0)
        for (; issued <= last && issued < q0 + S - 1; ++issued)
            march_issue<R, S>(M, bar, ring, issued, q0, k0, j0, issued == q0 ? extra : 0u);
    const uint32_t sj = g.pitch, si = g.ny * g.pitch;
    const uint32_t zoff = 4u + 4u * l;
    const uint32_t cm1 = row_ok ? P.cmask[1][j] : 0u;
    uint32_t cz[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) cz[e] = czs[zoff + e];
    // Row ids of the coefficient lanes (this plane's, the next one's loaded
    // one plane ahead), and for the node below the tile lanes 6, 7, 9, 10.
    uint32_t rid[12], ridn[12] = {}, zr[4] = {}, zrn[4] = {};
    if (row_ok) march_rids(P, q0 * g.ny + j, ridn);
    if (zfeed) {
        const uint32_t zrow = q0 * g.ny + (uint32_t)jz;
        const int zl[4] = {6, 7, 9, 10};
#pragma unroll
        for (int q = 0; q < 4; ++q) zrn[q] = P.lane[zl[q]].dense ? 0u : __ldg(P.lane[zl[q]].rid + zrow);
    }
    uint32_t cm0n = P.cmask[0][q0];
    for (uint32_t p = q0; p < xe; ++p) {
        bool ok = true;
        if (threadIdx.x == 0)
            ok = mbar_wait(&bar[(p - q0) % S], ((p - q0) / S) & 1u, limit) &&
                 mbar_wait(&bar[(p + 1 - q0) % S], ((p + 1 - q0) / S) & 1u, limit);
        if (march_any(!ok)) {
            if (threadIdx.x == 0) {
                atomicExch(P.status, 1);
                // Let the copies still in flight land (each wait bounded)
                // before the block's shared memory is given up.
                for (uint32_t q = p; q < issued; ++q) mbar_wait(&bar[(q - q0) % S], ((q - q0) / S) & 1u, limit);
            }
            return;
        }
        // Stage p − 1 is free: every thread has left the iteration that read it.
        if (threadIdx.x == 0 && p + S - 1 <= last) {
            march_issue<R, S>(M, bar, ring, issued, q0, k0, j0, 0u);
            ++issued;
        }
        // This plane's row ids and plane mask; the next plane's requested now.
#pragma unroll
        for (int ln = 0; ln < 12; ++ln) rid[ln] = ridn[ln];
#pragma unroll
        for (int q = 0; q < 4; ++q) zr[q] = zrn[q];
        const uint32_t cm0 = cm0n;
        if (p + 1 < xe) {
            if (row_ok) march_rids(P, (p + 1) * g.ny + j, ridn);
            if (zfeed) {
                const uint32_t zrow = (p + 1) * g.ny + (uint32_t)jz;
                const int zl[4] = {6, 7, 9, 10};
#pragma unroll
                for (int q = 0; q < 4; ++q) zrn[q] = P.lane[zl[q]].dense ? 0u : __ldg(P.lane[zl[q]].rid + zrow);
            }
            cm0n = P.cmask[0][p + 1];
        }
        float* st0 = ring + ((p - q0) % S) * (L::stage / 4);
        const float* st1 = ring + ((p + 1 - q0) % S) * (L::stage / 4);
        const bool warm = p < xs;  // the plane before the chunk: H values only
        const float* uw = st0 + w * kMW;   // the warp's row in plane p's u_x window
        const float* u1 = st1 + w * kMW;
        float* hrow = ht + w * kMW;
        float* hprow = hpt + w * kMW;
        const uint32_t cm = row_ok ? (cm0 | cm1) : 0u;
        // --- H update of the row, no hooks.
        if (row_ok && quad_ok) {
            const bool all = j + 1 < g.ny && p + 1 < g.nx && k + 4 < g.nz;
            const float* io = st0 + 3 * US + w * kMW + zoff;
            march_h_upd<0, OE, US, IS, HS>(P, p, j, k, all, rid, bgs + zoff, uw + zoff, u1 + zoff, io, hrow + zoff);
            march_h_upd<1, OE, US, IS, HS>(P, p, j, k, all, rid, bgs + zoff, uw + zoff, u1 + zoff, io, hrow + zoff);
            march_h_upd<2, OE, US, IS, HS>(P, p, j, k, all, rid, bgs + zoff, uw + zoff, u1 + zoff, io, hrow + zoff);
        } else if (quad_ok) {
            sts4(hrow + zoff, zq());
            sts4(hrow + HS + zoff, zq());
            sts4(hrow + 2 * HS + zoff, zq());
        }
        march_syncwarp();
        // --- H-side CPML of the row: every node of a row in a layer, else the
        // tile's z-layer nodes; one (node, component) per lane.
        if (row_ok) {
            MarchSpans sp{};
            if (cm & 0xfffu) sp.add(0u, tnodes);
            else sp = zl_h;
            const uint32_t items = 3u * sp.nodes;
            for (uint32_t b = 0; b < items; b += 32u) {
                const uint32_t it = b + l;
                if (it < items) {
                    const uint32_t z = sp.at(it / 3u);
                    march_h_fix<OE, US, HS>(P, owner && !warm, p, j, k0 + z, z, (int)(it % 3u), cm, czs, rid, bgs,
                                            uw, u1, hrow);
                }
            }
        }
        march_syncwarp();
        // --- The node below the tile (x, y) for rows 0..R−1 of the tile.
        if (w == 0 && l < R) {
            float zx = 0.0f, zy = 0.0f;
            if (zfeed) {
                const uint32_t tr = l + 1u;  // window row of row jz
                march_h_node<OE, US, IS>(P, p, (uint32_t)jz, k0 - 1u, zr, st0 + tr * kMW + 3u, st1 + tr * kMW + 3u,
                                         st0 + 3 * US + tr * kMW + 3u, zx, zy);
            }
            ht[(l + 1) * kMW + 3] = zx;  // zero where the tile starts at k = 0
            ht[HS + (l + 1) * kMW + 3] = zy;
        }
        if (warm) {
            // The y and z H values of this plane are the next plane's "before".
            if (owner && quad_ok) {
                sts4(hprow + zoff, lds4(hrow + HS + zoff));
                sts4(hprow + PS + zoff, lds4(hrow + 2 * HS + zoff));
            }
            continue;  // the next iteration's barrier orders the ring and the tiles
        }
        const uint32_t idx = p * si + j * sj + k;
        if (owner && quad_ok) {
            stq(P.in[0] + idx, lds4(hrow + zoff));
            stq(P.in[1] + idx, lds4(hrow + HS + zoff));
            stq(P.in[2] + idx, lds4(hrow + 2 * HS + zoff));
        }
        __syncthreads();
        if (owner) {
            // --- E update of the row into the E tile (the i window of plane p,
            // read by nobody any more), no hooks.
            float* erow = st0 + 3 * US + w * kMW;
            if (quad_ok) {
                const bool all = j + 1 < g.ny && p + 1 < g.nx && k + 4 < g.nz;
                march_e_upd<0, OE, US, HS, PS>(P, p, j, k, all, rid, bgs + zoff, uw + zoff, hrow + zoff,
                                               hprow + zoff, erow + zoff);
                march_e_upd<1, OE, US, HS, PS>(P, p, j, k, all, rid, bgs + zoff, uw + zoff, hrow + zoff,
                                               hprow + zoff, erow + zoff);
                march_e_upd<2, OE, US, HS, PS>(P, p, j, k, all, rid, bgs + zoff, uw + zoff, hrow + zoff,
                                               hprow + zoff, erow + zoff);
            }
            march_syncwarp();
            // --- E-side CPML of the row (as for H).
            MarchSpans sp{};
            if (cm & 0xfff000u) sp.add(0u, tnodes);
            else sp = zl_e;
            const uint32_t items = 3u * sp.nodes;
            for (uint32_t b = 0; b < items; b += 32u) {
                const uint32_t it = b + l;
                if (it < items) {
                    const uint32_t z = sp.at(it / 3u);
                    march_e_fix<OE, US, HS, PS>(P, p, j, k0 + z, z, (int)(it % 3u), cm, czs, rid, bgs, hrow, hprow,
                                                erow);
                }
            }
            march_syncwarp();
            if (quad_ok) {
                const Q4 ex = lds4(erow + zoff), ey = lds4(erow + HS + zoff), ez = lds4(erow + 2 * HS + zoff);
                stq(P.un[0] + idx, ex);
                stq(P.un[1] + idx, ey);
                stq(P.un[2] + idx, ez);
                march_check_finite(P, ex, ey, ez);
                // This plane's y and z H values become the next plane's
                // "before" (only this warp reads its row of that tile).
                sts4(hprow + zoff, lds4(hrow + HS + zoff));
                sts4(hprow + PS + zoff, lds4(hrow + 2 * HS + zoff));
            }
        }
    }
}

// Why a model cannot run the marching step ("" if it can): the hooks
// between the two updates (magnetic poles and sources), operators whose
// hooks read or write fields around the E update (lumped elements, Mur
// faces, openEMS PML layers), or the poles registered before the CPML (the
// pole kernel runs after the kernel's CPML correction).
inline std::string march_why(const ems_engine_desc* d) {
    int pos_cpml = -1, pos_poles = -1;
    for (size_t k = 0; k < d->n_ops; ++k) {
        const ems_op& op = d->ops[k];
        if (op.kind == EMS_OP_CPML) {
            pos_cpml = (int)k;
        } else if (op.kind == EMS_OP_POLES) {
            pos_poles = (int)k;
            if (((const ems_poles*)op.table)->magnetic.n_edges) return "magnetic poles";
        } else if (op.kind == EMS_OP_SOURCE) {
            const int kind = ((const ems_source*)op.table)->kind;
            if (kind == EMS_SOFT_H || kind == EMS_HARD_H) return "magnetic sources";
        } else if (op.kind != EMS_OP_PROBE) {
            return "lumped elements, Mur faces, openEMS PML layers or conducting sheets";
        }
    }
    if (pos_cpml >= 0 && pos_poles >= 0 && pos_poles < pos_cpml) return "poles registered before the CPML";
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
