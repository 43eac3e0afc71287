// split.cuh — the split step of the B200 FDTD engine (sm_100a).
//
// The H and E updates run as plain streaming kernels: four z-nodes per
// thread in 16-byte loads and stores, nothing in them but the Yee update of
// the three components, every load issued before any arithmetic and every
// store after it, so a warp keeps all of its loads in flight at once. Coefficients come from the pooled
// rows (a z-row's coefficient is one broadcast row id and one L2-resident
// row); in the common case of a uniform background that makes each update
// move 36 bytes per node (three components read, three read and written).
//
// The CPML correction of each side runs after its update as one kernel over
// the layer shell, cut once at set-up into boxes whose nodes all lie in the
// same slabs: a thread takes one node and applies its box's slabs in the
// slabs' order, with no per-node membership test. Dispersive, lumped, source and probe hooks run as
// in the per-operator schedule. All expressions are the reference's, so the
// results equal it bit for bit.
#pragma once

#include "separate.cuh"
#include <vector>

namespace emsk {

constexpr unsigned kSplitThreads = 128;  // quads (4 z-nodes) per block
constexpr unsigned kShellWarps = 8;      // shell segments per block

// Four consecutive z-nodes as registers (the element 4 of a 5-array is the
// z-neighbour beyond them, or below them for the E update).
struct Q4 {
    float v[4];
};
__device__ __forceinline__ Q4 ldq(const float* p) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    return Q4{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ Q4 ldq_rw(const float* p) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    return Q4{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ void stq(float* p, const Q4& q) {
    *reinterpret_cast<float4*>(p) = make_float4(q.v[0], q.v[1], q.v[2], q.v[3]);
}
__device__ __forceinline__ Q4 zq() { return Q4{{0.0f, 0.0f, 0.0f, 0.0f}}; }

// Whether the quad (i, j, k0..k0+3) lies in box B (the split kernels leave it
// to the interior kernel).
__host__ __device__ __forceinline__ bool in_interior(const InteriorBox& B, uint32_t i, uint32_t j, uint32_t k0) {
    return i >= B.lo[0] && i < B.hi[0] && j >= B.lo[1] && j < B.hi[1] && k0 >= B.lo[2] && k0 + 4u <= B.hi[2];
}

// The quad index (in the plane) of thread t of a split kernel (QuadMap);
// ~0u: none.
__device__ __forceinline__ uint32_t mapped_quad(const FusedParams& P, uint32_t t) {
    const QuadMap& M = P.qmap;
    if (M.count && t >= M.count) return ~0u;
    if (M.mode == 0) return M.q0 + t;
    const uint32_t r = t / M.nzl, c = t - r * M.nzl;
    return (M.row0 + r) * (P.g.pitch >> 2) + (c < M.zl ? c : M.zr + (c - M.zl));
}

// The quad a thread owns: plane i = blockIdx.y; quad q of the plane's
// ny·pitch/4 (rows are padded to a multiple of 32 floats, so a quad never
// straddles two rows). False for a quad that lies beyond the plane or in
// a row's padding.
__device__ __forceinline__ bool quad_of(const Grid& g, uint32_t q, uint32_t& j, uint32_t& k0) {
    const uint32_t qpr = g.pitch >> 2;
    if (q >= g.ny * qpr) return false;
    j = q / qpr;
    k0 = (q - j * qpr) * 4u;
    return k0 < g.nz;
}

// The CPML corrections of component C of the quad (i, j, k0..k0+3), applied
// to the updated values t before they are stored (mask bit e: node e has the
// component): for every slab of the side and component that holds the node,
// in the slabs' order, the chain of cpml_body on the curl differences the
// update just formed (s = A or −B by the slab's normal). The update kernels'
// CPML variant runs it over every quad that holds a layer node, so no shell
// kernel follows them.
template <int SIDE, int C>
__device__ __forceinline__ void row_cpml(const FusedParams& P, uint32_t i, uint32_t j, uint32_t k0, uint32_t mask,
                                         Q4& t, const Q4& coef, const Q4& A, const Q4& B) {
    constexpr uint32_t na = (C + 1) % 3;
    const int n = P.nslab[SIDE][C];
    for (int q = 0; q < n; ++q) {
        const FSlab& s = P.slab[SIDE][C][q];
        if (i < s.lo[0] || i >= s.hi[0] || j < s.lo[1] || j >= s.hi[1]) continue;
        const uint32_t base = ((i - s.lo[0]) * (s.hi[1] - s.lo[1]) + (j - s.lo[1])) * (s.hi[2] - s.lo[2]);
        // The slab's nodes of the quad; every load of them first (the four
        // ψ entries are distinct, so their loads need not wait for the
        // stores), then the four chains, then the stores.
        uint32_t in = 0;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const uint32_t k = k0 + e;
            in |= (((mask >> e) & 1u) && k >= s.lo[2] && k < s.hi[2] ? 1u : 0u) << e;
        }
        if (!in) continue;
        float psi[4], cb_[4], ca_[4], ck_[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            psi[e] = 0.0f;
            cb_[e] = ca_[e] = ck_[e] = 0.0f;
            if (!((in >> e) & 1u)) continue;
            const uint32_t k = k0 + e;
            const uint32_t d = s.normal == 0u ? i - s.lo[0] : (s.normal == 1u ? j - s.lo[1] : k - s.lo[2]);
            psi[e] = s.psi_old[base + (k - s.lo[2])];
            cb_[e] = __ldg(s.b + d);
            ca_[e] = __ldg(s.a + d);
            ck_[e] = __ldg(s.k + d);
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            if (!((in >> e) & 1u)) continue;
            const float sv = s.normal == na ? A.v[e] : __fmul_rn(-1.0f, B.v[e]);
            psi[e] = flush(__fadd_rn(__fmul_rn(cb_[e], psi[e]), __fmul_rn(ca_[e], sv)));
            t.v[e] = flush(__fadd_rn(t.v[e], __fmul_rn(coef.v[e], __fadd_rn(__fmul_rn(ck_[e], sv), psi[e]))));
        }
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if ((in >> e) & 1u) s.psi_new[base + (k0 + e - s.lo[2])] = psi[e];
    }
}

// H update of every dual edge (src/engine/kernel.rs:447-511, 571-618), four
// z-nodes per thread; with ENERGY each block writes its share of the energy
// invariant in units of dt/4 (src/engine/kernel.rs:132-244). Entries the
// update does not write (edges that do not exist, row padding) are stored
// back as read. OE: openEMS's summation order. Grid: (quads of a plane /
// kSplitThreads, nx).
template <bool ENERGY, bool OE, bool ROWCPML = false>
__device__ __forceinline__ double split_h_quad(const FusedParams& P, uint32_t i, uint32_t q) {
    const Grid& g = P.g;
    uint32_t j = 0, k0 = 0;
    double w = 0.0;
    if (quad_of(g, q, j, k0) && !in_interior(P.skip, i, j, k0)) {
        const uint32_t sj = g.pitch, si = g.ny * g.pitch;
        const uint32_t idx = i * si + j * sj + k0;
        const uint32_t row = i * g.ny + j;
        const bool jn = j + 1 < g.ny, in_ = i + 1 < g.nx;
        // Neighbour offsets; 0 where the neighbour does not exist (the value
        // read is then unused).
        const uint32_t oj = jn ? sj : 0u, oi = in_ ? si : 0u, o4 = k0 + 4 < g.nz ? 4u : 0u;
        const Q4 ux = ldq(P.uo[0] + idx), uy = ldq(P.uo[1] + idx), uz = ldq(P.uo[2] + idx);
        const Q4 uzj = ldq(P.uo[2] + idx + oj), uxj = ldq(P.uo[0] + idx + oj);
        const Q4 uzi = ldq(P.uo[2] + idx + oi), uyi = ldq(P.uo[1] + idx + oi);
        const float uy4 = __ldg(P.uo[1] + idx + o4), ux4 = __ldg(P.uo[0] + idx + o4);
        const Q4 hx = ldq_rw(P.io[0] + idx), hy = ldq_rw(P.io[1] + idx), hz = ldq_rw(P.io[2] + idx);
        const Q4 dax = ldq(lane_row(P, 6, row) + k0), dbx = ldq(lane_row(P, 9, row) + k0);
        const Q4 day = ldq(lane_row(P, 7, row) + k0), dby = ldq(lane_row(P, 10, row) + k0);
        const Q4 daz = ldq(lane_row(P, 8, row) + k0), dbz = ldq(lane_row(P, 11, row) + k0);
        Q4 nx_ = hx, ny_ = hy, nz_ = hz;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const uint32_t k = k0 + e;
            const bool kn = k + 1 < g.nz;
            const float uy1 = e < 3 ? uy.v[e + 1] : uy4, ux1 = e < 3 ? ux.v[e + 1] : ux4;
            if (jn && kn) nx_.v[e] = h_upd_t<OE>(dax.v[e], hx.v[e], dbx.v[e], uzj.v[e], uz.v[e], uy1, uy.v[e]);
            if (in_ && kn) ny_.v[e] = h_upd_t<OE>(day.v[e], hy.v[e], dby.v[e], ux1, ux.v[e], uzi.v[e], uz.v[e]);
            if (in_ && jn && k < g.nz)
                nz_.v[e] = h_upd_t<OE>(daz.v[e], hz.v[e], dbz.v[e], uyi.v[e], uy.v[e], uxj.v[e], ux.v[e]);
        }
        if (ENERGY) {
            const Q4 ca0 = ldq(lane_row(P, 0, row) + k0), cb0 = ldq(lane_row(P, 3, row) + k0);
            const Q4 ca1 = ldq(lane_row(P, 1, row) + k0), cb1 = ldq(lane_row(P, 4, row) + k0);
            const Q4 ca2 = ldq(lane_row(P, 2, row) + k0), cb2 = ldq(lane_row(P, 5, row) + k0);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const uint32_t k = k0 + e;
                if (k >= g.nz) break;
                const bool kn = k + 1 < g.nz;
                const double x = ux.v[e], y = uy.v[e], z = uz.v[e];
                w = __dadd_rn(w, weight(ca0.v[e], __dmul_rn(x, x), cb0.v[e]));
                w = __dadd_rn(w, weight(ca1.v[e], __dmul_rn(y, y), cb1.v[e]));
                w = __dadd_rn(w, weight(ca2.v[e], __dmul_rn(z, z), cb2.v[e]));
                if (jn && kn) w = __dadd_rn(w, weight(dax.v[e], __dmul_rn((double)hx.v[e], (double)nx_.v[e]), dbx.v[e]));
                if (in_ && kn) w = __dadd_rn(w, weight(day.v[e], __dmul_rn((double)hy.v[e], (double)ny_.v[e]), dby.v[e]));
                if (in_ && jn) w = __dadd_rn(w, weight(daz.v[e], __dmul_rn((double)hz.v[e], (double)nz_.v[e]), dbz.v[e]));
            }
        }
        if (ROWCPML) {
            // The curl differences of the shell kernel's H side (shell_node).
            Q4 A, B;
            uint32_t mx = 0, my = 0, mz = 0;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const uint32_t k = k0 + e;
                const bool kn = k + 1 < g.nz;
                mx |= (jn && kn ? 1u : 0u) << e;
                my |= (in_ && kn ? 1u : 0u) << e;
                mz |= (in_ && jn && k < g.nz ? 1u : 0u) << e;
            }
            const Q4 mdbx{{-dbx.v[0], -dbx.v[1], -dbx.v[2], -dbx.v[3]}};
            const Q4 mdby{{-dby.v[0], -dby.v[1], -dby.v[2], -dby.v[3]}};
            const Q4 mdbz{{-dbz.v[0], -dbz.v[1], -dbz.v[2], -dbz.v[3]}};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                A.v[e] = __fsub_rn(uzj.v[e], uz.v[e]);
                B.v[e] = __fsub_rn(e < 3 ? uy.v[e + 1] : uy4, uy.v[e]);
            }
            row_cpml<0, 0>(P, i, j, k0, mx, nx_, mdbx, A, B);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                A.v[e] = __fsub_rn(e < 3 ? ux.v[e + 1] : ux4, ux.v[e]);
                B.v[e] = __fsub_rn(uzi.v[e], uz.v[e]);
            }
            row_cpml<0, 1>(P, i, j, k0, my, ny_, mdby, A, B);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                A.v[e] = __fsub_rn(uyi.v[e], uy.v[e]);
                B.v[e] = __fsub_rn(uxj.v[e], ux.v[e]);
            }
            row_cpml<0, 2>(P, i, j, k0, mz, nz_, mdbz, A, B);
        }
        if (jn) stq(P.in[0] + idx, nx_);
        if (in_) stq(P.in[1] + idx, ny_);
        if (in_ && jn) stq(P.in[2] + idx, nz_);
    }
    return w;
}

// Grid: (quads of a plane / kSplitThreads, planes): planes i0 .. i0 +
// gridDim.y − 1 from the last to the first. An H update reads the u of the
// plane above its own; in descending order a plane's blocks find it in L2,
// loaded by the blocks just before them (as the E update, ascending, finds
// the i of the plane below), and the update ends on the planes the E update
// starts with. Seven blocks of 72 registers per SM.
template <bool ENERGY, bool OE = false, bool ROWCPML = false>
__global__ void __launch_bounds__(kSplitThreads, ENERGY ? 1 : (ROWCPML ? 4 : 7)) k_split_h(
    const __grid_constant__ FusedParams P, uint32_t i0) {
    const uint32_t i = i0 + (gridDim.y - 1u - blockIdx.y);
    const double w = split_h_quad<ENERGY, OE, ROWCPML>(P, i, mapped_quad(P, blockIdx.x * kSplitThreads + threadIdx.x));
    if (ENERGY) {
        const double s = block_sum<kSplitThreads>(w);
        if (threadIdx.x == 0) P.partials[(size_t)i * gridDim.x + blockIdx.x] = s;
    }
}

// E update of every edge (src/engine/kernel.rs:624-697), four z-nodes per
// thread; OE: openEMS's summation order. Grid: (quads of a plane /
// kSplitThreads, nx).
template <bool OE, bool ROWCPML = false>
__device__ __forceinline__ void split_e_quad(const FusedParams& P, uint32_t i, uint32_t q) {
    const Grid& g = P.g;
    uint32_t j = 0, k0 = 0;
    if (!quad_of(g, q, j, k0) || in_interior(P.skip, i, j, k0)) return;
    const uint32_t sj = g.pitch, si = g.ny * g.pitch;
    const uint32_t idx = i * si + j * sj + k0;
    const uint32_t row = i * g.ny + j;
    const Q4 ix = ldq(P.in[0] + idx), iy = ldq(P.in[1] + idx), iz = ldq(P.in[2] + idx);
    // Neighbours below the node; zero on the low faces (no edge there).
    const Q4 izj = j > 0 ? ldq(P.in[2] + idx - sj) : zq(), ixj = j > 0 ? ldq(P.in[0] + idx - sj) : zq();
    const Q4 izi = i > 0 ? ldq(P.in[2] + idx - si) : zq(), iyi = i > 0 ? ldq(P.in[1] + idx - si) : zq();
    const float iym = k0 > 0 ? __ldg(P.in[1] + idx - 1) : 0.0f, ixm = k0 > 0 ? __ldg(P.in[0] + idx - 1) : 0.0f;
    const Q4 ex = ldq_rw(P.uo[0] + idx), ey = ldq_rw(P.uo[1] + idx), ez = ldq_rw(P.uo[2] + idx);
    const Q4 cax = ldq(lane_row(P, 0, row) + k0), cbx = ldq(lane_row(P, 3, row) + k0);
    const Q4 cay = ldq(lane_row(P, 1, row) + k0), cby = ldq(lane_row(P, 4, row) + k0);
    const Q4 caz = ldq(lane_row(P, 2, row) + k0), cbz = ldq(lane_row(P, 5, row) + k0);
    const bool xi = i + 1 < g.nx, yj = j + 1 < g.ny;
    Q4 nx_ = ex, ny_ = ey, nz_ = ez;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const uint32_t k = k0 + e;
        if (k >= g.nz) break;
        const float iy0 = e > 0 ? iy.v[e - 1] : iym, ix0 = e > 0 ? ix.v[e - 1] : ixm;
        if (xi) nx_.v[e] = e_upd_t<OE>(cax.v[e], ex.v[e], cbx.v[e], iz.v[e], izj.v[e], iy.v[e], iy0);
        if (yj) ny_.v[e] = e_upd_t<OE>(cay.v[e], ey.v[e], cby.v[e], ix.v[e], ix0, iz.v[e], izi.v[e]);
        if (k + 1 < g.nz) nz_.v[e] = e_upd_t<OE>(caz.v[e], ez.v[e], cbz.v[e], iy.v[e], iyi.v[e], ix.v[e], ixj.v[e]);
    }
    if (ROWCPML) {
        // The curl differences of the shell kernel's E side (shell_node).
        Q4 A, B;
        uint32_t mx = 0, my = 0, mz = 0;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const uint32_t k = k0 + e;
            mx |= (xi && k < g.nz ? 1u : 0u) << e;
            my |= (yj && k < g.nz ? 1u : 0u) << e;
            mz |= (k + 1 < g.nz ? 1u : 0u) << e;
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            A.v[e] = __fsub_rn(iz.v[e], izj.v[e]);
            B.v[e] = __fsub_rn(iy.v[e], e > 0 ? iy.v[e - 1] : iym);
        }
        row_cpml<1, 0>(P, i, j, k0, mx, nx_, cbx, A, B);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            A.v[e] = __fsub_rn(ix.v[e], e > 0 ? ix.v[e - 1] : ixm);
            B.v[e] = __fsub_rn(iz.v[e], izi.v[e]);
        }
        row_cpml<1, 1>(P, i, j, k0, my, ny_, cby, A, B);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            A.v[e] = __fsub_rn(iy.v[e], iyi.v[e]);
            B.v[e] = __fsub_rn(ix.v[e], ixj.v[e]);
        }
        row_cpml<1, 2>(P, i, j, k0, mz, nz_, cbz, A, B);
    }
    if (xi) stq(P.un[0] + idx, nx_);
    if (yj) stq(P.un[1] + idx, ny_);
    stq(P.un[2] + idx, nz_);
}

template <bool OE = false, bool ROWCPML = false>
__global__ void __launch_bounds__(kSplitThreads, ROWCPML ? 4 : 7) k_split_e(const __grid_constant__ FusedParams P,
                                                                         uint32_t i0) {
    split_e_quad<OE, ROWCPML>(P, i0 + blockIdx.y, mapped_quad(P, blockIdx.x * kSplitThreads + threadIdx.x));
}

// Blocks of the split update kernels: (quads of a plane / kSplitThreads) × nx.
__host__ __device__ inline uint32_t split_blocks_x(const Grid& g) {
    return (g.ny * (g.pitch >> 2) + kSplitThreads - 1) / kSplitThreads;
}

// The layer shell of one side as the shell kernel reads it: boxes with one
// slab set per component (ShellBox), their nodes numbered box by box (z
// fastest), one thread per node.
struct ShellDev {
    const ShellBox* box;
    uint32_t n_box, total;  // boxes, and the nodes this launch covers
    uint32_t base;          // the first node of the launch (box starts count from 0)
    // Per window of kShellWindow nodes (node t in window t / kShellWindow),
    // the box holding the window's first node; null: binary search.
    const uint32_t* first_box = nullptr;
};

constexpr uint32_t kShellWindowLog = 8, kShellWindow = 1u << kShellWindowLog;

// The first_box table of a shell's boxes (sorted by start) covering `total`
// nodes.
inline std::vector<uint32_t> shell_windows(const std::vector<ShellBox>& boxes, uint32_t total) {
    std::vector<uint32_t> w((total + kShellWindow - 1) / kShellWindow + 1, 0);
    uint32_t q = 0;
    for (size_t b = 0; b < w.size(); ++b) {
        const uint64_t t = (uint64_t)b * kShellWindow;
        while (q + 1 < boxes.size() && boxes[q + 1].start <= t) ++q;
        w[b] = q;
    }
    return w;
}

// The CPML chain of one field value over the slabs of `list` (count | q…),
// in order: ψ = flush(b·ψ + a·s), t = flush(t + coef·(k·s + ψ)), with s = sA
// or sB by the slab's normal (the arithmetic of cpml_body; every listed
// slab holds the node).
template <int SIDE, int C>
__device__ __forceinline__ float shell_chain(const FusedParams& P, uint32_t list, uint32_t i, uint32_t j, uint32_t k,
                                             float t, float coef, float sA, float sB) {
    constexpr uint32_t na = (C + 1) % 3;
    const uint32_t cnt = list & 15u;
    for (uint32_t e = 0; e < cnt; ++e) {
        const FSlab& s = P.slab[SIDE][C][(list >> (4 + 4 * e)) & 15u];
        const uint32_t d = s.normal == 0 ? i - s.lo[0] : (s.normal == 1 ? j - s.lo[1] : k - s.lo[2]);
        const uint32_t at = ((i - s.lo[0]) * (s.hi[1] - s.lo[1]) + (j - s.lo[1])) * (s.hi[2] - s.lo[2]) + (k - s.lo[2]);
        const float sv = s.normal == na ? sA : sB;
        const float psi = flush(__fadd_rn(__fmul_rn(__ldg(s.b + d), s.psi_old[at]), __fmul_rn(__ldg(s.a + d), sv)));
        s.psi_new[at] = psi;
        t = flush(__fadd_rn(t, __fmul_rn(coef, __fadd_rn(__fmul_rn(__ldg(s.k + d), sv), psi))));
    }
    return t;
}

// CPML correction of the node (i, j, k) of box B on one side (0: H edges
// after the H update, 1: E edges after the E update)
// (src/engine/boundary/cpml.rs:445-520, 657-676). The curl differences are
// those of the update: A along next(c), B along prev(c); a slab takes s = A
// or −B by its normal.
template <int SIDE>
__device__ __forceinline__ void shell_node(const FusedParams& P, const ShellBox& Bx, uint32_t i, uint32_t j,
                                           uint32_t k) {
    const Grid& g = P.g;
    const uint32_t sj = g.pitch, si = g.ny * g.pitch;
    const uint32_t idx = i * si + j * sj + k, row = i * g.ny + j;
    const uint32_t l0 = Bx.list[0], l1 = Bx.list[1], l2 = Bx.list[2];
    if (SIDE == 0) {
        const float *ux = P.uo[0], *uy = P.uo[1], *uz = P.uo[2];
        if (l0 & 15u) {
            const float A = __fsub_rn(uz[idx + sj], uz[idx]), B = __fsub_rn(uy[idx + 1], uy[idx]);
            const float db = lane_row(P, 9, row)[k];
            P.in[0][idx] = shell_chain<0, 0>(P, l0, i, j, k, P.in[0][idx], -db, A, __fmul_rn(-1.0f, B));
        }
        if (l1 & 15u) {
            const float A = __fsub_rn(ux[idx + 1], ux[idx]), B = __fsub_rn(uz[idx + si], uz[idx]);
            const float db = lane_row(P, 10, row)[k];
            P.in[1][idx] = shell_chain<0, 1>(P, l1, i, j, k, P.in[1][idx], -db, A, __fmul_rn(-1.0f, B));
        }
        if (l2 & 15u) {
            const float A = __fsub_rn(uy[idx + si], uy[idx]), B = __fsub_rn(ux[idx + sj], ux[idx]);
            const float db = lane_row(P, 11, row)[k];
            P.in[2][idx] = shell_chain<0, 2>(P, l2, i, j, k, P.in[2][idx], -db, A, __fmul_rn(-1.0f, B));
        }
    } else {
        const float *ix = P.in[0], *iy = P.in[1], *iz = P.in[2];
        if (l0 & 15u) {
            const float A = __fsub_rn(iz[idx], j > 0 ? iz[idx - sj] : 0.0f);
            const float B = __fsub_rn(iy[idx], k > 0 ? iy[idx - 1] : 0.0f);
            const float cb = lane_row(P, 3, row)[k];
            P.un[0][idx] = shell_chain<1, 0>(P, l0, i, j, k, P.un[0][idx], cb, A, __fmul_rn(-1.0f, B));
        }
        if (l1 & 15u) {
            const float A = __fsub_rn(ix[idx], k > 0 ? ix[idx - 1] : 0.0f);
            const float B = __fsub_rn(iz[idx], i > 0 ? iz[idx - si] : 0.0f);
            const float cb = lane_row(P, 4, row)[k];
            P.un[1][idx] = shell_chain<1, 1>(P, l1, i, j, k, P.un[1][idx], cb, A, __fmul_rn(-1.0f, B));
        }
        if (l2 & 15u) {
            const float A = __fsub_rn(iy[idx], i > 0 ? iy[idx - si] : 0.0f);
            const float B = __fsub_rn(ix[idx], j > 0 ? ix[idx - sj] : 0.0f);
            const float cb = lane_row(P, 5, row)[k];
            P.un[2][idx] = shell_chain<1, 2>(P, l2, i, j, k, P.un[2][idx], cb, A, __fmul_rn(-1.0f, B));
        }
    }
}

// Node `block·256 + tid` of the side's shell: its box by binary search over
// the boxes' first nodes, then its (i, j, k) in the box (z fastest).
template <int SIDE>
__device__ __forceinline__ void shell_item(const FusedParams& P, const ShellDev& S, uint32_t block, uint32_t tid) {
    const uint32_t t0 = block * (32 * kShellWarps) + tid;
    if (t0 >= S.total) return;
    const uint32_t t = S.base + t0;
    uint32_t lo = 0;  // box[lo].start <= t < box[lo + 1].start
    if (S.first_box) {
        // The window's first box, then forward (a window spans few boxes).
        lo = __ldg(&S.first_box[t >> kShellWindowLog]);
        while (lo + 1 < S.n_box && __ldg(&S.box[lo + 1].start) <= t) ++lo;
    } else {
        uint32_t hi = S.n_box;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(&S.box[mid].start) <= t) lo = mid;
            else hi = mid;
        }
    }
    const ShellBox& Bx = S.box[lo];
    const uint32_t local = t - Bx.start;
    const uint32_t r = local / Bx.n[2];
    const uint32_t k = Bx.lo[2] + (local - r * Bx.n[2]);
    const uint32_t i = Bx.lo[0] + r / Bx.n[1];
    const uint32_t j = Bx.lo[1] + (r - (r / Bx.n[1]) * Bx.n[1]);
    shell_node<SIDE>(P, Bx, i, j, k);
}

template <int SIDE>
__global__ void __launch_bounds__(32 * kShellWarps) k_shell(const __grid_constant__ FusedParams P,
                                                            const __grid_constant__ ShellDev S) {
    shell_item<SIDE>(P, S, blockIdx.x, threadIdx.x);
}

// Blocks of the shell kernel for a side.
__host__ __device__ inline uint32_t shell_blocks(const ShellDev& S) {
    const uint32_t tb = 32 * kShellWarps;
    return (S.total + tb - 1) / tb;
}

// Dispersive correction of edge e of run R, one edge per thread, the
// constants read from the run (shared by consecutive edges of a row with
// equal poles) instead of per pole (src/engine/dispersive.rs:1392-1470): idx
// its padded node, ax its axis, p0 its first pole state. A leapfrog pole's
// new state does not depend on the corrected value and is stored at once; a
// trapezoidal pole's is formed from its old state after it. save_prev: also
// store the corrected value as the edge's saved value (the capture it
// replaces would read the same value; pole_prev_fold). prev_field: the field
// array holding u^n (the old buffer of a two-buffer step), read in place of
// the saved value; null: the saved value.
__device__ __forceinline__ void poles_edge_core(const Fields& f, const Coeffs& c, const PoleSideDev& p,
                                                const PoleRun& R, const double* sets, int electric, double dt,
                                                int save_prev, uint32_t e, uint32_t idx, int ax, uint32_t p0,
                                                const float* prev_field = nullptr) {
    const float prev32 = prev_field ? prev_field[idx] : p.prev[e];
    const double prev = (double)prev32;
    float* fld = electric ? f.u[ax] : f.i[ax];
    float u32 = fld[idx];
    const double cb = (double)(electric ? c.c[3 + ax][idx] : c.c[9 + ax][idx]);
    const double j0 = p.j[p0], q0 = p.q[p0];
    const double half_prev = __dmul_rn(0.5, prev);
    const double* cs = sets + R.set;
    if (R.oe & kOeDebye) {
        const float u_new = oe_debye_edge(cs, cs + 1, cs + 2, 3u, p.j + p0, R.np, prev32, u32);
        fld[idx] = u_new;
        if (save_prev) p.prev[e] = u_new;
        return;
    }
    double s = 0.0;
    for (uint32_t q = 0; q < R.np; ++q) {
        const double a = cs[3 * q], ic = cs[3 * q + 1], iz = cs[3 * q + 2];
        const double jq = q ? p.j[p0 + q] : j0, qq = q ? p.q[p0 + q] : q0;
        if ((R.oe >> q) & 1u) {
            u32 = oe_pole_step(a, ic, iz, p.j[p0 + q], p.q[p0 + q], prev32, u32);
        } else if ((R.kinds >> q) & 1u) {
            const double jn = __dadd_rn(__dmul_rn(a, jq), __dmul_rn(iz, __dsub_rn(prev, __dmul_rn(qq, ic))));
            p.j[p0 + q] = jn;
            p.q[p0 + q] = __dadd_rn(qq, __dmul_rn(dt, jn));
            s = __dadd_rn(s, jn);
        } else {
            s = __dadd_rn(s, __dmul_rn(__dadd_rn(__dsub_rn(__dmul_rn(a, jq), __dmul_rn(qq, ic)), half_prev), iz));
        }
    }
    // Without trapezoidal poles the denominator is exactly 1 (sum_inv_z = 0)
    // and the quotient is the numerator itself.
    const double num = __dsub_rn((double)u32, __dmul_rn(cb, s));
    const float u_new = R.sum_inv_z == 0.0
                            ? (float)num
                            : (float)__ddiv_rn(num, __dadd_rn(1.0, __dmul_rn(__dmul_rn(0.5, cb), R.sum_inv_z)));
    if (R.kinds != (1u << R.np) - 1u) {
        const double half_new = __dmul_rn(0.5, (double)u_new);
        for (uint32_t q = 0; q < R.np; ++q) {
            if ((R.kinds >> q) & 1u) continue;
            const double a = cs[3 * q], ic = cs[3 * q + 1], iz = cs[3 * q + 2];
            const double jq = p.j[p0 + q], qq = p.q[p0 + q];
            const double kk = __dadd_rn(__dsub_rn(__dmul_rn(a, jq), __dmul_rn(qq, ic)), half_prev);
            const double jb = __dmul_rn(__dadd_rn(kk, half_new), iz);
            p.j[p0 + q] = __dsub_rn(__dmul_rn(2.0, jb), jq);
            p.q[p0 + q] = __dadd_rn(qq, __dmul_rn(dt, jb));
        }
    }
    fld[idx] = u_new;
    if (save_prev) p.prev[e] = u_new;
}

// The correction of edge e found through its run index (edge tables first,
// independent of each other, so their latencies overlap).
__device__ __forceinline__ void poles_edge(const Fields& f, const Coeffs& c, const PoleSideDev& p, const PoleRun* runs,
                                           const double* sets, const uint32_t* run_of, int electric, double dt,
                                           int save_prev, uint32_t e, const Fields* old = nullptr) {
    if (e >= p.n_edges) return;
    const uint32_t r = __ldg(run_of + e);
    const uint32_t idx = __ldg(p.node + e);
    const int ax = (int)__ldg(p.axis + e);
    const uint32_t p0 = e ? __ldg(p.pole_end + e - 1) : 0u;
    poles_edge_core(f, c, p, runs[r], sets, electric, dt, save_prev, e, idx, ax, p0,
                    old ? (electric ? old->u[ax] : old->i[ax]) : nullptr);
}

constexpr uint32_t kPoleBlock = 256;

// Edges [e0, e1) of the side, kPoleBlock consecutive edges per block. The
// runs covering a block's edges (a contiguous range: a run holds
// consecutive edges) are staged in shared memory and each edge's node, axis
// and first pole state derived from its run, so the only per-edge traffic
// is the field, the saved value and the pole state. OLD: u^n comes from the
// old buffer `old` of a two-buffer step instead of the saved values.
template <bool OLD = false>
__global__ void __launch_bounds__(kPoleBlock) k_poles_blocks(const __grid_constant__ Fields f,
                                                             const __grid_constant__ Coeffs c,
                                                             const __grid_constant__ PoleSideDev p, const PoleRun* runs,
                                                             const double* sets, const uint32_t* run_of, int electric,
                                                             double dt, int save_prev, uint32_t e0, uint32_t e1,
                                                             const __grid_constant__ Fields old = Fields{}) {
    EMS_SHARED PoleRun sr[kPoleBlock];
    const uint32_t eb = e0 + blockIdx.x * kPoleBlock;
    if (eb >= e1) return;
    const uint32_t el = min(eb + kPoleBlock, e1) - 1;
    const uint32_t r0 = __ldg(run_of + eb), r1 = __ldg(run_of + el);
    const uint32_t e = eb + threadIdx.x;
    if (r1 < r0 || r1 - r0 >= kPoleBlock) {  // not a contiguous run range: per edge
        if (e <= el) poles_edge(f, c, p, runs, sets, run_of, electric, dt, save_prev, e, OLD ? &old : nullptr);
        return;
    }
    const uint32_t nr = r1 - r0 + 1;
    for (uint32_t t = threadIdx.x; t < nr; t += kPoleBlock) sr[t] = runs[r0 + t];
    __syncthreads();
    if (e > el) return;
    uint32_t lo = 0, hi = nr;  // sr[lo].e0 <= e < sr[lo + 1].e0
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (sr[mid].e0 <= e) lo = mid;
        else hi = mid;
    }
    const PoleRun& R = sr[lo];
    const uint32_t off = e - R.e0;
    poles_edge_core(f, c, p, R, sets, electric, dt, save_prev, e, R.node0 + off, (int)R.axis, R.p0 + off * R.np,
                    OLD ? (electric ? old.u[R.axis] : old.i[R.axis]) : nullptr);
}

}  // namespace emsk
