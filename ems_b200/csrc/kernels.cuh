// kernels.cuh — device kernels of the B200 FDTD engine (sm_100a).
//
// Every field update uses explicitly rounded IEEE operations (__fmul_rn,
// __fadd_rn, __fsub_rn and their f64 forms), so no multiply-add is ever
// contracted and each value is the reference's expression bit for bit.
#pragma once

#include <cfloat>
#include <cstdint>

#include "arith.cuh"

namespace emsk {

constexpr unsigned kRowThreads = 128;  // threads of a z-row block
constexpr uint32_t kMaxPoles = 16;     // poles per edge held in registers
constexpr uint32_t kOeDebye = 1u << 31;  // PoleRun::oe: an edge of openEMS Debye poles

struct Grid {
    uint32_t nx, ny, nz, pitch;  // pitch: padded z-row length (multiple of 32)
    uint64_t n, np;              // nodes, padded nodes
};

struct Fields {
    float* u[3];
    float* i[3];
};

struct Coeffs {
    const float* c[12];
};

struct SlabDev {
    int e_side, comp, normal, other;
    float sign;
    uint32_t lo[3], hi[3];
    const float* b;
    const float* a;
    const float* k;
    float* psi;
};

struct PoleSideDev {
    size_t n_edges = 0, n_poles = 0;
    const uint8_t* axis = nullptr;
    const uint32_t* node = nullptr;
    const double* sum_inv_z = nullptr;
    const uint32_t* pole_end = nullptr;
    const uint8_t* kind = nullptr;
    const double* a = nullptr;
    const double* inv_c = nullptr;
    const double* inv_z = nullptr;
    const double* half_l = nullptr;
    float* prev = nullptr;
    double* j = nullptr;
    double* q = nullptr;
};

struct LumpedDevT {
    uint32_t n = 0;
    double series = 1.0, columns = 0.0;
    int src_in_branch = 0, has_branch = 0, record = 0;
    const uint32_t* node = nullptr;
    const double* cb = nullptr;
    const double* g_src = nullptr;
    const double* src_w = nullptr;
    const double* two_l_dt = nullptr;
    const double* inv_c = nullptr;
    const double* z = nullptr;
    const double* rec_g = nullptr;
    const double* rec_c = nullptr;
    double* v = nullptr;
    double* bj = nullptr;
    double* bq = nullptr;
    double* bu_prev = nullptr;
    double* j_avg = nullptr;
    double* ru_prev = nullptr;
    int openems_order = 0;
    const float* oe_k = nullptr;   // openEMS's explicit inductor (f32 state oe_s)
    const double* oe_vi = nullptr;
    float* oe_s = nullptr;
};

struct ProbeDevT {
    uint32_t n = 0;
    int f32_sum = 0;
    const uint32_t* node = nullptr;
    const uint8_t* axis = nullptr;
    const double* weight = nullptr;
};

// H update of every dual edge (src/engine/kernel.rs:447-511, 571-618);
// with ENERGY each block also writes its share of the energy invariant
// Σ (1+ca)/cb·u² + Σ (1+da)/db·i_old·i_new in units of dt/4
// (src/engine/kernel.rs:132-244). OE: openEMS's summation order.
template <bool ENERGY, bool OE = false>
__global__ void __launch_bounds__(kRowThreads) k_update_h(const __grid_constant__ Grid g, const __grid_constant__ Fields f, const __grid_constant__ Coeffs c, double* partials) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t j = blockIdx.y, i = blockIdx.z;
    double w = 0.0;
    if (k < g.nz) {
        const uint32_t sj = g.pitch, si = g.ny * g.pitch;
        const uint32_t idx = i * si + j * sj + k;
        const float ux = f.u[0][idx], uy = f.u[1][idx], uz = f.u[2][idx];
        if (ENERGY) {
            w = __dadd_rn(w, weight(c.c[0][idx], __dmul_rn((double)ux, (double)ux), c.c[3][idx]));
            w = __dadd_rn(w, weight(c.c[1][idx], __dmul_rn((double)uy, (double)uy), c.c[4][idx]));
            w = __dadd_rn(w, weight(c.c[2][idx], __dmul_rn((double)uz, (double)uz), c.c[5][idx]));
        }
        if (j + 1 < g.ny && k + 1 < g.nz) {
            const float old = f.i[0][idx];
            const float da = c.c[6][idx], db = c.c[9][idx];
            const float nw = h_upd_t<OE>(da, old, db, f.u[2][idx + sj], uz, f.u[1][idx + 1], uy);
            f.i[0][idx] = nw;
            if (ENERGY) w = __dadd_rn(w, weight(da, __dmul_rn((double)old, (double)nw), db));
        }
        if (i + 1 < g.nx && k + 1 < g.nz) {
            const float old = f.i[1][idx];
            const float da = c.c[7][idx], db = c.c[10][idx];
            const float nw = h_upd_t<OE>(da, old, db, f.u[0][idx + 1], ux, f.u[2][idx + si], uz);
            f.i[1][idx] = nw;
            if (ENERGY) w = __dadd_rn(w, weight(da, __dmul_rn((double)old, (double)nw), db));
        }
        if (i + 1 < g.nx && j + 1 < g.ny) {
            const float old = f.i[2][idx];
            const float da = c.c[8][idx], db = c.c[11][idx];
            const float nw = h_upd_t<OE>(da, old, db, f.u[1][idx + si], uy, f.u[0][idx + sj], ux);
            f.i[2][idx] = nw;
            if (ENERGY) w = __dadd_rn(w, weight(da, __dmul_rn((double)old, (double)nw), db));
        }
    }
    if (ENERGY) {
        double s = block_sum<kRowThreads>(w);
        if (threadIdx.x == 0)
            partials[((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
    }
}

// Sums the per-block energy shares in a fixed order.
__global__ void __launch_bounds__(1024) k_reduce_partials(const double* partials, size_t n, double* out) {
    double s = 0.0;
    for (size_t q = threadIdx.x; q < n; q += blockDim.x) s = __dadd_rn(s, partials[q]);
    double t = block_sum<1024>(s);
    if (threadIdx.x == 0) out[0] = t;
}

// E update of every edge (src/engine/kernel.rs:624-697); OE: openEMS's
// summation order.
template <bool OE = false>
__global__ void __launch_bounds__(kRowThreads) k_update_e(const __grid_constant__ Grid g, const __grid_constant__ Fields f, const __grid_constant__ Coeffs c) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t j = blockIdx.y, i = blockIdx.z;
    if (k >= g.nz) return;
    const uint32_t sj = g.pitch, si = g.ny * g.pitch;
    const uint32_t idx = i * si + j * sj + k;
    const float ix = f.i[0][idx], iy = f.i[1][idx], iz = f.i[2][idx];
    if (i + 1 < g.nx) {
        const float b = j > 0 ? f.i[2][idx - sj] : 0.0f;
        const float d = k > 0 ? f.i[1][idx - 1] : 0.0f;
        f.u[0][idx] = e_upd_t<OE>(c.c[0][idx], f.u[0][idx], c.c[3][idx], iz, b, iy, d);
    }
    if (j + 1 < g.ny) {
        const float b = k > 0 ? f.i[0][idx - 1] : 0.0f;
        const float d = i > 0 ? f.i[2][idx - si] : 0.0f;
        f.u[1][idx] = e_upd_t<OE>(c.c[1][idx], f.u[1][idx], c.c[4][idx], ix, b, iz, d);
    }
    if (k + 1 < g.nz) {
        const float b = i > 0 ? f.i[1][idx - si] : 0.0f;
        const float d = j > 0 ? f.i[0][idx - sj] : 0.0f;
        f.u[2][idx] = e_upd_t<OE>(c.c[2][idx], f.u[2][idx], c.c[5][idx], iy, b, ix, d);
    }
}

// CPML correction of one slab (src/engine/boundary/cpml.rs:445-520, 657-676):
// s = sign·(h − l); ψ = flush(b·ψ + a·s); t = flush(t + scale·coef·(k·s + ψ)).
template <bool E_SIDE>
__global__ void k_cpml(const __grid_constant__ Grid g, const __grid_constant__ Fields f,
                       const __grid_constant__ Coeffs c, const __grid_constant__ SlabDev s) {
    const uint32_t k = s.lo[2] + blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t j = s.lo[1] + blockIdx.y, i = s.lo[0] + blockIdx.z;
    if (k >= s.hi[2]) return;
    const uint32_t si = g.ny * g.pitch;
    const uint32_t idx = i * si + j * g.pitch + k;
    const uint32_t step = s.normal == 0 ? si : (s.normal == 1 ? g.pitch : 1u);
    const uint32_t along = s.normal == 0 ? i : (s.normal == 1 ? j : k);
    const uint32_t d = along - s.lo[s.normal];
    float h, l;
    float* t;
    float coef;
    if (E_SIDE) {
        const float* src = f.i[s.other];
        h = src[idx];
        l = along == 0 ? 0.0f : src[idx - step];
        t = f.u[s.comp];
        coef = c.c[3 + s.comp][idx];
    } else {
        const float* src = f.u[s.other];
        h = src[idx + step];
        l = src[idx];
        t = f.i[s.comp];
        coef = -c.c[9 + s.comp][idx];
    }
    const uint32_t n1 = s.hi[1] - s.lo[1], n2 = s.hi[2] - s.lo[2];
    const uint32_t q = ((i - s.lo[0]) * n1 + (j - s.lo[1])) * n2 + (k - s.lo[2]);
    const float sv = __fmul_rn(s.sign, __fsub_rn(h, l));
    const float psi = flush(__fadd_rn(__fmul_rn(s.b[d], s.psi[q]), __fmul_rn(s.a[d], sv)));
    s.psi[q] = psi;
    t[idx] = flush(__fadd_rn(t[idx], __fmul_rn(coef, __fadd_rn(__fmul_rn(s.k[d], sv), psi))));
}

// Dispersive correction of one edge per thread (src/engine/dispersive.rs:1392-1470).
// A leapfrog pole's new state does not depend on the corrected value and is
// stored at once; a trapezoidal pole's is formed from its old state after it.
__global__ void k_poles_correct(const __grid_constant__ Grid g, const __grid_constant__ Fields f,
                                const __grid_constant__ Coeffs c, const __grid_constant__ PoleSideDev p, bool electric,
                                double dt) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= p.n_edges) return;
    (void)g;
    const int ax = p.axis[e];
    const uint32_t idx = p.node[e];
    float* fld = electric ? f.u[ax] : f.i[ax];
    const double cb = (double)(electric ? c.c[3 + ax][idx] : c.c[9 + ax][idx]);
    const uint32_t p0 = e ? p.pole_end[e - 1] : 0u, p1 = p.pole_end[e];
    const float prev_f = p.prev[e];
    if (p.kind[p0] == 3) {  // openEMS Debye edge
        fld[idx] = oe_debye_edge(p.a + p0, p.inv_c + p0, p.inv_z + p0, 1u, p.j + p0, p1 - p0, prev_f, fld[idx]);
        return;
    }
    const double prev = (double)prev_f;
    const double half_prev = __dmul_rn(0.5, prev);
    float u32 = fld[idx];
    double s = 0.0;
    bool trap = false;
    for (uint32_t q = p0; q < p1; ++q) {
        const double a = p.a[q], ic = p.inv_c[q], iz = p.inv_z[q], jq = p.j[q], qq = p.q[q];
        if (p.kind[q] == 2) {  // openEMS's f32 pole, before the others
            u32 = oe_pole_step(a, ic, iz, p.j[q], p.q[q], prev_f, u32);
        } else if (p.kind[q] == 1) {  // leapfrog: j^{n+1/2} from u^n, then q^{n+1}
            const double jn = __dadd_rn(__dmul_rn(a, jq), __dmul_rn(iz, __dsub_rn(prev, __dmul_rn(qq, ic))));
            p.j[q] = jn;
            p.q[q] = __dadd_rn(qq, __dmul_rn(dt, jn));
            s = __dadd_rn(s, jn);
        } else {
            trap = true;
            s = __dadd_rn(s, __dmul_rn(__dadd_rn(__dsub_rn(__dmul_rn(a, jq), __dmul_rn(qq, ic)), half_prev), iz));
        }
    }
    const double u_star = (double)u32;
    const float u_new = (float)__ddiv_rn(__dsub_rn(u_star, __dmul_rn(cb, s)),
                                         __dadd_rn(1.0, __dmul_rn(__dmul_rn(0.5, cb), p.sum_inv_z[e])));
    if (trap) {
        const double half_new = __dmul_rn(0.5, (double)u_new);
        for (uint32_t q = p0; q < p1; ++q) {
            if (p.kind[q] != 0) continue;
            const double a = p.a[q], ic = p.inv_c[q], iz = p.inv_z[q], jq = p.j[q], qq = p.q[q];
            const double kk = __dadd_rn(__dsub_rn(__dmul_rn(a, jq), __dmul_rn(qq, ic)), half_prev);
            const double jb = __dmul_rn(__dadd_rn(kk, half_new), iz);
            p.j[q] = __dsub_rn(__dmul_rn(2.0, jb), jq);
            p.q[q] = __dadd_rn(qq, __dmul_rn(dt, jb));
        }
    }
    fld[idx] = u_new;
}

// Saves the field value of every edge (src/engine/dispersive.rs:1173-1180).
__global__ void k_poles_capture(const __grid_constant__ Fields f, const __grid_constant__ PoleSideDev p, bool electric) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= p.n_edges) return;
    p.prev[e] = (electric ? f.u[p.axis[e]] : f.i[p.axis[e]])[p.node[e]];
}

// Edge source (src/engine/excite.rs:104-117): soft adds w·a, hard sets w·a.
__global__ void k_source(float* f0, float* f1, float* f2, const uint8_t* axis, const uint32_t* node,
                         const float* weight, size_t n, float a, bool hard) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    float* F = axis[e] == 0 ? f0 : (axis[e] == 1 ? f1 : f2);
    const float v = __fmul_rn(weight[e], a);
    F[node[e]] = hard ? v : __fadd_rn(F[node[e]], v);
}

// Probe sample: Σ w·x in entry order (src/engine/probe.rs:381-392).
__device__ __forceinline__ void probe_sample(const float* f0, const float* f1, const float* f2, const ProbeDevT& p,
                                             double* out) {
    if (p.f32_sum) {
        float s = 0.0f;
        for (uint32_t e = 0; e < p.n; ++e) {
            const float* F = p.axis[e] == 0 ? f0 : (p.axis[e] == 1 ? f1 : f2);
            s = __fadd_rn(s, __fmul_rn((float)p.weight[e], F[p.node[e]]));
        }
        out[0] = (double)s;
    } else {
        double s = 0.0;
        for (uint32_t e = 0; e < p.n; ++e) {
            const float* F = p.axis[e] == 0 ? f0 : (p.axis[e] == 1 ? f1 : f2);
            s = __dadd_rn(s, __dmul_rn(p.weight[e], (double)F[p.node[e]]));
        }
        out[0] = s;
    }
}

__global__ void k_probe(const float* f0, const float* f1, const float* f2, ProbeDevT p, double* out) {
    if (threadIdx.x != 0) return;
    probe_sample(f0, f1, f2, p, out);
}

// Lumped element pre_e: saves u^n (src/engine/lumped.rs:1106-1121).
__device__ __forceinline__ void lumped_pre_e_edge(const float* u, const LumpedDevT& d, uint32_t e) {
    const double x = (double)u[d.node[e]];
    if (d.has_branch && !d.openems_order) d.bu_prev[e] = x;  // openEMS's order keeps the post_e value
    if (d.record) d.ru_prev[e] = x;
}

__global__ void k_lumped_pre_e(const float* u, LumpedDevT d) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= d.n) return;
    lumped_pre_e_edge(u, d, e);
}

// Lumped element post_e (src/engine/lumped.rs:1123-1236) and, for a port,
// V = Σu/columns, I = −record (src/engine/port.rs:276-290). One block: the
// per-edge updates in parallel, the sums in edge order by thread 0.
__device__ __forceinline__ void lumped_post_e_block(float* u, const LumpedDevT& d, double val, int active, double dt,
                                                    double* rec_out, double* pv_out, double* pi_out) {
    for (uint32_t e = threadIdx.x; e < d.n; e += blockDim.x) {
        const uint32_t idx = d.node[e];
        if (d.src_w) d.v[e] = active ? __dadd_rn(0.0, __dmul_rn(d.src_w[e], val)) : 0.0;
        // In openEMS's order a resistor's source acts like a soft one, after
        // the branch.
        if (active && !d.src_in_branch && !d.openems_order) {
            const double add = __dmul_rn(__dmul_rn(d.cb[e], d.g_src[e]), d.v[e]);
            if (add != 0.0) u[idx] = (float)__dadd_rn((double)u[idx], add);
        }
        if (d.has_branch && d.oe_k) {
            // openEMS's explicit inductor in f32 (src/engine/lumped.rs:1168-1177).
            const float u_l = (float)d.bu_prev[e];
            d.oe_s[e] = flush(__fadd_rn(d.oe_s[e], flush(__fmul_rn(d.oe_k[e], u_l))));
            const float u_new = flush(__fsub_rn(u[idx], d.oe_s[e]));
            d.bj[e] = __ddiv_rn((double)d.oe_s[e], d.oe_vi[e]);
            d.j_avg[e] = d.bj[e];
            u[idx] = u_new;
            d.bu_prev[e] = (double)u_new;
        } else if (d.has_branch) {
            const double v_br = (active && d.src_in_branch) ? d.v[e] : 0.0;
            const double u_star = (double)u[idx];
            const double kk = __dadd_rn(__dsub_rn(__dsub_rn(__dmul_rn(d.two_l_dt[e], d.bj[e]), __dmul_rn(d.bq[e], d.inv_c[e])), v_br),
                                        __dmul_rn(0.5, d.bu_prev[e]));
            const double z = d.z[e], cb = d.cb[e];
            const double u_new = __ddiv_rn(__dsub_rn(__dmul_rn(z, u_star), __dmul_rn(cb, kk)), __dadd_rn(z, __dmul_rn(0.5, cb)));
            const double jb = __ddiv_rn(__dadd_rn(kk, __dmul_rn(0.5, u_new)), z);
            d.bj[e] = __dsub_rn(__dmul_rn(2.0, jb), d.bj[e]);
            d.bq[e] = __dadd_rn(d.bq[e], __dmul_rn(dt, jb));
            d.j_avg[e] = jb;
            u[idx] = (float)u_new;
            if (d.openems_order) d.bu_prev[e] = (double)(float)u_new;
        }
        if (active && !d.src_in_branch && d.openems_order) {
            const double add = __dmul_rn(__dmul_rn(d.cb[e], d.g_src[e]), d.v[e]);
            if (add != 0.0) u[idx] = (float)__dadd_rn((double)u[idx], add);
        }
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double rec = 0.0;
    if (d.record && rec_out) {
        double sum = 0.0;
        for (uint32_t e = 0; e < d.n; ++e) {
            const double u0 = d.ru_prev[e], u1 = (double)u[d.node[e]];
            const double v = (active && !d.src_in_branch) ? d.v[e] : 0.0;
            const double t1 = __dmul_rn(d.rec_g[e], __dsub_rn(__dmul_rn(0.5, __dadd_rn(u0, u1)), v));
            const double t2 = __ddiv_rn(__dmul_rn(d.rec_c[e], __dsub_rn(u1, u0)), dt);
            sum = __dadd_rn(sum, __dadd_rn(t1, t2));
            if (d.has_branch) sum = __dadd_rn(sum, d.j_avg[e]);
        }
        rec = __ddiv_rn(sum, d.series);
        rec_out[0] = rec;
    }
    if (pv_out) {
        pi_out[0] = -rec;
        double s = 0.0;
        for (uint32_t e = 0; e < d.n; ++e) s = __dadd_rn(s, (double)u[d.node[e]]);
        pv_out[0] = __ddiv_rn(s, d.columns);
    }
}

__global__ void __launch_bounds__(256) k_lumped_post_e(float* u, LumpedDevT d, double val, int active, double dt,
                                                       double* rec_out, double* pv_out, double* pi_out) {
    lumped_post_e_block(u, d, val, active, dt, rec_out, pv_out, pi_out);
}

// Σ ½·L·j² + ½·q²/C_p of the electric then the magnetic poles
// (src/engine/dispersive.rs:1488-1506, 2598-2618).
template <unsigned THREADS>
__device__ __forceinline__ double pole_energy_block(const PoleSideDev& e, const PoleSideDev& h) {
    double s = 0.0;
    for (int side = 0; side < 2; ++side) {
        const PoleSideDev& p = side == 0 ? e : h;
        for (size_t q = threadIdx.x; q < p.n_poles; q += blockDim.x) {
            if (p.kind[q] >= 2) continue;  // openEMS's poles hold no energy
            const double a = __dmul_rn(__dmul_rn(p.half_l[q], p.j[q]), p.j[q]);
            const double b = __dmul_rn(__dmul_rn(__dmul_rn(0.5, p.inv_c[q]), p.q[q]), p.q[q]);
            s = __dadd_rn(s, __dadd_rn(a, b));
        }
    }
    return block_sum<THREADS>(s);
}

__global__ void __launch_bounds__(1024) k_pole_energy(PoleSideDev e, PoleSideDev h, double* out) {
    double s = 0.0;
    for (int side = 0; side < 2; ++side) {
        const PoleSideDev& p = side == 0 ? e : h;
        for (size_t q = threadIdx.x; q < p.n_poles; q += blockDim.x) {
            if (p.kind[q] >= 2) continue;  // openEMS's poles hold no energy
            const double a = __dmul_rn(__dmul_rn(p.half_l[q], p.j[q]), p.j[q]);
            const double b = __dmul_rn(__dmul_rn(__dmul_rn(0.5, p.inv_c[q]), p.q[q]), p.q[q]);
            s = __dadd_rn(s, __dadd_rn(a, b));
        }
    }
    const double t = block_sum<1024>(s);
    if (threadIdx.x == 0) out[0] = t;
}

// Σ ½·L_e·j² + ½·q²/C_e of a lumped branch (src/engine/lumped.rs:1066-1077).
__device__ __forceinline__ double branch_energy(const LumpedDevT& d, double dt) {
    double s = 0.0;
    for (uint32_t e = 0; e < d.n; ++e) {
        const double half_l = __dmul_rn(__dmul_rn(0.25, d.two_l_dt[e]), dt);
        s = __dadd_rn(s, __dadd_rn(__dmul_rn(__dmul_rn(half_l, d.bj[e]), d.bj[e]),
                                   __dmul_rn(__dmul_rn(__dmul_rn(0.5, d.inv_c[e]), d.bq[e]), d.bq[e])));
    }
    return s;
}

__global__ void k_branch_energy(LumpedDevT d, double dt, double* out) {
    double s = 0.0;
    for (uint32_t e = 0; e < d.n; ++e) {
        const double half_l = __dmul_rn(__dmul_rn(0.25, d.two_l_dt[e]), dt);
        s = __dadd_rn(s, __dadd_rn(__dmul_rn(__dmul_rn(half_l, d.bj[e]), d.bj[e]),
                                   __dmul_rn(__dmul_rn(__dmul_rn(0.5, d.inv_c[e]), d.bq[e]), d.bq[e])));
    }
    out[0] = s;
}

// One side of openEMS's PML layers on the device (src/engine/boundary/
// upml.rs:260-420): per edge its axis, node, coefficients (co.x..co.w =
// (1 − a_p)/(1 + a_p), (1 − a_q)/(1 + a_q), (1 + a_a)/((1 + a_q)·m),
// (1 − a_a)/((1 + a_q)·m)), flux f and start value v.
struct UpmlSideDev {
    uint32_t n = 0;
    const uint8_t* axis = nullptr;
    const uint32_t* node = nullptr;
    const float4* co = nullptr;
    float* f = nullptr;
    float* v = nullptr;
};

// One slab hook of the layers (upml.rs:443-464): threads [0, r.n) take the
// start values of side r from the fields `src` (Run::refresh), threads
// [r.n, r.n + a.n) complete the update of side a in the fields `dst` from
// the flux increment the update kernel left there (Run::apply):
// F' = flush(flush(co.x·F) + t), x = flush(flush(flush(co.y·v) − flush(co.w·F)) + flush(co.z·F')).
__global__ void __launch_bounds__(256) k_upml_hook(const float* s0, const float* s1, const float* s2, UpmlSideDev r,
                                                   float* d0, float* d1, float* d2, UpmlSideDev a) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < r.n) {
        const uint8_t ax = r.axis[e];
        const float* F = ax == 0 ? s0 : (ax == 1 ? s1 : s2);
        r.v[e] = F[r.node[e]];
        return;
    }
    const uint32_t q = e - r.n;
    if (q >= a.n) return;
    const uint8_t ax = a.axis[q];
    float* F = ax == 0 ? d0 : (ax == 1 ? d1 : d2);
    const uint32_t idx = a.node[q];
    const float4 c = a.co[q];
    const float t = F[idx], f0 = a.f[q], v = a.v[q];
    const float f1 = flush(__fadd_rn(flush(__fmul_rn(c.x, f0)), t));
    const float x = flush(__fadd_rn(flush(__fsub_rn(flush(__fmul_rn(c.y, v)), flush(__fmul_rn(c.w, f0)))),
                                    flush(__fmul_rn(c.z, f1))));
    a.f[q] = f1;
    a.v[q] = x;
    F[idx] = x;
}

// A Mur boundary on the device (src/engine/boundary/mur.rs:103-139):
// entries [0, n_edges) face edges, [n_edges, n) edges shared by two faces;
// inner and k 2 per entry, saved 3 per entry (u_b^n, u_1^n of each
// neighbour), last the value after the last update (energy).
struct MurDevT {
    uint32_t n = 0, n_edges = 0;
    int openems_order = 0, openems_corners = 0;
    const uint8_t* axis = nullptr;
    const uint32_t* node = nullptr;
    const uint32_t* inner = nullptr;
    const float* k = nullptr;
    const uint64_t* hold = nullptr;  // null: no holds
    const double* cap = nullptr;     // null: energy not counted
    float* saved = nullptr;
    float* last = nullptr;
};

// src/engine/boundary/mur.rs:252-259 mur_1d, rounded step by step.
__device__ __forceinline__ float mur_1d(float i, float k, float x, float b, int openems) {
    return openems ? __fadd_rn(__fsub_rn(i, __fmul_rn(k, b)), __fmul_rn(k, x)) : __fadd_rn(i, __fmul_rn(k, __fsub_rn(x, b)));
}

// pre_e (src/engine/boundary/mur.rs:781-808): u_b^n, u_1^n of every entry.
__global__ void k_mur_save(float* f0, float* f1, float* f2, MurDevT m) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.n) return;
    const float* F = m.axis[e] == 0 ? f0 : (m.axis[e] == 1 ? f1 : f2);
    m.saved[3 * e] = F[m.node[e]];
    m.saved[3 * e + 1] = F[m.inner[2 * e]];
    if (e >= m.n_edges) m.saved[3 * e + 2] = F[m.inner[2 * e + 1]];
}

// post_e (src/engine/boundary/mur.rs:812-843) of the entries [e0, e1): the
// face edges in one launch, then the shared edges, whose neighbours are
// face edges, in a second one.
__global__ void k_mur_update(float* f0, float* f1, float* f2, MurDevT m, uint64_t step, uint32_t e0, uint32_t e1) {
    const uint32_t e = e0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= e1) return;
    if (m.hold && step < m.hold[e]) return;
    float* F = m.axis[e] == 0 ? f0 : (m.axis[e] == 1 ? f1 : f2);
    const float b = m.saved[3 * e], i0 = m.saved[3 * e + 1];
    float v;
    if (e < m.n_edges) {
        v = mur_1d(i0, m.k[2 * e], F[m.inner[2 * e]], b, m.openems_order);
    } else if (m.openems_corners) {
        v = __fsub_rn(i0, __fmul_rn(m.k[2 * e], b));
    } else {
        const float v0 = mur_1d(i0, m.k[2 * e], F[m.inner[2 * e]], b, m.openems_order);
        const float v1 = mur_1d(m.saved[3 * e + 2], m.k[2 * e + 1], F[m.inner[2 * e + 1]], b, m.openems_order);
        v = __fmul_rn(0.5f, __fadd_rn(v0, v1));
    }
    F[m.node[e]] = v;
    m.last[e] = v;
}

// Σ ½·C_e·u_e² over the last written values (src/engine/boundary/mur.rs:683-704).
__global__ void __launch_bounds__(1024) k_mur_energy(MurDevT m, double* out) {
    double s = 0.0;
    for (uint32_t e = threadIdx.x; e < m.n; e += blockDim.x) {
        const double x = (double)m.last[e];
        s = __dadd_rn(s, __dmul_rn(__dmul_rn(__dmul_rn(0.5, m.cap[e]), x), x));
    }
    const double t = block_sum<1024>(s);
    if (threadIdx.x == 0) out[0] = t;
}

// Frequency-domain dump (src/engine/dump.rs:1420-1700): one running-DFT
// update of every point of the box with the field of state m. The phase is
// f·(t0 + m·dt) reduced modulo one cycle with the product's exact rounding
// error (src/post/dft.rs:196-203), the phasor e^{−j2π·phase}.
struct DumpDev {
    const float* f[3];
    const double* inv_len[3];
    uint32_t lo[3], st[3], n[3];
    uint32_t pitch, ny, npts, nf;
    const double* freqs;
    double dt, t0;
    double* acc;  // [nf][npts][3] complex, re and im interleaved
    // A sampler's table (samp != 0; n holds its dims): taps, factors.
    int32_t samp = 0, roth = 0;
    uint32_t off[3];
    const uint32_t* tidx = nullptr;
    const double* tw = nullptr;
    uint32_t flo[3], fdim[3];
    const double* fac = nullptr;
};

__device__ __forceinline__ double dump_get(const DumpDev& d, int c, uint32_t i, uint32_t j, uint32_t k) {
    return (double)d.f[c][((size_t)i * d.ny + j) * d.pitch + k];
}

// The three components of point p: native (E = u/Δ or H = i/Δ* of the
// edge that starts at the node) or through a sampler (FieldSampler::
// sample_from, src/engine/dump.rs:846-906: Σ wx·wy·wz·m·x over the taps
// of nonzero weight, x the unknown or, for rot H, the circulation of i
// around the primary edge, dump.rs:814-834).
__device__ __forceinline__ void dump_point(const DumpDev& d, uint32_t p, double x[3]) {
    const uint32_t iz = p % d.n[2], r = p / d.n[2], iy = r % d.n[1], ix = r / d.n[1];
    if (!d.samp) {
        const uint32_t i = d.lo[0] + ix * d.st[0], j = d.lo[1] + iy * d.st[1], k = d.lo[2] + iz * d.st[2];
        const size_t idx = ((size_t)i * d.ny + j) * d.pitch + k;
        x[0] = __dmul_rn((double)d.f[0][idx], d.inv_len[0][i]);
        x[1] = __dmul_rn((double)d.f[1][idx], d.inv_len[1][j]);
        x[2] = __dmul_rn((double)d.f[2][idx], d.inv_len[2][k]);
        return;
    }
    const size_t vol = (size_t)d.fdim[0] * d.fdim[1] * d.fdim[2];
    for (int c = 0; c < 3; ++c) {
        const uint32_t ex = 2 * (d.off[0] + c * d.n[0] + ix), ey = 2 * (d.off[1] + c * d.n[1] + iy),
                       ez = 2 * (d.off[2] + c * d.n[2] + iz);
        double v = 0.0;
        for (int tx = 0; tx < 2; ++tx) {
            const double wx = d.tw[ex + tx];
            if (wx == 0.0) continue;
            for (int ty = 0; ty < 2; ++ty) {
                const double wy = d.tw[ey + ty];
                if (wy == 0.0) continue;
                for (int tz = 0; tz < 2; ++tz) {
                    const double wz = d.tw[ez + tz];
                    if (wz == 0.0) continue;
                    const uint32_t nd[3] = {d.tidx[ex + tx], d.tidx[ey + ty], d.tidx[ez + tz]};
                    double val;
                    if (d.roth) {
                        const int a = (c + 1) % 3, b = (c + 2) % 3;
                        val = __dsub_rn(dump_get(d, b, nd[0], nd[1], nd[2]), dump_get(d, a, nd[0], nd[1], nd[2]));
                        if (nd[a] > 0) {
                            uint32_t q[3] = {nd[0], nd[1], nd[2]};
                            q[a] -= 1;
                            val = __dsub_rn(val, dump_get(d, b, q[0], q[1], q[2]));
                        }
                        if (nd[b] > 0) {
                            uint32_t q[3] = {nd[0], nd[1], nd[2]};
                            q[b] -= 1;
                            val = __dadd_rn(val, dump_get(d, a, q[0], q[1], q[2]));
                        }
                    } else {
                        val = dump_get(d, c, nd[0], nd[1], nd[2]);
                    }
                    double m = 1.0;
                    if (d.fac)
                        m = d.fac[c * vol + ((size_t)(nd[0] - d.flo[0]) * d.fdim[1] + (nd[1] - d.flo[1])) * d.fdim[2] +
                                  (nd[2] - d.flo[2])];
                    v = __dadd_rn(v, __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(wx, wy), wz), m), val));
                }
            }
        }
        x[c] = v;
    }
}

// Time-domain snapshot (src/engine/dump.rs TimeDump): the three components
// of every point, in f64, into out[p·3 + component].
__global__ void __launch_bounds__(256) k_snapshot(const __grid_constant__ DumpDev d, double* out) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= d.npts) return;
    double x[3];
    dump_point(d, p, x);
    out[3 * (size_t)p] = x[0];
    out[3 * (size_t)p + 1] = x[1];
    out[3 * (size_t)p + 2] = x[2];
}

__device__ __forceinline__ double frac_toward_zero(double x) { return x - trunc(x); }

__global__ void __launch_bounds__(256) k_dump(const __grid_constant__ DumpDev d, double m) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= d.npts) return;
    double x[3];
    dump_point(d, p, x);
    for (uint32_t q = 0; q < d.nf; ++q) {
        const double fq = d.freqs[q];
        const double a = __dmul_rn(fq, d.dt);
        const double pr = __dmul_rn(a, m);
        const double e = __fma_rn(a, m, -pr);
        const double c = __dmul_rn(fq, d.t0);
        const double ph = frac_toward_zero(__dadd_rn(__dadd_rn(frac_toward_zero(pr), e), frac_toward_zero(c)));
        double sn, cs;
        sincospi(__dmul_rn(2.0, ph), &sn, &cs);
        double* a6 = d.acc + ((size_t)q * d.npts + p) * 6;
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
            a6[2 * cc] = __dadd_rn(a6[2 * cc], __dmul_rn(x[cc], cs));
            a6[2 * cc + 1] = __dsub_rn(a6[2 * cc + 1], __dmul_rn(x[cc], sn));
        }
    }
}

}  // namespace emsk
