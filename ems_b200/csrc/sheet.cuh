// sheet.cuh — conducting sheets as device operators (src/engine/sheet.rs).
//
// A sheet edge's ladder (node voltages u, layer currents h, f64) lives in
// device arrays; the constants of the distinct ladders are shared. Both
// hooks run one thread per item:
//   k_sheet_post_h: one thread per corrected dual edge (its corrections from
//     every sheet edge that touches it, applied in edge order, as the
//     reference's serial loop applies them), and one per sheet edge that
//     takes the + face voltage from the field array;
//   k_sheet_post_e: one thread per sheet edge (Ampère sums in coupling order,
//     the Thomas sweep over its ladder, the + face written back).
// The arithmetic is the reference's expression by expression, each double
// operation explicitly rounded.
#pragma once

#include <cstdint>

#include "arith.cuh"

namespace emsk {

struct SheetDevT {
    uint32_t n_edges = 0;
    const uint8_t* axis = nullptr;     // per edge
    const uint32_t* node = nullptr;    // per edge, device index
    const uint32_t* nn = nullptr;      // per edge: ladder nodes
    const uint32_t* k0 = nullptr;      // per edge: first node constant
    const uint32_t* a0 = nullptr;      // per edge: first layer constant
    const uint32_t* n0 = nullptr;      // per edge: first node of u
    const uint32_t* l0 = nullptr;      // per edge: first layer of h
    const uint32_t* c0 = nullptr;      // n_edges + 1: couplings [c0[e], c0[e+1])
    const double* c_edge = nullptr;
    const uint8_t* c_axis = nullptr;   // per coupling
    const uint32_t* c_node = nullptr;
    const double* w_up = nullptr;
    const double* w_dn = nullptr;
    const double* ecorr = nullptr;
    const double* two_c = nullptr;     // per node constant
    const double* cp = nullptr;
    const double* inv_den = nullptr;
    const double* a = nullptr;         // per layer constant
    double* u = nullptr;               // state: per ladder node
    double* h = nullptr;               // state: per ladder layer
    double* x = nullptr;               // scratch: per ladder node
    double* wcorr = nullptr;           // per edge: its term of the energy correction
    // post_h: corrected dual edges, entries [t0[t], t0[t+1]) (edge, corr).
    uint32_t n_targets = 0;
    const uint8_t* t_axis = nullptr;
    const uint32_t* t_node = nullptr;
    const uint32_t* t0 = nullptr;
    const uint32_t* t_edge = nullptr;
    const double* t_corr = nullptr;
};

// post_h (src/engine/sheet.rs:950-972): u_0 of every edge from the array;
// each dual edge on the - side gets i = flush(i + f32(corr·(u_{nn-1} - u_0)))
// from every sheet edge touching it, in edge order.
__global__ void __launch_bounds__(256) k_sheet_post_h(const float* __restrict__ ux, const float* __restrict__ uy,
                                                      const float* __restrict__ uz, float* ix, float* iy, float* iz,
                                                      SheetDevT d) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const float* U[3] = {ux, uy, uz};
    if (t < d.n_targets) {
        float* I = d.t_axis[t] == 0 ? ix : (d.t_axis[t] == 1 ? iy : iz);
        const uint32_t at = d.t_node[t];
        float v = I[at];
        for (uint32_t q = d.t0[t]; q < d.t0[t + 1]; ++q) {
            const uint32_t e = d.t_edge[q];
            const double stored = (double)U[d.axis[e]][d.node[e]];
            const double diff = __dsub_rn(d.u[d.n0[e] + d.nn[e] - 1], stored);
            v = flush(__fadd_rn(v, __double2float_rn(__dmul_rn(d.t_corr[q], diff))));
        }
        I[at] = v;
    } else if (t < d.n_targets + d.n_edges) {
        const uint32_t e = t - d.n_targets;
        d.u[d.n0[e]] = (double)U[d.axis[e]][d.node[e]];
    }
}

// post_e (src/engine/sheet.rs:974-1050): one edge per thread.
__global__ void __launch_bounds__(128) k_sheet_post_e(float* ux, float* uy, float* uz, const float* __restrict__ ix,
                                                      const float* __restrict__ iy, const float* __restrict__ iz,
                                                      SheetDevT d) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= d.n_edges) return;
    const float* I[3] = {ix, iy, iz};
    double s_up = 0.0, s_dn = 0.0, s_e = 0.0;
    for (uint32_t c = d.c0[e]; c < d.c0[e + 1]; ++c) {
        const double iv = (double)I[d.c_axis[c]][d.c_node[c]];
        s_up = __dadd_rn(s_up, __dmul_rn(d.w_up[c], iv));
        s_dn = __dadd_rn(s_dn, __dmul_rn(d.w_dn[c], iv));
        s_e = __dadd_rn(s_e, __dmul_rn(d.ecorr[c], iv));
    }
    const uint32_t nn = d.nn[e];
    const double* two_c = d.two_c + d.k0[e];
    const double* cp = d.cp + d.k0[e];
    const double* inv_den = d.inv_den + d.k0[e];
    const double* a = d.a + d.a0[e];
    double* U = d.u + d.n0[e];
    double* H = d.h + d.l0[e];
    double* X = d.x + d.n0[e];
    // Forward sweep: X holds d'_k.
    double xp = 0.0;
    for (uint32_t k = 0; k < nn; ++k) {
        double r = __dmul_rn(two_c[k], U[k]);
        if (k + 1 < nn) r = __dsub_rn(r, H[k]);
        if (k > 0) r = __dadd_rn(r, __dadd_rn(H[k - 1], __dmul_rn(a[k - 1], xp)));
        if (k == 0) r = __dadd_rn(r, s_up);
        if (k + 1 == nn) r = __dadd_rn(r, s_dn);
        xp = __dmul_rn(r, inv_den[k]);
        X[k] = xp;
    }
    // Back substitution: X holds the mean voltages.
    for (uint32_t k = nn - 1; k-- > 0;) {
        xp = __dsub_rn(X[k], __dmul_rn(cp[k], xp));
        X[k] = xp;
    }
    for (uint32_t j = 0; j + 1 < nn; ++j)
        H[j] = __dadd_rn(H[j], __dmul_rn(__dmul_rn(2.0, a[j]), __dsub_rn(X[j], X[j + 1])));
    for (uint32_t k = 0; k < nn; ++k) U[k] = __dsub_rn(__dmul_rn(2.0, X[k]), U[k]);
    const float up = flush(__double2float_rn(U[0]));
    float* F = d.axis[e] == 0 ? ux : (d.axis[e] == 1 ? uy : uz);
    F[d.node[e]] = up;
    d.wcorr[e] = __dmul_rn(s_e, __dsub_rn(U[nn - 1], (double)up));
}

// energy (src/engine/sheet.rs:1052-1083): per edge its ladder's electric
// and magnetic energy less ½·C·u_0², plus the correction term of the last
// post_e; summed over the edges in one block.
template <unsigned THREADS>
__device__ __forceinline__ double sheet_energy_block(const SheetDevT& d, double dt) {
    double s = 0.0;
    for (uint32_t e = threadIdx.x; e < d.n_edges; e += blockDim.x) {
        const uint32_t nn = d.nn[e];
        const double* two_c = d.two_c + d.k0[e];
        const double* a = d.a + d.a0[e];
        const double* U = d.u + d.n0[e];
        const double* H = d.h + d.l0[e];
        double w = 0.0;
        for (uint32_t k = 0; k < nn; ++k)
            w = __dadd_rn(w, __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(0.25, two_c[k]), dt), U[k]), U[k]));
        w = __dsub_rn(w, __dmul_rn(__dmul_rn(__dmul_rn(0.5, d.c_edge[e]), U[0]), U[0]));
        for (uint32_t j = 0; j + 1 < nn; ++j) {
            const double l = __ddiv_rn(dt, __dmul_rn(2.0, a[j]));
            w = __dadd_rn(w, __dmul_rn(__dmul_rn(__dmul_rn(0.5, l), H[j]), H[j]));
        }
        s = __dadd_rn(s, __dadd_rn(w, d.wcorr[e]));
    }
    return block_sum<THREADS>(s);
}

__global__ void __launch_bounds__(1024) k_sheet_energy(SheetDevT d, double dt, double* out) {
    const double t = sheet_energy_block<1024>(d, dt);
    if (threadIdx.x == 0) out[0] = t;
}

}  // namespace emsk
