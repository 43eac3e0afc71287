// batch.cuh — many models stepping together (sm_100a).
//
// A batch packs the split-schedule work of every model into one launch per
// kernel kind: each model's blocks occupy a range of a global block index
// (prefix sums per kernel kind), and a persistent grid walks the global
// index with a stride, finding a block's model by binary search in the
// prefix sums. Models of uneven sizes therefore share each launch, and a
// model that has met its end criterion (inactive) costs one early return per
// block. The serial hooks (sources, probes, lumped elements) run batched too,
// driven by per-model step counters on the device, so a whole step has no
// host dependency and is captured once as a CUDA graph.
//
// Every per-model expression is that of the single-model split schedule
// (split.cuh, kernels.cuh), so a batched model equals the same model run
// alone bit for bit.
#pragma once

#include "split.cuh"

namespace emsk {

constexpr uint32_t kMaxBatch = 1024;  // models per batch

// One model of a batch, as the batched kernels read it (device memory).
struct BatchModel {
    FusedParams P;         // split-schedule tables, fields in place
    ShellDev shell[2];     // CPML layer shell per side (0 H, 1 E)
    Fields f;
    Coeffs c;              // dense coefficients (pole corrections)
    PoleSideDev pe, ph;    // electric, magnetic poles (n_edges 0: none)
    const uint32_t* run_of[2];
    double dt;
    uint32_t bx;           // split-update blocks per plane
};

// Kernel kinds with a per-model block range.
enum BatchKind { BK_SPLIT = 0, BK_SHELL_H, BK_SHELL_E, BK_POLES_E, BK_POLES_H, BK_KINDS };

// The packed per-model offset table.
struct BatchTable {
    const BatchModel* models;
    const uint32_t* start[BK_KINDS];  // per kind: n + 1 prefix sums of blocks per model
    const int* active;                // per model: 1 steps, 0 frozen
    const uint32_t* steps;            // per model: completed steps
    uint32_t n;
};

// The model whose block range holds global block gb (start: n + 1 sums).
__device__ __forceinline__ uint32_t batch_model(const uint32_t* start, uint32_t n, uint32_t gb) {
    uint32_t lo = 0, hi = n;  // start[lo] <= gb < start[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(start + mid) <= gb) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Split H update of every active model; with ENERGY each block writes its
// energy share (units dt/4) to partials[gb].
template <bool ENERGY>
__global__ void __launch_bounds__(kSplitThreads, ENERGY ? 1 : 8) k_batch_h(const __grid_constant__ BatchTable T,
                                                                         double* partials) {
    const uint32_t total = T.start[BK_SPLIT][T.n];
    for (uint32_t gb = blockIdx.x; gb < total; gb += gridDim.x) {
        const uint32_t m = batch_model(T.start[BK_SPLIT], T.n, gb);
        if (!T.active[m]) continue;  // uniform per block
        const BatchModel& M = T.models[m];
        const uint32_t lb = gb - T.start[BK_SPLIT][m];
        const uint32_t i = lb / M.bx, bx = lb - i * M.bx;
        const double w = split_h_quad<ENERGY, false>(M.P, i, bx * kSplitThreads + threadIdx.x);
        if (ENERGY) {
            const double s = block_sum<kSplitThreads>(w);
            if (threadIdx.x == 0) partials[gb] = s;
            __syncthreads();  // the block sum's shared slots are reused next iteration
        }
    }
}

__global__ void __launch_bounds__(kSplitThreads) k_batch_e(const __grid_constant__ BatchTable T) {
    const uint32_t total = T.start[BK_SPLIT][T.n];
    for (uint32_t gb = blockIdx.x; gb < total; gb += gridDim.x) {
        const uint32_t m = batch_model(T.start[BK_SPLIT], T.n, gb);
        if (!T.active[m]) continue;
        const BatchModel& M = T.models[m];
        const uint32_t lb = gb - T.start[BK_SPLIT][m];
        const uint32_t i = lb / M.bx, bx = lb - i * M.bx;
        split_e_quad<false>(M.P, i, bx * kSplitThreads + threadIdx.x);
    }
}

template <int SIDE>
__global__ void __launch_bounds__(32 * kShellWarps) k_batch_shell(const __grid_constant__ BatchTable T) {
    const uint32_t* start = T.start[BK_SHELL_H + SIDE];
    const uint32_t total = start[T.n];
    for (uint32_t gb = blockIdx.x; gb < total; gb += gridDim.x) {
        const uint32_t m = batch_model(start, T.n, gb);
        if (!T.active[m]) continue;
        const BatchModel& M = T.models[m];
        shell_item<SIDE>(M.P, M.shell[SIDE], gb - start[m], threadIdx.x);
    }
}

// Pole correction of one side of every active model (256 edges per block).
template <int ELECTRIC>
__global__ void __launch_bounds__(256) k_batch_poles(const __grid_constant__ BatchTable T) {
    const uint32_t* start = T.start[ELECTRIC ? BK_POLES_E : BK_POLES_H];
    const uint32_t total = start[T.n];
    for (uint32_t gb = blockIdx.x; gb < total; gb += gridDim.x) {
        const uint32_t m = batch_model(start, T.n, gb);
        if (!T.active[m]) continue;
        const BatchModel& M = T.models[m];
        const uint32_t e = (gb - start[m]) * 256u + threadIdx.x;
        if (ELECTRIC)
            poles_edge(M.f, M.c, M.pe, M.P.runs, M.P.sets, M.run_of[0], 1, M.dt, 0, e);
        else
            poles_edge(M.f, M.c, M.ph, M.P.runs_h, M.P.sets_h, M.run_of[1], 0, M.dt, 0, e);
    }
}

// Saves the field value of every pole edge of one side (electric: after the
// H update's hooks; magnetic: after the E update) (src/engine/dispersive.rs:
// 1173-1180, 1730-1744).
template <int ELECTRIC>
__global__ void __launch_bounds__(256) k_batch_capture(const __grid_constant__ BatchTable T) {
    const uint32_t* start = T.start[ELECTRIC ? BK_POLES_E : BK_POLES_H];
    const uint32_t total = start[T.n];
    for (uint32_t gb = blockIdx.x; gb < total; gb += gridDim.x) {
        const uint32_t m = batch_model(start, T.n, gb);
        if (!T.active[m]) continue;
        const BatchModel& M = T.models[m];
        const PoleSideDev& p = ELECTRIC ? M.pe : M.ph;
        const uint32_t e = (gb - start[m]) * 256u + threadIdx.x;
        if (e < p.n_edges) p.prev[e] = (ELECTRIC ? M.f.u[p.axis[e]] : M.f.i[p.axis[e]])[p.node[e]];
    }
}

// An edge source entry of a batch (src/engine/excite.rs:104-117).
struct BatchSource {
    uint32_t model, node;
    uint32_t axis, hard;
    float weight;
    uint32_t n_amp;
    const float* amp;  // the source's amplitude table on the device
};

// Sources of one field (E or H) of every active model: soft adds w·a (not
// when a = 0, as the step skips a zero soft source), hard sets w·a. Edges
// are distinct within a model (checked at set-up).
template <int ELECTRIC>
__global__ void __launch_bounds__(256) k_batch_sources(const __grid_constant__ BatchTable T, const BatchSource* src,
                                                       uint32_t n) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const BatchSource s = src[q];
    if (!T.active[s.model]) return;
    const uint32_t step = T.steps[s.model];
    const float a = step < s.n_amp ? s.amp[step] : 0.0f;
    if (!s.hard && a == 0.0f) return;
    const BatchModel& M = T.models[s.model];
    float* F = ELECTRIC ? M.f.u[s.axis] : M.f.i[s.axis];
    const float v = __fmul_rn(s.weight, a);
    F[s.node] = s.hard ? v : __fadd_rn(F[s.node], v);
}

// A probe of a batch (src/engine/probe.rs:381-392): sample q = step/interval
// on steps with step % interval == 0.
struct BatchProbe {
    uint32_t model, interval, cap;
    ProbeDevT d;
    double* values;
};

template <int ELECTRIC>
__global__ void __launch_bounds__(128) k_batch_probes(const __grid_constant__ BatchTable T, const BatchProbe* pr,
                                                      uint32_t n) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const BatchProbe& p = pr[q];
    if (!T.active[p.model]) return;
    const uint32_t step = T.steps[p.model];
    if (step % p.interval != 0 || step / p.interval >= p.cap) return;
    const BatchModel& M = T.models[p.model];
    const Fields& f = M.f;
    if (ELECTRIC)
        probe_sample(f.u[0], f.u[1], f.u[2], p.d, p.values + step / p.interval);
    else
        probe_sample(f.i[0], f.i[1], f.i[2], p.d, p.values + step / p.interval);
}

// A lumped element of a batch (src/engine/lumped.rs:1106-1236; a port's
// V and I, src/engine/port.rs:276-290): series index = step.
struct BatchLumped {
    uint32_t model, axis, cap, has_src;
    LumpedDevT d;
    const double* amp;  // source values per step (n_amp), or null
    uint32_t n_amp;
    double* rec;        // terminal current record (record), or null
    double* pv;         // port V (port), or null
    double* pi;         // port I (port), or null
};

__global__ void __launch_bounds__(128) k_batch_lumped_pre(const __grid_constant__ BatchTable T, const BatchLumped* L,
                                                          uint32_t n) {
    const BatchLumped& l = L[blockIdx.x];
    if (blockIdx.x >= n || !T.active[l.model] || !(l.d.record || l.d.has_branch)) return;
    const float* u = T.models[l.model].f.u[l.axis];
    for (uint32_t e = threadIdx.x; e < l.d.n; e += blockDim.x) lumped_pre_e_edge(u, l.d, e);
}

__global__ void __launch_bounds__(256) k_batch_lumped_post(const __grid_constant__ BatchTable T, const BatchLumped* L,
                                                           uint32_t n) {
    const BatchLumped& l = L[blockIdx.x];
    if (blockIdx.x >= n || !T.active[l.model]) return;
    const BatchModel& M = T.models[l.model];
    const uint32_t step = T.steps[l.model];
    const double val = (l.has_src && step < l.n_amp) ? l.amp[step] : 0.0;
    const int active = l.has_src && val != 0.0;
    const bool room = step < l.cap;
    lumped_post_e_block(M.f.u[l.axis], l.d, val, active, M.dt, (l.rec && room) ? l.rec + step : nullptr,
                        (l.pv && room) ? l.pv + step : nullptr, (l.pi && room) ? l.pi + step : nullptr);
}

// Operator energies before an energy step: per model the poles' and the
// lumped branches' held energy (one block per model).
__global__ void __launch_bounds__(1024) k_batch_ops_energy(const __grid_constant__ BatchTable T, const BatchLumped* L,
                                                           uint32_t n_lumped, double* ops) {
    const uint32_t m = blockIdx.x;
    if (m >= T.n || !T.active[m]) return;
    const BatchModel& M = T.models[m];
    double w = pole_energy_block<1024>(M.pe, M.ph);
    if (threadIdx.x == 0) {
        for (uint32_t q = 0; q < n_lumped; ++q)
            if (L[q].model == m && L[q].d.has_branch) w = __dadd_rn(w, branch_energy(L[q].d, M.dt));
        ops[m] = w;
    }
}

// Each active model's energy: its blocks' shares (in block order) × dt/4 plus
// its operator energy (one block per model).
__global__ void __launch_bounds__(1024) k_batch_energy(const __grid_constant__ BatchTable T, const double* partials,
                                                       const double* ops, double* out) {
    const uint32_t m = blockIdx.x;
    if (m >= T.n || !T.active[m]) return;
    const uint32_t b0 = T.start[BK_SPLIT][m], b1 = T.start[BK_SPLIT][m + 1];
    double s = 0.0;
    for (uint32_t q = b0 + threadIdx.x; q < b1; q += blockDim.x) s = __dadd_rn(s, partials[q]);
    const double t = block_sum<1024>(s);
    if (threadIdx.x == 0) out[m] = __dadd_rn(__dmul_rn(__dmul_rn(0.25, T.models[m].dt), t), ops[m]);
}

// End of a step: the step counters of the active models advance.
__global__ void k_batch_advance(const __grid_constant__ BatchTable T, uint32_t* steps) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < T.n && T.active[m]) steps[m] += 1u;
}

}  // namespace emsk
