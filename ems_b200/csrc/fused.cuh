// fused.cuh — the single-pass step kernel of the B200 FDTD engine (sm_100a).
//
// One launch advances every field by one step: the H update, the CPML
// correction of the H edges, the E update, the CPML correction of the E
// edges and the electric-pole ADE correction, with the same expressions in
// the same order as the separate kernels (and the reference), so results
// are identical bit for bit. It reads the old fields and writes new ones
// into the other buffer (fields double-buffered), so a CTA never waits for
// another: it recomputes the few H values on its tile's low edge that its
// E update needs (one halo row, and one halo plane at the start of its x
// range) from the old state.
//
// Tiling: a CTA owns TJ consecutive y-rows × the whole z-row (one thread per
// z-node) and marches along x over a chunk of planes; work items (row tile,
// x chunk) are taken from an atomic counter by a persistent grid. The E
// voltages of the tile's window (TJ+2 rows, 3 components) are staged in
// shared memory by TMA bulk copies (cp.async.bulk, one row per copy) into a
// 3-stage ring, one plane ahead; H currents come straight to registers one
// plane ahead. Coefficients are pooled rows: the distinct z-rows of each
// array and a row id per (x, y) row; each array's most frequent row is held
// in shared memory, the ids of the next plane are staged there too.
#pragma once

#include "kernels.cuh"

namespace emsk {

constexpr int kStages = 3;
constexpr uint64_t kWaitNs = 2000000000ull;  // a bounded mbarrier wait gives up after 2 s

struct Lane {
    const float* dense;     // dense array (padded layout), or null if pooled
    const uint32_t* rid;    // pooled: row id per (x, y) row
    const float* rows;      // pooled: the distinct rows, pitch floats each
    uint32_t bg;            // pooled: the row held in shared memory
};

struct FSlab {
    uint32_t lo[3], hi[3];
    uint32_t normal;
    uint32_t pad;
    const float* b;
    const float* a;
    const float* k;
    const float* psi_old;
    float* psi_new;
};

// A box of the CPML layer shell in which every node has the same CPML
// slabs per component (split schedule): first node, extent, the index of its
// first node in the side's flat node list, and per component c the slabs in
// application order, list[c] = count | q0 << 4 | q1 << 8 | q2 << 12 | q3 << 16.
struct ShellBox {
    uint32_t lo[3], n[3];
    uint32_t start;
    uint32_t list[3];
};

struct PoleRun {
    uint32_t kb, ke;   // z range of the run's edges
    uint32_t p0;       // state index of the run's first pole
    uint32_t set;      // offset of the run's constants (np poles × {a, inv_c, inv_z})
    uint32_t np;       // poles per edge
    uint32_t kinds;    // bit q set: pole q is not trapezoidal (leapfrog or openEMS)
    uint32_t e0;       // edge index of the run's first edge (in the side's table)
    uint32_t axis;     // the edges' axis
    uint32_t node0;    // padded node index of the run's first edge
    uint32_t oe;       // bit q: pole q is openEMS's f32 pole; kOeDebye: an openEMS Debye edge
    double sum_inv_z;
};

// A box of nodes [lo, hi) per axis whose quads the split kernels leave to
// the one-pass interior kernel (interior.cuh): lo >= 1, hi <= n − 1, lo[2] and
// hi[2] multiples of 4. Empty (all 0): the split kernels update every quad.
struct InteriorBox {
    uint32_t lo[3], hi[3];
};

// Which quads of a plane a split-kernel thread takes (the interior
// schedule's launches over the nodes outside its box): mode 0, quad q0 + t
// for thread t; mode 1, the quads outside z range [zl, zr) of rows row0,
// row0 + 1, …: thread t takes row row0 + t / nzl and the (t mod nzl)-th of
// the row's quads below zl or from zr on. t >= count (if count) takes none.
struct QuadMap {
    uint32_t mode, q0, row0, nzl, zl, zr, count;
};

struct FusedParams {
    Grid g;
    const float* uo[3];
    const float* io[3];
    float* un[3];
    float* in[3];
    Lane lane[12];
    FSlab slab[2][3][4];   // [side: 0 H, 1 E][component][application order]
    int nslab[2][3];
    // Per axis and node index: bit side·12 + component·4 + q is set where the
    // index lies in the normal range of slab [side][component][q] (a slab
    // spans the grid on its other axes, so that decides membership).
    const uint32_t* cmask[3];
    const uint4* row_runs; // electric poles: per (x*3 + axis)*ny + y: (first run, count, z min, z end)
    const PoleRun* runs;
    const double* sets;
    double* pj;
    double* pq;
    int has_poles;
    const uint4* row_runs_h; // magnetic poles (two-kernel schedule only)
    const PoleRun* runs_h;
    const double* sets_h;
    double* pj_h;
    double* pq_h;
    const float* prev_h;   // saved i^{n−½} of each magnetic-pole edge
    int has_poles_h;
    int poles_first;       // the dispersive medium was registered before the CPML
    double dt;
    uint32_t tiles_j, chunk, n_chunks, n_items;
    uint32_t* counter;
    double* partials;      // per CTA energy share
    int energy;
    int* status;           // nonzero: a bounded wait ran out
    int* diverged;         // set by the marching kernel where it writes a non-finite E value
    uint64_t wait_ns;      // limit of the marching kernel's waits (0: kWaitNs)
    uint32_t test_extra_tx; // test hook: bytes the marching kernel's first block expects in excess
    InteriorBox skip;      // quads the split kernels leave to the interior kernel
    QuadMap qmap;          // which quads a split-kernel thread takes
};

#ifndef EMS_HOST_EMULATION
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase `parity` of the barrier; gives up (returns false) after
// `limit_ns` nanoseconds.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = kWaitNs) {
    uint32_t done = 0;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0;; ++it) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 63u) == 63u && global_ns() - t0 > limit_ns) return false;
    }
}

// One bulk copy global → shared, completing on `bar` (16-byte aligned, size multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
#define EMS_DYNAMIC_SMEM(name) extern __shared__ __align__(128) unsigned char name[]
#define EMS_SHARED __shared__
#else
// CPU emulation (tests): the bulk copies complete at once; a barrier is a
// phase counter and a wait that would not succeed is reported.
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t) { *bar = 0; }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) { emu::expect_tx(bar, bytes); }
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = kWaitNs) {
    return emu::wait(bar, parity, limit_ns);
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    emu::bulk(dst, src, bytes, bar);
}
__device__ __forceinline__ void fence_proxy_async() {}
__device__ __forceinline__ void fence_mbar_init() {}
#define EMS_DYNAMIC_SMEM(name) unsigned char* name = emu::dynamic_smem()
#define EMS_SHARED static
#endif

// The CPML correction of one field value t by every slab of `list` that
// contains the node, in order: ψ = flush(b·ψ + a·s), t = flush(t + coef·(k·s + ψ)),
// s the derivative term along the slab's normal (sA along next(c), sB along prev(c)).
template <bool WRITE>
__device__ __forceinline__ float cpml_body_inl(const FSlab* list, int n, uint32_t i, uint32_t j, uint32_t k, int c,
                                               float t, float coef, float sA, float sB) {
    const int na = (c + 1) % 3;
    for (int q = 0; q < n; ++q) {
        const FSlab& s = list[q];
        if (i < s.lo[0] || i >= s.hi[0] || j < s.lo[1] || j >= s.hi[1] || k < s.lo[2] || k >= s.hi[2]) continue;
        const uint32_t d = s.normal == 0 ? i - s.lo[0] : (s.normal == 1 ? j - s.lo[1] : k - s.lo[2]);
        const uint32_t idx = ((i - s.lo[0]) * (s.hi[1] - s.lo[1]) + (j - s.lo[1])) * (s.hi[2] - s.lo[2]) + (k - s.lo[2]);
        const float sv = (int)s.normal == na ? sA : sB;
        const float psi = flush(__fadd_rn(__fmul_rn(s.b[d], s.psi_old[idx]), __fmul_rn(s.a[d], sv)));
        if (WRITE) s.psi_new[idx] = psi;
        t = flush(__fadd_rn(t, __fmul_rn(coef, __fadd_rn(__fmul_rn(s.k[d], sv), psi))));
    }
    return t;
}

// The same, out of line (most nodes lie in no layer).
template <bool WRITE>
__device__ __noinline__ float cpml_body(const FSlab* list, int n, uint32_t i, uint32_t j, uint32_t k, int c, float t,
                                        float coef, float sA, float sB) {
    return cpml_body_inl<WRITE>(list, n, i, j, k, c, t, coef, sA, sB);
}

// The CPML slabs containing node (i, j, k): one bit per slab (cmask).
__device__ __forceinline__ uint32_t cpml_bits(const FusedParams& P, uint32_t i, uint32_t j, uint32_t k) {
    return P.cmask[0][i] | P.cmask[1][j] | P.cmask[2][k];
}

// The CPML correction of component C on side SIDE (0 H, 1 E) by the slabs
// whose bits are set in `bits`, in application order; out of line, as most
// nodes lie in no layer.
template <bool WRITE, int SIDE, int C>
__device__ __forceinline__ float cpml_apply(const FusedParams& P, uint32_t bits, uint32_t i, uint32_t j, uint32_t k,
                                            float t, float coef, float sA, float sB) {
    uint32_t m = (bits >> (SIDE * 12 + C * 4)) & 15u;
    while (m) {
        const int q = __ffs(m) - 1;
        m &= m - 1;
        t = cpml_body<WRITE>(&P.slab[SIDE][C][q], 1, i, j, k, C, t, coef, sA, sB);
    }
    return t;
}

// Electric-pole correction of the E edge (axis a, row (i, j), node k)
// (src/engine/dispersive.rs:1392-1470), if the edge has poles. A leapfrog
// pole's new state does not depend on the corrected voltage and is stored
// at once; a trapezoidal pole's is formed from its old state after it.
__device__ __forceinline__ float poles_run_inl(const PoleRun* runs, const double* sets, double* pj, double* pq,
                                               double dt, const uint4 rr, uint32_t k, float u_star, float prev_f,
                                               float cb_f, const float* prev_arr) {
    for (uint32_t q = 0; q < rr.y; ++q) {
        const PoleRun R = runs[rr.x + q];
        if (k < R.kb || k >= R.ke) continue;
        const uint32_t p0 = R.p0 + (k - R.kb) * R.np;
        const double* cs = sets + R.set;
        const double cb = (double)cb_f;
        // The field value the update starts from: the one given, or the
        // edge's saved value (magnetic poles, src/engine/dispersive.rs:1173).
        const float prev32 = prev_arr ? prev_arr[R.e0 + (k - R.kb)] : prev_f;
        if (R.oe & kOeDebye) return oe_debye_edge(cs, cs + 1, cs + 2, 3u, pj + p0, R.np, prev32, u_star);
        const double prev = (double)prev32;
        const double half_prev = __dmul_rn(0.5, prev);
        double s = 0.0;
        float u32 = u_star;
        for (uint32_t p = 0; p < R.np; ++p) {
            const double a = cs[3 * p], ic = cs[3 * p + 1], iz = cs[3 * p + 2];
            const double jq = pj[p0 + p], qq = pq[p0 + p];
            if ((R.oe >> p) & 1u) {
                u32 = oe_pole_step(a, ic, iz, pj[p0 + p], pq[p0 + p], prev32, u32);
            } else if ((R.kinds >> p) & 1u) {
                const double jn = __dadd_rn(__dmul_rn(a, jq), __dmul_rn(iz, __dsub_rn(prev, __dmul_rn(qq, ic))));
                pj[p0 + p] = jn;
                pq[p0 + p] = __dadd_rn(qq, __dmul_rn(dt, jn));
                s = __dadd_rn(s, jn);
            } else {
                s = __dadd_rn(s, __dmul_rn(__dadd_rn(__dsub_rn(__dmul_rn(a, jq), __dmul_rn(qq, ic)), half_prev), iz));
            }
        }
        // Without trapezoidal poles the denominator is exactly 1 and the
        // quotient the numerator itself.
        const double num = __dsub_rn((double)u32, __dmul_rn(cb, s));
        const float u_new = R.sum_inv_z == 0.0
                                ? (float)num
                                : (float)__ddiv_rn(num, __dadd_rn(1.0, __dmul_rn(__dmul_rn(0.5, cb), R.sum_inv_z)));
        if (R.kinds != (1u << R.np) - 1u) {
            const double half_new = __dmul_rn(0.5, (double)u_new);
            for (uint32_t p = 0; p < R.np; ++p) {
                if ((R.kinds >> p) & 1u) continue;
                const double a = cs[3 * p], ic = cs[3 * p + 1], iz = cs[3 * p + 2];
                const double jq = pj[p0 + p], qq = pq[p0 + p];
                const double kk = __dadd_rn(__dsub_rn(__dmul_rn(a, jq), __dmul_rn(qq, ic)), half_prev);
                const double jb = __dmul_rn(__dadd_rn(kk, half_new), iz);
                pj[p0 + p] = __dsub_rn(__dmul_rn(2.0, jb), jq);
                pq[p0 + p] = __dadd_rn(qq, __dmul_rn(dt, jb));
            }
        }
        return u_new;
    }
    return u_star;
}

// The same, out of line.
__device__ __noinline__ float poles_run(const PoleRun* runs, const double* sets, double* pj, double* pq, double dt,
                                        const uint4 rr, uint32_t k, float u_star, float prev_f, float cb_f,
                                        const float* prev_arr) {
    return poles_run_inl(runs, sets, pj, pq, dt, rr, k, u_star, prev_f, cb_f, prev_arr);
}

// The pole correction of one edge, if its row has runs (the common case,
// no runs, stays inline).
__device__ __forceinline__ float poles_apply(const FusedParams& P, const uint4 rr, uint32_t k, float u_star,
                                             float prev_f, float cb_f) {
    if (k < rr.z || k >= rr.w) return u_star;
    return poles_run(P.runs, P.sets, P.pj, P.pq, P.dt, rr, k, u_star, prev_f, cb_f, nullptr);
}

// Shared memory layout of the fused kernel (floats unless noted):
//   u stages: kStages × 3 × (TJ + 2) × pitch
//   H tile:   2 × TJ × pitch            (i_x, i_y of the owned rows, for the k−1 neighbour)
//   bg rows:  12 × pitch                (each lane's background row)
//   ids:      2 × 12 × (TJ + 1) u32     (row ids, current / next plane)
//   runs:     2 × 3 × TJ uint4          (pole runs of the owned rows, 16-byte aligned)
//   bars:     kStages u64
template <int TJ>
__host__ __device__ constexpr size_t fused_smem_bytes(uint32_t pitch) {
    return sizeof(float) * ((size_t)kStages * 3 * (TJ + 2) * pitch + 2 * (size_t)TJ * pitch + 12 * (size_t)pitch) +
           sizeof(uint32_t) * 2 * 12 * (TJ + 1) + 16 + sizeof(uint4) * 2 * 3 * TJ + 8 * kStages + 64;
}

template <int TJ, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) k_fused(const __grid_constant__ FusedParams P) {
    EMS_DYNAMIC_SMEM(smem_raw);
    const Grid g = P.g;
    const uint32_t pitch = g.pitch;
    const uint32_t k = threadIdx.x;
    const uint32_t nthr = blockDim.x;
    float* su = (float*)smem_raw;                                   // u stages
    float* sh = su + (size_t)kStages * 3 * (TJ + 2) * pitch;        // H tile
    float* sbg = sh + 2 * (size_t)TJ * pitch;                       // background rows
    uint32_t* sid = (uint32_t*)(sbg + 12 * (size_t)pitch);          // row ids [2][12][TJ+1]
    uint4* srun = (uint4*)(((uintptr_t)(sid + 2 * 12 * (TJ + 1)) + 15) & ~(uintptr_t)15);  // pole runs [2][3][TJ]
    uint64_t* bars = (uint64_t*)(srun + 2 * 3 * TJ);
    EMS_SHARED uint32_t s_item;
    EMS_SHARED int s_fail;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
        s_fail = 0;
    }
    for (int l = 0; l < 12; ++l)
        if (!P.lane[l].dense && k < pitch) sbg[l * pitch + k] = P.lane[l].rows[(size_t)P.lane[l].bg * pitch + k];
    __syncthreads();
    uint32_t uses[kStages] = {0, 0, 0};
    double w_acc = 0.0;
    const uint32_t si = g.ny * pitch;
    const size_t stage_floats = (size_t)3 * (TJ + 2) * pitch;

    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(P.counter, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= P.n_items || s_fail) break;
        const uint32_t tj = item % P.tiles_j, ch = item / P.tiles_j;
        const int j0 = (int)(tj * TJ);
        const uint32_t x0 = ch * P.chunk, x1 = min(g.nx, x0 + P.chunk);
        const uint32_t xs = x0 > 0 ? x0 - 1 : x0;  // first plane (a warm-up H plane before x0)

        // Issues the bulk copies of plane p's window into stage p % kStages.
        auto issue = [&](uint32_t p) {
            if (threadIdx.x != 0 || p >= g.nx) return;
            const int st = (int)(p % kStages);
            uint32_t bytes = 0;
            for (int r = 0; r < TJ + 2; ++r) {
                const int j = j0 - 1 + r;
                if (j >= 0 && j < (int)g.ny) bytes += 3 * pitch * 4;
            }
            fence_proxy_async();
            mbar_expect_tx(&bars[st], bytes);
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < TJ + 2; ++r) {
                    const int j = j0 - 1 + r;
                    if (j < 0 || j >= (int)g.ny) continue;
                    bulk_g2s(su + st * stage_floats + ((size_t)c * (TJ + 2) + r) * pitch,
                             P.uo[c] + (size_t)p * si + (size_t)j * pitch, pitch * 4, &bars[st]);
                }
        };
        // Row ids of plane p (rows j0−1..j0+TJ−1) and pole runs of its owned rows into buffer b.
        auto stage_ids = [&](uint32_t p, int b) {
            for (uint32_t t = threadIdx.x; t < 12 * (TJ + 1) + 3 * TJ; t += nthr) {
                if (t < 12 * (TJ + 1)) {
                    const int l = (int)(t / (TJ + 1)), r = (int)(t % (TJ + 1));
                    const int j = j0 - 1 + r;
                    uint32_t v = 0xffffffffu;
                    if (p < g.nx && j >= 0 && j < (int)g.ny && !P.lane[l].dense) v = P.lane[l].rid[(size_t)p * g.ny + j];
                    sid[(b * 12 + l) * (TJ + 1) + r] = v;
                } else {
                    const uint32_t q = t - 12 * (TJ + 1);
                    const int a = (int)(q / TJ), r = (int)(q % TJ);
                    const int j = j0 + r;
                    uint4 v = make_uint4(0, 0, 0, 0);
                    if (P.has_poles && p < g.nx && j < (int)g.ny) v = P.row_runs[((size_t)p * 3 + a) * g.ny + j];
                    srun[(b * 3 + a) * TJ + r] = v;
                }
            }
        };
        // Pointer to row r (plane p, y = j0−1+r) of lane l, from the ids in buffer b.
        auto row = [&](int l, int b, int r, uint32_t p) -> const float* {
            const Lane& L = P.lane[l];
            const int j = j0 - 1 + r;
            if (L.dense) return L.dense + (size_t)p * si + (size_t)j * pitch;
            const uint32_t id = sid[(b * 12 + l) * (TJ + 1) + r];
            return id == L.bg ? sbg + l * pitch : L.rows + (size_t)id * pitch;
        };

        issue(xs);
        issue(xs + 1);
        stage_ids(xs, xs & 1);
        __syncthreads();

        float hy_prev[TJ], hz_prev[TJ];
#pragma unroll
        for (int r = 0; r < TJ; ++r) hy_prev[r] = hz_prev[r] = 0.0f;
        // Old currents of the current plane (rows j0−1..j0+TJ−1), loaded a plane ahead.
        float io_c[3][TJ + 1];
        auto load_io = [&](uint32_t p, float (&dst)[3][TJ + 1]) {
#pragma unroll
            for (int r = 0; r < TJ + 1; ++r) {
                const int j = j0 - 1 + r;
                const bool ok = p < g.nx && j >= 0 && j < (int)g.ny && k < g.nz;
                const size_t idx = (size_t)p * si + (size_t)j * pitch + k;
#pragma unroll
                for (int c = 0; c < 3; ++c) dst[c][r] = ok ? P.io[c][idx] : 0.0f;
            }
        };
        load_io(xs, io_c);

        for (uint32_t i = xs; i < x1; ++i) {
            const bool warm = i < x0;
            const int st = (int)(i % kStages);
            const int st1 = (int)((i + 1) % kStages);
            const int b = (int)(i & 1);
            // The stage of plane i+2 was last read in iteration i−1 (synchronised since).
            issue(i + 2);
            if (i + 1 < g.nx) stage_ids(i + 1, b ^ 1);  // ready after this iteration's final sync
            bool ok = mbar_wait(&bars[st], uses[st] & 1u);
            uses[st]++;
            if (i + 1 < g.nx) {
                ok = ok && mbar_wait(&bars[st1], uses[st1] & 1u);
            }
            if (!ok) atomicExch(&s_fail, 1);
            const float* U0 = su + st * stage_floats;   // plane i:   [c][r][k]
            const float* U1 = su + st1 * stage_floats;  // plane i+1
            auto u0 = [&](int c, int r, uint32_t kk) { return U0[((size_t)c * (TJ + 2) + r) * pitch + kk]; };
            auto u1 = [&](int c, int r) { return U1[((size_t)c * (TJ + 2) + r) * pitch + k]; };
            const bool nxt = i + 1 < g.nx;
            float io_n[3][TJ + 1];
            load_io(i + 1, io_n);  // prefetch for the next plane

            // ---- H of rows j0−1 .. j0+TJ−1 (r = 0 .. TJ); r = 0 is the halo row.
            // Window row w of the staged voltages is y = j0 − 1 + w: row j is r, row j + 1 is r + 1.
            float hx[TJ + 1], hy[TJ + 1], hz[TJ + 1];
#pragma unroll
            for (int r = 0; r < TJ + 1; ++r) {
                const int j = j0 - 1 + r;
                hx[r] = hy[r] = hz[r] = 0.0f;
                if (j < 0 || j >= (int)g.ny || k >= g.nz) continue;
                const bool own = r >= 1 && !warm;
                const size_t idx = (size_t)i * si + (size_t)j * pitch + k;
                const uint32_t cbits = cpml_bits(P, i, j, k);
                const float ux = u0(0, r, k), uy = u0(1, r, k), uz = u0(2, r, k);
                // x: (uz[j+1] − uz[j]) − (uy[k+1] − uy[k])
                if (j + 1 < (int)g.ny && k + 1 < g.nz) {
                    const float da = row(6, b, r, i)[k], db = row(9, b, r, i)[k];
                    const float A = __fsub_rn(u0(2, r + 1, k), uz), B = __fsub_rn(u0(1, r, k + 1), uy);
                    const float old = io_c[0][r];
                    const float nw = flush(__fsub_rn(__fmul_rn(da, old), __fmul_rn(db, __fsub_rn(A, B))));
                    if (P.energy && own) w_acc = __dadd_rn(w_acc, weight(da, __dmul_rn((double)old, (double)nw), db));
                    float t = nw;
                    if (cbits) {
                        t = own ? cpml_apply<true, 0, 0>(P, cbits, i, j, k, t, -db, A, __fmul_rn(-1.0f, B))
                                : cpml_apply<false, 0, 0>(P, cbits, i, j, k, t, -db, A, __fmul_rn(-1.0f, B));
                    }
                    hx[r] = t;
                    if (own) P.in[0][idx] = t;
                }
                // y: (ux[k+1] − ux[k]) − (uz[i+1] − uz[i])   (owned rows only)
                if (r >= 1 && nxt && k + 1 < g.nz) {
                    const float da = row(7, b, r, i)[k], db = row(10, b, r, i)[k];
                    const float A = __fsub_rn(u0(0, r, k + 1), ux), B = __fsub_rn(u1(2, r), uz);
                    const float old = io_c[1][r];
                    const float nw = flush(__fsub_rn(__fmul_rn(da, old), __fmul_rn(db, __fsub_rn(A, B))));
                    if (P.energy && own) w_acc = __dadd_rn(w_acc, weight(da, __dmul_rn((double)old, (double)nw), db));
                    float t = nw;
                    if (cbits) {
                        t = own ? cpml_apply<true, 0, 1>(P, cbits, i, j, k, t, -db, A, __fmul_rn(-1.0f, B))
                                : cpml_apply<false, 0, 1>(P, cbits, i, j, k, t, -db, A, __fmul_rn(-1.0f, B));
                    }
                    hy[r] = t;
                    if (own) P.in[1][idx] = t;
                }
                // z: (uy[i+1] − uy[i]) − (ux[j+1] − ux[j])
                if (nxt && j + 1 < (int)g.ny) {
                    const float da = row(8, b, r, i)[k], db = row(11, b, r, i)[k];
                    const float A = __fsub_rn(u1(1, r), uy), B = __fsub_rn(u0(0, r + 1, k), ux);
                    const float old = io_c[2][r];
                    const float nw = flush(__fsub_rn(__fmul_rn(da, old), __fmul_rn(db, __fsub_rn(A, B))));
                    if (P.energy && own) w_acc = __dadd_rn(w_acc, weight(da, __dmul_rn((double)old, (double)nw), db));
                    float t = nw;
                    if (cbits) {
                        t = own ? cpml_apply<true, 0, 2>(P, cbits, i, j, k, t, -db, A, __fmul_rn(-1.0f, B))
                                : cpml_apply<false, 0, 2>(P, cbits, i, j, k, t, -db, A, __fmul_rn(-1.0f, B));
                    }
                    hz[r] = t;
                    if (own) P.in[2][idx] = t;
                }
            }
            if (!warm) {
                // i_x, i_y of the owned rows for the k − 1 neighbours.
#pragma unroll
                for (int r = 1; r < TJ + 1; ++r) {
                    sh[(size_t)(r - 1) * pitch + k] = hx[r];
                    sh[(size_t)(TJ + r - 1) * pitch + k] = hy[r];
                }
            }
            __syncthreads();
            if (s_fail) break;
            if (!warm) {
                // ---- E of the owned rows.
#pragma unroll
                for (int r = 1; r < TJ + 1; ++r) {
                    const int j = j0 - 1 + r;
                    if (j >= (int)g.ny || k >= g.nz) continue;
                    const size_t idx = (size_t)i * si + (size_t)j * pitch + k;
                    const float uxo = u0(0, r, k), uyo = u0(1, r, k), uzo = u0(2, r, k);
                    const uint32_t cbits = cpml_bits(P, i, j, k);
                    const float hxk1 = k > 0 ? sh[(size_t)(r - 1) * pitch + k - 1] : 0.0f;
                    const float hyk1 = k > 0 ? sh[(size_t)(TJ + r - 1) * pitch + k - 1] : 0.0f;
                    float ca, cb;
                    if (P.energy) {
                        for (int c = 0; c < 3; ++c) {
                            const float uo = c == 0 ? uxo : (c == 1 ? uyo : uzo);
                            w_acc = __dadd_rn(w_acc, weight(row(c, b, r, i)[k], __dmul_rn((double)uo, (double)uo),
                                                            row(3 + c, b, r, i)[k]));
                        }
                    }
                    // x: (iz[j] − iz[j−1]) − (iy[k] − iy[k−1])
                    if (nxt) {
                        ca = row(0, b, r, i)[k];
                        cb = row(3, b, r, i)[k];
                        const float A = __fsub_rn(hz[r], hz[r - 1]), B = __fsub_rn(hy[r], hyk1);
                        float t = flush(__fadd_rn(__fmul_rn(ca, uxo), __fmul_rn(cb, __fsub_rn(A, B))));
                        if (P.has_poles && P.poles_first) t = poles_apply(P, srun[(b * 3 + 0) * TJ + r - 1], k, t, uxo, cb);
                        if (cbits) t = cpml_apply<true, 1, 0>(P, cbits, i, j, k, t, cb, A, __fmul_rn(-1.0f, B));
                        if (P.has_poles && !P.poles_first) t = poles_apply(P, srun[(b * 3 + 0) * TJ + r - 1], k, t, uxo, cb);
                        P.un[0][idx] = t;
                    }
                    // y: (ix[k] − ix[k−1]) − (iz[i] − iz[i−1])
                    if (j + 1 < (int)g.ny) {
                        ca = row(1, b, r, i)[k];
                        cb = row(4, b, r, i)[k];
                        const float A = __fsub_rn(hx[r], hxk1), B = __fsub_rn(hz[r], hz_prev[r - 1]);
                        float t = flush(__fadd_rn(__fmul_rn(ca, uyo), __fmul_rn(cb, __fsub_rn(A, B))));
                        if (P.has_poles && P.poles_first) t = poles_apply(P, srun[(b * 3 + 1) * TJ + r - 1], k, t, uyo, cb);
                        if (cbits) t = cpml_apply<true, 1, 1>(P, cbits, i, j, k, t, cb, A, __fmul_rn(-1.0f, B));
                        if (P.has_poles && !P.poles_first) t = poles_apply(P, srun[(b * 3 + 1) * TJ + r - 1], k, t, uyo, cb);
                        P.un[1][idx] = t;
                    }
                    // z: (iy[i] − iy[i−1]) − (ix[j] − ix[j−1])
                    if (k + 1 < g.nz) {
                        ca = row(2, b, r, i)[k];
                        cb = row(5, b, r, i)[k];
                        const float A = __fsub_rn(hy[r], hy_prev[r - 1]), B = __fsub_rn(hx[r], hx[r - 1]);
                        float t = flush(__fadd_rn(__fmul_rn(ca, uzo), __fmul_rn(cb, __fsub_rn(A, B))));
                        if (P.has_poles && P.poles_first) t = poles_apply(P, srun[(b * 3 + 2) * TJ + r - 1], k, t, uzo, cb);
                        if (cbits) t = cpml_apply<true, 1, 2>(P, cbits, i, j, k, t, cb, A, __fmul_rn(-1.0f, B));
                        if (P.has_poles && !P.poles_first) t = poles_apply(P, srun[(b * 3 + 2) * TJ + r - 1], k, t, uzo, cb);
                        P.un[2][idx] = t;
                    }
                }
            }
#pragma unroll
            for (int r = 1; r < TJ + 1; ++r) {
                hy_prev[r - 1] = hy[r];
                hz_prev[r - 1] = hz[r];
            }
#pragma unroll
            for (int r = 0; r < TJ + 1; ++r)
                for (int c = 0; c < 3; ++c) io_c[c][r] = io_n[c][r];
            __syncthreads();
        }
        // Drain: planes x1 (waited as i + 1, not counted) and x1 + 1 (issued,
        // not waited) complete their phases before the stages are reused.
        for (uint32_t p = x1; p < x1 + 2 && p < g.nx; ++p) {
            const int st = (int)(p % kStages);
            if (!mbar_wait(&bars[st], uses[st] & 1u)) atomicExch(&s_fail, 1);
            uses[st]++;
        }
        __syncthreads();
    }
    if (P.energy) {
        const double s = block_sum<1024>(w_acc);
        if (threadIdx.x == 0) P.partials[blockIdx.x] = s;
    }
    if (threadIdx.x == 0 && s_fail) atomicExch(P.status, 1);
}

}  // namespace emsk
