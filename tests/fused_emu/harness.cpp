// harness.cpp — the fused step kernel (ems_b200/csrc/fused.cuh) run on the
// CPU through emu_shim.h. TEST INFRASTRUCTURE: compiled and called by
// tests/test_fused_emulation.py; shared memory is a heap buffer of exactly
// the size the engine requests, and every global array is bounds-checked by
// the surrounding tables' sizes (the tests run it under the same sizes).
#include "emu_shim.h"

#include <memory>

thread_local EmuDim threadIdx;
EmuDim blockIdx, blockDim, gridDim;
namespace emu {
Block* cur = nullptr;
void fail(const char* what) {
    if (cur && cur->errors.fetch_add(1) == 0) std::snprintf(cur->msg, sizeof cur->msg, "%s", what);
}
}  // namespace emu

#include "../../ems_b200/csrc/fused.cuh"
#include "../../ems_b200/csrc/fused_tables.h"
#include "../../ems_b200/csrc/separate.cuh"
#include "../../ems_b200/csrc/split.cuh"
#include "../../ems_b200/csrc/interior.cuh"
#include "../../ems_b200/csrc/march.cuh"

using namespace emsk;

static char g_err[256];

extern "C" const char* emu_error(void) { return g_err; }

// Runs `steps` fused steps from the fields given in reference layout
// (u_x, u_y, u_z, i_x, i_y, i_z; overwritten with the result). energies:
// the invariant's field part (×dt/4 applied) of each step, or NULL.
extern "C" int emu_fused_run(const ems_engine_desc* d, int tj, unsigned grid, uint64_t steps, float** fields,
                             double* energies) {
    g_err[0] = 0;
    Grid g{};
    g.nx = (uint32_t)d->nodes[0];
    g.ny = (uint32_t)d->nodes[1];
    g.nz = (uint32_t)d->nodes[2];
    g.pitch = (g.nz + 31u) & ~31u;
    g.n = (uint64_t)g.nx * g.ny * g.nz;
    g.np = (uint64_t)g.nx * g.ny * g.pitch;
    FusedTables T = build_fused_tables(d, g.pitch);
    if (!T.why.empty()) {
        std::snprintf(g_err, sizeof g_err, "not eligible: %s", T.why.c_str());
        return 1;
    }
    auto pad = [&](const float* src, std::vector<float>& dst) {
        dst.assign(g.np, 0.0f);
        for (size_t r = 0; r < (size_t)g.nx * g.ny; ++r) std::memcpy(&dst[r * g.pitch], src + r * g.nz, g.nz * 4);
    };
    std::vector<float> buf[2][6];
    for (int c = 0; c < 6; ++c) {
        pad(fields[c], buf[0][c]);
        buf[1][c].assign(g.np, 0.0f);
    }
    std::vector<float> dense[12];
    FusedParams P{};
    P.g = g;
    P.dt = d->dt;
    for (int l = 0; l < 12; ++l) {
        if (T.lane[l].pooled) {
            P.lane[l].rid = T.lane[l].rid.data();
            P.lane[l].rows = T.lane[l].rows.data();
            P.lane[l].bg = T.lane[l].bg;
        } else {
            pad(d->coeff[l], dense[l]);
            P.lane[l].dense = dense[l].data();
        }
    }
    std::vector<std::vector<float>> psi_e, psi_h0, psi_h1;
    std::vector<std::pair<int, int>> at_h;
    psi_e.reserve(T.slabs.size());
    psi_h0.reserve(T.slabs.size());
    psi_h1.reserve(T.slabs.size());
    for (int side = 0; side < 2; ++side)
        for (int c = 0; c < 3; ++c) P.nslab[side][c] = T.nslab[side][c];
    for (const FusedSlabSpec& sp : T.slabs) {
        FSlab& f = P.slab[sp.side][sp.comp][sp.q];
        for (int a = 0; a < 3; ++a) {
            f.lo[a] = (uint32_t)sp.src->lo[a];
            f.hi[a] = (uint32_t)sp.src->hi[a];
        }
        f.normal = (uint32_t)sp.src->normal;
        f.b = sp.src->b;
        f.a = sp.src->a;
        f.k = sp.src->k;
        if (sp.side) {
            psi_e.emplace_back(sp.len, 0.0f);
            f.psi_old = psi_e.back().data();
            f.psi_new = psi_e.back().data();
        } else {
            psi_h0.emplace_back(sp.len, 0.0f);
            psi_h1.emplace_back(sp.len, 0.0f);
            at_h.push_back({sp.comp, sp.q});
        }
    }
    std::vector<double> pj, pq;
    if (T.has_poles) {
        size_t np = 0;
        for (size_t k = 0; k < d->n_ops; ++k)
            if (d->ops[k].kind == EMS_OP_POLES) np = ((const ems_poles*)d->ops[k].table)->electric.n_poles;
        pj.assign(np, 0.0);
        pq.assign(np, 0.0);
        P.has_poles = 1;
        P.runs = T.runs.data();
        P.sets = T.sets.data();
        P.row_runs = T.row_runs.data();
        P.pj = pj.data();
        P.pq = pq.data();
    }
    P.poles_first = T.poles_first ? 1 : 0;
    for (int a = 0; a < 3; ++a) P.cmask[a] = T.cmask[a].data();
    fused_work(P, g.nx, g.ny, tj, grid);
    uint32_t counter = 0;
    int status = 0;
    std::vector<double> partials(grid, 0.0);
    P.counter = &counter;
    P.status = &status;
    P.partials = partials.data();
    size_t smem_bytes = 0;
    switch (tj) {
    case 2: smem_bytes = fused_smem_bytes<2>(g.pitch); break;
    case 4: smem_bytes = fused_smem_bytes<4>(g.pitch); break;
    case 6: smem_bytes = fused_smem_bytes<6>(g.pitch); break;
    default: std::snprintf(g_err, sizeof g_err, "tj must be 2, 4 or 6"); return 1;
    }
    std::vector<unsigned char> smem(smem_bytes + 128);
    unsigned char* sm = smem.data() + (128 - ((uintptr_t)smem.data() & 127)) % 128;
    int cur = 0;
    for (uint64_t s = 0; s < steps; ++s) {
        for (int a = 0; a < 3; ++a) {
            P.uo[a] = buf[cur][a].data();
            P.io[a] = buf[cur][3 + a].data();
            P.un[a] = buf[cur ^ 1][a].data();
            P.in[a] = buf[cur ^ 1][3 + a].data();
        }
        for (size_t q = 0; q < at_h.size(); ++q) {
            FSlab& f = P.slab[0][at_h[q].first][at_h[q].second];
            f.psi_old = (s & 1) ? psi_h1[q].data() : psi_h0[q].data();
            f.psi_new = (s & 1) ? psi_h0[q].data() : psi_h1[q].data();
        }
        P.energy = energies ? 1 : 0;
        counter = 0;
        blockDim = EmuDim{g.pitch, 1, 1};
        gridDim = EmuDim{grid, 1, 1};
        double w = 0.0;
        for (unsigned b = 0; b < grid; ++b) {
            blockIdx = EmuDim{b, 0, 0};
            emu::Block blk;
            std::barrier<> bar((std::ptrdiff_t)g.pitch);
            blk.bar = &bar;
            blk.smem = sm;
            blk.smem_bytes = smem_bytes;
            blk.sums.assign(g.pitch, 0.0);
            std::memset(sm, 0xA5, smem_bytes);  // stale shared memory must not matter
            emu::cur = &blk;
            std::vector<std::thread> th;
            for (unsigned t = 0; t < g.pitch; ++t)
                th.emplace_back([&, t] {
                    threadIdx.x = t;
                    switch (tj) {
                    case 2: k_fused<2, 1024>(P); break;
                    case 4: k_fused<4, 1024>(P); break;
                    default: k_fused<6, 1024>(P); break;
                    }
                });
            for (auto& x : th) x.join();
            emu::cur = nullptr;
            if (blk.errors.load()) {
                std::snprintf(g_err, sizeof g_err, "step %llu block %u: %s", (unsigned long long)s, b, blk.msg);
                return 2;
            }
            if (energies) w += partials[b];
        }
        if (status) {
            std::snprintf(g_err, sizeof g_err, "status flag set at step %llu", (unsigned long long)s);
            return 3;
        }
        if (energies) energies[s] = 0.25 * d->dt * w;
        cur ^= 1;
    }
    for (int c = 0; c < 6; ++c)
        for (size_t r = 0; r < (size_t)g.nx * g.ny; ++r)
            std::memcpy(fields[c] + r * g.nz, &buf[cur][c][r * g.pitch], g.nz * 4);
    return 0;
}

// Runs `steps` steps of the two-kernel schedule (separate.cuh) in place from
// the given fields (reference layout, overwritten). energies as above.
extern "C" int emu_two_run(const ems_engine_desc* d, uint64_t steps, float** fields, double* energies) {
    g_err[0] = 0;
    Grid g{};
    g.nx = (uint32_t)d->nodes[0];
    g.ny = (uint32_t)d->nodes[1];
    g.nz = (uint32_t)d->nodes[2];
    g.pitch = (g.nz + 31u) & ~31u;
    g.n = (uint64_t)g.nx * g.ny * g.nz;
    g.np = (uint64_t)g.nx * g.ny * g.pitch;
    FusedTables T = build_fused_tables(d, g.pitch);
    if (!T.why.empty()) {
        std::snprintf(g_err, sizeof g_err, "not eligible: %s", T.why.c_str());
        return 1;
    }
    auto pad = [&](const float* src, std::vector<float>& dst) {
        dst.assign(g.np, 0.0f);
        for (size_t r = 0; r < (size_t)g.nx * g.ny; ++r) std::memcpy(&dst[r * g.pitch], src + r * g.nz, g.nz * 4);
    };
    std::vector<float> buf[6];
    for (int c = 0; c < 6; ++c) pad(fields[c], buf[c]);
    std::vector<float> dense[12];
    FusedParams P{};
    P.g = g;
    P.dt = d->dt;
    for (int l = 0; l < 12; ++l) {
        if (T.lane[l].pooled) {
            P.lane[l].rid = T.lane[l].rid.data();
            P.lane[l].rows = T.lane[l].rows.data();
            P.lane[l].bg = T.lane[l].bg;
        } else {
            pad(d->coeff[l], dense[l]);
            P.lane[l].dense = dense[l].data();
        }
    }
    std::vector<std::vector<float>> psi;
    psi.reserve(T.slabs.size());
    for (int side = 0; side < 2; ++side)
        for (int c = 0; c < 3; ++c) P.nslab[side][c] = T.nslab[side][c];
    for (const FusedSlabSpec& sp : T.slabs) {
        FSlab& f = P.slab[sp.side][sp.comp][sp.q];
        for (int a = 0; a < 3; ++a) {
            f.lo[a] = (uint32_t)sp.src->lo[a];
            f.hi[a] = (uint32_t)sp.src->hi[a];
        }
        f.normal = (uint32_t)sp.src->normal;
        f.b = sp.src->b;
        f.a = sp.src->a;
        f.k = sp.src->k;
        psi.emplace_back(sp.len, 0.0f);
        f.psi_old = f.psi_new = psi.back().data();
    }
    std::vector<double> pj, pq, pjh, pqh;
    for (size_t k = 0; k < d->n_ops; ++k)
        if (d->ops[k].kind == EMS_OP_POLES) {
            const auto* p = (const ems_poles*)d->ops[k].table;
            pj.assign(p->electric.n_poles, 0.0);
            pq.assign(p->electric.n_poles, 0.0);
            pjh.assign(p->magnetic.n_poles, 0.0);
            pqh.assign(p->magnetic.n_poles, 0.0);
        }
    if (T.has_poles) {
        P.has_poles = 1;
        P.runs = T.runs.data();
        P.sets = T.sets.data();
        P.row_runs = T.row_runs.data();
        P.pj = pj.data();
        P.pq = pq.data();
    }
    std::vector<float> prev_h;
    const ems_pole_side* mside = nullptr;
    for (size_t k = 0; k < d->n_ops; ++k)
        if (d->ops[k].kind == EMS_OP_POLES) mside = &((const ems_poles*)d->ops[k].table)->magnetic;
    if (T.has_poles_h) {
        P.has_poles_h = 1;
        P.runs_h = T.h.runs.data();
        P.sets_h = T.h.sets.data();
        P.row_runs_h = T.h.row_runs.data();
        P.pj_h = pjh.data();
        P.pq_h = pqh.data();
        prev_h.assign(mside->n_edges, 0.0f);
        P.prev_h = prev_h.data();
    }
    P.poles_first = T.poles_first ? 1 : 0;
    for (int a = 0; a < 3; ++a) P.cmask[a] = T.cmask[a].data();
    for (int a = 0; a < 3; ++a) {
        P.uo[a] = P.un[a] = buf[a].data();
        P.io[a] = P.in[a] = buf[3 + a].data();
    }
    const unsigned gx = (g.nz + kSepJ * kSeg - 1) / (kSepJ * kSeg), gy = (g.ny + kSepK - 1) / kSepK, gz = g.nx;
    std::vector<double> partials((size_t)gx * gy * gz, 0.0);
    P.partials = partials.data();
    auto launch = [&](auto body) -> bool {
        blockDim = EmuDim{kSepK, kSepJ, 1};
        gridDim = EmuDim{gx, gy, gz};
        for (unsigned bz = 0; bz < gz; ++bz)
            for (unsigned by = 0; by < gy; ++by)
                for (unsigned bx = 0; bx < gx; ++bx) {
                    blockIdx = EmuDim{bx, by, bz};
                    emu::Block blk;
                    std::barrier<> bar((std::ptrdiff_t)(kSepK * kSepJ));
                    blk.bar = &bar;
                    blk.sums.assign(kSepK * kSepJ, 0.0);
                    emu::cur = &blk;
                    std::vector<std::thread> th;
                    for (unsigned ty = 0; ty < kSepJ; ++ty)
                        for (unsigned tx = 0; tx < kSepK; ++tx)
                            th.emplace_back([&, tx, ty] {
                                threadIdx.x = tx;
                                threadIdx.y = ty;
                                body();
                            });
                    for (auto& x : th) x.join();
                    emu::cur = nullptr;
                    if (blk.errors.load()) {
                        std::snprintf(g_err, sizeof g_err, "%s", blk.msg);
                        return false;
                    }
                }
        return true;
    };
    for (uint64_t s = 0; s < steps; ++s) {
        bool ok = energies ? launch([&] { k_step_h<true>(P); }) : launch([&] { k_step_h<false>(P); });
        if (!ok) return 2;
        if (energies) {
            double w = 0.0;
            for (double x : partials) w += x;
            energies[s] = 0.25 * d->dt * w;
        }
        if (!launch([&] { k_step_e(P); })) return 2;
        // The magnetic-pole edges save their current after the E update.
        if (T.has_poles_h)
            for (size_t e = 0; e < mside->n_edges; ++e) {
                const uint64_t idx = mside->node[e];
                const uint64_t k = idx % g.nz, r = idx / g.nz;
                prev_h[e] = buf[3 + mside->axis[e]][r * g.pitch + k];
            }
    }
    for (int c = 0; c < 6; ++c)
        for (size_t r = 0; r < (size_t)g.nx * g.ny; ++r)
            std::memcpy(fields[c] + r * g.nz, &buf[c][r * g.pitch], g.nz * 4);
    return 0;
}

// Runs a kernel body over a grid (gx, gy, gz) of blocks of (bx, by) threads,
// one host thread per CUDA thread. False (and g_err set) on a shim error.
template <class F>
static bool emu_launch(unsigned gx, unsigned gy, unsigned gz, unsigned bx, unsigned by, F body) {
    blockDim = EmuDim{bx, by, 1};
    gridDim = EmuDim{gx, gy, gz};
    for (unsigned z = 0; z < gz; ++z)
        for (unsigned y = 0; y < gy; ++y)
            for (unsigned x = 0; x < gx; ++x) {
                blockIdx = EmuDim{x, y, z};
                emu::Block blk;
                std::barrier<> bar((std::ptrdiff_t)(bx * by));
                blk.bar = &bar;
                blk.sums.assign(bx * by, 0.0);
                emu::cur = &blk;
                std::vector<std::thread> th;
                for (unsigned ty = 0; ty < by; ++ty)
                    for (unsigned tx = 0; tx < bx; ++tx)
                        th.emplace_back([&, tx, ty] {
                            threadIdx.x = tx;
                            threadIdx.y = ty;
                            body();
                        });
                for (auto& t : th) t.join();
                emu::cur = nullptr;
                if (blk.errors.load()) {
                    std::snprintf(g_err, sizeof g_err, "%s", blk.msg);
                    return false;
                }
            }
    return true;
}

// Runs `steps` steps of the split schedule (split.cuh: streaming H and E
// updates, one CPML shell kernel per side) from the fields given in reference
// layout (overwritten with the result); models without dispersive media,
// lumped elements or sources (those hooks are the per-operator kernels).
static int split_run(const ems_engine_desc* d, uint64_t steps, float** fields, double* energies, bool rows);

extern "C" int emu_split_run(const ems_engine_desc* d, uint64_t steps, float** fields, double* energies) {
    return split_run(d, steps, fields, energies, false);
}

// The same with the row CPML of the engine's split steps (launch_split_rows
// in engine.cu): the update kernels' CPML variant over every quad holding a
// layer node, the plain one elsewhere, no shell. Steps without energy (the
// engine's energy steps take the shell).
extern "C" int emu_split_rows_run(const ems_engine_desc* d, uint64_t steps, float** fields) {
    return split_run(d, steps, fields, nullptr, true);
}

static int split_run(const ems_engine_desc* d, uint64_t steps, float** fields, double* energies, bool rows) {
    g_err[0] = 0;
    for (size_t k = 0; k < d->n_ops; ++k)
        if (d->ops[k].kind != EMS_OP_CPML && d->ops[k].kind != EMS_OP_PROBE) {
            std::snprintf(g_err, sizeof g_err, "only CPML and probes are emulated");
            return 1;
        }
    Grid g{};
    g.nx = (uint32_t)d->nodes[0];
    g.ny = (uint32_t)d->nodes[1];
    g.nz = (uint32_t)d->nodes[2];
    g.pitch = (g.nz + 31u) & ~31u;
    g.n = (uint64_t)g.nx * g.ny * g.nz;
    g.np = (uint64_t)g.nx * g.ny * g.pitch;
    FusedTables T = build_fused_tables(d, g.pitch);
    if (!T.why.empty()) {
        std::snprintf(g_err, sizeof g_err, "not eligible: %s", T.why.c_str());
        return 1;
    }
    auto pad = [&](const float* src, std::vector<float>& dst) {
        dst.assign(g.np, 0.0f);
        for (size_t r = 0; r < (size_t)g.nx * g.ny; ++r) std::memcpy(&dst[r * g.pitch], src + r * g.nz, g.nz * 4);
    };
    std::vector<float> buf[6];
    for (int c = 0; c < 6; ++c) pad(fields[c], buf[c]);
    std::vector<float> dense[12];
    FusedParams P{};
    P.g = g;
    P.dt = d->dt;
    for (int l = 0; l < 12; ++l) {
        if (T.lane[l].pooled) {
            P.lane[l].rid = T.lane[l].rid.data();
            P.lane[l].rows = T.lane[l].rows.data();
        } else {
            pad(d->coeff[l], dense[l]);
            P.lane[l].dense = dense[l].data();
        }
    }
    std::vector<std::vector<float>> psi;
    psi.reserve(T.slabs.size());
    for (int side = 0; side < 2; ++side)
        for (int c = 0; c < 3; ++c) P.nslab[side][c] = T.nslab[side][c];
    for (const FusedSlabSpec& sp : T.slabs) {
        FSlab& f = P.slab[sp.side][sp.comp][sp.q];
        for (int a = 0; a < 3; ++a) {
            f.lo[a] = (uint32_t)sp.src->lo[a];
            f.hi[a] = (uint32_t)sp.src->hi[a];
        }
        f.normal = (uint32_t)sp.src->normal;
        f.b = sp.src->b;
        f.a = sp.src->a;
        f.k = sp.src->k;
        psi.emplace_back(sp.len, 0.0f);
        f.psi_old = f.psi_new = psi.back().data();
    }
    for (int a = 0; a < 3; ++a) P.cmask[a] = T.cmask[a].data();
    for (int a = 0; a < 3; ++a) {
        P.uo[a] = P.un[a] = buf[a].data();
        P.io[a] = P.in[a] = buf[3 + a].data();
    }
    std::vector<ShellBox> st[2];
    std::vector<uint32_t> win[2];
    ShellDev sd[2];
    RowCpml R;
    if (rows) {
        R = row_cpml_plan(slab_geometry(T), d->nodes);
        if (!R.ok) {
            std::snprintf(g_err, sizeof g_err, "row CPML plan does not apply");
            return 1;
        }
    }
    for (int side = 0; side < 2; ++side) {
        uint32_t total = 0;
        st[side] = shell_boxes(T, d->nodes, side, &total);
        win[side] = shell_windows(st[side], total);
        sd[side] = ShellDev{st[side].data(), (uint32_t)st[side].size(), total, 0u, win[side].data()};
    }
    const unsigned gx = split_blocks_x(g);
    std::vector<double> partials((size_t)gx * g.nx, 0.0);
    P.partials = partials.data();
    // launch_split_rows of engine.cu, emulated.
    auto rows_update = [&](int side) -> bool {
        const uint32_t qpr = g.pitch >> 2, qrow = (g.nz + 3u) / 4u;
        const uint32_t xl = R.lo[side][0], xh = R.hi[side][0], yl = R.lo[side][1], yh = R.hi[side][1];
        const uint32_t zl = (R.lo[side][2] + 3u) / 4u, zr = std::max(zl, R.hi[side][2] / 4u);
        auto go = [&](bool cpml, uint32_t i0, uint32_t planes, const QuadMap& M) -> bool {
            if (!planes || !M.count) return true;
            FusedParams Q = P;
            Q.qmap = M;
            const unsigned bx = (M.count + kSplitThreads - 1) / kSplitThreads;
            if (side == 0)
                return cpml ? emu_launch(bx, planes, 1, kSplitThreads, 1, [&] { k_split_h<false, false, true>(Q, i0); })
                            : emu_launch(bx, planes, 1, kSplitThreads, 1, [&] { k_split_h<false>(Q, i0); });
            return cpml ? emu_launch(bx, planes, 1, kSplitThreads, 1, [&] { k_split_e<false, true>(Q, i0); })
                        : emu_launch(bx, planes, 1, kSplitThreads, 1, [&] { k_split_e(Q, i0); });
        };
        const uint32_t mid = xh > xl ? xh - xl : 0u, nrows = yh > yl ? yh - yl : 0u;
        const uint32_t ends = zl + (qrow > zr ? qrow - zr : 0u), inner = zr - zl;
        return go(true, 0u, xl, QuadMap{0u, 0u, 0u, 0u, 0u, 0u, g.ny * qpr}) &&
               go(true, xh, g.nx - xh, QuadMap{0u, 0u, 0u, 0u, 0u, 0u, g.ny * qpr}) &&
               go(true, xl, mid, QuadMap{0u, 0u, 0u, 0u, 0u, 0u, yl * qpr}) &&
               go(true, xl, mid, QuadMap{0u, yh * qpr, 0u, 0u, 0u, 0u, (g.ny - yh) * qpr}) &&
               go(true, xl, mid, QuadMap{1u, 0u, yl, ends, zl, zr, nrows * ends}) &&
               go(false, xl, mid, QuadMap{1u, 0u, yl, inner, 0u, zl, nrows * inner});
    };
    auto shell = [&](int side) -> bool {
        const uint32_t blocks = shell_blocks(sd[side]);
        if (!blocks) return true;
        const ShellDev S = sd[side];
        return side ? emu_launch(blocks, 1, 1, 32 * kShellWarps, 1, [&] { k_shell<1>(P, S); })
                    : emu_launch(blocks, 1, 1, 32 * kShellWarps, 1, [&] { k_shell<0>(P, S); });
    };
    for (uint64_t s = 0; s < steps; ++s) {
        if (rows) {
            if (!rows_update(0) || !rows_update(1)) return 2;
            continue;
        }
        bool ok = energies ? emu_launch(gx, g.nx, 1, kSplitThreads, 1, [&] { k_split_h<true>(P, 0u); })
                           : emu_launch(gx, g.nx, 1, kSplitThreads, 1, [&] { k_split_h<false>(P, 0u); });
        if (!ok || !shell(0)) return 2;
        if (energies) {
            double w = 0.0;
            for (double x : partials) w += x;
            energies[s] = 0.25 * d->dt * w;
        }
        if (!emu_launch(gx, g.nx, 1, kSplitThreads, 1, [&] { k_split_e(P, 0u); }) || !shell(1)) return 2;
    }
    for (int c = 0; c < 6; ++c)
        for (size_t r = 0; r < (size_t)g.nx * g.ny; ++r)
            std::memcpy(fields[c] + r * g.nz, &buf[c][r * g.pitch], g.nz * 4);
    return 0;
}

// Runs `steps` steps of the interior schedule (interior.cuh: the split H
// update and CPML correction outside the interior box, the one-pass kernel
// inside it, the split E update and CPML correction outside it, old and new
// fields in two buffers) from the fields given in reference layout
// (overwritten with the result); models with CPML layers and probes only.
extern "C" int emu_interior_run(const ems_engine_desc* d, uint64_t steps, float** fields, uint32_t* box) {
    g_err[0] = 0;
    for (size_t k = 0; k < d->n_ops; ++k)
        if (d->ops[k].kind != EMS_OP_CPML && d->ops[k].kind != EMS_OP_PROBE) {
            std::snprintf(g_err, sizeof g_err, "only CPML and probes are emulated");
            return 1;
        }
    Grid g{};
    g.nx = (uint32_t)d->nodes[0];
    g.ny = (uint32_t)d->nodes[1];
    g.nz = (uint32_t)d->nodes[2];
    g.pitch = (g.nz + 31u) & ~31u;
    g.n = (uint64_t)g.nx * g.ny * g.nz;
    g.np = (uint64_t)g.nx * g.ny * g.pitch;
    FusedTables T = build_fused_tables(d, g.pitch);
    if (!T.why.empty()) {
        std::snprintf(g_err, sizeof g_err, "not eligible: %s", T.why.c_str());
        return 1;
    }
    auto pad = [&](const float* src, std::vector<float>& dst) {
        dst.assign(g.np, 0.0f);
        for (size_t r = 0; r < (size_t)g.nx * g.ny; ++r) std::memcpy(&dst[r * g.pitch], src + r * g.nz, g.nz * 4);
    };
    std::vector<float> buf[6], buf2[6];
    for (int c = 0; c < 6; ++c) pad(fields[c], buf[c]);
    for (int c = 0; c < 6; ++c) buf2[c] = buf[c];
    InteriorBox IB{};
    const std::string why = interior_box(d, g, IB);
    if (!why.empty()) {
        std::snprintf(g_err, sizeof g_err, "no interior schedule: %s", why.c_str());
        return 1;
    }
    for (int a = 0; a < 3; ++a) {
        box[a] = IB.lo[a];
        box[3 + a] = IB.hi[a];
    }
    std::vector<float> dense[12];
    FusedParams P{};
    P.g = g;
    P.dt = d->dt;
    for (int l = 0; l < 12; ++l) {
        if (T.lane[l].pooled) {
            P.lane[l].rid = T.lane[l].rid.data();
            P.lane[l].rows = T.lane[l].rows.data();
        } else {
            pad(d->coeff[l], dense[l]);
            P.lane[l].dense = dense[l].data();
        }
    }
    std::vector<std::vector<float>> psi;
    psi.reserve(T.slabs.size());
    for (int side = 0; side < 2; ++side)
        for (int c = 0; c < 3; ++c) P.nslab[side][c] = T.nslab[side][c];
    for (const FusedSlabSpec& sp : T.slabs) {
        FSlab& f = P.slab[sp.side][sp.comp][sp.q];
        for (int a = 0; a < 3; ++a) {
            f.lo[a] = (uint32_t)sp.src->lo[a];
            f.hi[a] = (uint32_t)sp.src->hi[a];
        }
        f.normal = (uint32_t)sp.src->normal;
        f.b = sp.src->b;
        f.a = sp.src->a;
        f.k = sp.src->k;
        psi.emplace_back(sp.len, 0.0f);
        f.psi_old = f.psi_new = psi.back().data();
    }
    for (int a = 0; a < 3; ++a) P.cmask[a] = T.cmask[a].data();
    std::vector<ShellBox> st[2];
    std::vector<uint32_t> win[2];
    ShellDev sd[2];
    for (int side = 0; side < 2; ++side) {
        uint32_t total = 0;
        st[side] = shell_boxes(T, d->nodes, side, &total);
        win[side] = shell_windows(st[side], total);
        sd[side] = ShellDev{st[side].data(), (uint32_t)st[side].size(), total, 0u, win[side].data()};
    }
    const unsigned gx = split_blocks_x(g);
    std::vector<double> partials((size_t)gx * g.nx, 0.0);
    P.partials = partials.data();
    auto shell = [&](int side) -> bool {
        const uint32_t blocks = shell_blocks(sd[side]);
        if (!blocks) return true;
        const ShellDev S = sd[side];
        return side ? emu_launch(blocks, 1, 1, 32 * kShellWarps, 1, [&] { k_shell<1>(P, S); })
                    : emu_launch(blocks, 1, 1, 32 * kShellWarps, 1, [&] { k_shell<0>(P, S); });
    };
    uint32_t ib[3];
    const uint32_t planes = 5;  // chunks that start inside the box
    interior_blocks(IB, planes, ib);
    for (uint64_t s = 0; s < steps; ++s) {
        for (int a = 0; a < 3; ++a) {
            P.uo[a] = buf[a].data();
            P.io[a] = buf[3 + a].data();
            P.un[a] = buf2[a].data();
            P.in[a] = buf2[3 + a].data();
        }
        P.skip = IB;
        // The engine's launches over the nodes outside the box: planes
        // before and after it, rows before and after it, quads before and
        // after it in its rows (QuadMap).
        const uint32_t qpr = g.pitch >> 2, zl = IB.lo[2] / 4u, zr = IB.hi[2] / 4u, nzl = zl + (qpr - zr);
        const uint32_t xn = IB.hi[0] - IB.lo[0];
        auto outer = [&](bool h_side) -> bool {
            auto go = [&](unsigned bx, unsigned by, uint32_t i0) {
                return h_side ? emu_launch(bx, by, 1, kSplitThreads, 1, [&] { k_split_h<false>(P, i0); })
                              : emu_launch(bx, by, 1, kSplitThreads, 1, [&] { k_split_e(P, i0); });
            };
            auto nb = [](uint32_t n) { return (n + kSplitThreads - 1) / kSplitThreads; };
            bool ok = true;
            P.qmap = QuadMap{};
            ok = ok && go(gx, IB.lo[0], 0u);
            ok = ok && go(gx, g.nx - IB.hi[0], IB.hi[0]);
            P.qmap = QuadMap{0u, 0u, 0u, 1u, 0u, 0u, IB.lo[1] * qpr};
            ok = ok && go(nb(P.qmap.count), xn, IB.lo[0]);
            P.qmap = QuadMap{0u, IB.hi[1] * qpr, 0u, 1u, 0u, 0u, (g.ny - IB.hi[1]) * qpr};
            ok = ok && (P.qmap.count == 0 || go(nb(P.qmap.count), xn, IB.lo[0]));
            P.qmap = QuadMap{1u, 0u, IB.lo[1], nzl, zl, zr, (IB.hi[1] - IB.lo[1]) * nzl};
            ok = ok && go(nb(P.qmap.count), xn, IB.lo[0]);
            P.qmap = QuadMap{};
            return ok;
        };
        if (!outer(true) || !shell(0)) return 2;
        if (!emu_launch(ib[0], ib[1], ib[2], 32 * kInWarps, 1, [&] { k_interior<false>(P, IB, planes); })) return 2;
        if (!outer(false) || !shell(1)) return 2;
        for (int c = 0; c < 6; ++c) std::swap(buf[c], buf2[c]);
    }
    for (int c = 0; c < 6; ++c)
        for (size_t r = 0; r < (size_t)g.nx * g.ny; ++r)
            std::memcpy(fields[c] + r * g.nz, &buf[c][r * g.pitch], g.nz * 4);
    return 0;
}

// pole_prev_fold of fused_tables.h for a model (1: the side's pole kernel
// may store its saved values itself).
extern "C" int emu_pole_prev_fold(const ems_engine_desc* d, int electric) {
    int pos_cpml = -1, pos_poles = -1;
    for (size_t k = 0; k < d->n_ops; ++k) {
        if (d->ops[k].kind == EMS_OP_CPML) pos_cpml = (int)k;
        if (d->ops[k].kind == EMS_OP_POLES) pos_poles = (int)k;
    }
    const bool poles_first = pos_poles >= 0 && pos_cpml >= 0 && pos_poles < pos_cpml;
    return pole_prev_fold(d, electric != 0, poles_first) ? 1 : 0;
}

// Runs `steps` steps of the marching kernel (march.cuh) with R rows per
// block, an S-stage ring and x chunks of `planes` from the fields given in
// reference layout (overwritten with the result); models with CPML layers
// and probes only (the pole and hook kernels are the split schedule's).
// Old and new fields in two buffers, H ψ in two buffers, E ψ in place; the
// tensor copies of the ring are bounds- and alignment-checked.
template <uint32_t R, uint32_t S>
static int march_run(const ems_engine_desc* d, uint64_t steps, float** fields, uint32_t planes,
                     uint32_t test_extra_tx = 0, uint64_t wait_ns = 0) {
    g_err[0] = 0;
    for (size_t k = 0; k < d->n_ops; ++k)
        if (d->ops[k].kind != EMS_OP_CPML && d->ops[k].kind != EMS_OP_PROBE) {
            std::snprintf(g_err, sizeof g_err, "only CPML and probes are emulated");
            return 1;
        }
    const std::string why = march_why(d);
    if (!why.empty()) {
        std::snprintf(g_err, sizeof g_err, "no marching step: %s", why.c_str());
        return 1;
    }
    Grid g{};
    g.nx = (uint32_t)d->nodes[0];
    g.ny = (uint32_t)d->nodes[1];
    g.nz = (uint32_t)d->nodes[2];
    g.pitch = (g.nz + 31u) & ~31u;
    g.n = (uint64_t)g.nx * g.ny * g.nz;
    g.np = (uint64_t)g.nx * g.ny * g.pitch;
    FusedTables T = build_fused_tables(d, g.pitch);
    if (!T.why.empty()) {
        std::snprintf(g_err, sizeof g_err, "not eligible: %s", T.why.c_str());
        return 1;
    }
    auto pad = [&](const float* src, std::vector<float>& dst) {
        dst.assign(g.np, 0.0f);
        for (size_t r = 0; r < (size_t)g.nx * g.ny; ++r) std::memcpy(&dst[r * g.pitch], src + r * g.nz, g.nz * 4);
    };
    std::vector<float> buf[2][6];
    for (int c = 0; c < 6; ++c) {
        pad(fields[c], buf[0][c]);
        buf[1][c] = buf[0][c];
    }
    std::vector<float> dense[12];
    FusedParams P{};
    P.g = g;
    P.dt = d->dt;
    for (int l = 0; l < 12; ++l) {
        if (T.lane[l].pooled) {
            P.lane[l].rid = T.lane[l].rid.data();
            P.lane[l].rows = T.lane[l].rows.data();
            P.lane[l].bg = T.lane[l].bg;
        } else {
            pad(d->coeff[l], dense[l]);
            P.lane[l].dense = dense[l].data();
        }
    }
    std::vector<std::vector<float>> psi_e, psi_h0, psi_h1;
    std::vector<std::pair<int, int>> at_h;
    psi_e.reserve(T.slabs.size());
    psi_h0.reserve(T.slabs.size());
    psi_h1.reserve(T.slabs.size());
    for (int side = 0; side < 2; ++side)
        for (int c = 0; c < 3; ++c) P.nslab[side][c] = T.nslab[side][c];
    for (const FusedSlabSpec& sp : T.slabs) {
        FSlab& f = P.slab[sp.side][sp.comp][sp.q];
        for (int a = 0; a < 3; ++a) {
            f.lo[a] = (uint32_t)sp.src->lo[a];
            f.hi[a] = (uint32_t)sp.src->hi[a];
        }
        f.normal = (uint32_t)sp.src->normal;
        f.b = sp.src->b;
        f.a = sp.src->a;
        f.k = sp.src->k;
        if (sp.side) {
            psi_e.emplace_back(sp.len, 0.0f);
            f.psi_old = f.psi_new = psi_e.back().data();
        } else {
            psi_h0.emplace_back(sp.len, 0.0f);
            psi_h1.emplace_back(sp.len, 0.0f);
            at_h.push_back({sp.comp, sp.q});
        }
    }
    for (int a = 0; a < 3; ++a) P.cmask[a] = T.cmask[a].data();
    std::vector<double> pj, pq;
    if (T.has_poles) {
        size_t np = 0;
        for (size_t k = 0; k < d->n_ops; ++k)
            if (d->ops[k].kind == EMS_OP_POLES) np = ((const ems_poles*)d->ops[k].table)->electric.n_poles;
        pj.assign(np, 0.0);
        pq.assign(np, 0.0);
        P.has_poles = 1;
        P.runs = T.runs.data();
        P.sets = T.sets.data();
        P.row_runs = T.row_runs.data();
        P.pj = pj.data();
        P.pq = pq.data();
    }
    P.poles_first = T.poles_first ? 1 : 0;
    int status = 0, diverged = 0;
    P.status = &status;
    P.diverged = &diverged;
    P.test_extra_tx = test_extra_tx;
    P.wait_ns = wait_ns;
    using LT = MarchLayout<R>;
    const size_t smem_bytes = LT::bytes(S);
    std::vector<unsigned char> smem(smem_bytes + 128);
    unsigned char* sm = smem.data() + (128 - ((uintptr_t)smem.data() & 127)) % 128;
    uint32_t nb[3];
    march_blocks(g, R, planes, nb);
    const unsigned threads = 32 * (R + 1);
    int cur = 0;
    for (uint64_t s = 0; s < steps; ++s) {
        MarchMaps M{};
        for (int a = 0; a < 3; ++a) {
            P.uo[a] = buf[cur][a].data();
            P.io[a] = buf[cur][3 + a].data();
            P.un[a] = buf[cur ^ 1][a].data();
            P.in[a] = buf[cur ^ 1][3 + a].data();
            M.u[a] = CUtensorMap{P.uo[a], {g.pitch, g.ny, g.nx}, {g.pitch, (uint64_t)g.ny * g.pitch}, {kMW, R + 2, 1}};
            M.i[a] = CUtensorMap{P.io[a], {g.pitch, g.ny, g.nx}, {g.pitch, (uint64_t)g.ny * g.pitch}, {kMW, R + 1, 1}};
        }
        for (size_t q = 0; q < at_h.size(); ++q) {
            FSlab& f = P.slab[0][at_h[q].first][at_h[q].second];
            f.psi_old = (s & 1) ? psi_h1[q].data() : psi_h0[q].data();
            f.psi_new = (s & 1) ? psi_h0[q].data() : psi_h1[q].data();
        }
        blockDim = EmuDim{threads, 1, 1};
        gridDim = EmuDim{nb[0], nb[1], nb[2]};
        for (unsigned bz = 0; bz < nb[2]; ++bz)
            for (unsigned by = 0; by < nb[1]; ++by)
                for (unsigned bx = 0; bx < nb[0]; ++bx) {
                    blockIdx = EmuDim{bx, by, bz};
                    emu::Block blk;
                    std::barrier<> bar((std::ptrdiff_t)threads);
                    blk.bar = &bar;
                    std::vector<std::unique_ptr<std::barrier<>>> wbars;
                    for (unsigned q = 0; q < threads / 32; ++q) wbars.emplace_back(new std::barrier<>(32));
                    for (unsigned q = 0; q < threads / 32; ++q) blk.wbar[q] = wbars[q].get();
                    blk.smem = sm;
                    blk.smem_bytes = smem_bytes;
                    blk.sums.assign(threads, 0.0);
                    std::memset(sm, 0xA5, smem_bytes);  // stale shared memory must not matter
                    emu::cur = &blk;
                    std::vector<std::thread> th;
                    for (unsigned t = 0; t < threads; ++t)
                        th.emplace_back([&, t] {
                            threadIdx.x = t;
                            k_march<R, S, false>(P, M, planes);
                        });
                    for (auto& x : th) x.join();
                    emu::cur = nullptr;
                    if (blk.errors.load()) {
                        std::snprintf(g_err, sizeof g_err, "step %llu block (%u, %u, %u): %s",
                                      (unsigned long long)s, bx, by, bz, blk.msg);
                        return 2;
                    }
                }
        if (status) {
            std::snprintf(g_err, sizeof g_err, "status flag set at step %llu", (unsigned long long)s);
            return 3;
        }
        if (diverged) {
            std::snprintf(g_err, sizeof g_err, "divergence flag set at step %llu", (unsigned long long)s);
            return 4;
        }
        cur ^= 1;
    }
    for (int c = 0; c < 6; ++c)
        for (size_t r = 0; r < (size_t)g.nx * g.ny; ++r)
            std::memcpy(fields[c] + r * g.nz, &buf[cur][c][r * g.pitch], g.nz * 4);
    return 0;
}

// One marching step with the bounded-wait test hook armed (the first block
// expects 16 bytes more than its copies deliver; waits give up after
// `wait_ns`): 3 when the kernel reports the timeout as the engine reads it.
extern "C" int emu_march_timeout(const ems_engine_desc* d, float** fields, uint64_t wait_ns) {
    return march_run<7, 3>(d, 1, fields, 4, 16u, wait_ns);
}

extern "C" int emu_march_run(const ems_engine_desc* d, uint64_t steps, float** fields, uint32_t rows, uint32_t planes) {
    if (rows == 7) return march_run<7, 3>(d, steps, fields, planes);
    if (rows == 8) return march_run<8, 4>(d, steps, fields, planes);
    if (rows == 3) return march_run<3, 4>(d, steps, fields, planes);
    std::snprintf(g_err, sizeof g_err, "rows must be 3, 7 or 8");
    return 1;
}
