// fused_tables.h — host-side tables of the fused step kernel (fused.cuh).
//
// Pure host code (no CUDA calls): from an engine descriptor it decides
// whether the fused schedule can run, pools the coefficient rows, orders the
// CPML slabs per (side, component) and turns the electric poles into runs
// along z. The engine uploads the result; the CPU emulation of the kernel
// used by the tests reads it in place.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/ems_gpu.h"

namespace emsk {

// Pools the rows of one coefficient array (src/engine/coeffs.rs:395-599,
// Lane::Pooled): the distinct z-rows and a row id per (x, y) row; pooled only
// when at most a quarter of the rows are distinct (coeffs.rs POOL_RATIO).
struct Pooled {
    bool pooled = false;
    std::vector<uint32_t> rid;
    std::vector<float> rows;  // pitch floats each, zero beyond nz
    uint32_t bg = 0;          // the most frequent row
};

inline Pooled pool_lane(const float* a, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t pitch) {
    Pooled P;
    const size_t nrows = (size_t)nx * ny;
    std::unordered_map<uint64_t, std::vector<uint32_t>> seen;
    std::vector<size_t> first;  // source row of each distinct id
    std::vector<uint32_t> count;
    P.rid.resize(nrows);
    for (size_t r = 0; r < nrows; ++r) {
        const float* row = a + r * nz;
        uint64_t hsh = 1469598103934665603ull;
        for (size_t k = 0; k < nz; ++k) {
            uint32_t b;
            std::memcpy(&b, &row[k], 4);
            hsh = (hsh ^ b) * 1099511628211ull;
        }
        auto& cand = seen[hsh];
        uint32_t id = 0xffffffffu;
        for (uint32_t c : cand)
            if (std::memcmp(a + first[c] * nz, row, (size_t)nz * 4) == 0) {
                id = c;
                break;
            }
        if (id == 0xffffffffu) {
            id = (uint32_t)first.size();
            first.push_back(r);
            count.push_back(0);
            cand.push_back(id);
            if (first.size() * 4 > nrows) {
                P.rid.clear();
                return P;  // not pooled
            }
        }
        count[id]++;
        P.rid[r] = id;
    }
    P.pooled = true;
    P.rows.assign(first.size() * pitch, 0.0f);
    for (size_t d = 0; d < first.size(); ++d) std::memcpy(&P.rows[d * pitch], a + first[d] * nz, (size_t)nz * 4);
    P.bg = (uint32_t)(std::max_element(count.begin(), count.end()) - count.begin());
    return P;
}

struct FusedSlabSpec {
    int side, comp, q;             // place in FusedParams::slab[side][comp][q]
    size_t op_slab;                // index of the slab in the CPML table
    const ems_cpml_slab* src;
    size_t len;                    // ψ values of the slab
};

struct PoleRuns {
    std::vector<PoleRun> runs;
    std::vector<double> sets;
    std::vector<uint4> row_runs;  // per (x*3 + axis)*ny + y: first run, count, z min, z end
    std::vector<uint32_t> run_of; // per edge: its run
};

// The poles of one side as runs along z (edges are in (plane, axis, y, z)
// order): consecutive edges of one row with the same constants share a run.
// Returns "" or why the side cannot be held as runs.
inline std::string pole_runs(const ems_pole_side* pe, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t pitch,
                             PoleRuns& R) {
    std::unordered_map<std::string, uint32_t> set_of;
    R.row_runs.assign((size_t)nx * 3 * ny, uint4{0, 0, 0, 0});
    uint64_t last_row = ~0ull;
    uint32_t last_k = 0;
    for (size_t e = 0; e < pe->n_edges; ++e) {
        const uint64_t idx = pe->node[e];
        const uint64_t kk = idx % nz, rr = idx / nz;
        const uint64_t jj = rr % ny, ii = rr / ny;
        const uint64_t row_key = (ii * 3 + pe->axis[e]) * ny + jj;
        if (last_row != ~0ull && row_key < last_row) return "pole edges out of order";
        const uint32_t p0 = e ? pe->pole_end[e - 1] : 0, p1 = pe->pole_end[e];
        const uint32_t np = p1 - p0;
        if (np > kMaxPoles || np == 0) return "more than 16 poles on an edge";
        std::string key((size_t)np * 24 + 16, '\0');
        uint32_t kinds = 0, oe = 0;
        for (uint32_t q = 0; q < np; ++q) {
            const double c3[3] = {pe->a[p0 + q], pe->inv_c[p0 + q], pe->inv_z[p0 + q]};
            std::memcpy(&key[(size_t)q * 24], c3, 24);
            const uint8_t kd = pe->kind[p0 + q];
            if (kd != EMS_POLE_TRAPEZOIDAL) kinds |= 1u << q;
            if (kd == EMS_POLE_OPENEMS) oe |= 1u << q;
            if (kd == EMS_POLE_OPENEMS_DEBYE) oe |= kOeDebye;
        }
        std::memcpy(&key[(size_t)np * 24], &pe->sum_inv_z[e], 8);
        std::memcpy(&key[(size_t)np * 24 + 8], &kinds, 4);
        std::memcpy(&key[(size_t)np * 24 + 12], &oe, 4);
        auto it = set_of.find(key);
        uint32_t set;
        if (it == set_of.end()) {
            set = (uint32_t)R.sets.size();
            for (uint32_t q = 0; q < np; ++q) {
                R.sets.push_back(pe->a[p0 + q]);
                R.sets.push_back(pe->inv_c[p0 + q]);
                R.sets.push_back(pe->inv_z[p0 + q]);
            }
            set_of.emplace(key, set);
        } else {
            set = it->second;
        }
        const bool extend = !R.runs.empty() && row_key == last_row && kk == (uint64_t)last_k + 1 &&
                            R.runs.back().set == set && R.runs.back().np == np && R.runs.back().kinds == kinds &&
                            R.runs.back().oe == oe &&
                            R.runs.back().p0 + (R.runs.back().ke - R.runs.back().kb) * np == p0 &&
                            R.runs.back().e0 + (R.runs.back().ke - R.runs.back().kb) == e;
        if (extend) {
            R.runs.back().ke = (uint32_t)kk + 1;
        } else {
            if (row_key != last_row) R.row_runs[row_key] = uint4{(uint32_t)R.runs.size(), 0, (uint32_t)kk, 0};
            R.runs.push_back(PoleRun{(uint32_t)kk, (uint32_t)kk + 1, p0, set, np, kinds, (uint32_t)e, (uint32_t)pe->axis[e],
                                     (uint32_t)((ii * ny + jj) * pitch + kk), oe, pe->sum_inv_z[e]});
            R.row_runs[row_key].y++;
        }
        R.run_of.push_back((uint32_t)R.runs.size() - 1);
        R.row_runs[row_key].w = (uint32_t)kk + 1;  // the row's edges are in z order
        last_row = row_key;
        last_k = (uint32_t)kk;
    }
    return "";
}

// Tables of the table-driven schedules (the fused kernel and the two-kernel
// schedule): pooled coefficient rows, CPML slabs per (side, component) in
// application order, poles as runs.
struct FusedTables {
    std::string why;               // why the table-driven schedules cannot run ("" if they can)
    std::string fused_why;         // why the fused kernel cannot run ("" if it can)
    Pooled lane[12];
    std::vector<FusedSlabSpec> slabs;
    int nslab[2][3] = {{0, 0, 0}, {0, 0, 0}};
    std::vector<uint32_t> cmask[3];  // per axis and node index: the slabs whose normal range holds it
    bool poles_first = false;
    bool has_poles = false, has_poles_h = false;
    std::vector<PoleRun> runs;
    std::vector<double> sets;
    std::vector<uint4> row_runs;
    std::vector<uint32_t> run_of;  // electric poles: per edge, its run
    PoleRuns h;                    // magnetic poles
};

// Why the fused schedule cannot run this model ("" if it can).
inline std::string fused_ineligible(const ems_engine_desc* d, uint32_t pitch) {
    for (size_t k = 0; k < d->n_ops; ++k) {
        const int kind = d->ops[k].kind;
        if (kind == EMS_OP_POLES) {
            const auto* p = (const ems_poles*)d->ops[k].table;
            if (p->magnetic.n_edges) return "magnetic poles";
        }
        if (kind == EMS_OP_SOURCE) {
            const auto* s = (const ems_source*)d->ops[k].table;
            if (s->kind == EMS_SOFT_H || s->kind == EMS_HARD_H) return "magnetic sources";
        }
        if (kind == EMS_OP_SHEET) return "conducting sheets";
    }
    if (pitch > 1024) return "z rows longer than 1024 nodes";
    return "";
}

inline FusedTables build_fused_tables(const ems_engine_desc* d, uint32_t pitch) {
    FusedTables T;
    int n_cpml = 0, n_poles = 0;
    for (size_t k = 0; k < d->n_ops; ++k) {
        n_cpml += d->ops[k].kind == EMS_OP_CPML;
        n_poles += d->ops[k].kind == EMS_OP_POLES;
    }
    if (n_cpml > 1 || n_poles > 1) {
        T.why = T.fused_why = "several CPML or dispersive operators";
        return T;
    }
    T.fused_why = fused_ineligible(d, pitch);
    const uint32_t nx = (uint32_t)d->nodes[0], ny = (uint32_t)d->nodes[1], nz = (uint32_t)d->nodes[2];
    {
        std::vector<std::thread> th;
        for (int l = 0; l < 12; ++l)
            th.emplace_back([&, l] { T.lane[l] = pool_lane(d->coeff[l], nx, ny, nz, pitch); });
        for (auto& t : th) t.join();
    }
    int pos_cpml = -1, pos_poles = -1;
    const ems_poles* poles = nullptr;
    for (size_t k = 0; k < d->n_ops; ++k) {
        if (d->ops[k].kind == EMS_OP_CPML) {
            pos_cpml = (int)k;
            const auto* c = (const ems_cpml*)d->ops[k].table;
            for (size_t q = 0; q < c->n_slabs; ++q) {
                const ems_cpml_slab& s = c->slabs[q];
                const size_t len = (size_t)(s.hi[0] - s.lo[0]) * (s.hi[1] - s.lo[1]) * (s.hi[2] - s.lo[2]);
                if (!len) continue;
                const int side = s.e_side ? 1 : 0;
                int& n = T.nslab[side][s.comp];
                if (n >= 4) {
                    T.why = T.fused_why = "more than four CPML slabs per component";
                    return T;
                }
                // The kernels test a node's membership along the normal only:
                // the slab must span the grid on its other axes (as the
                // reference's layers do, less the padding index).
                for (int a = 0; a < 3; ++a) {
                    if (a == s.normal) continue;
                    if (s.lo[a] != 0 || s.hi[a] + 1 < d->nodes[a]) {
                        T.why = T.fused_why = "a CPML slab that does not span the grid";
                        return T;
                    }
                }
                if (T.cmask[0].empty())
                    for (int a = 0; a < 3; ++a) T.cmask[a].assign(d->nodes[a], 0u);
                for (uint64_t x = s.lo[s.normal]; x < s.hi[s.normal]; ++x)
                    T.cmask[s.normal][x] |= 1u << (side * 12 + s.comp * 4 + n);
                T.slabs.push_back({side, (int)s.comp, n, q, &s, len});
                ++n;
            }
        }
        if (d->ops[k].kind == EMS_OP_POLES) {
            pos_poles = (int)k;
            poles = (const ems_poles*)d->ops[k].table;
        }
    }
    if (T.cmask[0].empty())
        for (int a = 0; a < 3; ++a) T.cmask[a].assign(d->nodes[a], 0u);
    T.poles_first = pos_poles >= 0 && pos_cpml >= 0 && pos_poles < pos_cpml;
    if (poles && poles->electric.n_edges) {
        PoleRuns R;
        std::string w = pole_runs(&poles->electric, nx, ny, nz, pitch, R);
        if (!w.empty()) {
            T.why = T.fused_why = w;
            return T;
        }
        T.runs = std::move(R.runs);
        T.sets = std::move(R.sets);
        T.row_runs = std::move(R.row_runs);
        T.run_of = std::move(R.run_of);
        T.has_poles = true;
    }
    if (poles && poles->magnetic.n_edges) {
        std::string w = pole_runs(&poles->magnetic, nx, ny, nz, pitch, T.h);
        if (!w.empty()) {
            T.why = T.fused_why = w;
            return T;
        }
        T.has_poles_h = true;
    }
    return T;
}

// The CPML layer shell of one side (0 H, 1 E) as boxes with one slab set
// per component each. Along every axis the slabs' bounds and n − 1, n cut the
// grid into intervals; in a product of intervals every node lies in the same
// slabs and has the same components (a component is missing on the high
// faces, as in the update), so a box needs no per-node test. Boxes with no
// correction are dropped; they come x-interval by x-interval, so the boxes
// of an x range between two cuts are consecutive. Returns the boxes and the
// total node count.
// A slab's place and extent, kept by the engine to re-cut the shell.
struct SlabGeo {
    int side, comp, q;
    uint32_t lo[3], hi[3];
    int normal;
};

inline std::vector<SlabGeo> slab_geometry(const FusedTables& T) {
    std::vector<SlabGeo> out;
    for (const FusedSlabSpec& sp : T.slabs) {
        SlabGeo g{sp.side, sp.comp, sp.q, {}, {}, (int)sp.src->normal};
        for (int a = 0; a < 3; ++a) {
            g.lo[a] = (uint32_t)sp.src->lo[a];
            g.hi[a] = (uint32_t)sp.src->hi[a];
        }
        out.push_back(g);
    }
    return out;
}

inline std::vector<ShellBox> shell_boxes(const std::vector<SlabGeo>& slabs, const int nslab[3],
                                         const uint64_t nodes[3], int side, uint32_t* total,
                                         const std::vector<uint32_t>& xcuts = {}) {
    std::vector<uint32_t> bp[3];
    for (int a = 0; a < 3; ++a) bp[a] = {0u, (uint32_t)nodes[a] - 1u, (uint32_t)nodes[a]};
    bp[0].insert(bp[0].end(), xcuts.begin(), xcuts.end());  // extra cuts: no box straddles an x chunk
    for (const SlabGeo& sp : slabs) {
        if (sp.side != side) continue;
        for (int a = 0; a < 3; ++a) {
            bp[a].push_back(sp.lo[a]);
            bp[a].push_back(sp.hi[a]);
        }
    }
    for (int a = 0; a < 3; ++a) {
        std::sort(bp[a].begin(), bp[a].end());
        bp[a].erase(std::unique(bp[a].begin(), bp[a].end()), bp[a].end());
    }
    // Slabs of this side per component, in application order.
    std::vector<const SlabGeo*> by[3];
    for (int c = 0; c < 3; ++c) by[c].assign(nslab[c], nullptr);
    for (const SlabGeo& sp : slabs)
        if (sp.side == side) by[sp.comp][sp.q] = &sp;
    std::vector<ShellBox> out;
    uint64_t sum = 0;
    for (size_t xi = 0; xi + 1 < bp[0].size(); ++xi)
        for (size_t yi = 0; yi + 1 < bp[1].size(); ++yi)
            for (size_t zi = 0; zi + 1 < bp[2].size(); ++zi) {
                const uint32_t lo[3] = {bp[0][xi], bp[1][yi], bp[2][zi]};
                const uint32_t hi[3] = {bp[0][xi + 1], bp[1][yi + 1], bp[2][zi + 1]};
                ShellBox B{};
                bool any = false;
                for (int c = 0; c < 3; ++c) {
                    // The component exists in the box (the update's conditions:
                    // E_c needs index c + 1 < n_c, H_c both other indices + 1 < n;
                    // n − 1 is a cut, so lo decides for the whole box).
                    const int p1 = (c + 1) % 3, p2 = (c + 2) % 3;
                    const bool valid = side ? lo[c] + 1 < nodes[c]
                                            : (lo[p1] + 1 < nodes[p1]) && (lo[p2] + 1 < nodes[p2]);
                    uint32_t cnt = 0, list = 0;
                    for (int q = 0; valid && q < (int)by[c].size(); ++q) {
                        const SlabGeo* sl = by[c][q];
                        if (!sl) continue;  // a slab left out of this shell
                        bool in = true;
                        for (int a = 0; a < 3; ++a) in = in && sl->lo[a] <= lo[a] && hi[a] <= sl->hi[a];
                        if (!in) continue;
                        list |= (uint32_t)q << (4 + 4 * cnt);
                        ++cnt;
                    }
                    B.list[c] = list | cnt;
                    any = any || cnt;
                }
                if (!any) continue;
                for (int a = 0; a < 3; ++a) {
                    B.lo[a] = lo[a];
                    B.n[a] = hi[a] - lo[a];
                }
                B.start = (uint32_t)sum;
                sum += (uint64_t)B.n[0] * B.n[1] * B.n[2];
                out.push_back(B);
            }
    *total = (uint32_t)sum;
    return out;
}

// The split schedule's row CPML (split.cuh row_cpml): the update kernels'
// CPML variant applies every slab's correction itself over the quads that
// hold layer nodes, so no shell kernel runs. Per side: the planes [0, x_lo)
// and [x_hi, nx), the rows [0, y_lo) and [y_hi, ny) and the z-nodes [0, z_lo)
// and [z_hi, nz) hold the slabs normal to x, y and z (every slab lies on a
// face: it starts at 0 or ends at the last node or its padding).
struct RowCpml {
    bool ok = false;
    uint32_t lo[2][3] = {}, hi[2][3] = {};
};

inline RowCpml row_cpml_plan(const std::vector<SlabGeo>& slabs, const uint64_t nodes[3]) {
    RowCpml R;
    for (int side = 0; side < 2; ++side)
        for (int a = 0; a < 3; ++a) {
            R.lo[side][a] = 0;
            R.hi[side][a] = (uint32_t)nodes[a];
        }
    for (const SlabGeo& sp : slabs) {
        const int a = sp.normal, side = sp.side;
        if (a < 0 || a > 2 || side < 0 || side > 1) return RowCpml{};
        const uint32_t n = (uint32_t)nodes[a];
        if (sp.lo[a] == 0) R.lo[side][a] = std::max(R.lo[side][a], sp.hi[a]);
        else if (sp.hi[a] + 1 >= n) R.hi[side][a] = std::min(R.hi[side][a], sp.lo[a]);
        else return RowCpml{};
    }
    for (int side = 0; side < 2; ++side)
        for (int a = 0; a < 3; ++a)
            if (R.lo[side][a] > R.hi[side][a]) R.lo[side][a] = R.hi[side][a];
    R.ok = true;
    return R;
}

inline std::vector<ShellBox> shell_boxes(const FusedTables& T, const uint64_t nodes[3], int side, uint32_t* total,
                                         const std::vector<uint32_t>& xcuts = {}) {
    return shell_boxes(slab_geometry(T), T.nslab[side], nodes, side, total, xcuts);
}

// Whether a side's dispersive correction may store its corrected value as
// the edge's saved field value, in place of the capture the reference makes
// one hook later (E edges: after the next H update; H edges: after the E
// update; src/engine/dispersive.rs:1173-1180, 1730-1744). True when nothing
// that runs between the correction and that capture writes a pole edge of
// the side: no lumped element, Mur boundary edge or source of that field on
// one, and, when the
// CPML hooks run after the dispersive ones, no CPML slab of that side over
// one. The side's edges are in (plane, axis, row, z) order, so membership is
// a binary search.
inline bool pole_prev_fold(const ems_engine_desc* d, bool electric, bool poles_first) {
    for (size_t k = 0; k < d->n_ops; ++k)
        if (d->ops[k].kind == EMS_OP_UPML) return false;  // its layer update may write pole edges
    const ems_pole_side* ps = nullptr;
    for (size_t k = 0; k < d->n_ops; ++k)
        if (d->ops[k].kind == EMS_OP_POLES) {
            const auto* p = (const ems_poles*)d->ops[k].table;
            ps = electric ? &p->electric : &p->magnetic;
        }
    if (!ps || !ps->n_edges) return false;
    const uint64_t ny = d->nodes[1], nz = d->nodes[2];
    auto key = [&](uint64_t node, uint64_t axis) {
        const uint64_t k = node % nz, r = node / nz, j = r % ny, i = r / ny;
        return ((i * 3 + axis) * ny + j) * nz + k;
    };
    auto is_pole_edge = [&](uint64_t node, uint64_t axis) {
        const uint64_t want = key(node, axis);
        size_t lo = 0, hi = ps->n_edges;
        while (lo < hi) {
            const size_t mid = lo + (hi - lo) / 2;
            const uint64_t k = key(ps->node[mid], ps->axis[mid]);
            if (k == want) return true;
            if (k < want) lo = mid + 1;
            else hi = mid;
        }
        return false;
    };
    for (size_t k = 0; k < d->n_ops; ++k) {
        const int kind = d->ops[k].kind;
        if (kind == EMS_OP_LUMPED && electric) {
            const auto* l = (const ems_lumped*)d->ops[k].table;
            for (size_t e = 0; e < l->n_edges; ++e)
                if (is_pole_edge(l->node[e], (uint64_t)l->axis)) return false;
        } else if (kind == EMS_OP_MUR && electric) {
            const auto* m = (const ems_mur*)d->ops[k].table;
            for (size_t e = 0; e < m->n; ++e)
                if (is_pole_edge(m->node[e], m->axis[e])) return false;
        } else if (kind == EMS_OP_SOURCE) {
            const auto* sr = (const ems_source*)d->ops[k].table;
            const bool e_src = sr->kind == EMS_SOFT_E || sr->kind == EMS_HARD_E;
            if (e_src != electric) continue;
            for (size_t e = 0; e < sr->n_edges; ++e)
                if (is_pole_edge(sr->node[e], sr->axis[e])) return false;
        } else if (kind == EMS_OP_CPML && poles_first) {
            const auto* c = (const ems_cpml*)d->ops[k].table;
            for (size_t q = 0; q < c->n_slabs; ++q) {
                const ems_cpml_slab& sl = c->slabs[q];
                if ((sl.e_side != 0) != electric) continue;
                for (size_t e = 0; e < ps->n_edges; ++e) {
                    if ((int)ps->axis[e] != sl.comp) continue;
                    const uint64_t n = ps->node[e], kk = n % nz, r = n / nz, jj = r % ny, ii = r / ny;
                    if (ii >= sl.lo[0] && ii < sl.hi[0] && jj >= sl.lo[1] && jj < sl.hi[1] && kk >= sl.lo[2] &&
                        kk < sl.hi[2])
                        return false;
                }
            }
        }
    }
    return true;
}

// Work items (row tile, x chunk): about eight per CTA of the persistent grid,
// chunks of at least eight planes.
inline void fused_work(FusedParams& P, uint32_t nx, uint32_t ny, int tj, unsigned grid) {
    P.tiles_j = (ny + tj - 1) / tj;
    const uint32_t want = 8u * grid;
    const uint32_t chunks = std::max<uint32_t>(1, (want + P.tiles_j - 1) / P.tiles_j);
    const uint32_t chunk = std::max<uint32_t>(8, (nx + chunks - 1) / chunks);
    P.chunk = chunk;
    P.n_chunks = (nx + chunk - 1) / chunk;
    P.n_items = P.tiles_j * P.n_chunks;
}

}  // namespace emsk
