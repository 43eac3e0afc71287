// oracle.cpp — CPU restatement of the ems engine step (test infrastructure).
//
// TEST INFRASTRUCTURE ONLY: the checker of the CUDA engine and the timed
// CPU baseline. Each function below cites the reference source it restates;
// the arithmetic follows it expression by expression (f32 fields, f64 branch
// state, no fused multiply-add: build with -ffp-contract=off), and for any
// thread count each value has one writer and one expression.
//
// Pinning: the reference (Rust, with an un-vendored csx dependency) cannot be
// built here, so the oracle is pinned by the reference's own known-answer
// tests restated on it (tests/test_oracle_known_answers.py: cavity modes,
// energy invariant and decay, run-loop stop, thread determinism, CPML
// reflection levels as printed, dispersive energy;
// tests/test_oracle_dispersive_validation.py: poles against the continuum
// and the discrete susceptibilities; tests/test_oracle_lumped.py: lumped
// elements and ports; tests/test_oracle_sheet.py: conducting sheets against
// the exact slab; tests/test_mur.py: Mur reflection, stability,
// determinism) and by the reference's golden vectors, the
// openEMS probe files of its XML fixtures, which the oracle reproduces to
// 1e-4 or better on every fixture whose features the openEMS front end
// (ems_b200/openems.py) restates (tests/test_openems_fixtures.py).
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

// src/engine/kernel.rs:30-33 — subnormal results rounded to zero.
inline float flush(float x) { return std::fabs(x) < 1.17549435e-38f ? 0.0f : x; }

// openEMS's summation order with every operation flushed (CurlOrder::OpenEms,
// src/engine/kernel.rs:35-50 oe_h, oe_e).
inline float oe_h(float da, float h, float db, float a, float b, float c, float d) {
    const float curl = flush(flush(flush(a - b) + d) - c);
    return flush(flush(da * h) - flush(db * curl));
}
inline float oe_e(float ca, float u, float cb, float a, float b, float c, float d) {
    const float curl = flush(flush(flush(a - b) - c) + d);
    return flush(flush(ca * u) + flush(cb * curl));
}

// src/engine/kernel.rs:116-120 — (1 + a)·p/b, 0 where b = 0.
inline double weight(float a, double p, float b) {
    double w = (1.0 + (double)a) * p / (double)b;
    return b != 0.0f ? w : 0.0;
}

// Persistent worker pool: the caller runs slab 0, workers slabs 1..n-1
// (src/engine/pool.rs:1-16, one x-slab per thread, a barrier per phase).
class Pool {
public:
    explicit Pool(int n) : n_(n) {
        for (int t = 1; t < n; ++t) workers_.emplace_back([this, t] { loop(t); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (auto& w : workers_) w.join();
    }
    int size() const { return n_; }
    void run(const std::function<void(int)>& f) {
        if (n_ == 1) { f(0); return; }
        {
            std::lock_guard<std::mutex> g(m_);
            job_ = &f;
            done_.store(0);
            ++gen_;
        }
        cv_.notify_all();
        f(0);
        while (done_.load(std::memory_order_acquire) != n_ - 1) std::this_thread::yield();
    }

private:
    void loop(int t) {
        uint64_t seen = 0;
        for (;;) {
            const std::function<void(int)>* job;
            {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [&] { return gen_ != seen; });
                seen = gen_;
                if (stop_) return;
                job = job_;
            }
            (*job)(t);
            done_.fetch_add(1, std::memory_order_release);
        }
    }
    int n_;
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_;
    uint64_t gen_ = 0;
    bool stop_ = false;
    const std::function<void(int)>* job_ = nullptr;
    std::atomic<int> done_{0};
};

struct CpmlSlab {
    ems_cpml_slab s;
    std::vector<float> b, a, k, psi;
};

struct PoleSide {
    std::vector<uint8_t> axis;
    std::vector<uint64_t> node;
    std::vector<uint32_t> plane;
    std::vector<double> sum_inv_z;
    std::vector<uint32_t> pole_end;
    std::vector<uint8_t> kind;
    std::vector<double> a, inv_c, inv_z, half_l;
    std::vector<float> prev;
    std::vector<double> j, q;
};

struct Lumped {
    int axis = 0;
    std::vector<uint64_t> node;
    std::vector<double> cb, g_src, src_w, src_amp, two_l_dt, inv_c, z, rec_g, rec_c;
    uint64_t series = 1;
    bool src_in_branch = false, has_src = false, has_branch = false, record = false;
    uint64_t port_columns = 0;
    bool openems_order = false;
    std::vector<float> oe_k, oe_s;  // openEMS's explicit inductor: f32 constant and state
    std::vector<double> oe_vi;
    std::vector<double> v, bj, bq, bu_prev, j_avg, ru_prev;
    std::vector<double> rec, port_v, port_i;
};

struct Source {
    int kind = 0;
    std::vector<uint8_t> axis;
    std::vector<uint64_t> node;
    std::vector<float> weight, amp;
};

struct Probe {
    int quantity = 0;
    std::vector<uint8_t> axis;
    std::vector<uint64_t> node;
    std::vector<double> weight;
    uint64_t interval = 1;
    bool f32_sum = false;
    std::vector<double> values;
};

// A Mur boundary (src/engine/boundary/mur.rs:103-139): face edges first,
// then the edges shared by two Mur faces.
struct Mur {
    size_t n_edges = 0;
    std::vector<uint8_t> axis;
    std::vector<uint64_t> node, inner, hold;  // inner: 2 per entry
    std::vector<float> k;                     // 2 per entry
    std::vector<double> cap;
    bool openems_order = false, openems_corners = false, count_energy = false;
    std::vector<float> saved;                 // 3 per entry: u_b^n, u_1^n (both neighbours)
    std::vector<float> last;                  // value after the last update
};

// openEMS's PML layers (src/engine/boundary/upml.rs:260-420 Run): per
// side (0 E, 1 H) the edges, their coefficients, flux F and start value v,
// and the edges of each x-plane (by_plane[pstart[i]..pstart[i + 1]]).
struct Upml {
    std::vector<uint8_t> axis[2];
    std::vector<uint64_t> node[2];
    std::vector<float> co[2];
    std::vector<float> f[2], v[2];
    std::vector<uint32_t> by_plane[2], pstart[2];
};

// Conducting sheets (src/engine/sheet.rs:403-522): per edge its ladder
// (nodes n0..n0+nn of u, layers l0..l0+nn-1 of h), its constants from k0
// (per node) and a0 (per layer), its couplings [c0, c1).
struct Sheet {
    std::vector<uint8_t> axis, c_axis;
    std::vector<uint64_t> node, c_node;
    std::vector<uint32_t> nn, k0, a0, c0, c1, n0, l0;
    std::vector<double> c_edge, w_up, w_dn, corr, ecorr, two_c, cp, inv_den, a;
    std::vector<double> u, h, x;
    double w_corr = 0.0;
};

struct Op {
    int kind = 0;
    std::vector<CpmlSlab> cpml;
    PoleSide pe, ph;
    Lumped lumped;
    Source source;
    Probe probe;
    Mur mur;
    Upml upml;
    Sheet sheet;
};

// src/engine/boundary/mur.rs:252-259 mur_1d: u_b^{n+1} from u_1^n (i),
// k, u_1^{n+1} (x) and u_b^n (b), in ems's or openEMS's order.
inline float mur_1d(float i, float k, float x, float b, bool openems) {
    return openems ? (i - k * b) + k * x : i + k * (x - b);
}

}  // namespace

struct oracle_engine {
    size_t nx, ny, nz, plane, n;
    double dt;
    std::vector<float> co[12];
    std::vector<float> u[3], i[3];
    std::vector<float> zero;
    std::vector<Op> ops;
    uint64_t step = 0;
    std::vector<size_t> slab_start;
    std::vector<double> plane_w;
    Pool* pool = nullptr;
    bool oe = false;  // CurlOrder::OpenEms

    // ---- H update of one x-plane (src/engine/kernel.rs:447-511 h_plane,
    // 58-79 h_row, 132-174 h_row_energy). Returns the plane's H energy
    // share in units of dt/4 when ENERGY.
    template <bool ENERGY>
    double h_plane(size_t gi) {
        const size_t base = gi * plane;
        float* ix = &i[0][base];
        float* iy = &i[1][base];
        float* iz = &i[2][base];
        const float* ux = &u[0][base];
        const float* uy = &u[1][base];
        const float* uz = &u[2][base];
        const bool next = gi + 1 < nx;
        const float* uyn = next ? &u[1][base + plane] : nullptr;
        const float* uzn = next ? &u[2][base + plane] : nullptr;
        double wh = 0.0;
        // One row: h = flush(da·h − db·((a − b) − (c − d))), energy entry k
        // into accumulator k & 3 (groups of four, then the tail).
        auto row = [&](float* h, const float* da, const float* db, const float* a, const float* b,
                       const float* c, const float* d, size_t m) -> double {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            for (size_t k = 0; k < m; ++k) {
                float old = h[k];
                float nw = oe ? oe_h(da[k], old, db[k], a[k], b[k], c[k], d[k])
                              : flush(da[k] * old - db[k] * ((a[k] - b[k]) - (c[k] - d[k])));
                if (ENERGY) acc[k & 3] += weight(da[k], (double)old * (double)nw, db[k]);
                h[k] = nw;
            }
            return (acc[0] + acc[1]) + (acc[2] + acc[3]);
        };
        const size_t m = nz - 1;
        for (size_t j = 0; j + 1 < ny; ++j) {
            size_t r = j * nz;
            double w = row(ix + r, &co[6][base + r], &co[9][base + r], uz + r + nz, uz + r, uy + r + 1,
                           uy + r, m);
            if (ENERGY) wh += 1.0 * w;
        }
        if (next) {
            for (size_t j = 0; j < ny; ++j) {
                size_t r = j * nz;
                double w = row(iy + r, &co[7][base + r], &co[10][base + r], ux + r + 1, ux + r, uzn + r,
                               uz + r, m);
                if (ENERGY) wh += 1.0 * w;
            }
            for (size_t j = 0; j + 1 < ny; ++j) {
                size_t r = j * nz;
                double w = row(iz + r, &co[8][base + r], &co[11][base + r], uyn + r, uy + r, ux + r + nz,
                               ux + r, nz);
                if (ENERGY) wh += w * 1.0;
            }
        }
        return wh;
    }

    // E part of a plane's energy (src/engine/kernel.rs:211-244
    // e_energy_row, 393-408 in h_slab): entry with in-plane index r + k into
    // accumulator (r + k) & 3, per component.
    double e_energy_plane(size_t gi) {
        const size_t base = gi * plane;
        double we = 0.0;
        for (int a = 0; a < 3; ++a) {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            const float* uc = &u[a][base];
            const float* ca = &co[a][base];
            const float* cb = &co[3 + a][base];
            for (size_t p = 0; p < plane; ++p) {
                double x = (double)uc[p];
                acc[p & 3] += weight(ca[p], x * x, cb[p]);
            }
            we += (acc[0] + acc[1]) + (acc[2] + acc[3]);
        }
        return we;
    }

    // ---- E update of one x-plane (src/engine/kernel.rs:624-697 e_rows,
    // 252-273 e_row): u = flush(ca·u + cb·((a − b) − (c − d))).
    void e_plane(size_t gi) {
        const size_t base = gi * plane;
        float* ux = &u[0][base];
        float* uy = &u[1][base];
        float* uz = &u[2][base];
        const float* ix = &i[0][base];
        const float* iy = &i[1][base];
        const float* iz = &i[2][base];
        const float* iyp = gi == 0 ? zero.data() : &i[1][base - plane];
        const float* izp = gi == 0 ? zero.data() : &i[2][base - plane];
        const bool o = oe;
        auto e1 = [o](float ca, float u0, float cb, float a, float b, float c, float d) {
            return o ? oe_e(ca, u0, cb, a, b, c, d) : flush(ca * u0 + cb * ((a - b) - (c - d)));
        };
        for (size_t j = 0; j < ny; ++j) {
            const size_t r = j * nz;
            if (gi + 1 < nx) {
                const float* ca = &co[0][base + r];
                const float* cb = &co[3][base + r];
                const float* izm = j == 0 ? zero.data() : iz + r - nz;
                ux[r] = e1(ca[0], ux[r], cb[0], iz[r], izm[0], iy[r], 0.0f);
                for (size_t k = 1; k < nz; ++k)
                    ux[r + k] = e1(ca[k], ux[r + k], cb[k], iz[r + k], izm[k], iy[r + k], iy[r + k - 1]);
            }
            if (j + 1 < ny) {
                const float* ca = &co[1][base + r];
                const float* cb = &co[4][base + r];
                uy[r] = e1(ca[0], uy[r], cb[0], ix[r], 0.0f, iz[r], izp[r]);
                for (size_t k = 1; k < nz; ++k)
                    uy[r + k] = e1(ca[k], uy[r + k], cb[k], ix[r + k], ix[r + k - 1], iz[r + k], izp[r + k]);
            }
            {
                const float* ca = &co[2][base + r];
                const float* cb = &co[5][base + r];
                const float* ixm = j == 0 ? zero.data() : ix + r - nz;
                for (size_t k = 0; k + 1 < nz; ++k)
                    uz[r + k] = e1(ca[k], uz[r + k], cb[k], iy[r + k], iyp[r + k], ix[r + k], ixm[k]);
            }
        }
    }

    // ---- CPML slab correction on the x-planes [x0, x1)
    // (src/engine/boundary/cpml.rs:445-520 Slab::apply, 657-676 row_uniform).
    void cpml_apply(CpmlSlab& c, size_t x0, size_t x1) {
        const ems_cpml_slab& s = c.s;
        const size_t lo0 = std::max<size_t>(s.lo[0], x0), hi0 = std::min<size_t>(s.hi[0], x1);
        if (lo0 >= hi0) return;
        const bool e = s.e_side != 0;
        float* t = e ? u[s.comp].data() : i[s.comp].data();
        const float* src = e ? i[s.other].data() : u[s.other].data();
        const float* coef = e ? co[3 + s.comp].data() : co[9 + s.comp].data();
        const float scale = e ? 1.0f : -1.0f;
        const size_t n1 = s.hi[1] - s.lo[1], n2 = s.hi[2] - s.lo[2];
        const size_t step_n = s.normal == 0 ? plane : (s.normal == 1 ? nz : 1);
        for (size_t x = lo0; x < hi0; ++x)
            for (size_t y = s.lo[1]; y < s.hi[1]; ++y)
                for (size_t z = s.lo[2]; z < s.hi[2]; ++z) {
                    const size_t idx = (x * ny + y) * nz + z;
                    const size_t node[3] = {x, y, z};
                    const size_t d = node[s.normal] - s.lo[s.normal];
                    float h, l;
                    if (e) {
                        h = src[idx];
                        l = node[s.normal] == 0 ? 0.0f : src[idx - step_n];
                    } else {
                        h = src[idx + step_n];
                        l = src[idx];
                    }
                    const size_t q = ((x - s.lo[0]) * n1 + (y - s.lo[1])) * n2 + (z - s.lo[2]);
                    const float sv = s.sign * (h - l);
                    c.psi[q] = flush(c.b[d] * c.psi[q] + c.a[d] * sv);
                    t[idx] = flush(t[idx] + scale * coef[idx] * (c.k[d] * sv + c.psi[q]));
                }
    }

    // ---- dispersive correction of the edges in planes [x0, x1)
    // (src/engine/dispersive.rs:1392-1470 step_edge, 1183-1343 correct).
    // Edges of the x-planes [x0, x1) (edges are in plane order).
    static std::pair<size_t, size_t> edges_in(const PoleSide& p, size_t x0, size_t x1) {
        auto lo = std::lower_bound(p.plane.begin(), p.plane.end(), (uint32_t)x0);
        auto hi = std::lower_bound(p.plane.begin(), p.plane.end(), (uint32_t)x1);
        return {size_t(lo - p.plane.begin()), size_t(hi - p.plane.begin())};
    }

    void poles_correct(PoleSide& p, bool electric, size_t x0, size_t x1) {
        const auto [e0, e1] = edges_in(p, x0, x1);
        for (size_t e = e0; e < e1; ++e) {
            const int ax = p.axis[e];
            float* f = electric ? u[ax].data() : i[ax].data();
            const size_t idx = p.node[e];
            const double cb = (double)(electric ? co[3 + ax][idx] : co[9 + ax][idx]);
            const size_t p0 = e ? p.pole_end[e - 1] : 0, p1 = p.pole_end[e];
            const float prev32 = p.prev[e];
            if (p1 > p0 && p.kind[p0] == EMS_POLE_OPENEMS_DEBYE) {
                // openems_debye_step (src/engine/dispersive.rs:930-960): the
                // explicit halves P first, their increments summed in pole
                // order, then u_new = F·(u* − S) and Q = P + b·u_new; every
                // operation f32, flushed.
                const float F = (float)p.a[p0], us = f[idx];
                float sum = 0.0f;
                for (size_t q = p0; q < p1; ++q) {
                    const float om = (float)p.inv_c[q], b = (float)p.inv_z[q], Q = (float)p.j[q];
                    const float P = flush(flush(om * Q) + flush(b * prev32));
                    sum = flush(sum + flush(P - Q));
                    p.j[q] = P;
                }
                const float un = flush(F * flush(us - sum));
                for (size_t q = p0; q < p1; ++q) p.j[q] = flush((float)p.j[q] + flush((float)p.inv_z[q] * un));
                f[idx] = flush(us - flush(us - un));
                continue;
            }
            const double prev = (double)prev32;
            const double half_prev = 0.5 * prev;
            float u32 = f[idx];
            double s = 0.0;
            double nj[64], nq[64];
            for (size_t q = p0; q < p1; ++q) {
                if (p.kind[q] == EMS_POLE_OPENEMS) {
                    // OpenEmsPole (src/engine/dispersive.rs:846-899, 1414-1425):
                    // V <- A·V + B·(u^n − W), W <- W + K·V, u <- u − V (f32).
                    const float A = (float)p.a[q], K = (float)p.inv_c[q], B = (float)p.inv_z[q];
                    const float w = (float)p.q[q];
                    const float v = flush(flush(A * (float)p.j[q]) + flush(B * flush(prev32 - w)));
                    nj[q - p0] = v;
                    nq[q - p0] = flush(w + flush(K * v));
                    u32 = flush(u32 - v);
                } else if (p.kind[q] == EMS_POLE_LEAPFROG) {
                    double jn = p.a[q] * p.j[q] + p.inv_z[q] * (prev - p.q[q] * p.inv_c[q]);
                    nj[q - p0] = jn;
                    nq[q - p0] = p.q[q] + dt * jn;
                    s += jn;
                } else {
                    s += (p.a[q] * p.j[q] - p.q[q] * p.inv_c[q] + half_prev) * p.inv_z[q];
                }
            }
            const double u_star = (double)u32;
            const float u_new = (float)((u_star - cb * s) / (1.0 + 0.5 * cb * p.sum_inv_z[e]));
            const double half_new = 0.5 * (double)u_new;
            for (size_t q = p0; q < p1; ++q) {
                if (p.kind[q] == EMS_POLE_LEAPFROG || p.kind[q] == EMS_POLE_OPENEMS) {
                    p.j[q] = nj[q - p0];
                    p.q[q] = nq[q - p0];
                } else {
                    double k = p.a[q] * p.j[q] - p.q[q] * p.inv_c[q] + half_prev;
                    double jb = (k + half_new) * p.inv_z[q];
                    p.j[q] = 2.0 * jb - p.j[q];
                    p.q[q] = p.q[q] + dt * jb;
                }
            }
            f[idx] = u_new;
        }
    }

    // Saves the current field value of the edges (src/engine/dispersive.rs:1173-1180).
    void poles_capture(PoleSide& p, bool electric, size_t x0, size_t x1) {
        const auto [e0, e1] = edges_in(p, x0, x1);
        for (size_t e = e0; e < e1; ++e) {
            p.prev[e] = (electric ? u : i)[p.axis[e]][p.node[e]];
        }
    }

    // Σ ½·L·j² + ½·q²/C_p in pole order (src/engine/dispersive.rs:1488-1506).
    static void pole_energy(const PoleSide& p, double& w) {
        for (size_t q = 0; q < p.kind.size(); ++q)
            if (p.kind[q] < EMS_POLE_OPENEMS) w += p.half_l[q] * p.j[q] * p.j[q] + 0.5 * p.inv_c[q] * p.q[q] * p.q[q];
    }

    double operator_energy() const {
        double w = 0.0;
        for (const Op& op : ops) {
            double x = 0.0;
            if (op.kind == EMS_OP_POLES) {
                double we = 0.0, wm = 0.0;
                pole_energy(op.pe, we);
                pole_energy(op.ph, wm);
                x = we + wm;
            } else if (op.kind == EMS_OP_MUR && op.mur.count_energy) {
                // src/engine/boundary/mur.rs:683-704 boundary_energy, in entry order.
                const Mur& m = op.mur;
                for (size_t e = 0; e < m.node.size(); ++e)
                    x += 0.5 * m.cap[e] * (double)m.last[e] * (double)m.last[e];
            } else if (op.kind == EMS_OP_SHEET) {
                x = sheet_energy(op.sheet);
            } else if (op.kind == EMS_OP_LUMPED && op.lumped.has_branch) {
                // src/engine/lumped.rs:1066-1077 branch_energy
                const Lumped& l = op.lumped;
                for (size_t e = 0; e < l.node.size(); ++e) {
                    double half_l = 0.25 * l.two_l_dt[e] * dt;
                    x += half_l * l.bj[e] * l.bj[e] + 0.5 * l.inv_c[e] * l.bq[e] * l.bq[e];
                }
            }
            w += x;
        }
        return w;
    }

    // ---- conducting sheets
    // post_h (src/engine/sheet.rs:950-972): the + face voltage from the
    // array, then the dual edges on the - side see u- - u+.
    void sheet_post_h(Sheet& s) {
        for (size_t e = 0; e < s.axis.size(); ++e) {
            const size_t n0 = s.n0[e], nn = s.nn[e];
            s.u[n0] = (double)u[s.axis[e]][s.node[e]];
            const double diff = s.u[n0 + nn - 1] - s.u[n0];
            for (uint32_t c = s.c0[e]; c < s.c1[e]; ++c)
                if (s.corr[c] != 0.0) {
                    float& v = i[s.c_axis[c]][s.c_node[c]];
                    v = flush(v + (float)(s.corr[c] * diff));
                }
        }
    }

    // post_e (src/engine/sheet.rs:974-1050): the ladder and both faces by
    // the trapezoidal rule, one tridiagonal solve per edge (Thomas, the
    // factorisation precomputed), the + face written back.
    void sheet_post_e(Sheet& s) {
        double w_corr = 0.0;
        for (size_t e = 0; e < s.axis.size(); ++e) {
            double s_up = 0.0, s_dn = 0.0, s_e = 0.0;
            for (uint32_t c = s.c0[e]; c < s.c1[e]; ++c) {
                const double iv = (double)i[s.c_axis[c]][s.c_node[c]];
                s_up += s.w_up[c] * iv;
                s_dn += s.w_dn[c] * iv;
                s_e += s.ecorr[c] * iv;
            }
            const size_t nn = s.nn[e], k0 = s.k0[e], ka = s.a0[e];
            double* U = s.u.data() + s.n0[e];
            double* H = s.h.data() + s.l0[e];
            double* X = s.x.data();
            for (size_t k = 0; k < nn; ++k) {
                double r = s.two_c[k0 + k] * U[k];
                if (k + 1 < nn) r -= H[k];
                if (k > 0) r += H[k - 1] + s.a[ka + k - 1] * X[k - 1];
                if (k == 0) r += s_up;
                if (k + 1 == nn) r += s_dn;
                X[k] = r * s.inv_den[k0 + k];
            }
            for (size_t k = nn - 1; k-- > 0;) X[k] -= s.cp[k0 + k] * X[k + 1];
            for (size_t j = 0; j + 1 < nn; ++j) H[j] += 2.0 * s.a[ka + j] * (X[j] - X[j + 1]);
            for (size_t k = 0; k < nn; ++k) U[k] = 2.0 * X[k] - U[k];
            const float up = flush((float)U[0]);
            u[s.axis[e]][s.node[e]] = up;
            w_corr += s_e * (U[nn - 1] - (double)up);
        }
        s.w_corr = w_corr;
    }

    // energy (src/engine/sheet.rs:1052-1083), edge by edge.
    double sheet_energy(const Sheet& s) const {
        double w = 0.0;
        for (size_t e = 0; e < s.axis.size(); ++e) {
            const size_t nn = s.nn[e], k0 = s.k0[e], ka = s.a0[e];
            const double* U = s.u.data() + s.n0[e];
            const double* H = s.h.data() + s.l0[e];
            for (size_t k = 0; k < nn; ++k) w += 0.25 * s.two_c[k0 + k] * dt * U[k] * U[k];
            const double stored = U[0];
            w -= 0.5 * s.c_edge[e] * stored * stored;
            for (size_t j = 0; j + 1 < nn; ++j) {
                const double l = dt / (2.0 * s.a[ka + j]);
                w += 0.5 * l * H[j] * H[j];
            }
        }
        return w + s.w_corr;
    }

    // ---- serial hooks
    void source_apply(Source& s, bool magnetic_phase) {
        const bool mag = s.kind == EMS_SOFT_H || s.kind == EMS_HARD_H;
        if (mag != magnetic_phase) return;
        const float a = step < s.amp.size() ? s.amp[step] : 0.0f;
        const bool hard = s.kind == EMS_HARD_E || s.kind == EMS_HARD_H;
        // src/engine/excite.rs:104-117 apply, 136-150 hooks_at (soft: skipped at 0).
        if (!hard && a == 0.0f) return;
        auto& F = mag ? i : u;
        for (size_t e = 0; e < s.axis.size(); ++e) {
            float& x = F[s.axis[e]][s.node[e]];
            if (hard) x = s.weight[e] * a;
            else x += s.weight[e] * a;
        }
    }

    void probe_sample(Probe& p, bool current_phase) {
        if ((p.quantity == EMS_PROBE_CURRENT) != current_phase) return;
        if (step % p.interval != 0) return;
        auto& F = current_phase ? i : u;
        // src/engine/probe.rs:381-392 (f64 sum in entry order; f32 variant).
        if (p.f32_sum) {
            float s = 0.0f;
            for (size_t e = 0; e < p.axis.size(); ++e) s = s + (float)p.weight[e] * F[p.axis[e]][p.node[e]];
            p.values.push_back((double)s);
        } else {
            double s = 0.0;
            for (size_t e = 0; e < p.axis.size(); ++e) s += p.weight[e] * (double)F[p.axis[e]][p.node[e]];
            p.values.push_back(s);
        }
    }

    // Run::refresh (upml.rs:380-392): the start values of side `sd` from
    // the fields, planes [x0, x1).
    void upml_refresh(Upml& L, int sd, size_t x0, size_t x1) {
        const auto& F = sd == 0 ? u : i;
        for (uint32_t q = L.pstart[sd][x0]; q < L.pstart[sd][x1]; ++q) {
            const uint32_t e = L.by_plane[sd][q];
            L.v[sd][e] = F[L.axis[sd][e]][L.node[sd][e]];
        }
    }

    // Run::apply (upml.rs:394-418): the layer update of side `sd` from the
    // flux increment the kernel left in the field, planes [x0, x1).
    void upml_apply(Upml& L, int sd, size_t x0, size_t x1) {
        auto& F = sd == 0 ? u : i;
        for (uint32_t q = L.pstart[sd][x0]; q < L.pstart[sd][x1]; ++q) {
            const uint32_t e = L.by_plane[sd][q];
            const float* c = &L.co[sd][4 * (size_t)e];
            float& t = F[L.axis[sd][e]][L.node[sd][e]];
            const float f0 = L.f[sd][e];
            const float f1 = flush(flush(c[0] * f0) + t);
            const float x = flush(flush(flush(c[1] * L.v[sd][e]) - flush(c[3] * f0)) + flush(c[2] * f1));
            L.f[sd][e] = f1;
            L.v[sd][e] = x;
            t = x;
        }
    }

    // src/engine/boundary/mur.rs:781-808 pre_e: u_b^n and u_1^n.
    void mur_pre_e(Mur& m) {
        for (size_t e = 0; e < m.node.size(); ++e) {
            const std::vector<float>& f = u[m.axis[e]];
            m.saved[3 * e] = f[m.node[e]];
            m.saved[3 * e + 1] = f[m.inner[2 * e]];
            if (e >= m.n_edges) m.saved[3 * e + 2] = f[m.inner[2 * e + 1]];
        }
    }

    // src/engine/boundary/mur.rs:812-843 post_e: the face edges, then the
    // shared edges, whose neighbours are face edges updated just before.
    void mur_post_e(Mur& m) {
        for (size_t e = 0; e < m.node.size(); ++e) {
            if (step < m.hold[e]) continue;
            std::vector<float>& f = u[m.axis[e]];
            const float b = m.saved[3 * e], i0 = m.saved[3 * e + 1];
            float v;
            if (e < m.n_edges) {
                v = mur_1d(i0, m.k[2 * e], f[m.inner[2 * e]], b, m.openems_order);
            } else if (m.openems_corners) {
                v = i0 - m.k[2 * e] * b;
            } else {
                const float i1 = m.saved[3 * e + 2];
                const float v0 = mur_1d(i0, m.k[2 * e], f[m.inner[2 * e]], b, m.openems_order);
                const float v1 = mur_1d(i1, m.k[2 * e + 1], f[m.inner[2 * e + 1]], b, m.openems_order);
                v = 0.5f * (v0 + v1);
            }
            f[m.node[e]] = v;
            m.last[e] = v;
        }
    }

    void lumped_pre_e(Lumped& l) {
        // src/engine/lumped.rs:1106-1121 pre_e_impl.
        for (size_t e = 0; e < l.node.size(); ++e) {
            double x = (double)u[l.axis][l.node[e]];
            if (l.has_branch && !l.openems_order) l.bu_prev[e] = x;
            if (l.record) l.ru_prev[e] = x;
        }
    }

    void lumped_post_e(Lumped& l) {
        // src/engine/lumped.rs:1123-1236 post_e_impl (openEMS's order: the
        // branch driven by its own previous result, the source after it;
        // its explicit f32 inductor), src/engine/port.rs:276-290
        // LumpedPort::post_e.
        float* U = u[l.axis].data();
        const size_t ne = l.node.size();
        bool active = false;
        if (l.has_src) {
            std::fill(l.v.begin(), l.v.end(), 0.0);
            const double val = step < l.src_amp.size() ? l.src_amp[step] : 0.0;
            if (val != 0.0) {
                active = true;
                for (size_t e = 0; e < ne; ++e) l.v[e] += l.src_w[e] * val;
            }
        }
        auto add_sources = [&]() {
            for (size_t e = 0; e < ne; ++e) {
                double add = l.cb[e] * l.g_src[e] * l.v[e];
                if (add != 0.0) U[l.node[e]] = (float)((double)U[l.node[e]] + add);
            }
        };
        if (active && !l.src_in_branch && !l.openems_order) add_sources();
        if (l.has_branch) {
            for (size_t e = 0; e < ne; ++e) {
                if (!l.oe_k.empty()) {
                    const float u_l = (float)l.bu_prev[e];
                    l.oe_s[e] = flush(l.oe_s[e] + flush(l.oe_k[e] * u_l));
                    const float u_new = flush(U[l.node[e]] - l.oe_s[e]);
                    l.bj[e] = (double)l.oe_s[e] / l.oe_vi[e];
                    l.j_avg[e] = l.bj[e];
                    U[l.node[e]] = u_new;
                    l.bu_prev[e] = (double)u_new;
                    continue;
                }
                double v_br = (active && l.src_in_branch) ? l.v[e] : 0.0;
                double u_star = (double)U[l.node[e]];
                double k = l.two_l_dt[e] * l.bj[e] - l.bq[e] * l.inv_c[e] - v_br + 0.5 * l.bu_prev[e];
                double z = l.z[e];
                double cb = l.cb[e];
                double u_new = (z * u_star - cb * k) / (z + 0.5 * cb);
                double jb = (k + 0.5 * u_new) / z;
                l.bj[e] = 2.0 * jb - l.bj[e];
                l.bq[e] += dt * jb;
                l.j_avg[e] = jb;
                U[l.node[e]] = (float)u_new;
                if (l.openems_order) l.bu_prev[e] = (double)(float)u_new;
            }
        }
        if (active && !l.src_in_branch && l.openems_order) add_sources();
        if (l.record) {
            double sum = 0.0;
            for (size_t e = 0; e < ne; ++e) {
                double u0 = l.ru_prev[e], u1 = (double)U[l.node[e]];
                double v = (active && !l.src_in_branch) ? l.v[e] : 0.0;
                sum += l.rec_g[e] * (0.5 * (u0 + u1) - v) + l.rec_c[e] * (u1 - u0) / dt;
                if (l.has_branch) sum += l.j_avg[e];
            }
            l.rec.push_back(sum / (double)l.series);
        }
        if (l.port_columns > 0) {
            double i_last = l.rec.empty() ? 0.0 : l.rec.back();
            l.port_i.push_back(-i_last);
            double s = 0.0;
            for (size_t e = 0; e < ne; ++e) s += (double)U[l.node[e]];
            l.port_v.push_back(s / (double)l.port_columns);
        }
    }

    // One step (src/engine/pool.rs Shared::h / Shared::e with the serial
    // gaps of src/engine/mod.rs:833-992).
    void one_step(bool energy) {
        const int ns = pool->size();
        // H half-step with its slab hooks.
        pool->run([&](int sl) {
            const size_t p0 = slab_start[sl], p1 = slab_start[sl + 1];
            for (size_t gi = p0; gi < p1; ++gi) {
                if (energy) {
                    double wh = h_plane<true>(gi);
                    double we = e_energy_plane(gi);
                    plane_w[gi] = we + wh;
                } else {
                    h_plane<false>(gi);
                }
            }
            for (Op& op : ops) {
                if (op.kind == EMS_OP_CPML) {
                    for (CpmlSlab& c : op.cpml)
                        if (!c.s.e_side) cpml_apply(c, p0, p1);
                } else if (op.kind == EMS_OP_POLES) {
                    poles_correct(op.ph, false, p0, p1);
                    poles_capture(op.pe, true, p0, p1);
                } else if (op.kind == EMS_OP_UPML) {
                    // upml.rs:443-454 post_h_slab.
                    upml_refresh(op.upml, 0, p0, p1);
                    upml_apply(op.upml, 1, p0, p1);
                }
            }
        });
        (void)ns;
        for (Op& op : ops) {
            if (op.kind == EMS_OP_SOURCE) source_apply(op.source, true);
            else if (op.kind == EMS_OP_PROBE) probe_sample(op.probe, true);
            else if (op.kind == EMS_OP_SHEET) sheet_post_h(op.sheet);
        }
        for (Op& op : ops) {
            if (op.kind == EMS_OP_LUMPED) lumped_pre_e(op.lumped);
            else if (op.kind == EMS_OP_MUR) mur_pre_e(op.mur);
        }
        // E half-step with its slab hooks.
        pool->run([&](int sl) {
            const size_t p0 = slab_start[sl], p1 = slab_start[sl + 1];
            for (size_t gi = p0; gi < p1; ++gi) e_plane(gi);
            for (Op& op : ops) {
                if (op.kind == EMS_OP_CPML) {
                    for (CpmlSlab& c : op.cpml)
                        if (c.s.e_side) cpml_apply(c, p0, p1);
                } else if (op.kind == EMS_OP_POLES) {
                    poles_correct(op.pe, true, p0, p1);
                    poles_capture(op.ph, false, p0, p1);
                } else if (op.kind == EMS_OP_UPML) {
                    // upml.rs:456-464 post_e_slab.
                    upml_refresh(op.upml, 1, p0, p1);
                    upml_apply(op.upml, 0, p0, p1);
                }
            }
        });
        for (Op& op : ops) {
            if (op.kind == EMS_OP_LUMPED) lumped_post_e(op.lumped);
            else if (op.kind == EMS_OP_MUR) mur_post_e(op.mur);
            else if (op.kind == EMS_OP_SOURCE) source_apply(op.source, false);
            else if (op.kind == EMS_OP_PROBE) probe_sample(op.probe, false);
            else if (op.kind == EMS_OP_SHEET) sheet_post_e(op.sheet);
        }
        ++step;
    }
};

namespace {

int default_threads(size_t nx, size_t cells) {
    unsigned hw = std::thread::hardware_concurrency();
    size_t t = hw ? hw : 1;
    t = std::min<size_t>(t, cells / 4096);
    t = std::min<size_t>(t, nx / 5);
    return (int)std::max<size_t>(t, 1);
}

template <class T>
std::vector<T> vec(const T* p, size_t n) {
    return p ? std::vector<T>(p, p + n) : std::vector<T>();
}

void load_side(PoleSide& s, const ems_pole_side& t, size_t ny, size_t nz) {
    s.axis = vec(t.axis, t.n_edges);
    s.node = vec(t.node, t.n_edges);
    s.sum_inv_z = vec(t.sum_inv_z, t.n_edges);
    s.pole_end = vec(t.pole_end, t.n_edges);
    s.kind = vec(t.kind, t.n_poles);
    s.a = vec(t.a, t.n_poles);
    s.inv_c = vec(t.inv_c, t.n_poles);
    s.inv_z = vec(t.inv_z, t.n_poles);
    s.half_l = vec(t.half_l, t.n_poles);
    s.prev.assign(t.n_edges, 0.0f);
    s.j.assign(t.n_poles, 0.0);
    s.q.assign(t.n_poles, 0.0);
    s.plane.resize(t.n_edges);
    for (size_t e = 0; e < t.n_edges; ++e) s.plane[e] = (uint32_t)(s.node[e] / (ny * nz));
}

// An edge's poles are at most this many (the per-edge scratch of poles_correct).
constexpr size_t MAX_POLES = 64;

bool side_ok(const ems_pole_side& t, size_t n) {
    if (t.n_edges && (!t.axis || !t.node || !t.sum_inv_z || !t.pole_end)) return false;
    if (t.n_poles && (!t.kind || !t.a || !t.inv_c || !t.inv_z || !t.half_l)) return false;
    uint32_t prev = 0;
    for (size_t e = 0; e < t.n_edges; ++e) {
        if (t.node[e] >= n || t.axis[e] > 2 || t.pole_end[e] < prev || t.pole_end[e] - prev > MAX_POLES)
            return false;
        prev = t.pole_end[e];
    }
    return prev == t.n_poles;
}

}  // namespace

extern "C" {

int oracle_create(const ems_engine_desc* d, int threads, oracle_engine** out) {
    if (!d || !out) return EMS_ERR_INVALID;
    if (d->nodes[0] < 2 || d->nodes[1] < 2 || d->nodes[2] < 2 || !(d->dt > 0)) return EMS_ERR_INVALID;
    auto* e = new oracle_engine();
    e->nx = d->nodes[0];
    e->ny = d->nodes[1];
    e->nz = d->nodes[2];
    e->plane = e->ny * e->nz;
    e->n = e->nx * e->plane;
    e->dt = d->dt;
    for (int l = 0; l < 12; ++l) {
        if (!d->coeff[l]) { delete e; return EMS_ERR_INVALID; }
        e->co[l].assign(d->coeff[l], d->coeff[l] + e->n);
    }
    for (int a = 0; a < 3; ++a) {
        e->u[a].assign(e->n, 0.0f);
        e->i[a].assign(e->n, 0.0f);
    }
    e->zero.assign(e->plane, 0.0f);
    e->plane_w.assign(e->nx, 0.0);
    for (size_t k = 0; k < d->n_ops; ++k) {
        Op op;
        op.kind = d->ops[k].kind;
        const void* t = d->ops[k].table;
        switch (op.kind) {
        case EMS_OP_CPML: {
            const auto* c = (const ems_cpml*)t;
            for (size_t s = 0; s < c->n_slabs; ++s) {
                CpmlSlab cs;
                cs.s = c->slabs[s];
                size_t depth = cs.s.hi[cs.s.normal] - cs.s.lo[cs.s.normal];
                cs.b = vec(cs.s.b, depth);
                cs.a = vec(cs.s.a, depth);
                cs.k = vec(cs.s.k, depth);
                size_t len = (cs.s.hi[0] - cs.s.lo[0]) * (cs.s.hi[1] - cs.s.lo[1]) * (cs.s.hi[2] - cs.s.lo[2]);
                cs.psi.assign(len, 0.0f);
                op.cpml.push_back(std::move(cs));
            }
            break;
        }
        case EMS_OP_POLES: {
            const auto* p = (const ems_poles*)t;
            if (!side_ok(p->electric, e->n) || !side_ok(p->magnetic, e->n)) { delete e; return EMS_ERR_INVALID; }
            load_side(op.pe, p->electric, e->ny, e->nz);
            load_side(op.ph, p->magnetic, e->ny, e->nz);
            break;
        }
        case EMS_OP_LUMPED: {
            const auto* l = (const ems_lumped*)t;
            Lumped& L = op.lumped;
            size_t ne = l->n_edges;
            L.axis = l->axis;
            L.node = vec(l->node, ne);
            L.cb = vec(l->cb, ne);
            L.g_src = vec(l->g_src, ne);
            L.series = l->series ? l->series : 1;
            L.src_in_branch = l->src_in_branch != 0;
            L.has_src = l->src_w != nullptr;
            L.src_w = vec(l->src_w, ne);
            L.src_amp = vec(l->src_amp, l->n_src_amp);
            L.has_branch = l->has_branch != 0;
            if (L.has_branch) {
                L.two_l_dt = vec(l->two_l_dt, ne);
                L.inv_c = vec(l->inv_c, ne);
                L.z = vec(l->z, ne);
            }
            L.record = l->record != 0;
            if (L.record) {
                L.rec_g = vec(l->rec_g, ne);
                L.rec_c = vec(l->rec_c, ne);
            }
            L.port_columns = l->port_columns;
            L.openems_order = l->openems_order != 0;
            if (l->oe_k) {
                if (!L.has_branch || !l->oe_vi || !L.openems_order) { delete e; return EMS_ERR_INVALID; }
                L.oe_k.assign(l->oe_k, l->oe_k + ne);
                L.oe_vi = vec(l->oe_vi, ne);
                L.oe_s.assign(ne, 0.0f);
            }
            L.v.assign(ne, 0.0);
            L.bj.assign(ne, 0.0);
            L.bq.assign(ne, 0.0);
            L.bu_prev.assign(ne, 0.0);
            L.j_avg.assign(ne, 0.0);
            L.ru_prev.assign(ne, 0.0);
            break;
        }
        case EMS_OP_SOURCE: {
            const auto* s = (const ems_source*)t;
            op.source.kind = s->kind;
            op.source.axis = vec(s->axis, s->n_edges);
            op.source.node = vec(s->node, s->n_edges);
            op.source.weight = vec(s->weight, s->n_edges);
            op.source.amp = vec(s->amp, s->n_amp);
            break;
        }
        case EMS_OP_PROBE: {
            const auto* p = (const ems_probe*)t;
            op.probe.quantity = p->quantity;
            op.probe.axis = vec(p->axis, p->n_entries);
            op.probe.node = vec(p->node, p->n_entries);
            op.probe.weight = vec(p->weight, p->n_entries);
            op.probe.interval = p->interval ? p->interval : 1;
            op.probe.f32_sum = p->f32_sum != 0;
            break;
        }
        case EMS_OP_UPML: {
            const auto* pm = (const ems_upml*)t;
            Upml& L = op.upml;
            for (int sd = 0; sd < 2; ++sd) {
                const size_t n = pm->n[sd];
                if (n && (!pm->axis[sd] || !pm->node[sd] || !pm->co[sd])) { delete e; return EMS_ERR_INVALID; }
                L.axis[sd] = vec(pm->axis[sd], n);
                L.node[sd] = vec(pm->node[sd], n);
                L.co[sd] = vec(pm->co[sd], 4 * n);
                L.f[sd].assign(n, 0.0f);
                L.v[sd].assign(n, 0.0f);
                std::vector<uint32_t> cnt(e->nx + 1, 0);
                for (size_t q = 0; q < n; ++q) {
                    if (L.axis[sd][q] > 2 || L.node[sd][q] >= e->n) { delete e; return EMS_ERR_INVALID; }
                    ++cnt[L.node[sd][q] / e->plane + 1];
                }
                for (size_t x = 0; x < e->nx; ++x) cnt[x + 1] += cnt[x];
                L.pstart[sd] = cnt;
                L.by_plane[sd].assign(n, 0);
                std::vector<uint32_t> fill(cnt.begin(), cnt.end() - 1);
                for (size_t q = 0; q < n; ++q) L.by_plane[sd][fill[L.node[sd][q] / e->plane]++] = (uint32_t)q;
            }
            break;
        }
        case EMS_OP_MUR: {
            const auto* m = (const ems_mur*)t;
            Mur& M = op.mur;
            if (m->n_edges > m->n || (m->n && (!m->axis || !m->node || !m->inner || !m->k)) ||
                (m->count_energy && !m->cap)) {
                delete e;
                return EMS_ERR_INVALID;
            }
            for (size_t q = 0; q < m->n; ++q) {
                bool ok = m->axis[q] < 3 && m->node[q] < e->n && m->inner[2 * q] < e->n;
                if (q >= m->n_edges) ok = ok && m->inner[2 * q + 1] < e->n;
                if (!ok) { delete e; return EMS_ERR_INVALID; }
            }
            M.n_edges = m->n_edges;
            M.axis = vec(m->axis, m->n);
            M.node = vec(m->node, m->n);
            M.inner = vec(m->inner, 2 * m->n);
            M.k = vec(m->k, 2 * m->n);
            M.hold = m->hold ? vec(m->hold, m->n) : std::vector<uint64_t>(m->n, 0);
            M.cap = m->count_energy ? vec(m->cap, m->n) : std::vector<double>(m->n, 0.0);
            M.openems_order = m->openems_order != 0;
            M.openems_corners = m->openems_corners != 0;
            M.count_energy = m->count_energy != 0;
            M.saved.assign(3 * m->n, 0.0f);
            M.last.assign(m->n, 0.0f);
            break;
        }
        case EMS_OP_SHEET: {
            const auto* st = (const ems_sheet*)t;
            Sheet& S = op.sheet;
            const size_t ne = st->n_edges, nc = st->n_couplings;
            S.axis = vec(st->axis, ne);
            S.node = vec(st->node, ne);
            S.nn = vec(st->nn, ne);
            S.k0 = vec(st->konst0, ne);
            S.a0 = vec(st->a0, ne);
            S.c_edge = vec(st->c_edge, ne);
            S.c_axis = vec(st->c_axis, nc);
            S.c_node = vec(st->c_node, nc);
            S.w_up = vec(st->w_up, nc);
            S.w_dn = vec(st->w_dn, nc);
            S.corr = vec(st->corr, nc);
            S.ecorr = vec(st->ecorr, nc);
            S.two_c = vec(st->two_c, st->n_konst);
            S.cp = vec(st->cp, st->n_konst);
            S.inv_den = vec(st->inv_den, st->n_konst);
            S.a = vec(st->a, st->n_a);
            uint32_t nodes_total = 0, layers_total = 0, c = 0, max_nn = 0;
            for (size_t q = 0; q < ne; ++q) {
                const uint32_t nn = S.nn[q], end = st->coupling_end[q];
                if (nn < 2 || S.axis[q] > 2 || S.node[q] >= e->n || end < c || end > nc ||
                    S.k0[q] + (size_t)nn > st->n_konst || S.a0[q] + (size_t)nn - 1 > st->n_a) {
                    delete e;
                    return EMS_ERR_INVALID;
                }
                S.c0.push_back(c);
                S.c1.push_back(end);
                c = end;
                S.n0.push_back(nodes_total);
                S.l0.push_back(layers_total);
                nodes_total += nn;
                layers_total += nn - 1;
                max_nn = std::max(max_nn, nn);
            }
            for (size_t q = 0; q < nc; ++q)
                if (S.c_axis[q] > 2 || S.c_node[q] >= e->n) {
                    delete e;
                    return EMS_ERR_INVALID;
                }
            S.u.assign(nodes_total, 0.0);
            S.h.assign(layers_total, 0.0);
            S.x.assign(max_nn, 0.0);
            break;
        }
        default:
            delete e;
            return EMS_ERR_INVALID;
        }
        e->ops.push_back(std::move(op));
    }
    size_t cells = (e->nx - 1) * (e->ny - 1) * (e->nz - 1);
    int nt = threads > 0 ? threads : default_threads(e->nx, cells);
    nt = (int)std::min<size_t>((size_t)nt, e->nx);
    // src/engine/fields.rs:38-58 Layout::new — contiguous x-slabs.
    size_t q = e->nx / nt, r = e->nx % nt, p = 0;
    for (int s = 0; s < nt; ++s) {
        e->slab_start.push_back(p);
        p += q + ((size_t)s < r ? 1 : 0);
    }
    e->slab_start.push_back(e->nx);
    e->pool = new Pool(nt);
    *out = e;
    return EMS_OK;
}

int oracle_destroy(oracle_engine* e) {
    if (!e) return EMS_ERR_INVALID;
    delete e->pool;
    delete e;
    return EMS_OK;
}

int oracle_threads(const oracle_engine* e) { return e ? e->pool->size() : 0; }

int oracle_upml_state(oracle_engine* e, size_t op, int side, float* f, float* v, size_t cap) {
    if (!e || op >= e->ops.size() || e->ops[op].kind != EMS_OP_UPML || side < 0 || side > 1) return EMS_ERR_INVALID;
    const Upml& L = e->ops[op].upml;
    if (cap < L.f[side].size()) return EMS_ERR_INVALID;
    std::memcpy(f, L.f[side].data(), L.f[side].size() * sizeof(float));
    std::memcpy(v, L.v[side].data(), L.v[side].size() * sizeof(float));
    return EMS_OK;
}

int oracle_set_curl_order(oracle_engine* e, int order) {
    if (!e || order < 0 || order > 1) return EMS_ERR_INVALID;
    e->oe = order == 1;
    return EMS_OK;
}

int oracle_run(oracle_engine* e, uint64_t n) {
    if (!e) return EMS_ERR_INVALID;
    for (uint64_t s = 0; s < n; ++s) e->one_step(false);
    return EMS_OK;
}

int oracle_step_with_energy(oracle_engine* e, double* energy) {
    if (!e || !energy) return EMS_ERR_INVALID;
    // src/engine/mod.rs:819-823 and pool.rs:675-692 (planes summed in order, ×dt/4).
    double w_ops = e->operator_energy();
    e->one_step(true);
    double s = 0.0;
    for (size_t gi = 0; gi < e->nx; ++gi) s += e->plane_w[gi];
    *energy = 0.25 * e->dt * s + w_ops;
    return EMS_OK;
}

int oracle_download_field(oracle_engine* e, int field, int axis, float* host) {
    if (!e || !host || axis < 0 || axis > 2 || field < 0 || field > 1) return EMS_ERR_INVALID;
    const auto& v = field == 0 ? e->u[axis] : e->i[axis];
    std::memcpy(host, v.data(), v.size() * sizeof(float));
    return EMS_OK;
}

int oracle_upload_field(oracle_engine* e, int field, int axis, const float* host) {
    if (!e || !host || axis < 0 || axis > 2 || field < 0 || field > 1) return EMS_ERR_INVALID;
    auto& v = field == 0 ? e->u[axis] : e->i[axis];
    std::memcpy(v.data(), host, v.size() * sizeof(float));
    return EMS_OK;
}

int oracle_sample(oracle_engine* e, const ems_sampler* s, double* out) {
    if (!e || !s || !out) return EMS_ERR_INVALID;
    const uint64_t nd[3] = {e->nx, e->ny, e->nz};
    const bool cur = s->quantity == EMS_DUMP_H || s->quantity == EMS_DUMP_B || s->quantity == EMS_DUMP_ROTH;
    const bool roth = s->quantity == EMS_DUMP_ROTH;
    const auto& F = cur ? e->i : e->u;
    auto get = [&](int c, const uint64_t p[3]) -> double { return (double)F[c][(p[0] * e->ny + p[1]) * e->nz + p[2]]; };
    // circulation (src/engine/dump.rs:814-834): i around the primary edge c.
    auto circ = [&](int c, const uint64_t p[3]) {
        const int a = (c + 1) % 3, b = (c + 2) % 3;
        double v = get(b, p) - get(a, p);
        if (p[a] > 0) {
            uint64_t q[3] = {p[0], p[1], p[2]};
            q[a] -= 1;
            v -= get(b, q);
        }
        if (p[b] > 0) {
            uint64_t q[3] = {p[0], p[1], p[2]};
            q[b] -= 1;
            v += get(a, q);
        }
        return v;
    };
    const uint64_t* dims = s->dims;
    const uint64_t off[3] = {0, 3 * dims[0], 3 * (dims[0] + dims[1])};
    const uint64_t vol = s->fac_dims[0] * s->fac_dims[1] * s->fac_dims[2];
    for (int a = 0; a < 3; ++a)
        for (uint64_t q = 0; q < 6 * dims[a]; ++q)
            if (s->tap_w[2 * off[a] + q] != 0.0 && s->tap_idx[2 * off[a] + q] >= nd[a]) return EMS_ERR_INVALID;
    size_t at = 0;
    for (uint64_t p = 0; p < dims[0]; ++p)
        for (uint64_t q = 0; q < dims[1]; ++q)
            for (uint64_t r = 0; r < dims[2]; ++r, ++at)
                for (int c = 0; c < 3; ++c) {
                    const uint64_t ex = 2 * (off[0] + c * dims[0] + p), ey = 2 * (off[1] + c * dims[1] + q),
                                   ez = 2 * (off[2] + c * dims[2] + r);
                    double v = 0.0;
                    for (int tx = 0; tx < 2; ++tx) {
                        const double wx = s->tap_w[ex + tx];
                        if (wx == 0.0) continue;
                        for (int ty = 0; ty < 2; ++ty) {
                            const double wy = s->tap_w[ey + ty];
                            if (wy == 0.0) continue;
                            for (int tz = 0; tz < 2; ++tz) {
                                const double wz = s->tap_w[ez + tz];
                                if (wz == 0.0) continue;
                                const uint64_t node[3] = {s->tap_idx[ex + tx], s->tap_idx[ey + ty], s->tap_idx[ez + tz]};
                                const double x = roth ? circ(c, node) : get(c, node);
                                double m = 1.0;
                                if (s->factors)
                                    m = s->factors[c * vol + ((node[0] - s->fac_lo[0]) * s->fac_dims[1] +
                                                              (node[1] - s->fac_lo[1])) * s->fac_dims[2] +
                                                   (node[2] - s->fac_lo[2])];
                                v += wx * wy * wz * m * x;
                            }
                        }
                    }
                    out[3 * at + c] = v;
                }
    return EMS_OK;
}

int oracle_samples(oracle_engine* e, size_t op, int which, double* out, size_t cap, size_t* n) {
    if (!e || !n || op >= e->ops.size()) return EMS_ERR_INVALID;
    const Op& o = e->ops[op];
    const std::vector<double>* v = nullptr;
    if (o.kind == EMS_OP_PROBE && which == 0) v = &o.probe.values;
    else if (o.kind == EMS_OP_LUMPED && which == 0) v = &o.lumped.rec;
    else if (o.kind == EMS_OP_LUMPED && which == 1) v = &o.lumped.port_v;
    else if (o.kind == EMS_OP_LUMPED && which == 2) v = &o.lumped.port_i;
    else if (o.kind == EMS_OP_SHEET && which == 0) v = &o.sheet.u;
    else if (o.kind == EMS_OP_SHEET && which == 1) v = &o.sheet.h;
    else return EMS_ERR_INVALID;
    *n = v->size();
    if (out) std::memcpy(out, v->data(), std::min(cap, v->size()) * sizeof(double));
    return EMS_OK;
}

}  // extern "C"
