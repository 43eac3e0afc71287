// host.cpp — host-side model set-up for the B200 engine (see include/ems_host.h).
//
// Restates the reference's set-up arithmetic expression by expression
// (f64, no contraction: built with -ffp-contract=off) so the tables handed
// to the engine are the ones the reference's own host would compute.
#include "../../include/ems_host.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <numeric>
#include <unordered_map>
#include <tuple>
#include <string>
#include <thread>
#include <vector>

namespace {

// src/constants.rs:9-18.
constexpr double C0 = 299792458.0;
constexpr double MU0 = 1.25663706127e-6;
const double EPS0 = 1.0 / (MU0 * C0 * C0);
// openEMS's vacuum constants (src/constants.rs OPENEMS_EPS0, OPENEMS_MU0).
constexpr double OE_EPS0 = 8.85418781762e-12;
constexpr double OE_MU0 = 1.256637062e-6;
const double Z0 = MU0 * C0;
constexpr double PI = 3.14159265358979323846;
constexpr double TAU = 6.28318530717958647692;
constexpr double LN_10 = 2.30258509299404568402;

inline int next_axis(int a) { return (a + 1) % 3; }
inline int prev_axis(int a) { return (a + 2) % 3; }

struct Material {
    double eps_r[3], mu_r[3], kappa[3], sigma_m[3];
};

struct Pole {
    int kind;  // 0 Lorentz, 1 Drude, 2 Debye
    double p1, p2, p3;
    // Pole::scaled (src/engine/dispersive.rs:306-327).
    Pole scaled(double s) const {
        Pole q = *this;
        if (kind == 0 || kind == 1) q.p1 = p1 * std::sqrt(s);
        else q.p1 = p1 * s;
        return q;
    }
};

struct Entry {
    int field, axis;
    uint64_t node[3];
    Pole pole;
};

void run_threads(size_t n, const std::function<void(size_t, size_t)>& f);

}  // namespace

struct ems_cellset {
    uint64_t c[3];
    std::vector<uint8_t> mask;
    uint64_t lo[3], hi[3];  // bounding box of the set (cells, half-open)
    bool any = false;
    bool at(uint64_t i, uint64_t j, uint64_t k) const { return mask[(i * c[1] + j) * c[2] + k] != 0; }
    void grow(const uint64_t l[3], const uint64_t h[3]) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = any ? std::min(lo[a], l[a]) : l[a];
            hi[a] = any ? std::max(hi[a], h[a]) : h[a];
        }
        any = true;
    }
};

struct ems_dispersive {
    std::vector<Entry> entries;
};

namespace {

struct OpStore {
    int kind = 0;
    // CPML
    std::vector<ems_cpml_slab> slabs;
    std::vector<std::vector<float>> arrays;
    ems_cpml cpml{};
    double index[6] = {0, 0, 0, 0, 0, 0};
    // poles
    struct Side {
        std::vector<uint8_t> axis, kind;
        std::vector<uint64_t> node;
        std::vector<double> sum_inv_z, a, inv_c, inv_z, half_l;
        std::vector<uint32_t> pole_end;
        void fill(ems_pole_side& t) const {
            t.n_edges = axis.size();
            t.axis = axis.data();
            t.node = node.data();
            t.sum_inv_z = sum_inv_z.data();
            t.pole_end = pole_end.data();
            t.n_poles = kind.size();
            t.kind = kind.data();
            t.a = a.data();
            t.inv_c = inv_c.data();
            t.inv_z = inv_z.data();
            t.half_l = half_l.data();
        }
    } pe, ph;
    ems_poles poles{};
    // lumped
    std::vector<uint64_t> lnode;
    std::vector<double> lcb, lg, lw, lamp, lrg, lrc, ltl, linvc, lz, loevi;
    std::vector<float> loek;
    ems_lumped lumped{};
    // source / probe
    std::vector<uint8_t> axis;
    std::vector<uint64_t> node;
    std::vector<float> fw, famp;
    std::vector<double> dw;
    ems_source source{};
    ems_probe probe{};
    // Mur
    std::vector<uint64_t> inner, hold;
    std::vector<float> mk;
    std::vector<double> mcap;
    ems_mur mur{};
    // openEMS PML (side 0 E, 1 H)
    std::vector<uint8_t> pax[2];
    std::vector<uint64_t> pnode[2];
    std::vector<float> pco[2];
    ems_upml upml{};
    // conducting sheets
    std::vector<uint8_t> sax, cax;
    std::vector<uint64_t> snode, cnode;
    std::vector<uint32_t> snn, sk0, sa0, send;
    std::vector<double> scedge, cwup, cwdn, ccorr, cecorr, two_c, cp, inv_den, sa;
    ems_sheet sheet{};
};

}  // namespace

struct ems_model {
    std::vector<double> lines[3];
    uint64_t n[3];
    uint64_t c[3];
    std::vector<Material> table;
    std::vector<uint16_t> cell;
    std::vector<uint8_t> pec[3];
    int faces[6] = {0, 0, 0, 0, 0, 0};
    bool built = false;
    bool oe_round = false;  // built with openEMS's coefficient rounding
    // Per-edge materials given by the caller (ems_model_set_edge_materials)
    // in place of the averages of the cells: [axis][0 eps_r or mu_r, 1
    // kappa or sigma_m], reference layout; empty: from the cells.
    std::vector<double> emat[3][2], hmat[3][2];
    // Per-edge phase velocities of local-medium Mur faces (MurMedia), keyed
    // face·3 + axis, one value per node of the face plane (0: none).
    std::map<int, std::vector<double>> mur_v;
    // Capacitances that replaced an E edge's medium (ems_model_set_edge_circuit),
    // keyed axis·N + node index: the circuit openEMS's poles of that edge
    // are formed with (src/sim/map.rs:1583-1588).
    std::unordered_map<uint64_t, double> edge_cap;
    double dt = 0.0;
    std::vector<float> co[12];
    std::vector<std::unique_ptr<OpStore>> ops;
    std::vector<ems_op> op_list;
    ems_engine_desc desc{};
    std::string err;

    uint64_t index(uint64_t i, uint64_t j, uint64_t k) const { return (i * n[1] + j) * n[2] + k; }
    // src/engine/grid.rs:562-597.
    double delta(int a, uint64_t i) const { return lines[a][i + 1] - lines[a][i]; }
    double dual_delta(int a, uint64_t i) const {
        double lo = i > 0 ? delta(a, i - 1) : 0.0;
        double hi = i + 1 < n[a] ? delta(a, i) : 0.0;
        return 0.5 * (lo + hi);
    }
    double min_delta(int a) const {
        double m = INFINITY;
        for (uint64_t i = 0; i + 1 < n[a]; ++i) m = std::fmin(m, delta(a, i));
        return m;
    }
    const Material& mat(uint64_t i, uint64_t j, uint64_t k) const {
        return table[cell[(i * c[1] + j) * c[2] + k]];
    }
    // primary_edge_cg (src/engine/coeffs.rs:264-292).
    void primary_edge_cg(int a, const uint64_t p[3], double& cap_out, double& cond_out) const {
        const int b = next_axis(a), cc = prev_axis(a);
        const double l = delta(a, p[a]);
        double cap = 0.0, cond = 0.0;
        for (int db = -1; db <= 0; ++db) {
            if (p[b] == 0 && db < 0) continue;
            uint64_t cb = p[b] + db;
            if (cb >= n[b] - 1) continue;
            for (int dc = -1; dc <= 0; ++dc) {
                if (p[cc] == 0 && dc < 0) continue;
                uint64_t ccell = p[cc] + dc;
                if (ccell >= n[cc] - 1) continue;
                uint64_t q[3];
                q[a] = p[a];
                q[b] = cb;
                q[cc] = ccell;
                double area = 0.25 * delta(b, cb) * delta(cc, ccell);
                const Material& m = mat(q[0], q[1], q[2]);
                cap += EPS0 * m.eps_r[a] * area;
                cond += m.kappa[a] * area;
            }
        }
        cap_out = cap / l;
        cond_out = cond / l;
    }
    // dual_edge_lr (src/engine/coeffs.rs:300-325).
    void dual_edge_lr(int a, const uint64_t p[3], double& l_out, double& r_out) const {
        const int b = next_axis(a), cc = prev_axis(a);
        const double area = delta(b, p[b]) * delta(cc, p[cc]);
        double inv_l = 0.0, r_over_l2 = 0.0;
        for (int da = -1; da <= 0; ++da) {
            if (p[a] == 0 && da < 0) continue;
            uint64_t ca = p[a] + da;
            if (ca >= n[a] - 1) continue;
            uint64_t q[3] = {p[0], p[1], p[2]};
            q[a] = ca;
            double half = 0.5 * delta(a, ca);
            const Material& m = mat(q[0], q[1], q[2]);
            double lc = MU0 * m.mu_r[a] * area / half;
            double rc = m.sigma_m[a] * area / half;
            inv_l += 1.0 / lc;
            r_over_l2 += rc / (lc * lc);
        }
        double l = 1.0 / inv_l;
        l_out = l;
        r_out = l * l * r_over_l2;
    }

    void refresh_desc() {
        desc.nodes[0] = n[0];
        desc.nodes[1] = n[1];
        desc.nodes[2] = n[2];
        desc.dt = dt;
        for (int l = 0; l < 12; ++l) desc.coeff[l] = co[l].empty() ? nullptr : co[l].data();
        op_list.clear();
        for (auto& o : ops) {
            ems_op e;
            e.kind = o->kind;
            switch (o->kind) {
            case EMS_OP_CPML: e.table = &o->cpml; break;
            case EMS_OP_POLES: e.table = &o->poles; break;
            case EMS_OP_LUMPED: e.table = &o->lumped; break;
            case EMS_OP_SOURCE: e.table = &o->source; break;
            case EMS_OP_MUR: e.table = &o->mur; break;
            case EMS_OP_UPML: e.table = &o->upml; break;
            case EMS_OP_SHEET: e.table = &o->sheet; break;
            default: e.table = &o->probe; break;
            }
            op_list.push_back(e);
        }
        desc.n_ops = op_list.size();
        desc.ops = op_list.data();
    }
};

namespace {

void run_threads(size_t n, const std::function<void(size_t, size_t)>& f) {
    unsigned hw = std::thread::hardware_concurrency();
    size_t t = std::max<size_t>(1, std::min<size_t>(hw ? hw : 1, 64));
    t = std::min(t, n);
    if (t <= 1) { f(0, n); return; }
    std::vector<std::thread> th;
    size_t q = n / t, r = n % t, p = 0;
    for (size_t s = 0; s < t; ++s) {
        size_t len = q + (s < r ? 1 : 0);
        th.emplace_back(f, p, p + len);
        p += len;
    }
    for (auto& x : th) x.join();
}

// CpmlCoefficients::in_medium (src/engine/boundary/cpml.rs:350-387).
struct CpmlCo {
    double b, a, direct;
};
CpmlCo cpml_in_medium(double m, double sigma_factor, double kappa_max, double alpha_max, bool linear, double rho,
                      double delta, double dt, double n) {
    double g = std::pow(rho, m);
    double eta = n * Z0;
    double sigma = sigma_factor * 0.8 * (m + 1.0) / (eta * delta) * g;
    double kappa = 1.0 + (kappa_max - 1.0) * g;
    double alpha = alpha_max * (1.0 - rho);
    double b = std::exp(-(sigma / kappa + alpha) * dt / EPS0);
    double den = sigma * kappa + kappa * kappa * alpha;
    double x = (sigma / kappa + alpha) * dt / EPS0;
    double a, shift;
    if (!(sigma > 0.0 && den > 0.0)) {
        a = 0.0;
        shift = 0.0;
    } else if (linear && x <= 8.0) {
        double cdt = sigma * dt / (EPS0 * kappa * kappa);
        double gg = x < 1e-3 ? 0.5 - x / 3.0 + x * x / 8.0 : (-std::expm1(-x) - x * b) / (x * x);
        double a1 = -cdt * gg;
        double a0 = cdt * std::expm1(-x) / x - a1;
        a = a0 + a1 / b;
        shift = a1 / b;
    } else {
        a = sigma * (b - 1.0) / den;
        shift = 0.0;
    }
    return {b, a, 1.0 / kappa - 1.0 - shift};
}

// Waveform::Gaussian (src/waveform.rs:241-248, 455-463).
double gaussian_tau(double fc) { return std::sqrt(LN_10) / (PI * fc); }
double gaussian_delay(double fc) { return gaussian_tau(fc) * std::sqrt(6.0 * LN_10); }

bool set_err(ems_model* m, const std::string& s) {
    m->err = s;
    return false;
}

}  // namespace

extern "C" {

double ems_const_eps0(void) { return EPS0; }
double ems_const_mu0(void) { return MU0; }
double ems_const_c0(void) { return C0; }

double ems_waveform_value(int kind, double f0, double fc, double t, double dt) {
    (void)dt;
    if (kind != 0) return 0.0;
    double delay = gaussian_delay(fc);
    if (!(t >= 0.0 && t <= 2.0 * delay)) return 0.0;
    double x = (t - delay) / gaussian_tau(fc);
    return std::cos(TAU * f0 * (t - delay)) * std::exp(-x * x);
}

double ems_waveform_duration(int kind, double f0, double fc) {
    (void)f0;
    return kind == 0 ? 2.0 * gaussian_delay(fc) : 0.0;
}

ems_model* ems_model_new(const double* x, size_t nx, const double* y, size_t ny, const double* z, size_t nz) {
    const double* l[3] = {x, y, z};
    size_t nn[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a) {
        if (!l[a] || nn[a] < 2) return nullptr;
        for (size_t i = 0; i < nn[a]; ++i)
            if (!std::isfinite(l[a][i]) || (i && !(l[a][i] > l[a][i - 1]))) return nullptr;
    }
    auto* m = new ems_model();
    for (int a = 0; a < 3; ++a) {
        m->lines[a].assign(l[a], l[a] + nn[a]);
        m->n[a] = nn[a];
        m->c[a] = nn[a] - 1;
    }
    m->table.push_back(Material{{1, 1, 1}, {1, 1, 1}, {0, 0, 0}, {0, 0, 0}});
    m->cell.assign(m->c[0] * m->c[1] * m->c[2], 0);
    for (int a = 0; a < 3; ++a) m->pec[a].assign(m->n[0] * m->n[1] * m->n[2], 0);
    m->refresh_desc();
    return m;
}

void ems_model_free(ems_model* m) { delete m; }
const char* ems_model_error(const ems_model* m) { return m ? m->err.c_str() : "null model"; }
void ems_model_nodes(const ems_model* m, uint64_t nodes[3]) {
    for (int a = 0; a < 3; ++a) nodes[a] = m->n[a];
}

int ems_model_material(ems_model* m, const double eps_r[3], const double mu_r[3], const double kappa[3],
                       const double sigma_m[3]) {
    Material t;
    for (int a = 0; a < 3; ++a) {
        t.eps_r[a] = eps_r[a];
        t.mu_r[a] = mu_r[a];
        t.kappa[a] = kappa[a];
        t.sigma_m[a] = sigma_m[a];
        // Material::validate (src/engine/material.rs).
        if (!(std::isfinite(eps_r[a]) && eps_r[a] > 0 && std::isfinite(mu_r[a]) && mu_r[a] > 0 &&
              std::isfinite(kappa[a]) && kappa[a] >= 0 && std::isfinite(sigma_m[a]) && sigma_m[a] >= 0)) {
            set_err(m, "invalid material");
            return -1;
        }
    }
    if (m->table.size() >= 65535) return -1;
    m->table.push_back(t);
    return (int)m->table.size() - 1;
}

ems_cellset* ems_cellset_new(const ems_model* m) {
    auto* s = new ems_cellset();
    for (int a = 0; a < 3; ++a) s->c[a] = m->c[a];
    s->mask.assign(s->c[0] * s->c[1] * s->c[2], 0);
    return s;
}
void ems_cellset_free(ems_cellset* s) { delete s; }

int ems_cellset_box(ems_cellset* s, const uint64_t lo[3], const uint64_t hi[3]) {
    for (int a = 0; a < 3; ++a)
        if (lo[a] > hi[a] || hi[a] > s->c[a]) return EMS_ERR_INVALID;
    if (lo[0] == hi[0] || lo[1] == hi[1] || lo[2] == hi[2]) return EMS_OK;
    for (uint64_t i = lo[0]; i < hi[0]; ++i)
        for (uint64_t j = lo[1]; j < hi[1]; ++j)
            std::memset(&s->mask[(i * s->c[1] + j) * s->c[2] + lo[2]], 1, hi[2] - lo[2]);
    s->grow(lo, hi);
    return EMS_OK;
}

int ems_cellset_sphere(ems_cellset* s, const double ctr[3], double r) {
    // Cells whose centre (index + 1/2, in cell units) lies within r.
    uint64_t lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        double l = std::floor(ctr[a] - r - 1.0), h = std::ceil(ctr[a] + r + 1.0);
        lo[a] = (uint64_t)std::max(0.0, l);
        hi[a] = (uint64_t)std::min((double)s->c[a], std::max(0.0, h));
        if (lo[a] >= hi[a]) return EMS_OK;
    }
    bool any = false;
    for (uint64_t i = lo[0]; i < hi[0]; ++i)
        for (uint64_t j = lo[1]; j < hi[1]; ++j)
            for (uint64_t k = lo[2]; k < hi[2]; ++k) {
                double dx = (double)i + 0.5 - ctr[0], dy = (double)j + 0.5 - ctr[1], dz = (double)k + 0.5 - ctr[2];
                if (dx * dx + dy * dy + dz * dz <= r * r) {
                    s->mask[(i * s->c[1] + j) * s->c[2] + k] = 1;
                    any = true;
                }
            }
    if (any) s->grow(lo, hi);
    return EMS_OK;
}

uint64_t ems_cellset_count(const ems_cellset* s) {
    uint64_t n = 0;
    for (uint8_t v : s->mask) n += v;
    return n;
}

int ems_model_fill(ems_model* m, const ems_cellset* s, int mat) {
    if (mat < 0 || (size_t)mat >= m->table.size() || m->built) return EMS_ERR_INVALID;
    for (size_t q = 0; q < s->mask.size(); ++q)
        if (s->mask[q]) m->cell[q] = (uint16_t)mat;
    return EMS_OK;
}

int ems_model_pec_edges(ems_model* m, int axis, const uint64_t lo[3], const uint64_t hi[3]) {
    if (axis < 0 || axis > 2 || m->built) return EMS_ERR_INVALID;
    for (int a = 0; a < 3; ++a)
        if (lo[a] > hi[a] || hi[a] >= m->n[a]) return EMS_ERR_INVALID;
    for (uint64_t i = lo[0]; i <= hi[0]; ++i)
        for (uint64_t j = lo[1]; j <= hi[1]; ++j)
            for (uint64_t k = lo[2]; k <= hi[2]; ++k) m->pec[axis][m->index(i, j, k)] = 1;
    return EMS_OK;
}

int ems_model_faces(ems_model* m, const int faces[6]) {
    if (m->built) return EMS_ERR_INVALID;
    for (int f = 0; f < 6; ++f) {
        if (faces[f] != 0 && faces[f] != 1) return EMS_ERR_INVALID;
        m->faces[f] = faces[f];
    }
    return EMS_OK;
}

double ems_model_courant_limit(const ems_model* m) {
    // courant_limit (src/engine/coeffs.rs:254-262).
    double s = 0.0;
    for (int a = 0; a < 3; ++a) {
        double d = m->min_delta(a);
        s += 1.0 / (d * d);
    }
    return 1.0 / (C0 * std::sqrt(s));
}

// EdgeMaterials::from_cells (src/engine/edge_material.rs:376-413): eps_r
// and kappa of the E edge along a at p, mu_r and sigma_m of the H dual edge
// along a through p (vacuum where the edge does not exist).
static void edge_eps(const ems_model* m, int a, const uint64_t p[3], double& eps, double& kap) {
    eps = 1.0;
    kap = 0.0;
    if (p[a] + 1 >= m->n[a]) return;
    if (!m->emat[a][0].empty()) {
        const uint64_t idx = m->index(p[0], p[1], p[2]);
        eps = m->emat[a][0][idx];
        kap = m->emat[a][1][idx];
        return;
    }
    const int b = next_axis(a), c = prev_axis(a);
    double cap_c, g_c;
    m->primary_edge_cg(a, p, cap_c, g_c);
    const double k_ = m->delta(a, p[a]) / (m->dual_delta(b, p[b]) * m->dual_delta(c, p[c]));
    eps = cap_c * k_ / EPS0;
    kap = g_c * k_;
}

static void edge_mu(const ems_model* m, int a, const uint64_t p[3], double& mu, double& sig) {
    mu = 1.0;
    sig = 0.0;
    const int b = next_axis(a), c = prev_axis(a);
    if (p[b] + 1 >= m->n[b] || p[c] + 1 >= m->n[c]) return;
    if (!m->hmat[a][0].empty()) {
        const uint64_t idx = m->index(p[0], p[1], p[2]);
        mu = m->hmat[a][0][idx];
        sig = m->hmat[a][1][idx];
        return;
    }
    double l_c, r_c;
    m->dual_edge_lr(a, p, l_c, r_c);
    const double k_ = m->dual_delta(a, p[a]) / (m->delta(b, p[b]) * m->delta(c, p[c]));
    mu = l_c * k_ / MU0;
    sig = r_c * k_;
}

// openEMS's magnetic conductivity of the H dual edge along a through p
// (openems_sigma_m and sigma_m_average, src/compile/openems.rs:580-650):
// the length-weighted harmonic mean of the two half cells along a, 0 when
// the upper half is lossless, a lossless lower half left out.
static double oe_sigma_m(const ems_model* m, int a, const uint64_t p[3]) {
    const int b = next_axis(a), c = prev_axis(a);
    uint64_t q[3] = {p[0], p[1], p[2]};
    double len = 0.0, inv = 0.0;
    bool hi_zero = false;
    for (int side = 0; side < 2; ++side) {
        if (side == 0 && p[a] == 0) continue;
        if (side == 1 && p[a] + 1 >= m->n[a]) continue;
        q[a] = side == 0 ? p[a] - 1 : p[a];
        q[b] = p[b];
        q[c] = p[c];
        const double h = 0.5 * m->delta(a, q[a]);
        const double sg = m->mat(q[0], q[1], q[2]).sigma_m[a];
        len += h;
        if (sg != 0.0) inv += h / sg;
        else if (side == 1) hi_zero = true;
    }
    if (hi_zero || inv == 0.0) return 0.0;
    return len / inv;
}

// Coefficients::from_edges_rounded (src/engine/coeffs.rs:879-966) from the
// per-edge materials of EdgeMaterials::from_cells; `openems`: the circuit
// quantities C, G, L, R rounded to f32 and formed with openEMS's vacuum
// constants (CoeffRounding::OpenEms, coeffs.rs:705-760); `oe_sigma`: the
// magnetic conductivities by openEMS's average (oe_sigma_m). One x-plane
// range per thread.
static void compute_coefficients(ems_model* m, double dt, bool openems, bool oe_sigma = false) {
    const uint64_t N = m->n[0] * m->n[1] * m->n[2];
    for (int l = 0; l < 12; ++l) m->co[l].assign(N, 0.0f);
    m->edge_cap.clear();
    bool pec_face[3][2];
    for (int t = 0; t < 3; ++t)
        for (int s = 0; s < 2; ++s) pec_face[t][s] = m->faces[2 * t + s] == 0;
    const double eps0 = openems ? OE_EPS0 : EPS0, mu0 = openems ? OE_MU0 : MU0;
    auto store = [openems](double x) { return openems ? (double)(float)x : x; };
    run_threads(m->n[0], [&](size_t i0, size_t i1) {
        for (uint64_t i = i0; i < i1; ++i)
            for (uint64_t j = 0; j < m->n[1]; ++j)
                for (uint64_t k = 0; k < m->n[2]; ++k) {
                    const uint64_t p[3] = {i, j, k};
                    const uint64_t idx = m->index(i, j, k);
                    for (int a = 0; a < 3; ++a) {
                        const int b = next_axis(a), c = prev_axis(a);
                        if (p[a] + 1 < m->n[a]) {
                            bool on_pec_face = false;
                            for (int t : {b, c})
                                if ((p[t] == 0 && pec_face[t][0]) || (p[t] == m->n[t] - 1 && pec_face[t][1]))
                                    on_pec_face = true;
                            if (!(on_pec_face || m->pec[a][idx])) {
                                double eps, kap;
                                edge_eps(m, a, p, eps, kap);
                                double geo = m->dual_delta(b, p[b]) * m->dual_delta(c, p[c]) / m->delta(a, p[a]);
                                double cap = store(eps0 * eps * geo);
                                double g = store(kap * geo);
                                double den = cap + 0.5 * g * dt;
                                m->co[a][idx] = (float)((cap - 0.5 * g * dt) / den);
                                m->co[3 + a][idx] = (float)(dt / den);
                            }
                        }
                        if (p[b] + 1 < m->n[b] && p[c] + 1 < m->n[c]) {
                            double mu, sig;
                            edge_mu(m, a, p, mu, sig);
                            if (oe_sigma && m->hmat[a][1].empty()) sig = oe_sigma_m(m, a, p);
                            double geo = m->delta(b, p[b]) * m->delta(c, p[c]) / m->dual_delta(a, p[a]);
                            double l = store(mu0 * mu * geo);
                            double r = store(sig * geo);
                            double den = l + 0.5 * r * dt;
                            m->co[6 + a][idx] = (float)((l - 0.5 * r * dt) / den);
                            m->co[9 + a][idx] = (float)(dt / den);
                        }
                    }
                }
    });
    m->dt = dt;
    m->built = true;
    m->refresh_desc();
}

int ems_model_set_mur_media(ems_model* m, int face, int axis, const double* v) {
    if (face < 0 || face > 5 || axis < 0 || axis > 2 || axis == face / 2 || !v)
        return set_err(m, "invalid Mur media"), EMS_ERR_INVALID;
    const int a = face / 2, u = a == 0 ? 1 : 0, w = a == 2 ? 1 : 2;
    const size_t N = (size_t)(m->n[u] * m->n[w]);
    for (size_t q = 0; q < N; ++q)
        if (!(std::isfinite(v[q]) && v[q] >= 0.0)) return set_err(m, "Mur media velocities must be finite and >= 0"), EMS_ERR_INVALID;
    m->mur_v[face * 3 + axis].assign(v, v + N);
    return EMS_OK;
}

int ems_model_set_edge_materials(ems_model* m, int field, int axis, const double* v0, const double* v1) {
    if (m->built) return set_err(m, "set edge materials before build"), EMS_ERR_INVALID;
    if ((field != 0 && field != 1) || axis < 0 || axis > 2 || !v0 || !v1)
        return set_err(m, "invalid edge material arrays"), EMS_ERR_INVALID;
    const size_t N = (size_t)(m->n[0] * m->n[1] * m->n[2]);
    std::vector<double>* dst = field ? m->hmat[axis] : m->emat[axis];
    for (size_t q = 0; q < N; ++q)
        if (!(std::isfinite(v0[q]) && v0[q] > 0.0 && std::isfinite(v1[q]) && v1[q] >= 0.0))
            return set_err(m, "edge materials must be finite, eps_r/mu_r > 0, kappa/sigma_m >= 0"), EMS_ERR_INVALID;
    dst[0].assign(v0, v0 + N);
    dst[1].assign(v1, v1 + N);
    return EMS_OK;
}

int ems_model_build(ems_model* m, double courant, double fixed_dt) {
    if (m->built) return set_err(m, "model already built"), EMS_ERR_INVALID;
    // TimeStep::resolve (src/engine/coeffs.rs:220-240).
    double max = ems_model_courant_limit(m);
    double dt;
    if (fixed_dt != 0.0) {  // NaN and negative values included: TimeStep::Fixed
        if (!(std::isfinite(fixed_dt) && fixed_dt > 0.0)) return set_err(m, "time step must be finite and > 0"), EMS_ERR_INVALID;
        if (!(fixed_dt <= max)) return set_err(m, "time step above the stability limit"), EMS_ERR_INVALID;
        dt = fixed_dt;
    } else {
        if (!(std::isfinite(courant) && courant > 0.0 && courant <= 1.0)) return set_err(m, "Courant factor must be in (0, 1]"), EMS_ERR_INVALID;
        dt = courant * max;
    }
    compute_coefficients(m, dt, false);
    return EMS_OK;
}

int ems_model_build_bound(ems_model* m, double dt, int flags) {
    if (m->built) return set_err(m, "model already built"), EMS_ERR_INVALID;
    // TimeStep::Bound (src/engine/coeffs.rs:233-236): any positive step.
    if (!(std::isfinite(dt) && dt > 0.0)) return set_err(m, "time step must be positive and finite"), EMS_ERR_INVALID;
    if (flags & ~3) return set_err(m, "unknown build flags"), EMS_ERR_INVALID;
    compute_coefficients(m, dt, (flags & 1) != 0, (flags & 2) != 0);
    m->oe_round = (flags & 1) != 0;
    return EMS_OK;
}

namespace {

// openEMS's time-step criteria (src/engine/timestep.rs:127-320): the
// circuit values C (E edges) and L (H dual edges) in f32 with openEMS's
// constants and full dual lengths at the boundary; a lookup clamps every
// index into its table.
struct OeCircuit {
    uint64_t n[3];
    uint64_t dc[3][3], dl[3][3];
    std::vector<float> c[3], l[3];
    float get(const std::vector<float>& v, const uint64_t* d, const int64_t q[3]) const {
        uint64_t k[3];
        for (int a = 0; a < 3; ++a) k[a] = (uint64_t)std::min<int64_t>(std::max<int64_t>(q[a], 0), (int64_t)d[a] - 1);
        return v[(k[0] * d[1] + k[1]) * d[2] + k[2]];
    }
    float C(int a, const int64_t q[3]) const { return get(c[a], dc[a], q); }
    float L(int a, const int64_t q[3]) const { return get(l[a], dl[a], q); }
};

OeCircuit oe_circuit(const ems_model* m) {
    OeCircuit cir;
    std::vector<double> pl[3], dl[3];
    for (int a = 0; a < 3; ++a) {
        cir.n[a] = m->n[a];
        const uint64_t na = m->n[a];
        if (na < 2) pl[a] = {1.0};
        else for (uint64_t i = 0; i + 1 < na; ++i) pl[a].push_back(m->delta(a, i));
        for (uint64_t i = 0; i < na; ++i) {
            const bool lo = i >= 1 && i - 1 < pl[a].size(), hi = i < pl[a].size() && na >= 2 && i + 1 < na;
            if (lo && hi) dl[a].push_back(0.5 * (pl[a][i - 1] + pl[a][i]));
            else if (lo) dl[a].push_back(pl[a][i - 1]);
            else if (i < pl[a].size()) dl[a].push_back(pl[a][i]);
            else dl[a].push_back(1.0);
        }
    }
    for (int a = 0; a < 3; ++a) {
        const int b = (a + 1) % 3, c = (a + 2) % 3;
        for (int edge = 1; edge >= 0; --edge) {
            uint64_t* d = edge ? cir.dc[a] : cir.dl[a];
            for (int q = 0; q < 3; ++q)
                d[q] = ((q == a) == (edge != 0)) ? std::max<uint64_t>(m->n[q] - 1, 1) : m->n[q];
            std::vector<float>& v = edge ? cir.c[a] : cir.l[a];
            v.resize(d[0] * d[1] * d[2]);
            for (uint64_t i = 0; i < d[0]; ++i)
                for (uint64_t j = 0; j < d[1]; ++j)
                    for (uint64_t k = 0; k < d[2]; ++k) {
                        const uint64_t q[3] = {i, j, k};
                        double x;
                        if (edge) {
                            double eps, kap;
                            edge_eps(m, a, q, eps, kap);
                            const double geo = dl[b][q[b]] * dl[c][q[c]] / pl[a][q[a]];
                            x = OE_EPS0 * eps * geo;
                        } else {
                            double mu, sig;
                            edge_mu(m, a, q, mu, sig);
                            const double geo = pl[b][q[b]] * pl[c][q[c]] / dl[a][q[a]];
                            x = OE_MU0 * mu * geo;
                        }
                        v[(i * d[1] + j) * d[2] + k] = (float)x;
                    }
        }
    }
    return cir;
}

inline float oe_x(float c, float l) { return 1.0f / (c * l); }

}  // namespace

double ems_model_openems_timestep(const ems_model* m, int method) {
    if (method != 1 && method != 3) return 0.0;
    const OeCircuit cir = oe_circuit(m);
    const uint64_t* n = m->n;
    double w2max = 0.0;
    auto sh = [](const int64_t q[3], int a, int64_t k, int64_t out[3]) {
        out[0] = q[0];
        out[1] = q[1];
        out[2] = q[2];
        out[a] += k;
    };
    for (int a = 0; a < 3; ++a) {
        for (uint64_t i = 0; i < n[0]; ++i)
            for (uint64_t j = 0; j < n[1]; ++j)
                for (uint64_t k = 0; k < n[2]; ++k) {
                    const int64_t q[3] = {(int64_t)i, (int64_t)j, (int64_t)k};
                    int64_t t0[3], t1[3];
                    if (method == 1) {
                        // gershgorin (timestep.rs:225-246).
                        if ((uint64_t)q[a] + 1 >= n[a]) continue;
                        const int b = (a + 1) % 3, c = (a + 2) % 3;
                        float s = 0.0f;
                        for (int t : {c, b}) {
                            const int o = 3 - a - t;
                            s += 1.0f / cir.L(o, q);
                            sh(q, t, -1, t0);
                            s += 1.0f / cir.L(o, t0);
                        }
                        w2max = std::max(w2max, (double)s / (double)cir.C(a, q));
                        continue;
                    }
                    // rennings (timestep.rs:248-287).
                    const int bs[2] = {(a + 1) % 3, (a + 2) % 3};
                    double tt[2];
                    float lm[2], l0[2];
                    for (int slot = 0; slot < 2; ++slot) {
                        const int b = bs[slot], c = 3 - a - b;
                        sh(q, b, -1, t0);
                        lm[slot] = cir.L(c, t0);
                        l0[slot] = cir.L(c, q);
                        float below;
                        if ((b + 3 - a) % 3 == 2) {
                            int64_t f[3];
                            sh(t0, c, -1, f);
                            const float lb = cir.L(c, f);
                            sh(q, c, -1, t1);
                            below = oe_x(cir.C(a, f), lb) + oe_x(cir.C(a, t1), lb);
                        } else {
                            below = oe_x(cir.C(a, t0), lm[slot]) + oe_x(cir.C(a, q), lm[slot]);
                        }
                        sh(q, b, 1, t1);
                        const float above = oe_x(cir.C(a, q), l0[slot]) + oe_x(cir.C(a, t1), l0[slot]);
                        tt[slot] = 0.25 * ((double)below + (double)above);
                    }
                    double own = 0.0;
                    for (int e = 0; e < 2; ++e) {
                        int64_t mm[3];
                        sh(q, a, e, mm);
                        const float c0 = cir.C(bs[0], mm), c1 = cir.C(bs[1], mm);
                        const double x0m = oe_x(c0, lm[0]), x00 = oe_x(c0, l0[0]);
                        const double x1m = oe_x(c1, lm[1]), x10 = oe_x(c1, l0[1]);
                        const double lc0 = 0.5 * (x0m + x00), dc0 = 0.5 * (x0m - x00);
                        const double lc1 = 0.5 * (x1m + x10), dc1 = 0.5 * (x1m - x10);
                        own += std::max(lc1 + std::fabs(dc0), lc0 + std::fabs(dc1));
                    }
                    w2max = std::max(w2max, tt[0] + tt[1] + 0.5 * own);
                }
    }
    if (method == 1) return (double)(1.0f / std::sqrt((float)w2max));
    return 1.0 / std::sqrt(w2max);
}

// compiler-rt's __powidf2: a^b by repeated squaring (the f64 powi of the
// reference's grading).
static double powi(double a, int b) {
    const bool recip = b < 0;
    double r = 1.0;
    for (;;) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? 1.0 / r : r;
}

// openems_pml_sigma (src/engine/boundary/upml.rs:143-150).
static double oe_pml_sigma(double depth, double width, uint64_t cells) {
    if (depth <= 0.0 || cells == 0 || width <= 0.0) return 0.0;
    const double dl = width / (double)cells;
    const double g = 2.5;
    return std::log(1e6) * std::log(g) / (2.0 * dl * Z0 * (powi(g, (int)cells) - 1.0)) * std::pow(g, depth / dl);
}

int ems_model_add_openems_pml(ems_model* m, const uint64_t cells[6]) {
    if (!m->built) return set_err(m, "build the model first"), -1;
    const uint64_t* n = m->n;
    const double dt = m->dt;
    // Profile::new (upml.rs:165-196): a = sigma*dt/(2 eps0) at the lines
    // and the cell midpoints, summed over the faces.
    std::vector<double> at_node[3], at_mid[3];
    for (int a = 0; a < 3; ++a) {
        at_node[a].assign(n[a], 0.0);
        at_mid[a].assign(n[a], 0.0);
    }
    bool any = false;
    for (int f = 0; f < 6; ++f) {
        const uint64_t c = cells[f];
        if (!c) continue;
        const int ax = f / 2;
        const bool is_max = f & 1;
        const uint64_t last = n[ax] - 1;
        if (c > last) return set_err(m, "PML thicker than the mesh"), -1;
        const std::vector<double>& l = m->lines[ax];
        const double inner = is_max ? l[last - c] : l[c], outer = is_max ? l[last] : l[0];
        const double width = std::fabs(outer - inner);
        auto a_of = [&](double x) {
            const double depth = is_max ? x - inner : inner - x;
            return oe_pml_sigma(depth, width, c) * dt / (2.0 * EPS0);
        };
        for (uint64_t k = 0; k <= last; ++k) {
            at_node[ax][k] += a_of(l[k]);
            if (k < last) at_mid[ax][k] += a_of(0.5 * (l[k] + l[k + 1]));
        }
        any = true;
    }
    if (!any) return set_err(m, "no PML face"), -1;
    const double OE_PML_EPS0 = 8.854187817620389e-12, OE_PML_MU0 = 1.256637062e-6;
    auto op = std::make_unique<OpStore>();
    op->kind = EMS_OP_UPML;
    // OpenEmsPml::build (upml.rs:660-724): E then H, component, node order.
    for (int side = 0; side < 2; ++side) {
        const bool e_side = side == 0;
        for (int comp = 0; comp < 3; ++comp) {
            const int p = next_axis(comp), q = prev_axis(comp);
            std::vector<float>& ca = m->co[(e_side ? 0 : 6) + comp];
            std::vector<float>& cb = m->co[(e_side ? 3 : 9) + comp];
            const std::vector<double>* own = e_side ? at_mid : at_node;
            const std::vector<double>* other = e_side ? at_node : at_mid;
            for (uint64_t i = 0; i < n[0]; ++i)
                for (uint64_t j = 0; j < n[1]; ++j)
                    for (uint64_t k = 0; k < n[2]; ++k) {
                        const uint64_t node[3] = {i, j, k};
                        const uint64_t idx = m->index(i, j, k);
                        if (cb[idx] == 0.0f) continue;  // PEC, padding or no edge
                        const double aa = own[comp][node[comp]], ap = other[p][node[p]], aq = other[q][node[q]];
                        if (aa == 0.0 && ap == 0.0 && aq == 0.0) continue;
                        double geo, mm;
                        if (e_side) {
                            geo = m->dual_delta(p, node[p]) * m->dual_delta(q, node[q]) / m->delta(comp, node[comp]);
                            double eps, kap;
                            edge_eps(m, comp, node, eps, kap);
                            mm = OE_PML_EPS0 * eps;
                        } else {
                            geo = m->delta(p, node[p]) * m->delta(q, node[q]) / m->dual_delta(comp, node[comp]);
                            double mu, sig;
                            edge_mu(m, comp, node, mu, sig);
                            mm = OE_PML_MU0 * mu;
                        }
                        ca[idx] = 0.0f;
                        cb[idx] = (float)(dt / ((1.0 + ap) * geo));
                        op->pax[side].push_back((uint8_t)comp);
                        op->pnode[side].push_back(idx);
                        op->pco[side].push_back((float)((1.0 - ap) / (1.0 + ap)));
                        op->pco[side].push_back((float)((1.0 - aq) / (1.0 + aq)));
                        op->pco[side].push_back((float)((1.0 + aa) / ((1.0 + aq) * mm)));
                        op->pco[side].push_back((float)((1.0 - aa) / ((1.0 + aq) * mm)));
                    }
        }
    }
    for (int side = 0; side < 2; ++side) {
        op->upml.n[side] = op->pnode[side].size();
        op->upml.axis[side] = op->pax[side].data();
        op->upml.node[side] = op->pnode[side].data();
        op->upml.co[side] = op->pco[side].data();
    }
    m->ops.push_back(std::move(op));
    m->refresh_desc();
    return (int)m->ops.size() - 1;
}

int ems_model_set_edge_circuit(ems_model* m, int axis, const uint64_t node[3], double cap, double cond) {
    if (!m->built) return set_err(m, "build the model first"), EMS_ERR_INVALID;
    if (axis < 0 || axis > 2) return set_err(m, "invalid axis"), EMS_ERR_INVALID;
    for (int a = 0; a < 3; ++a)
        if (node[a] >= m->n[a] || (a == axis && node[a] + 1 >= m->n[a]))
            return set_err(m, "edge outside the grid"), EMS_ERR_INVALID;
    // replace_medium (src/sim/map.rs:1525-1606): the element's C and 1/R
    // replace the medium's, each rounded like the model's circuit values;
    // e_coefficients (src/engine/coeffs.rs:395-410).
    const bool oe = m->oe_round;
    auto store = [oe](double x) { return oe ? (double)(float)x : x; };
    const int b = next_axis(axis), c = prev_axis(axis);
    double eps, kap;
    edge_eps(m, axis, node, eps, kap);
    const double geo = m->dual_delta(b, node[b]) * m->dual_delta(c, node[c]) / m->delta(axis, node[axis]);
    const double C = cap >= 0.0 ? store(cap) : store((oe ? OE_EPS0 : EPS0) * eps * geo);
    const double G = cond >= 0.0 ? store(cond) : store(kap * geo);
    if (!(C > 0.0 && std::isfinite(C) && G >= 0.0 && std::isfinite(G)))
        return set_err(m, "edge circuit must have C > 0 and G >= 0"), EMS_ERR_INVALID;
    const double dt = m->dt, den = C + 0.5 * G * dt;
    const uint64_t idx = m->index(node[0], node[1], node[2]);
    m->co[axis][idx] = (float)((C - 0.5 * G * dt) / den);
    m->co[3 + axis][idx] = (float)(dt / den);
    m->edge_cap[(uint64_t)axis * m->co[0].size() + idx] = C;
    return EMS_OK;
}

int ems_model_zero_edges(ems_model* m, int field, int axis, const uint64_t lo[3], const uint64_t hi[3]) {
    if (!m->built) return set_err(m, "build the model first"), EMS_ERR_INVALID;
    if ((field != 0 && field != 1) || axis < 0 || axis > 2) return set_err(m, "invalid field or axis"), EMS_ERR_INVALID;
    for (int a = 0; a < 3; ++a)
        if (lo[a] > hi[a] || hi[a] >= m->n[a]) return set_err(m, "box outside the grid"), EMS_ERR_INVALID;
    std::vector<float>& c0 = m->co[(field ? 6 : 0) + axis];
    std::vector<float>& c1 = m->co[(field ? 9 : 3) + axis];
    for (uint64_t i = lo[0]; i <= hi[0]; ++i)
        for (uint64_t j = lo[1]; j <= hi[1]; ++j)
            for (uint64_t k = lo[2]; k <= hi[2]; ++k) {
                const uint64_t idx = m->index(i, j, k);
                c0[idx] = 0.0f;
                c1[idx] = 0.0f;
            }
    return EMS_OK;
}

double ems_model_dt(const ems_model* m) { return m->dt; }
const float* ems_model_coeff(const ems_model* m, int lane) {
    if (!m->built || lane < 0 || lane > 11) return nullptr;
    return m->co[lane].data();
}

// Mean refractive index of a layer, layer_index (src/engine/boundary/cpml.rs:1056-1120).
static double layer_index(const ems_model* m, int face, uint64_t cells) {
    const int p = face / 2;
    const bool is_max = face % 2 == 1;
    const uint64_t np = m->n[p];
    const uint64_t inner = is_max ? np - 1 - cells : cells;
    const uint64_t l0 = is_max ? inner : 0, l1 = is_max ? np : inner + 1;  // lines
    const uint64_t c0 = is_max ? inner : 0, c1 = is_max ? np - 1 : inner;  // cells
    const double dt = m->dt;
    double we = 0.0, se = 0.0, wh = 0.0, sh = 0.0;
    const int comps[2] = {next_axis(p), prev_axis(p)};
    uint64_t lo[3] = {0, 0, 0}, hi[3] = {m->n[0], m->n[1], m->n[2]};
    lo[p] = std::min(l0, c0);
    hi[p] = std::max(l1, c1);
    for (int comp : comps) {
        const int a = comp, b = next_axis(comp), c = prev_axis(comp);
        for (uint64_t i = lo[0]; i < hi[0]; ++i)
            for (uint64_t j = lo[1]; j < hi[1]; ++j)
                for (uint64_t k = lo[2]; k < hi[2]; ++k) {
                    const uint64_t node[3] = {i, j, k};
                    const uint64_t idx = m->index(i, j, k);
                    const uint64_t along = node[p];
                    const float ca = m->co[a][idx], cb = m->co[3 + a][idx];
                    if (along >= l0 && along < l1 && node[a] + 1 < m->n[a] && cb != 0.0f) {
                        double area = m->dual_delta(b, node[b]) * m->dual_delta(c, node[c]);
                        double l = m->delta(a, node[a]);
                        double cap = dt * (1.0 + (double)ca) / (2.0 * (double)cb);
                        double vol = area * l;
                        we += vol;
                        se += vol * cap * l / (EPS0 * area);
                    }
                    const float da = m->co[6 + a][idx], db = m->co[9 + a][idx];
                    if (along >= c0 && along < c1 && node[b] + 1 < m->n[b] && node[c] + 1 < m->n[c] && db != 0.0f) {
                        double area = m->delta(b, node[b]) * m->delta(c, node[c]);
                        double l = m->dual_delta(a, node[a]);
                        double ind = dt * (1.0 + (double)da) / (2.0 * (double)db);
                        double vol = area * l;
                        wh += vol;
                        sh += vol * ind * l / (MU0 * area);
                    }
                }
    }
    double eps = we > 0.0 ? se / we : 1.0;
    double mu = wh > 0.0 ? sh / wh : 1.0;
    double n_r = std::sqrt(eps * mu);
    if (std::fabs(n_r - 1.0) < 1e-6 || !std::isfinite(n_r) || n_r <= 0.0) return 1.0;
    return n_r;
}

int ems_model_add_cpml(ems_model* m, const uint64_t cells[6], double grading, double sigma_factor, double kappa_max,
                       double alpha_max, int linear) {
    if (!m->built) return set_err(m, "build the model first"), -1;
    // Cpml::validate (src/fdtd.rs:275-295).
    if (!(std::isfinite(grading) && grading >= 0 && std::isfinite(sigma_factor) && sigma_factor >= 0 &&
          std::isfinite(kappa_max) && kappa_max >= 1 && std::isfinite(alpha_max) && alpha_max >= 0))
        return set_err(m, "invalid CPML parameters"), -1;
    for (int p = 0; p < 3; ++p) {
        if (cells[2 * p] > m->n[p] - 1 || cells[2 * p + 1] > m->n[p] - 1) return set_err(m, "CPML thicker than the mesh"), -1;
        if (cells[2 * p] + cells[2 * p + 1] > m->n[p] - 1) return set_err(m, "opposite CPML layers overlap"), -1;
    }
    auto op = std::make_unique<OpStore>();
    op->kind = EMS_OP_CPML;
    // CpmlBoundary::build + Layer::new (src/engine/boundary/cpml.rs:979-1035, 1122-1196).
    for (int face = 0; face < 6; ++face) {
        const uint64_t c = cells[face];
        if (c == 0) continue;
        const int p = face / 2;
        const bool is_max = face % 2 == 1;
        const uint64_t np = m->n[p];
        const double n_face = layer_index(m, face, c);
        op->index[face] = n_face;
        const uint64_t inner = is_max ? np - 1 - c : c;
        auto rho = [&](double x) { return std::min(1.0, std::max(0.0, std::fabs(x - (double)inner) / (double)c)); };
        std::vector<uint64_t> e_idx, h_idx;
        if (is_max) {
            for (uint64_t k = inner + 1; k < np; ++k) e_idx.push_back(k);
            for (uint64_t k = inner; k < np - 1; ++k) h_idx.push_back(k);
        } else {
            for (uint64_t k = 0; k < inner; ++k) e_idx.push_back(k);
            for (uint64_t k = 0; k < inner; ++k) h_idx.push_back(k);
        }
        auto node_delta = [&](uint64_t k) {
            bool has_lo = k > 0, has_hi = k + 1 < np;
            if (has_lo && has_hi) return 0.5 * (m->delta(p, k - 1) + m->delta(p, k));
            return has_lo ? m->delta(p, k - 1) : m->delta(p, k);
        };
        std::vector<float> eb, ea, ek, hb, ha, hk;
        for (uint64_t k : e_idx) {
            CpmlCo q = cpml_in_medium(grading, sigma_factor, kappa_max, alpha_max, linear != 0, rho((double)k),
                                      node_delta(k), m->dt, n_face);
            eb.push_back((float)q.b);
            ea.push_back((float)q.a);
            ek.push_back((float)q.direct);
        }
        for (uint64_t k : h_idx) {
            CpmlCo q = cpml_in_medium(grading, sigma_factor, kappa_max, alpha_max, linear != 0, rho((double)k + 0.5),
                                      m->delta(p, k), m->dt, n_face);
            hb.push_back((float)q.b);
            ha.push_back((float)q.a);
            hk.push_back((float)q.direct);
        }
        const int a1 = next_axis(p), a2 = prev_axis(p);
        auto slab = [&](int comp, bool e_side) {
            ems_cpml_slab s{};
            s.e_side = e_side ? 1 : 0;
            s.comp = comp;
            s.normal = p;
            // Slab::new (src/engine/boundary/cpml.rs:412-437).
            if (p == next_axis(comp)) {
                s.sign = 1.0f;
                s.other = prev_axis(comp);
            } else {
                s.sign = -1.0f;
                s.other = next_axis(comp);
            }
            for (int t = 0; t < 3; ++t) {
                s.lo[t] = 0;
                s.hi[t] = m->n[t];
            }
            const auto& idx = e_side ? e_idx : h_idx;
            if (e_side) {
                s.hi[comp] = m->n[comp] - 1;
            } else {
                int o = comp == a1 ? a2 : a1;
                s.hi[o] = m->n[o] - 1;
            }
            s.lo[p] = idx.empty() ? 0 : idx.front();
            s.hi[p] = idx.empty() ? 0 : idx.back() + 1;
            op->arrays.push_back(e_side ? eb : hb);
            op->arrays.push_back(e_side ? ea : ha);
            op->arrays.push_back(e_side ? ek : hk);
            op->slabs.push_back(s);
        };
        slab(a1, true);
        slab(a2, true);
        slab(a1, false);
        slab(a2, false);
    }
    for (size_t s = 0; s < op->slabs.size(); ++s) {
        op->slabs[s].b = op->arrays[3 * s].data();
        op->slabs[s].a = op->arrays[3 * s + 1].data();
        op->slabs[s].k = op->arrays[3 * s + 2].data();
    }
    op->cpml.n_slabs = op->slabs.size();
    op->cpml.slabs = op->slabs.data();
    m->ops.push_back(std::move(op));
    m->refresh_desc();
    return (int)m->ops.size() - 1;
}

double ems_model_cpml_index(const ems_model* m, int face) {
    for (auto& o : m->ops)
        if (o->kind == EMS_OP_CPML && face >= 0 && face < 6) return o->index[face];
    return 0.0;
}

ems_dispersive* ems_dispersive_new(void) { return new ems_dispersive(); }
void ems_dispersive_free(ems_dispersive* d) { delete d; }

int ems_dispersive_fill(ems_dispersive* d, const ems_model* m, const ems_cellset* s, int field, size_t n_poles,
                        const int* kind, const double* p1, const double* p2, const double* p3) {
    std::vector<Pole> poles;
    for (size_t q = 0; q < n_poles; ++q) {
        Pole p{kind[q], p1[q], p2 ? p2[q] : 0.0, p3 ? p3[q] : 0.0};
        // Pole::validate (src/engine/dispersive.rs:339-358).
        double v[3] = {p.p1, p.p2, p.kind == 0 ? p.p3 : 0.0};
        for (double x : v)
            if (!(std::isfinite(x) && x >= 0.0)) return EMS_ERR_INVALID;
        if (p.kind < 0 || p.kind > 2) return EMS_ERR_INVALID;
        poles.push_back(p);
    }
    if (!s->any || poles.empty()) return EMS_OK;
    // Dispersive::fill_cells (src/engine/dispersive.rs:1896-1985) with the
    // box test replaced by the cell set's membership; edges touching the
    // set's bounding box, in the reference's axis / node order.
    for (int axis = 0; axis < 3; ++axis) {
        const int a = axis, b = next_axis(axis), c = prev_axis(axis);
        uint64_t lo[3], hi[3];
        for (int t = 0; t < 3; ++t) {
            bool along = field == 0 ? t == a : t != a;
            lo[t] = s->lo[t];
            hi[t] = along ? s->hi[t] : std::min(s->hi[t] + 1, m->n[t]);
        }
        uint64_t node[3];
        for (node[a] = lo[a]; node[a] < hi[a]; ++node[a])
            for (node[b] = lo[b]; node[b] < hi[b]; ++node[b])
                for (node[c] = lo[c]; node[c] < hi[c]; ++node[c]) {
                    double share;
                    if (field == 0) {
                        double w_in = 0.0, w = 0.0;
                        for (int db = -1; db <= 0; ++db) {
                            if (node[b] == 0 && db < 0) continue;
                            uint64_t cb = node[b] + db;
                            if (cb >= m->n[b] - 1) continue;
                            for (int dc = -1; dc <= 0; ++dc) {
                                if (node[c] == 0 && dc < 0) continue;
                                uint64_t cc = node[c] + dc;
                                if (cc >= m->n[c] - 1) continue;
                                double area = m->delta(b, cb) * m->delta(c, cc);
                                w += area;
                                uint64_t q[3];
                                q[a] = node[a];
                                q[b] = cb;
                                q[c] = cc;
                                if (s->at(q[0], q[1], q[2])) w_in += area;
                            }
                        }
                        share = w > 0.0 ? w_in / w : 0.0;
                    } else {
                        if (node[b] + 1 >= m->n[b] || node[c] + 1 >= m->n[c]) continue;
                        double w_in = 0.0, w = 0.0;
                        for (int da = -1; da <= 0; ++da) {
                            if (node[a] == 0 && da < 0) continue;
                            uint64_t ca = node[a] + da;
                            if (ca >= m->n[a] - 1) continue;
                            double len = m->delta(a, ca);
                            w += len;
                            uint64_t q[3] = {node[0], node[1], node[2]};
                            q[a] = ca;
                            if (s->at(q[0], q[1], q[2])) w_in += len;
                        }
                        share = w > 0.0 ? w_in / w : 0.0;
                    }
                    if (share > 0.0)
                        for (const Pole& p : poles) {
                            Pole q = p.scaled(share);
                            if (q.p1 == 0.0) continue;  // Pole::is_null
                            d->entries.push_back(Entry{field, axis, {node[0], node[1], node[2]}, q});
                        }
                }
    }
    return EMS_OK;
}

int ems_dispersive_add_edge(ems_dispersive* d, int field, int axis, const uint64_t node[3], int kind, double p1,
                            double p2, double p3) {
    if ((field != 0 && field != 1) || axis < 0 || axis > 2 || kind < 0 || kind > 3) return EMS_ERR_INVALID;
    const double v[3] = {p1, p2, kind == 0 ? p3 : 0.0};
    for (double x : v)
        if (!(std::isfinite(x) && x >= 0.0)) return EMS_ERR_INVALID;
    if (kind == 3 && (field != 0 || !(p1 > 0.0))) return EMS_ERR_INVALID;  // a branch: L > 0, R >= 0, E edges
    if (p1 == 0.0) return EMS_OK;  // Pole::is_null
    d->entries.push_back(Entry{field, axis, {node[0], node[1], node[2]}, Pole{kind, p1, p2, p3}});
    return EMS_OK;
}

int ems_model_edge_material(const ems_model* m, int field, int axis, const uint64_t node[3], double out[2]) {
    if ((field != 0 && field != 1) || axis < 0 || axis > 2) return EMS_ERR_INVALID;
    for (int a = 0; a < 3; ++a)
        if (node[a] >= m->n[a]) return EMS_ERR_INVALID;
    if (field == 0) edge_eps(m, axis, node, out[0], out[1]);
    else edge_mu(m, axis, node, out[0], out[1]);
    return EMS_OK;
}

int ems_model_add_dispersive(ems_model* m, ems_dispersive* d, int scheme) {
    if (!m->built) return set_err(m, "build the model first"), -1;
    if (scheme < 0 || scheme > 2) return set_err(m, "unknown pole scheme"), -1;
    for (const Entry& e : d->entries) {
        bool exists = e.node[0] < m->n[0] && e.node[1] < m->n[1] && e.node[2] < m->n[2];
        int a = e.axis, b = next_axis(a), c = prev_axis(a);
        exists = exists && (e.field == 0 ? e.node[a] + 1 < m->n[a] : (e.node[b] + 1 < m->n[b] && e.node[c] + 1 < m->n[c]));
        if (!exists) return set_err(m, "dispersive edge outside the grid"), -1;
    }
    // Dispersive::install (src/engine/dispersive.rs:2054-2300): entries in
    // edge order (stable: an edge keeps its insertion order), branch
    // constants from the pole and the edge geometry.
    std::vector<uint32_t> order(d->entries.size());
    for (size_t q = 0; q < order.size(); ++q) order[q] = (uint32_t)q;
    auto key = [&](uint32_t q) {
        const Entry& e = d->entries[q];
        return std::make_tuple(e.node[0], e.field, e.axis, e.node[1], e.node[2]);
    };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return key(x) < key(y); });
    if (scheme == 2) {
        // openEMS's poles come first on their edge (src/engine/dispersive.rs:
        // 2195-2215: the OpenEmsPole list precedes the other entries).
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
            const int ox = d->entries[x].pole.kind == 2, oy = d->entries[y].pole.kind == 2;
            return std::make_tuple(key(x), ox) < std::make_tuple(key(y), oy);
        });
    }
    // Per edge (scheme 2): whether all of its poles are Debye poles, for
    // openEMS's Debye update (with_openems_debye, electric edges only).
    std::vector<char> all_debye(order.size(), 0);
    if (scheme == 2)
        for (size_t s0 = 0; s0 < order.size();) {
            size_t s1 = s0;
            bool deb = d->entries[order[s0]].field == 0;
            while (s1 < order.size() && key(order[s1]) == key(order[s0])) {
                deb = deb && d->entries[order[s1]].pole.kind == 2;
                ++s1;
            }
            for (size_t t = s0; t < s1; ++t) all_debye[t] = deb;
            s0 = s1;
        }
    auto op = std::make_unique<OpStore>();
    op->kind = EMS_OP_POLES;
    const double dt = m->dt;
    bool have_last = false;
    std::tuple<uint64_t, int, int, uint64_t, uint64_t> last;
    bool skip_edge = false;
    double debye_f = 0.0;  // openEMS Debye edge: F of the edge's poles
    for (size_t oi = 0; oi < order.size(); ++oi) {
        const uint32_t q = order[oi];
        const Entry& e = d->entries[q];
        auto k = key(q);
        const bool new_edge = !have_last || last != k;
        last = k;
        have_last = true;
        const int a = e.axis, b = next_axis(a), c = prev_axis(a);
        const uint64_t idx = m->index(e.node[0], e.node[1], e.node[2]);
        double geo, x0;
        float coef;
        if (e.field == 0) {
            coef = m->co[3 + a][idx];
            x0 = EPS0;
            geo = m->dual_delta(b, e.node[b]) * m->dual_delta(c, e.node[c]) / m->delta(a, e.node[a]);
        } else {
            coef = m->co[9 + a][idx];
            x0 = MU0;
            geo = m->delta(b, e.node[b]) * m->delta(c, e.node[c]) / m->dual_delta(a, e.node[a]);
        }
        const double mm = x0 * geo;
        if (new_edge) skip_edge = coef == 0.0f;
        if (skip_edge) continue;
        OpStore::Side& side = e.field == 0 ? op->pe : op->ph;
        if (new_edge) {
            side.axis.push_back((uint8_t)a);
            side.node.push_back(idx);
            side.sum_inv_z.push_back(0.0);
            side.pole_end.push_back(side.pole_end.empty() ? 0 : side.pole_end.back());
        }
        const Pole& p = e.pole;
        if (scheme == 2 && all_debye[oi]) {
            // openems_debye_coefficients (src/engine/dispersive.rs:900-928):
            // beta_p = cb·cp·de_p/(2·tau_p + dt) with cp = eps0·A*/l
            // (openEMS's eps0), F = f32(1/(1 + sum beta)) over the edge.
            const double cp = OE_EPS0 * geo;
            auto beta = [&](const Pole& x) { return (double)coef * cp * x.p1 / (2.0 * x.p2 + dt); };
            if (new_edge) {
                double sum = 0.0;
                for (size_t t = oi; t < order.size() && key(order[t]) == k; ++t) sum += beta(d->entries[order[t]].pole);
                debye_f = (double)(float)(1.0 / (1.0 + sum));
            }
            side.kind.push_back(EMS_POLE_OPENEMS_DEBYE);
            side.a.push_back(debye_f);
            side.inv_c.push_back((double)(float)(1.0 - dt / (p.p2 + 0.5 * dt)));
            side.inv_z.push_back((double)(float)beta(p));
            side.half_l.push_back(0.0);
            side.pole_end.back() += 1;
            continue;
        }
        if (p.kind == 3) {
            // An openEMS conducting-sheet branch of inductance L = p1 and
            // resistance R = p2 (src/engine/openems_sheet.rs:56-80): the
            // f32 state x = cb·j with x <- ka·x + kb·u^n before the E update
            // and u <- u − x after it, ka = f32((L/dt − R/2)/(L/dt + R/2)),
            // kb = f32(cb/(L/dt + R/2)) with the edge's f32 coefficient cb:
            // an openEMS pole step with K = 0. It adds no energy.
            if (scheme != 2) return set_err(m, "conducting-sheet branches need the openEMS pole scheme"), -1;
            const double den = p.p1 / dt + 0.5 * p.p2;
            side.kind.push_back(EMS_POLE_OPENEMS);
            side.a.push_back((double)(float)((p.p1 / dt - 0.5 * p.p2) / den));
            side.inv_c.push_back(0.0);
            side.inv_z.push_back((double)(float)((double)coef / den));
            side.half_l.push_back(0.0);
            side.pole_end.back() += 1;
            continue;
        }
        if (scheme == 2 && p.kind != 2) {
            // OpenEmsPole::coefficients (src/engine/dispersive.rs:888-899):
            // omega_p as given (the material's 2·pi·f_plasma), the edge's
            // f32 coefficient vi and its f32 capacitance (inductance) with
            // openEMS's vacuum constants (e_edge_circuit / h_edge_inductance,
            // src/engine/coeffs.rs:776-810).
            double circuit;
            if (e.field == 0) {
                // The edge's capacitance: a parallel R/C lumped element folded
                // into it replaced the medium's (openEMS forms the poles from
                // the edge with the element folded in).
                const auto it = m->edge_cap.find((uint64_t)a * m->co[0].size() + idx);
                double eps, kap;
                edge_eps(m, a, e.node, eps, kap);
                circuit = it != m->edge_cap.end() ? it->second : (double)(float)(OE_EPS0 * eps * geo);
            } else {
                double mu, sig;
                edge_mu(m, a, e.node, mu, sig);
                circuit = (double)(float)(OE_MU0 * mu * geo);
            }
            const double vi = (double)coef;
            const double w0 = p.kind == 0 ? p.p2 : 0.0, gamma = p.kind == 0 ? p.p3 : p.p2;
            const double half = gamma * dt / 2.0, dd = 1.0 + half, wp2 = p.p1 * p.p1;
            side.kind.push_back(EMS_POLE_OPENEMS);
            side.a.push_back((double)(float)((1.0 - half) / dd));
            side.inv_c.push_back((double)(float)(w0 * w0 * dt / (wp2 * circuit * vi)));
            side.inv_z.push_back((double)(float)(vi * dt * wp2 * circuit / dd));
            side.half_l.push_back(0.0);
            side.pole_end.back() += 1;
            continue;
        }
        double l = 0.0, r = 0.0, inv_c = 0.0;
        if (p.kind == 0) {  // Lorentz
            l = 1.0 / (mm * p.p1 * p.p1);
            r = p.p3 * l;
            inv_c = p.p2 * p.p2 * l;
        } else if (p.kind == 1) {  // Drude (omega_p, gamma)
            l = 1.0 / (mm * p.p1 * p.p1);
            r = p.p2 * l;
            inv_c = 0.0;
        }
        if (scheme == 1 && p.kind != 2) {
            // Pole::leapfrog (src/engine/dispersive.rs:391-407).
            double dd = l / dt + 0.5 * r;
            side.kind.push_back(EMS_POLE_LEAPFROG);
            side.a.push_back((l / dt - 0.5 * r) / dd);
            side.inv_c.push_back(inv_c);
            side.inv_z.push_back(1.0 / dd);
            side.half_l.push_back(0.5 * l);
        } else {
            // Pole::branch (src/engine/dispersive.rs:361-384).
            if (p.kind == 2) {
                double cc = mm * p.p1;
                l = 0.0;
                r = p.p2 / cc;
                inv_c = 1.0 / cc;
            }
            double aa = 2.0 * l / dt;
            double z = aa + r + 0.5 * dt * inv_c;
            double inv_z = 1.0 / z;
            side.kind.push_back(EMS_POLE_TRAPEZOIDAL);
            side.a.push_back(aa);
            side.inv_c.push_back(inv_c);
            side.inv_z.push_back(inv_z);
            side.half_l.push_back(0.25 * aa * dt);
            side.sum_inv_z.back() += inv_z;
        }
        side.pole_end.back() += 1;
    }
    op->pe.fill(op->poles.electric);
    op->ph.fill(op->poles.magnetic);
    m->ops.push_back(std::move(op));
    m->refresh_desc();
    return (int)m->ops.size() - 1;
}

int ems_model_add_lumped(ems_model* m, int axis, const uint64_t lo[3], const uint64_t hi[3], double r, double l,
                         double c, int series_topology, int record, int port, const double* amp, uint64_t n_amp) {
    if (!m->built) return set_err(m, "build the model first"), -1;
    if (axis < 0 || axis > 2) return set_err(m, "invalid lumped element axis"), -1;
    // LumpedElement::validate (src/engine/lumped.rs:700-760): values finite
    // and > 0 where present (<= 0 here means absent), at least one of them,
    // a source on a parallel element only with a resistor.
    const bool has_r = r > 0.0, has_l = l > 0.0, has_c = c > 0.0;
    for (double v : {r, l, c})
        if (!(v <= 0.0) && !(std::isfinite(v) && v > 0.0)) return set_err(m, "invalid lumped value"), -1;
    if (!(has_r || has_l || has_c)) return set_err(m, "lumped element needs at least one of R, L, C"), -1;
    const bool has_src = amp != nullptr && n_amp > 0;
    if (has_src && !series_topology && !has_r) return set_err(m, "a source on a parallel lumped element needs a resistance"), -1;
    if (port && !(has_r && !has_l && !has_c && !series_topology)) return set_err(m, "a lumped port is a resistor"), -1;
    // LumpedBox::new / check_fits (src/engine/lumped.rs:145-215).
    for (int t = 0; t < 3; ++t)
        if (lo[t] > hi[t] || hi[t] >= m->n[t]) return set_err(m, "lumped box outside the grid"), -1;
    if (lo[axis] >= hi[axis]) return set_err(m, "lumped box degenerate along its axis"), -1;
    const int a = axis, b = next_axis(axis), cc = prev_axis(axis);
    std::vector<uint64_t> edges;
    for (uint64_t pb = lo[b]; pb <= hi[b]; ++pb)
        for (uint64_t pc = lo[cc]; pc <= hi[cc]; ++pc)
            for (uint64_t pa = lo[a]; pa < hi[a]; ++pa) {
                uint64_t p[3];
                p[a] = pa;
                p[b] = pb;
                p[cc] = pc;
                edges.push_back(m->index(p[0], p[1], p[2]));
            }
    for (uint64_t e : edges)
        if (m->co[3 + a][e] == 0.0f) return set_err(m, "lumped element edge is PEC"), -1;
    // edge_parts for a box (src/engine/lumped.rs:820-860): Z_e = N·Z/M, so
    // g_e = M/(N·R), C_e = M·C/N, L_e = N·L/M, R_e = N·R/M.
    const double mm = (double)(hi[a] - lo[a]);
    const double nn = (double)((hi[b] - lo[b] + 1) * (hi[cc] - lo[cc] + 1));
    const bool has_branch = series_topology ? (has_l || has_c) : has_l;
    const double inf = std::numeric_limits<double>::infinity();
    double g_e = 0.0, c_e = 0.0, br_r = 0.0, br_l = 0.0, br_c = inf;
    if (!series_topology) {
        g_e = has_r ? mm / (nn * r) : 0.0;
        c_e = has_c ? mm * c / nn : 0.0;
        br_l = has_l ? nn * l / mm : 0.0;
    } else if (!has_branch) {
        g_e = has_r ? mm / (nn * r) : 0.0;
    } else {
        br_r = has_r ? nn * r / mm : 0.0;
        br_l = has_l ? nn * l / mm : 0.0;
        br_c = has_c ? mm * c / nn : inf;
    }
    const double dt = m->dt;
    auto op = std::make_unique<OpStore>();
    op->kind = EMS_OP_LUMPED;
    const bool src_in_branch = has_branch && series_topology;
    for (uint64_t e : edges) {
        // fold_parallel (src/engine/lumped.rs:275-282).
        if (g_e != 0.0 || c_e != 0.0) {
            double ca = (double)m->co[a][e], cb = (double)m->co[3 + a][e];
            double cap = dt * (1.0 + ca) / (2.0 * cb) + c_e;
            double cond = (1.0 - ca) / cb + g_e;
            double den = cap + 0.5 * cond * dt;
            m->co[a][e] = (float)((cap - 0.5 * cond * dt) / den);
            m->co[3 + a][e] = (float)(dt / den);
        }
        op->lnode.push_back(e);
        op->lcb.push_back((double)m->co[3 + a][e]);
        op->lg.push_back(src_in_branch ? 0.0 : g_e);
        op->lw.push_back(1.0 / mm);
        op->lrg.push_back(g_e);
        op->lrc.push_back(c_e);
        if (has_branch) {
            // The branch constants of install (src/engine/lumped.rs:960-970).
            const double inv_c = std::isfinite(br_c) ? 1.0 / br_c : 0.0;
            op->ltl.push_back(2.0 * br_l / dt);
            op->linvc.push_back(inv_c);
            op->lz.push_back(2.0 * br_l / dt + br_r + 0.5 * dt * inv_c);
        }
    }
    if (has_src) op->lamp.assign(amp, amp + n_amp);
    ems_lumped& L = op->lumped;
    L.axis = a;
    L.n_edges = edges.size();
    L.node = op->lnode.data();
    L.cb = op->lcb.data();
    L.g_src = op->lg.data();
    L.series = hi[a] - lo[a];
    L.src_in_branch = src_in_branch ? 1 : 0;
    L.src_w = has_src ? op->lw.data() : nullptr;
    L.n_src_amp = op->lamp.size();
    L.src_amp = op->lamp.empty() ? nullptr : op->lamp.data();
    L.has_branch = has_branch ? 1 : 0;
    L.two_l_dt = has_branch ? op->ltl.data() : nullptr;
    L.inv_c = has_branch ? op->linvc.data() : nullptr;
    L.z = has_branch ? op->lz.data() : nullptr;
    L.record = (record || port) ? 1 : 0;
    L.rec_g = op->lrg.data();
    L.rec_c = op->lrc.data();
    L.port_columns = port ? (uint64_t)nn : 0;
    m->ops.push_back(std::move(op));
    m->refresh_desc();
    return (int)m->ops.size() - 1;
}

int ems_model_add_lumped_openems(ems_model* m, int axis, const uint64_t lo[3], const uint64_t hi[3], double r,
                                 double l, double c, int series_topology, double omega, int explicit_inductor,
                                 const double* src_w, const double* amp, uint64_t n_amp) {
    if (!m->built || !m->oe_round) return set_err(m, "build the model with openEMS's rounding first"), -1;
    if (axis < 0 || axis > 2) return set_err(m, "invalid lumped element axis"), -1;
    const bool has_r = r > 0.0, has_l = l > 0.0, has_c = c > 0.0;
    for (double v : {r, l, c})
        if (!(v <= 0.0) && !(std::isfinite(v) && v > 0.0)) return set_err(m, "invalid lumped value"), -1;
    if (!(has_l || series_topology)) return set_err(m, "an element with an inductor or in series"), -1;
    const bool has_src = src_w != nullptr && amp != nullptr && n_amp > 0;
    if (has_src && (series_topology || !has_r)) return set_err(m, "the element's source needs a parallel resistor"), -1;
    for (int t = 0; t < 3; ++t)
        if (lo[t] > hi[t] || hi[t] >= m->n[t]) return set_err(m, "lumped box outside the grid"), -1;
    if (lo[axis] >= hi[axis]) return set_err(m, "lumped box degenerate along its axis"), -1;
    const int a = axis, b = next_axis(axis), cc = prev_axis(axis);
    std::vector<uint64_t> edges;
    std::vector<std::array<uint64_t, 3>> pos;
    for (uint64_t pb = lo[b]; pb <= hi[b]; ++pb)
        for (uint64_t pc = lo[cc]; pc <= hi[cc]; ++pc)
            for (uint64_t pa = lo[a]; pa < hi[a]; ++pa) {
                std::array<uint64_t, 3> p{};
                p[a] = pa;
                p[b] = pb;
                p[cc] = pc;
                edges.push_back(m->index(p[0], p[1], p[2]));
                pos.push_back(p);
            }
    for (uint64_t e : edges)
        if (m->co[3 + a][e] == 0.0f) return set_err(m, "lumped element edge is PEC"), -1;
    // csx's equal parts per edge (src/sim/map.rs:198-205): R·p/s, L·p/s,
    // C·s/p with p edges in parallel and s in series.
    const double s_n = (double)(hi[a] - lo[a]);
    const double p_n = (double)((hi[b] - lo[b] + 1) * (hi[cc] - lo[cc] + 1));
    const double r_e = has_r ? r * p_n / s_n : 0.0, l_e = has_l ? l * p_n / s_n : 0.0;
    const double c_e = has_c ? c * s_n / p_n : 0.0;
    const bool series = series_topology != 0;
    const double dt = m->dt, inf = std::numeric_limits<double>::infinity();
    auto store = [](double x) { return (double)(float)x; };
    // capacitance_limit (src/sim/map.rs:1608-1632).
    double limit = inf;
    if (omega > 0.0 && std::isfinite(omega)) {
        if (!series) {
            if (has_r) limit = std::min(limit, 1.0 / (20.0 * omega * r_e));
            if (has_l) limit = std::min(limit, 1.0 / (20.0 * omega * omega * l_e));
        } else {
            const double x = (has_l ? omega * l_e : 0.0) - (has_c ? 1.0 / (omega * c_e) : 0.0);
            const double z = std::hypot(has_r ? r_e : 0.0, x);
            if (z > 0.0) limit = 1.0 / (20.0 * omega * z);
        }
    }
    auto op = std::make_unique<OpStore>();
    op->kind = EMS_OP_LUMPED;
    std::vector<double> den(edges.size());
    for (size_t q = 0; q < edges.size(); ++q) {
        // replace_medium (src/sim/map.rs:1525-1606): the element's C and 1/R
        // replace the medium's, the capacitance limited at omega.
        const uint64_t i = edges[q];
        const float fa = m->co[a][i], fb = m->co[3 + a][i];
        const double ca = fa, cb = fb;
        if ((!series && !has_c && !has_r && !(omega > 0.0)) || !std::isfinite(cb)) {
            den[q] = dt * (1.0 + ca) / (2.0 * cb);
            continue;
        }
        double eps, kap;
        edge_eps(m, a, pos[q].data(), eps, kap);
        const double geo = m->dual_delta(b, pos[q][b]) * m->dual_delta(cc, pos[q][cc]) / m->delta(a, pos[q][a]);
        double cap = store(OE_EPS0 * eps * geo), cond = store(kap * geo);
        const double dd = cap + 0.5 * cond * dt;
        if (!((float)((cap - 0.5 * cond * dt) / dd) == fa && (float)(dt / dd) == fb)) {
            cap = dt * (1.0 + ca) / (2.0 * cb);
            cond = (1.0 - ca) / cb;
        }
        if (!series && has_c) cap = store(c_e);
        if (series) cond = 0.0;
        if (!series && has_r) cond = store(1.0 / r_e);
        double c_own = (!series && has_c) ? c_e : cap;
        if (cap > limit) {
            cap = store(limit);
            c_own = limit;
        }
        const double d2 = cap + 0.5 * cond * dt;
        m->co[a][i] = (float)((cap - 0.5 * cond * dt) / d2);
        m->co[3 + a][i] = (float)(dt / d2);
        den[q] = c_own + ((!series && has_r) ? 0.5 * (dt / r_e) : 0.0);
    }
    // install (src/engine/lumped.rs:880-1000) with the medium folded: the
    // branch (r, l, c) of a series element, (0, l, inf) of a parallel one;
    // openEMS's order; its explicit inductor for a parallel one.
    const double br_r = series && has_r ? r_e : 0.0, br_l = has_l ? l_e : 0.0;
    const double br_c = series && has_c ? c_e : inf;
    const double g_e = (!series && has_r) ? 1.0 / r_e : 0.0;
    // openEMS's explicit inductor is stable while dt²/(L_e·C_e) = dt·cb/L_e
    // stays at most 1 on every edge; beyond, the trapezoidal branch
    // (src/sim/map.rs:928-958).
    double worst = 0.0;
    for (uint64_t e : edges) worst = std::max(worst, dt * (double)m->co[3 + a][e] / l_e);
    const bool oe = explicit_inductor && !series && has_l && worst <= 1.0;
    for (size_t q = 0; q < edges.size(); ++q) {
        const uint64_t e = edges[q];
        op->lnode.push_back(e);
        op->lcb.push_back((double)m->co[3 + a][e]);
        op->lg.push_back(series ? 0.0 : g_e);
        op->lw.push_back(has_src ? src_w[q] : 0.0);
        op->lrg.push_back(g_e);
        op->lrc.push_back(!series ? c_e : 0.0);
        const double inv_c = std::isfinite(br_c) ? 1.0 / br_c : 0.0;
        op->ltl.push_back(2.0 * br_l / dt);
        op->linvc.push_back(inv_c);
        op->lz.push_back(2.0 * br_l / dt + br_r + 0.5 * dt * inv_c);
        if (oe) {
            op->loek.push_back((float)(dt / br_l) * (float)(dt / den[q]));
            op->loevi.push_back(dt / den[q]);
        }
    }
    if (has_src) op->lamp.assign(amp, amp + n_amp);
    ems_lumped& L = op->lumped;
    L.axis = a;
    L.n_edges = edges.size();
    L.node = op->lnode.data();
    L.cb = op->lcb.data();
    L.g_src = op->lg.data();
    L.series = hi[a] - lo[a];
    L.src_in_branch = series ? 1 : 0;
    L.src_w = has_src ? op->lw.data() : nullptr;
    L.n_src_amp = op->lamp.size();
    L.src_amp = op->lamp.empty() ? nullptr : op->lamp.data();
    L.has_branch = 1;
    L.two_l_dt = op->ltl.data();
    L.inv_c = op->linvc.data();
    L.z = op->lz.data();
    L.record = 0;
    L.rec_g = op->lrg.data();
    L.rec_c = op->lrc.data();
    L.port_columns = 0;
    L.openems_order = 1;
    L.oe_k = oe ? op->loek.data() : nullptr;
    L.oe_vi = oe ? op->loevi.data() : nullptr;
    m->ops.push_back(std::move(op));
    m->refresh_desc();
    return (int)m->ops.size() - 1;
}

int ems_model_add_lumped_port(ems_model* m, int axis, const uint64_t lo[3], const uint64_t hi[3], double r, int wave,
                              double f0, double fc, double amplitude, uint64_t n_steps) {
    if (!m->built) return set_err(m, "build the model first"), -1;
    if (axis < 0 || axis > 2 || !(r > 0.0) || !std::isfinite(r)) return set_err(m, "invalid lumped port"), -1;
    // LumpedPort::new(region, r).excite_waveform(w, amplitude): a recorded
    // resistor whose Thevenin source is amplitude·w(t) at (n + 1/2)·dt
    // (src/engine/port.rs:102-155, src/engine/lumped.rs:1136-1148).
    std::vector<double> amps;
    for (uint64_t s = 0; s < n_steps; ++s)
        amps.push_back(amplitude * ems_waveform_value(wave, f0, fc, ((double)s + 0.5) * m->dt, m->dt));
    return ems_model_add_lumped(m, axis, lo, hi, r, 0.0, 0.0, 0, 1, 1, amps.data(), amps.size());
}

int ems_model_add_source(ems_model* m, int kind, size_t n, const int* axis, const uint64_t* nodes, const double* weight,
                         int wave, double f0, double fc, uint64_t n_steps) {
    if (!m->built) return set_err(m, "build the model first"), -1;
    if (kind < 0 || kind > 3) return set_err(m, "invalid source kind"), -1;
    auto op = std::make_unique<OpStore>();
    op->kind = EMS_OP_SOURCE;
    for (size_t e = 0; e < n; ++e) {
        const uint64_t* p = nodes + 3 * e;
        if (axis[e] < 0 || axis[e] > 2 || p[0] >= m->n[0] || p[1] >= m->n[1] || p[2] >= m->n[2])
            return set_err(m, "source edge outside the grid"), -1;
        op->axis.push_back((uint8_t)axis[e]);
        op->node.push_back(m->index(p[0], p[1], p[2]));
        op->fw.push_back((float)weight[e]);
    }
    const double dt = m->dt;
    // Sample time of each kind (src/engine/excite.rs:104-173).
    for (uint64_t s = 0; s < n_steps; ++s) {
        double t = kind == EMS_SOFT_E ? ((double)s + 0.5) * dt
                   : kind == EMS_HARD_E ? ((double)s + 1.0) * dt
                   : kind == EMS_SOFT_H ? (double)s * dt
                                        : ((double)s + 0.5) * dt;
        op->famp.push_back((float)ems_waveform_value(wave, f0, fc, t, dt));
    }
    ems_source& S = op->source;
    S.kind = kind;
    S.n_edges = n;
    S.axis = op->axis.data();
    S.node = op->node.data();
    S.weight = op->fw.data();
    S.n_amp = op->famp.size();
    S.amp = op->famp.data();
    m->ops.push_back(std::move(op));
    m->refresh_desc();
    return (int)m->ops.size() - 1;
}

int ems_model_add_source_table(ems_model* m, int kind, size_t n, const int* axis, const uint64_t* nodes,
                               const double* weight, const double* amp, uint64_t n_steps) {
    if (!amp && n_steps) return set_err(m, "missing amplitude table"), -1;
    int k = ems_model_add_source(m, kind, n, axis, nodes, weight, -1, 0.0, 0.0, 0);
    if (k < 0) return k;
    OpStore& op = *m->ops[(size_t)k];
    // EdgeSource::apply: amplitude(t) as f32 (src/engine/excite.rs:104-106).
    op.famp.resize(n_steps);
    for (uint64_t s = 0; s < n_steps; ++s) op.famp[s] = (float)amp[s];
    op.source.n_amp = op.famp.size();
    op.source.amp = op.famp.data();
    m->refresh_desc();
    return k;
}

int ems_model_add_probe(ems_model* m, int quantity, size_t n, const int* axis, const uint64_t* nodes,
                        const double* weight, uint64_t interval) {
    if (quantity < 0 || quantity > 1) return set_err(m, "invalid probe quantity"), -1;
    auto op = std::make_unique<OpStore>();
    op->kind = EMS_OP_PROBE;
    for (size_t e = 0; e < n; ++e) {
        const uint64_t* p = nodes + 3 * e;
        if (axis[e] < 0 || axis[e] > 2 || p[0] >= m->n[0] || p[1] >= m->n[1] || p[2] >= m->n[2])
            return set_err(m, "probe entry outside the grid"), -1;
        op->axis.push_back((uint8_t)axis[e]);
        op->node.push_back(m->index(p[0], p[1], p[2]));
        op->dw.push_back(weight[e]);
    }
    ems_probe& P = op->probe;
    P.quantity = quantity;
    P.n_entries = n;
    P.axis = op->axis.data();
    P.node = op->node.data();
    P.weight = op->dw.data();
    P.interval = interval ? interval : 1;
    P.f32_sum = 0;
    m->ops.push_back(std::move(op));
    m->refresh_desc();
    return (int)m->ops.size() - 1;
}

// MurBoundary::build (src/engine/boundary/mur.rs:403-604), hold_faces
// (619-637), openems_order / openems_corners / count_energy (649-679).
int ems_model_add_mur(ems_model* m, const int mode[6], const double velocity[6], const uint64_t hold_until[6],
                      int flags) {
    if (!m->built) return set_err(m, "build the model before adding operators"), -1;
    const uint64_t* n = m->n;
    const double dt = m->dt;
    // MurBoundary::coefficient (mur.rs:725-727).
    auto coefficient = [](double v, double dt_, double delta) { return (v * dt_ - delta) / (v * dt_ + delta); };
    auto face_delta = [&](int f) {
        const int a = f / 2;
        return (f & 1) ? m->delta(a, n[a] - 2) : m->delta(a, 0);
    };
    bool on[6] = {};
    float k_face[6] = {};
    for (int f = 0; f < 6; ++f) {
        if (mode[f] == 0) continue;
        if (mode[f] != 1 && mode[f] != 2) return set_err(m, "Mur boundary: face mode must be 0, 1 or 2"), -1;
        const int a = f / 2;
        if (mode[f] == 1) {
            const double v = velocity[f];
            if (!(std::isfinite(v) && v > 0.0))
                return set_err(m, "Mur boundary: phase velocity must be finite and > 0"), -1;
            k_face[f] = (float)coefficient(v, dt, face_delta(f));
        }
        if (n[a] < 3) return set_err(m, "Mur boundary: needs at least 3 mesh lines along the face normal"), -1;
        on[f] = true;
    }
    auto plane = [&](int f) -> uint64_t { return (f & 1) ? n[f / 2] - 1 : 0; };
    auto inner_of = [&](int f, std::array<uint64_t, 3> p) {
        const int a = f / 2;
        p[a] = (f & 1) ? p[a] - 1 : p[a] + 1;
        return p;
    };
    auto idx = [&](const std::array<uint64_t, 3>& p) { return m->index(p[0], p[1], p[2]); };
    // Local phase velocity c0/sqrt(eps_r mu_r) of the edge along t at node on
    // face f: eps_r of the interior neighbour edge, mu_r of the H face
    // between them (mur.rs:487-510), both the per-edge values of
    // EdgeMaterials::from_cells (src/engine/edge_material.rs:376-413).
    std::string bad;
    auto local = [&](int f, int t, int o, const std::array<uint64_t, 3>& node) -> float {
        const int a = f / 2;
        const auto given = m->mur_v.find(f * 3 + t);
        if (given != m->mur_v.end()) {
            const int u = a == 0 ? 1 : 0, w = a == 2 ? 1 : 2;
            const double v = given->second[node[u] * n[w] + node[w]];
            if (v > 0.0) return (float)coefficient(v, dt, face_delta(f));
        }
        const auto in = inner_of(f, node);
        auto hf = node;
        hf[a] = std::min(node[a], in[a]);
        const uint64_t pi[3] = {in[0], in[1], in[2]};
        double eps, kap;
        edge_eps(m, t, pi, eps, kap);
        const uint64_t ph[3] = {hf[0], hf[1], hf[2]};
        double mu, sig;
        edge_mu(m, o, ph, mu, sig);
        const double v = C0 / std::sqrt(eps * mu);
        if (!(std::isfinite(v) && v > 0.0)) {
            bad = "Mur boundary: local phase velocity must be finite and > 0";
            return 0.0f;
        }
        return (float)coefficient(v, dt, face_delta(f));
    };
    auto coef = [&](int f, int t, int o, const std::array<uint64_t, 3>& node) {
        return mode[f] == 1 ? k_face[f] : local(f, t, o, node);
    };
    // Capacitance of a boundary edge with full dual cells on the outer
    // planes (mur.rs:469-482), from the interior neighbour's ca, cb
    // (Coefficients::capacitance, src/engine/coeffs.rs:1066-1076).
    auto full_c = [&](int t, const std::array<uint64_t, 3>& node, const std::array<uint64_t, 3>& in) {
        const size_t i = idx(in);
        const float ca = m->co[t][i], cb = m->co[3 + t][i];
        const double c = cb == 0.0f ? 0.0 : dt * (1.0 + (double)ca) / (2.0 * (double)cb);
        double fac = 1.0;
        for (int b = 0; b < 3; ++b) {
            if (b == t) continue;
            const uint64_t k = node[b], ki = in[b], nb = n[b];
            if (k == 0 || k + 1 == nb) {
                const double cell = m->delta(b, k == 0 ? 0 : nb - 2);
                fac *= cell / m->dual_delta(b, ki);
            }
        }
        return std::isfinite(c) ? c * fac : 0.0;
    };
    struct Ent {
        int t;
        std::array<uint64_t, 3> node, in0, in1;
        float k0, k1;
        double c;
        bool corner;
    };
    std::vector<Ent> edges, corners;
    for (int f = 0; f < 6; ++f) {
        if (!on[f]) continue;
        const int a = f / 2;
        for (int t = 0; t < 3; ++t) {
            if (t == a) continue;
            const int o = 3 - a - t;
            const float* ca = m->co[t].data();
            const float* cb = m->co[3 + t].data();
            for (uint64_t p = 0; p + 1 < n[t]; ++p) {
                for (uint64_t q = 0; q < n[o]; ++q) {
                    std::array<uint64_t, 3> node{};
                    node[a] = plane(f);
                    node[t] = p;
                    node[o] = q;
                    const size_t id = idx(node);
                    if (ca[id] != 0.0f || cb[id] != 0.0f)
                        return set_err(m, "Mur boundary: the face must be PEC (its tangential edges have ca = cb = 0)"), -1;
                    int g = -1;
                    for (int mx = 0; mx < 2; ++mx)
                        if (on[2 * o + mx] && plane(2 * o + mx) == q) {
                            g = 2 * o + mx;
                            break;
                        }
                    if (g < 0) {
                        const auto in = inner_of(f, node);
                        edges.push_back({t, node, in, in, coef(f, t, o, node), 0.0f, full_c(t, node, in), false});
                    } else if (f < g) {
                        const auto i0 = inner_of(f, node), i1 = inner_of(g, node);
                        corners.push_back({t, node, i0, i1, coef(f, t, o, node), coef(g, t, a, node),
                                           full_c(t, node, inner_of(g, i0)), true});
                    }
                    if (!bad.empty()) return set_err(m, bad.c_str()), -1;
                }
            }
        }
    }
    // hold_faces: an entry whose node-to-neighbour step crosses a held
    // face's plane is held (mur.rs:619-637).
    auto held = [&](const std::array<uint64_t, 3>& node, const std::array<uint64_t, 3>& in) -> uint64_t {
        uint64_t until = 0;
        if (!hold_until) return 0;
        for (int f = 0; f < 6; ++f) {
            if (!hold_until[f]) continue;
            const int a = f / 2;
            if (node[a] != in[a] && (node[a] == 0) != ((f & 1) != 0)) until = std::max(until, hold_until[f]);
        }
        return until;
    };
    auto op = std::make_unique<OpStore>();
    op->kind = EMS_OP_MUR;
    for (const auto* list : {&edges, &corners}) {
        for (const Ent& e : *list) {
            op->axis.push_back((uint8_t)e.t);
            op->node.push_back(idx(e.node));
            op->inner.push_back(idx(e.in0));
            op->inner.push_back(e.corner ? idx(e.in1) : idx(e.in0));
            op->mk.push_back(e.k0);
            op->mk.push_back(e.k1);
            op->mcap.push_back(e.c);
            op->hold.push_back(e.corner ? std::max(held(e.node, e.in0), held(e.node, e.in1)) : held(e.node, e.in0));
        }
    }
    ems_mur& M = op->mur;
    M.n = op->node.size();
    M.n_edges = edges.size();
    M.axis = op->axis.data();
    M.node = op->node.data();
    M.inner = op->inner.data();
    M.k = op->mk.data();
    M.hold = hold_until ? op->hold.data() : nullptr;
    M.count_energy = (flags & 4) ? 1 : 0;
    M.cap = M.count_energy ? op->mcap.data() : nullptr;
    M.openems_order = (flags & 1) ? 1 : 0;
    M.openems_corners = (flags & 2) ? 1 : 0;
    m->ops.push_back(std::move(op));
    m->refresh_desc();
    return (int)m->ops.size() - 1;
}

// An absorbing sheet inside the domain (AbsorbingSheet::new,
// src/engine/boundary/abc.rs:131-240): the tangential E edges of the
// rectangle start..stop on mesh plane `plane` normal to `normal`, each with
// its neighbour one node against the outward normal (positive: +normal) and
// the first-order Mur coefficient (v·dt − Δ)/(v·dt + Δ) with v·dt rounded to
// f32 in openEMS's order; v the given velocity or, for velocity <= 0, the
// local c0/sqrt(eps_r·mu_r) of the neighbour edge and the H face spanning
// both. Edges kept at zero (metal) are left out unless the plane is outer.
// The update is a Mur face's (pre_e saves u_b^n and u_1^n, post_e writes
// u_b), so the sheet is an EMS_OP_MUR table of face edges.
int ems_model_add_absorbing_sheet(ems_model* m, int normal, uint64_t plane, int positive, const uint64_t start[3],
                                  const uint64_t stop[3], double velocity, int openems_order) {
    if (!m->built) return set_err(m, "build the model before adding operators"), -1;
    if (normal < 0 || normal > 2) return set_err(m, "absorbing sheet: invalid normal"), -1;
    const uint64_t* n = m->n;
    const int a = normal;
    if (plane >= n[a]) return set_err(m, "absorbing sheet: plane outside the mesh"), -1;
    if (positive ? plane == 0 : plane + 1 >= n[a])
        return set_err(m, "absorbing sheet: no mesh plane on its absorbing side"), -1;
    const uint64_t inner_plane = positive ? plane - 1 : plane + 1;
    for (int d = 0; d < 3; ++d)
        if (d != a && (start[d] > stop[d] || stop[d] >= n[d])) return set_err(m, "absorbing sheet: invalid range"), -1;
    const uint64_t lo = std::min(plane, inner_plane);
    const double delta = m->delta(a, lo), dt = m->dt;
    const bool outer = plane == 0 || plane == n[a] - 1;
    auto op = std::make_unique<OpStore>();
    op->kind = EMS_OP_MUR;
    for (int t = 0; t < 3; ++t) {
        if (t == a) continue;
        const int o = 3 - a - t;
        for (uint64_t p = start[t]; p < stop[t]; ++p)
            for (uint64_t q = start[o]; q <= stop[o]; ++q) {
                uint64_t node[3], inner[3];
                node[a] = plane;
                node[t] = p;
                node[o] = q;
                const uint64_t idx = m->index(node[0], node[1], node[2]);
                if (!outer && m->co[t][idx] == 0.0f && m->co[3 + t][idx] == 0.0f) continue;
                for (int d = 0; d < 3; ++d) inner[d] = node[d];
                inner[a] = inner_plane;
                double v = velocity;
                if (!(velocity > 0.0)) {
                    double eps, kap, mu, sig;
                    edge_eps(m, t, inner, eps, kap);
                    uint64_t face[3] = {node[0], node[1], node[2]};
                    face[a] = lo;
                    edge_mu(m, o, face, mu, sig);
                    v = C0 / std::sqrt(eps * mu);
                }
                if (!(std::isfinite(v) && v > 0.0)) return set_err(m, "absorbing sheet: invalid phase velocity"), -1;
                const double vdt = openems_order ? (double)(float)(v * dt) : v * dt;
                const float k = (float)((vdt - delta) / (vdt + delta));
                const uint64_t in_idx = m->index(inner[0], inner[1], inner[2]);
                op->axis.push_back((uint8_t)t);
                op->node.push_back(idx);
                op->inner.push_back(in_idx);
                op->inner.push_back(in_idx);
                op->mk.push_back(k);
                op->mk.push_back(k);
                op->mcap.push_back(0.0);
            }
    }
    ems_mur& M = op->mur;
    M.n = op->node.size();
    M.n_edges = M.n;
    M.axis = op->axis.data();
    M.node = op->node.data();
    M.inner = op->inner.data();
    M.k = op->mk.data();
    M.hold = nullptr;
    M.count_energy = 0;
    M.cap = nullptr;
    M.openems_order = openems_order ? 1 : 0;
    M.openems_corners = 0;
    m->ops.push_back(std::move(op));
    m->refresh_desc();
    return (int)m->ops.size() - 1;
}

// ---------------------------------------------------------------------------
// Field samplers (src/engine/dump.rs:281-760).

struct ems_sampler_host {
    ems_sampler t{};
    std::vector<uint32_t> idx;
    std::vector<double> w, fac, coords[3];
};

namespace {

// A sample position along one axis (dump.rs:291-303): node j, centre of
// cell j (j = n - 1: the virtual cell beyond the last node), raw node j.
enum class Pos { Node, Mid, Raw };
struct PosJ {
    Pos k;
    uint64_t j;
};
struct Tap2 {
    uint64_t i[2];
    double w[2];
};

// dual_coord (dump.rs:305-317).
double dual_coord(const ems_model* m, int a, uint64_t j) {
    const auto& l = m->lines[a];
    const uint64_t n = l.size();
    if (j + 1 < n) return 0.5 * (l[j] + l[j + 1]);
    if (n >= 2) return l[n - 1] + 0.5 * (l[n - 1] - l[n - 2]);
    return l[n - 1];
}

// oe_dual (dump.rs:319-329): the dual length with full outer cells.
double oe_dual(const ems_model* m, int a, uint64_t j) {
    const uint64_t n = m->n[a];
    const double d = m->dual_delta(a, j);
    return (n >= 2 && (j == 0 || j == n - 1)) ? 2.0 * d : d;
}

// taps (dump.rs:331-433), Cartesian grids.
Tap2 sampler_taps(const ems_model* m, bool dual, int comp, int a, PosJ pos, bool oe) {
    const uint64_t n = m->n[a];
    auto d = [&](uint64_t i) { return m->delta(a, i); };
    auto one = [](uint64_t i, double w) { return Tap2{{i, i}, {w, 0.0}}; };
    const Tap2 zero{{0, 0}, {0.0, 0.0}};
    if (n < 2) return (!dual && comp == a) ? zero : one(0, 1.0);
    auto lin = [&](uint64_t j) {
        if (j == 0) return one(0, 1.0);
        if (j == n - 1) return one(n - 2, 1.0);
        const double dl = d(j - 1), dh = d(j);
        return Tap2{{j - 1, j}, {dh / (dl + dh), dl / (dl + dh)}};
    };
    const uint64_t j = pos.j;
    if (pos.k == Pos::Mid && j + 1 >= n) return zero;
    const bool own = comp == a;
    if (!dual && own) {
        if (pos.k == Pos::Node) {
            Tap2 t = lin(j);
            t.w[0] = t.w[0] / d(t.i[0]);
            t.w[1] = t.w[1] / d(t.i[1]);
            return t;
        }
        if (pos.k == Pos::Mid) return one(j, 1.0 / d(j));
        return j + 1 < n ? one(j, 1.0 / d(j)) : zero;
    }
    if (!dual) {
        if (pos.k == Pos::Mid) return Tap2{{j, j + 1}, {0.5, 0.5}};
        return one(j, 1.0);
    }
    if (own) {
        if (pos.k != Pos::Mid) return one(j, 1.0 / m->dual_delta(a, j));
        if (oe) {
            const double x = oe_dual(m, a, j), y = oe_dual(m, a, j + 1);
            return Tap2{{j, j + 1}, {y / (x + y) / m->dual_delta(a, j), x / (x + y) / m->dual_delta(a, j + 1)}};
        }
        return Tap2{{j, j + 1}, {0.5 / m->dual_delta(a, j), 0.5 / m->dual_delta(a, j + 1)}};
    }
    if (pos.k == Pos::Node) {
        if (oe) return (j == 0 || j == n - 1) ? zero : Tap2{{j - 1, j}, {0.5, 0.5}};
        return lin(j);
    }
    return one(j, 1.0);
}

ems_sampler_host* sampler_build(ems_model* m, int q, const std::vector<PosJ> pos[3], bool oe) {
    const bool dual = q == EMS_DUMP_H || q == EMS_DUMP_B;
    auto s = std::make_unique<ems_sampler_host>();
    for (int a = 0; a < 3; ++a)
        for (const PosJ& p : pos[a]) {
            double c;
            if (p.k == Pos::Node || (p.k == Pos::Raw && !dual)) c = m->lines[a][p.j];
            else c = dual_coord(m, a, p.j);
            s->coords[a].push_back(c);
        }
    const uint64_t dims[3] = {pos[0].size(), pos[1].size(), pos[2].size()};
    const uint64_t off[3] = {0, 3 * dims[0], 3 * (dims[0] + dims[1])};
    const uint64_t total = 3 * (dims[0] + dims[1] + dims[2]);
    s->idx.assign(2 * total, 0);
    s->w.assign(2 * total, 0.0);
    uint64_t lo[3] = {UINT64_MAX, UINT64_MAX, UINT64_MAX}, hi[3] = {0, 0, 0};
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a)
            for (uint64_t k = 0; k < dims[a]; ++k) {
                const Tap2 t = sampler_taps(m, dual, c, a, pos[a][k], oe);
                const uint64_t e = 2 * (off[a] + (uint64_t)c * dims[a] + k);
                for (int u = 0; u < 2; ++u) {
                    s->idx[e + u] = (uint32_t)t.i[u];
                    s->w[e + u] = t.w[u];
                    if (t.w[u] != 0.0) {
                        lo[a] = std::min(lo[a], t.i[u]);
                        hi[a] = std::max(hi[a], t.i[u]);
                    }
                }
            }
    for (int a = 0; a < 3; ++a)
        if (lo[a] > hi[a]) lo[a] = hi[a] = 0;
    ems_sampler& T = s->t;
    T.quantity = q;
    for (int a = 0; a < 3; ++a) {
        T.dims[a] = dims[a];
        T.fac_lo[a] = lo[a];
        T.fac_dims[a] = hi[a] - lo[a] + 1;
    }
    T.tap_idx = s->idx.data();
    T.tap_w = s->w.data();
    T.factors = nullptr;
    // Factors (dump.rs:626-660 rot H, 700-750 prepare): per component over
    // the tap box, z fastest.
    if (q == EMS_DUMP_ROTH || q == EMS_DUMP_J || q == EMS_DUMP_D || q == EMS_DUMP_B) {
        const uint64_t vol = T.fac_dims[0] * T.fac_dims[1] * T.fac_dims[2];
        s->fac.assign(3 * vol, 0.0);
        const double dt = m->dt;
        for (int c = 0; c < 3; ++c) {
            const int ob = next_axis(c), oc = prev_axis(c);
            uint64_t at = (uint64_t)c * vol;
            for (uint64_t i = lo[0]; i <= hi[0]; ++i)
                for (uint64_t j = lo[1]; j <= hi[1]; ++j)
                    for (uint64_t k = lo[2]; k <= hi[2]; ++k, ++at) {
                        const uint64_t p[3] = {i, j, k};
                        const uint64_t idx = m->index(i, j, k);
                        double f = 0.0;
                        if (q == EMS_DUMP_ROTH) {
                            if (p[c] + 1 < m->n[c]) {
                                double area = m->dual_delta(ob, p[ob]) * m->dual_delta(oc, p[oc]);
                                if (oe)
                                    for (int t : {ob, oc})
                                        if (m->n[t] >= 2 && (p[t] == 0 || p[t] == m->n[t] - 1)) area *= 2.0;
                                f = area > 0.0 ? m->delta(c, p[c]) / area : 0.0;
                            }
                        } else if (q == EMS_DUMP_B) {
                            if (p[ob] + 1 < m->n[ob] && p[oc] + 1 < m->n[oc]) {
                                const float da = m->co[6 + c][idx], db = m->co[9 + c][idx];
                                const double area = m->delta(ob, p[ob]) * m->delta(oc, p[oc]);
                                if (db != 0.0f && area > 0.0) {
                                    const double l = dt * (1.0 + (double)da) / (2.0 * (double)db);
                                    f = l * m->dual_delta(c, p[c]) / area;
                                }
                            }
                        } else if (p[c] + 1 < m->n[c]) {
                            const float ca = m->co[c][idx], cb = m->co[3 + c][idx];
                            const double area = m->dual_delta(ob, p[ob]) * m->dual_delta(oc, p[oc]);
                            if (cb != 0.0f && area > 0.0) {
                                const double a = (double)ca, b = (double)cb;
                                const double v = q == EMS_DUMP_D ? dt * (1.0 + a) / (2.0 * b) : (1.0 - a) / b;
                                f = v * m->delta(c, p[c]) / area;
                            }
                        }
                        s->fac[at] = f;
                    }
        }
        T.factors = s->fac.data();
    }
    return s.release();
}

}  // namespace

ems_sampler_host* ems_sampler_new(ems_model* m, int quantity, int position, const uint64_t a[3], const uint64_t b[3],
                                  const uint64_t stride[3]) {
    if (quantity < EMS_DUMP_E || quantity > EMS_DUMP_B || position < 0 || position > 2)
        return set_err(m, "sampler: invalid quantity or position"), nullptr;
    if ((quantity == EMS_DUMP_J || quantity == EMS_DUMP_D || quantity == EMS_DUMP_B) && !m->built)
        return set_err(m, "sampler: J, D and B need the built model's coefficients"), nullptr;
    std::vector<PosJ> pos[3];
    for (int x = 0; x < 3; ++x) {
        const uint64_t lo = std::min(a[x], b[x]), hi = std::max(a[x], b[x]);
        const uint64_t st = (stride && stride[x]) ? stride[x] : 1;
        // DumpRegion::check_fits (dump.rs:210-225).
        if (hi >= m->n[x]) return set_err(m, "dump box exceeds the grid"), nullptr;
        if (position == 1 && hi > lo) {
            for (uint64_t j = lo; j < hi; j += st) pos[x].push_back({Pos::Mid, j});
        } else {
            for (uint64_t j = lo; j <= hi; j += st) pos[x].push_back({position == 2 ? Pos::Raw : Pos::Node, j});
        }
    }
    return sampler_build(m, quantity, pos, false);
}

ems_sampler_host* ems_sampler_new_indices(ems_model* m, int quantity, int position, const uint64_t* const idx[3],
                                          const size_t n[3]) {
    if (quantity < EMS_DUMP_E || quantity > EMS_DUMP_B || position < 0 || position > 2)
        return set_err(m, "sampler: invalid quantity or position"), nullptr;
    if ((quantity == EMS_DUMP_J || quantity == EMS_DUMP_D || quantity == EMS_DUMP_B) && !m->built)
        return set_err(m, "sampler: J, D and B need the built model's coefficients"), nullptr;
    std::vector<PosJ> pos[3];
    for (int x = 0; x < 3; ++x) {
        if (!n[x] || !idx[x]) return set_err(m, "dump sample indices must be increasing and inside the grid"), nullptr;
        for (size_t q = 0; q < n[x]; ++q) {
            if (idx[x][q] >= m->n[x] || (q && idx[x][q] <= idx[x][q - 1]))
                return set_err(m, "dump sample indices must be increasing and inside the grid"), nullptr;
            pos[x].push_back({position == 1 ? Pos::Mid : (position == 2 ? Pos::Raw : Pos::Node), idx[x][q]});
        }
    }
    return sampler_build(m, quantity, pos, true);
}

const ems_sampler* ems_sampler_table(const ems_sampler_host* s) { return s ? &s->t : nullptr; }

const double* ems_sampler_coords(const ems_sampler_host* s, int axis, size_t* n) {
    if (!s || axis < 0 || axis > 2) return nullptr;
    if (n) *n = s->coords[axis].size();
    return s->coords[axis].data();
}

void ems_sampler_free(ems_sampler_host* s) { delete s; }

// ---------------------------------------------------------------------------
// Conducting sheets (src/engine/sheet.rs).

namespace {

constexpr double kSurfaceLayer = 0.15;  // SURFACE_LAYER, sheet.rs:224
constexpr double kGrowth = 1.15;        // GROWTH, sheet.rs:233

// skin_depth (sheet.rs:237-239): sqrt(2/(ω μ0 σ)).
double skin_depth(double sigma, double f) { return std::sqrt(2.0 / (2.0 * PI * f * MU0 * sigma)); }

// layer_profile (sheet.rs:244-271): outer layers 0.15 skin depths at f_max
// thick, each further one 1.15 times thicker up to the middle, mirrored; a
// sheet thinner than two outer layers gets uniform layers of at most one
// outer layer each.
std::vector<double> layer_profile(double sigma, double t, double f_max) {
    const double s = kSurfaceLayer * skin_depth(sigma, f_max);
    const bool ok = std::isfinite(s) && s > 0.0;
    if (!ok || t <= 2.0 * s) {
        size_t n = 1;
        if (ok) {
            const double q = std::ceil(t / s);
            n = q >= 1.0 ? (size_t)q : 1;
        }
        return std::vector<double>(n, t / (double)n);
    }
    const double half_t = 0.5 * t;
    std::vector<double> half;
    double acc = 0.0, dz = s;
    while (acc + dz < half_t) {
        half.push_back(dz);
        acc += dz;
        dz *= kGrowth;
    }
    const double rem = half_t - acc;
    if (!half.empty() && rem < 0.5 * half.back()) half.back() += rem;
    else half.push_back(rem);
    std::vector<double> out = half;
    out.insert(out.end(), half.rbegin(), half.rend());
    return out;
}

// sheet_geometry on a Cartesian grid (sheet.rs:352-400): g = w/l (w the
// dual length across the edge in the sheet, l the edge length) and the
// share f_up of the crossing dual edges on the + side of the normal.
void sheet_geometry(const ems_model* m, int d, int nrm, const uint64_t node[3], double& g, double& f_up) {
    const int t = 3 - nrm - d;
    const uint64_t k = node[nrm];
    const double up = k + 1 < m->n[nrm] ? m->delta(nrm, k) : 0.0;
    const double dn = k > 0 ? m->delta(nrm, k - 1) : 0.0;
    f_up = up / (up + dn);
    g = m->dual_delta(t, node[t]) / m->delta(d, node[d]);
}

}  // namespace

size_t ems_sheet_layer_profile(double sigma, double thickness, double f_max, double* out, size_t cap) {
    const std::vector<double> v = layer_profile(sigma, thickness, f_max);
    for (size_t q = 0; q < v.size() && q < cap; ++q) out[q] = v[q];
    return v.size();
}

int ems_model_add_sheet(ems_model* m, size_t n, const int* axis, const uint64_t* nodes, const int* normal,
                        const double* sigma, const double* thickness, const double* share_c, const double* share_g,
                        double f_max, uint64_t* installed, uint64_t* skipped) {
    if (!m->built) return set_err(m, "build the model first"), -1;
    if (n && (!axis || !nodes || !normal || !sigma || !thickness)) return set_err(m, "conducting sheet: missing arrays"), -1;
    auto has_share = [&](size_t e) { return share_c && share_g && (share_c[e] >= 0.0 || share_g[e] >= 0.0); };
    // ConductingSheet::validate (sheet.rs:635-656).
    for (size_t e = 0; e < n; ++e) {
        const int a = axis[e], nr = normal[e];
        const uint64_t* p = nodes + 3 * e;
        if (a < 0 || a > 2 || nr < 0 || nr > 2 || a == nr)
            return set_err(m, "conducting sheet edge: the edge is not tangential to the sheet"), -1;
        if (!(std::isfinite(sigma[e]) && sigma[e] > 0.0))
            return set_err(m, "conducting sheet edge: conductivity must be finite and > 0"), -1;
        if (!(std::isfinite(thickness[e]) && thickness[e] > 0.0))
            return set_err(m, "conducting sheet edge: thickness must be finite and > 0"), -1;
        if (has_share(e) && !(share_c[e] >= 0.0 && share_c[e] <= 1.0 && share_g[e] >= 0.0 && share_g[e] <= 1.0))
            return set_err(m, "conducting sheet edge: shares must be in [0, 1]"), -1;
        if (p[0] >= m->n[0] || p[1] >= m->n[1] || p[2] >= m->n[2] || p[a] + 1 >= m->n[a])
            return set_err(m, "conducting sheet edge: not an edge of the grid"), -1;
    }
    if (f_max != 0.0 && !(std::isfinite(f_max) && f_max > 0.0))
        return set_err(m, "conducting sheet: f_max must be finite and > 0"), -1;
    const double dt = m->dt;
    const double fm = f_max > 0.0 ? f_max : 0.1 / dt;
    // install (sheet.rs:658-933): edges sorted by (node, axis), stable.
    std::vector<size_t> order(n);
    std::iota(order.begin(), order.end(), (size_t)0);
    auto key = [&](size_t e) { return std::make_tuple(nodes[3 * e], nodes[3 * e + 1], nodes[3 * e + 2], axis[e]); };
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return key(x) < key(y); });
    auto op = std::make_unique<OpStore>();
    op->kind = EMS_OP_SHEET;
    std::map<std::vector<uint64_t>, std::pair<uint32_t, uint32_t>> ladders;
    uint64_t n_skip = 0;
    bool have_last = false;
    uint64_t last_idx = 0;
    int last_axis = -1;
    auto bits = [](double v) {
        uint64_t b;
        std::memcpy(&b, &v, 8);
        return b;
    };
    for (size_t q : order) {
        const int d = axis[q], nrm = normal[q];
        const uint64_t* p = nodes + 3 * q;
        const uint64_t idx = m->index(p[0], p[1], p[2]);
        if (have_last && last_idx == idx && last_axis == d) {  // a duplicate
            ++n_skip;
            continue;
        }
        have_last = true;
        last_idx = idx;
        last_axis = d;
        const double ca = (double)m->co[d][idx], cb = (double)m->co[3 + d][idx];
        if (cb == 0.0) {  // PEC
            ++n_skip;
            continue;
        }
        const double c_edge = dt * (1.0 + ca) / (2.0 * cb);
        const double g_edge = (1.0 - ca) / cb;
        double geo, f_up;
        sheet_geometry(m, d, nrm, p, geo, f_up);
        const double sc = has_share(q) ? share_c[q] : f_up;
        const double sg = has_share(q) ? share_g[q] : f_up;
        // The ladder: shunt G_k, C_k on the nodes (half layers around
        // each), series L_j per layer, the split edge C and G on the faces.
        const std::vector<double> dz = layer_profile(sigma[q], thickness[q], fm);
        const size_t nn = dz.size() + 1;
        std::vector<double> a, g_node(nn, 0.0), c_node(nn, 0.0);
        for (size_t j = 0; j < dz.size(); ++j) {
            const double z = dz[j];
            for (size_t kk : {j, j + 1}) {
                g_node[kk] += 0.5 * sigma[q] * z * geo;
                c_node[kk] += 0.5 * EPS0 * z * geo;
            }
            a.push_back(dt * geo / (2.0 * MU0 * z));
        }
        c_node[0] += sc * c_edge;
        g_node[0] += sg * g_edge;
        c_node[nn - 1] += (1.0 - sc) * c_edge;
        g_node[nn - 1] += (1.0 - sg) * g_edge;
        // Thomas factorisation of the constant tridiagonal matrix.
        std::vector<double> konst;
        double prev_cp = 0.0;
        for (size_t kk = 0; kk < nn; ++kk) {
            const double a_up = kk + 1 < nn ? a[kk] : 0.0;
            const double a_dn = kk > 0 ? a[kk - 1] : 0.0;
            const double tc = 2.0 * c_node[kk] / dt;
            const double diag = tc + g_node[kk] + a_up + a_dn;
            const double den = diag + a_dn * prev_cp;
            const double cpk = -a_up / den;
            konst.insert(konst.end(), {tc, cpk, 1.0 / den});
            prev_cp = cpk;
        }
        // Edges with bit-identical constants share them.
        std::vector<uint64_t> kb;
        for (double v : a) kb.push_back(bits(v));
        for (double v : konst) kb.push_back(bits(v));
        auto it = ladders.find(kb);
        if (it == ladders.end()) {
            std::pair<uint32_t, uint32_t> at((uint32_t)op->two_c.size(), (uint32_t)op->sa.size());
            for (size_t kk = 0; kk < nn; ++kk) {
                op->two_c.push_back(konst[3 * kk]);
                op->cp.push_back(konst[3 * kk + 1]);
                op->inv_den.push_back(konst[3 * kk + 2]);
            }
            op->sa.insert(op->sa.end(), a.begin(), a.end());
            it = ladders.emplace(kb, at).first;
        }
        // The four dual edges around the dual face, with their sign in the
        // E update and their shares of the two faces.
        const int b = next_axis(d), c = prev_axis(d);
        const std::array<std::tuple<int, int, double>, 4> around = {
            {{c, -1, 1.0}, {c, b, -1.0}, {b, -1, -1.0}, {b, c, 1.0}}};
        for (const auto& [ax, off, sgn] : around) {
            uint64_t mm[3] = {p[0], p[1], p[2]};
            if (off >= 0) {
                if (mm[off] == 0) continue;
                mm[off] -= 1;
            }
            const int pp = next_axis(ax), qq = prev_axis(ax);
            if (mm[pp] + 1 >= m->n[pp] || mm[qq] + 1 >= m->n[qq]) continue;
            double w_up = 1.0, w_dn = 0.0;
            if (ax == nrm) {
                w_up = f_up;
                w_dn = 1.0 - f_up;
            } else if (off == nrm) {
                w_up = 0.0;
                w_dn = 1.0;
            }
            const uint64_t mi = m->index(mm[0], mm[1], mm[2]);
            const double da = (double)m->co[6 + ax][mi], db = (double)m->co[9 + ax][mi];
            const double corr = -db * sgn * w_dn;
            const double ecorr = db == 0.0 ? 0.0 : 0.5 * dt * (1.0 + da) / (2.0 * db) * corr;
            op->cax.push_back((uint8_t)ax);
            op->cnode.push_back(mi);
            op->cwup.push_back(sgn * w_up);
            op->cwdn.push_back(sgn * w_dn);
            op->ccorr.push_back(corr);
            op->cecorr.push_back(ecorr);
        }
        op->sax.push_back((uint8_t)d);
        op->snode.push_back(idx);
        op->snn.push_back((uint32_t)nn);
        op->sk0.push_back(it->second.first);
        op->sa0.push_back(it->second.second);
        op->send.push_back((uint32_t)op->cax.size());
        op->scedge.push_back(c_edge);
    }
    if (installed) *installed = op->sax.size();
    if (skipped) *skipped = n_skip;
    ems_sheet& S = op->sheet;
    S.n_edges = op->sax.size();
    S.axis = op->sax.data();
    S.node = op->snode.data();
    S.nn = op->snn.data();
    S.konst0 = op->sk0.data();
    S.a0 = op->sa0.data();
    S.coupling_end = op->send.data();
    S.c_edge = op->scedge.data();
    S.n_couplings = op->cax.size();
    S.c_axis = op->cax.data();
    S.c_node = op->cnode.data();
    S.w_up = op->cwup.data();
    S.w_dn = op->cwdn.data();
    S.corr = op->ccorr.data();
    S.ecorr = op->cecorr.data();
    S.n_konst = op->two_c.size();
    S.two_c = op->two_c.data();
    S.cp = op->cp.data();
    S.inv_den = op->inv_den.data();
    S.n_a = op->sa.size();
    S.a = op->sa.data();
    m->ops.push_back(std::move(op));
    m->refresh_desc();
    return (int)m->ops.size() - 1;
}

int ems_model_probe_f32(ems_model* m, int op, int on) {
    if (op < 0 || (size_t)op >= m->ops.size() || m->ops[(size_t)op]->kind != EMS_OP_PROBE)
        return set_err(m, "not a probe"), EMS_ERR_INVALID;
    m->ops[(size_t)op]->probe.f32_sum = on ? 1 : 0;
    return EMS_OK;
}

const ems_engine_desc* ems_model_desc(ems_model* m) {
    if (!m->built) return nullptr;
    m->refresh_desc();
    return &m->desc;
}

// phase_cycles (src/post/dft.rs:190-203): f·(t0 + n·dt) modulo one cycle.
static double phase_cycles(double f, double t0, double dt, double n) {
    double a = f * dt;
    double p = a * n;
    double e = std::fma(a, n, -p);
    double c = f * t0;
    double x = (p - std::trunc(p)) + e + (c - std::trunc(c));
    return x - std::trunc(x);
}

void ems_dft(double t0, double dt, const double* x, size_t n, const double* freqs, size_t nf, double* re, double* im) {
    for (size_t q = 0; q < nf; ++q) {
        double sr = 0.0, si = 0.0;
        for (size_t s = 0; s < n; ++s) {
            double ph = -TAU * phase_cycles(freqs[q], t0, dt, (double)s);
            sr += x[s] * std::cos(ph);
            si += x[s] * std::sin(ph);
        }
        re[q] = sr * dt;
        im[q] = si * dt;
    }
}

// drive (src/engine/run.rs:424-540), the invariant measure without a settle test.
int ems_drive(const ems_stepper* s, const ems_run_limits* lim, ems_run_outcome* out) {
    if (!s || !lim || !out) return EMS_ERR_INVALID;
    const uint64_t interval = lim->check_interval ? lim->check_interval : 50;
    const uint64_t max = lim->max_timesteps;
    uint64_t steps = 0, checks = 0;
    double w = 0.0, w_max = 0.0, ratio_db = 0.0;
    int reason;
    for (;;) {
        if (steps >= max) { reason = 1; break; }
        const uint64_t n = steps;  // timestep of a fresh engine
        // A stepper that reports divergence (EMS_ERR_DIVERGED) ends the run
        // as a non-finite energy does (src/engine/run.rs:156-161).
        if (const int rc = s->step_with_energy(s->ctx, &w)) { reason = rc == EMS_ERR_DIVERGED ? 2 : 3; break; }
        ++steps;
        ++checks;
        w_max = std::max(w_max, w);
        double ratio = w_max > 0.0 ? w / w_max : 1.0;
        ratio_db = ratio > 0.0 ? 10.0 * std::log10(ratio) : -INFINITY;
        double t = (double)n * lim->dt;
        if (!std::isfinite(w) || w < -1e-12 * w_max) { reason = 2; break; }
        if (lim->has_end_criteria && (!lim->has_excitation_end || t > lim->excitation_end) && w_max > 0.0 &&
            ratio < lim->energy_ratio) {
            reason = 0;
            break;
        }
        uint64_t chunk = std::min(interval - 1, max - steps);
        if (chunk && s->run(s->ctx, chunk) != 0) { reason = 3; break; }
        steps += chunk;
    }
    out->reason = reason;
    out->steps = steps;
    out->energy = w;
    out->max_energy = w_max;
    out->ratio_db = ratio_db;
    out->checks = checks;
    return EMS_OK;
}

// drive for a batch: ems_drive's loop per model, the models stepping
// together; a model whose loop ends is frozen and the rest go on.
int ems_batch_drive(const ems_batch_stepper* s, const ems_run_limits* lim, ems_run_outcome* out) {
    if (!s || !lim || !out || !s->n_models) return EMS_ERR_INVALID;
    const size_t n = s->n_models;
    const uint64_t interval = lim[0].check_interval ? lim[0].check_interval : 50;
    for (size_t m = 0; m < n; ++m)
        if ((lim[m].check_interval ? lim[m].check_interval : 50) != interval) return EMS_ERR_INVALID;
    struct State {
        bool done = false;
        double w = 0.0, w_max = 0.0, ratio_db = 0.0;
        uint64_t checks = 0;
    };
    std::vector<State> st(n);
    std::vector<double> e(n, 0.0);
    uint64_t steps = 0;
    size_t left = n;
    auto finish = [&](size_t m, int reason) {
        State& x = st[m];
        x.done = true;
        --left;
        out[m].reason = reason;
        out[m].steps = steps;
        out[m].energy = x.w;
        out[m].max_energy = x.w_max;
        out[m].ratio_db = x.ratio_db;
        out[m].checks = x.checks;
        s->set_active(s->ctx, m, 0);
    };
    auto finish_maxed = [&] {
        for (size_t m = 0; m < n; ++m)
            if (!st[m].done && steps >= lim[m].max_timesteps) finish(m, 1);
    };
    auto fail_all = [&] {
        for (size_t m = 0; m < n; ++m)
            if (!st[m].done) finish(m, 3);
    };
    for (;;) {
        finish_maxed();
        if (!left) break;
        const uint64_t t_step = steps;  // timestep of every active model
        if (s->step_with_energy(s->ctx, e.data()) != 0) {
            fail_all();
            break;
        }
        ++steps;
        for (size_t m = 0; m < n; ++m) {
            State& x = st[m];
            if (x.done) continue;
            x.w = e[m];
            ++x.checks;
            x.w_max = std::max(x.w_max, x.w);
            const double ratio = x.w_max > 0.0 ? x.w / x.w_max : 1.0;
            x.ratio_db = ratio > 0.0 ? 10.0 * std::log10(ratio) : -INFINITY;
            const double t = (double)t_step * lim[m].dt;
            if (!std::isfinite(x.w) || x.w < -1e-12 * x.w_max) {
                finish(m, 2);
            } else if (lim[m].has_end_criteria && (!lim[m].has_excitation_end || t > lim[m].excitation_end) &&
                       x.w_max > 0.0 && ratio < lim[m].energy_ratio) {
                finish(m, 0);
            }
        }
        // The steps up to the next check, stopping at each model's limit.
        uint64_t remaining = interval - 1;
        while (remaining && left) {
            uint64_t c = remaining;
            for (size_t m = 0; m < n; ++m)
                if (!st[m].done) c = std::min(c, lim[m].max_timesteps - std::min(lim[m].max_timesteps, steps));
            if (c && s->run(s->ctx, c) != 0) {
                fail_all();
                break;
            }
            steps += c;
            remaining -= c;
            finish_maxed();
        }
    }
    return EMS_OK;
}

}  // extern "C"
