// engine.cu — the B200 FDTD time-stepping engine behind include/ems_gpu.h.
//
// Replaces the reference engine's step (src/engine/pool.rs drive, kernel.rs
// h_row/e_row, boundary/cpml.rs Slab::apply, dispersive.rs Side::correct,
// lumped.rs post_e_impl, excite.rs, probe.rs) with CUDA kernels for sm_100a.
//
// Arithmetic: every field value is produced by the reference's expression in
// the reference's order, in IEEE f32 without contraction (built with
// --fmad=false, denormals kept, results flushed like kernel.rs flush), the
// branch state in f64 with IEEE division. So fields, probes and port series
// equal the reference's bit for bit; only the energy sums (a reduction)
// differ in order.
//
// Layout in HBM: the reference's node layout (i*ny + j)*nz + k with the row
// pitch padded to a multiple of 32 floats (128 B) so every z-row starts on a
// sector boundary; one array per field component and per coefficient lane.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/ems_gpu.h"
#include "kernels.cuh"
#include "fused.cuh"
#include "fused_tables.h"
#include "separate.cuh"
#include "split.cuh"
#include "interior.cuh"
#include "march.cuh"
#include "batch.cuh"
#include "sheet.cuh"

#include <cudaTypedefs.h>

#include <thread>
#include <unordered_map>

using namespace emsk;

namespace {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    bool chunk = false;  // an arena chunk: freed only with the engine
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

}  // namespace

struct ems_gpu {
    int device = 0;
    cudaStream_t stream = nullptr;
    Grid g{};
    double dt = 0.0;
    uint64_t step = 0;
    uint64_t launches = 0;
    int schedule = 0;
    bool oe_curl = false;  // openEMS's summation order of the curl (ems_gpu_set_curl_order)
    bool has_upml = false; // openEMS PML layers: per-operator and split schedules only
    std::string err;
    // Autotuning (ems_gpu_autotune): candidate schedules timed over real
    // steps (every schedule gives the same bits), the pick cached by key.
    struct Tune {
        bool active = false;
        std::string cache, key;
        std::vector<int> cand;
        std::vector<double> ms;
        size_t at = 0;       // candidate being timed
        int done = 0;        // steps of it run (the first is a warm-up)
        cudaEvent_t e0 = nullptr, e1 = nullptr;
    } tune;
    std::vector<std::unique_ptr<DevBuf>> bufs;
    float* u[3] = {nullptr, nullptr, nullptr};
    float* i[3] = {nullptr, nullptr, nullptr};
    float* co[12] = {};
    double* partials = nullptr;   // energy partial sums per block
    size_t n_partials = 0;
    double* d_energy = nullptr;   // [0] field part, [1] operator part
    int* diverged = nullptr;      // set on the device where a marching step writes a non-finite value
    uint64_t test_wait_ns = 0;    // ems_gpu_test_wait_timeout: the next marching step's waits run out
    struct CpmlDev {
        SlabDev s;
    };
    struct PoleDev {
        PoleSideDev e, h;
    };
    struct LumpedDev {
        LumpedDevT d;
        int axis = 0;
        size_t n_edges = 0;
        size_t n_amp = 0;
        std::vector<double> amp;   // host copy of the source values (activity test)
        bool has_src = false, record = false, has_branch = false;
        uint64_t columns = 0;
        size_t count = 0, cap = 0, vcap = 0, icap = 0;
        double* rec = nullptr;
        double* pv = nullptr;
        double* pi = nullptr;
    };
    struct SourceDev {
        int kind = 0;
        size_t n = 0;
        uint32_t* node = nullptr;
        uint8_t* axis = nullptr;
        float* weight = nullptr;
        std::vector<float> amp;
    };
    struct ProbeDev {
        ProbeDevT d;
        int quantity = 0;
        uint64_t interval = 1;
        size_t count = 0, cap = 0;
        double* values = nullptr;
    };
    struct Op {
        int kind = 0;
        std::vector<SlabDev> cpml;
        PoleDev poles;
        LumpedDev lumped;
        SourceDev source;
        ProbeDev probe;
        MurDevT mur;
        bool mur_energy = false;
        UpmlSideDev upml[2];  // openEMS PML layers: E, H
        SheetDevT sheet;
        size_t sheet_nodes = 0, sheet_layers = 0;
    };
    std::vector<Op> ops;
    // Frequency-domain dumps (ems_gpu_freq_dump_add).
    struct FreqDump {
        DumpDev d;
        int field = 0;
        uint64_t interval = 1;
        bool started = false;
    };
    std::vector<FreqDump> dumps;
    // Time-domain snapshots (ems_gpu_time_dump_add): the sampled states
    // stored one after another on the device.
    struct TimeDump {
        DumpDev d;
        int field = 0;
        uint64_t interval = 1;
        bool started = false;
        double* buf = nullptr;
        size_t used = 0, cap = 0;     // doubles
        std::vector<uint64_t> states; // the state m of each snapshot
    };
    std::vector<TimeDump> tdumps;
    // ---- the fused single-pass schedule
    bool fused_ok = false;
    bool tables_ok = false;         // the table-driven two-kernel schedule can run
    std::string fused_why;          // why the fused schedule is unavailable
    std::string tables_why;         // why the two-kernel schedule is unavailable
    double* spartials = nullptr;    // energy shares of the two-kernel H update
    size_t n_spartials = 0;
    int fused_tj = 0;
    void (*fused_launch)(const emsk::FusedParams&, unsigned, unsigned, size_t, cudaStream_t) = nullptr;
    size_t fused_smem = 0;
    unsigned fused_grid = 0;
    float* u2[3] = {nullptr, nullptr, nullptr};
    float* i2[3] = {nullptr, nullptr, nullptr};
    FusedParams fp{};               // everything but the field pointers and ψ_H parity
    std::vector<std::pair<float*, float*>> psi_h;  // ψ of each H slab: (current, other)
    std::vector<std::pair<int, int>> psi_h_at;     // its place in fp.slab[0][c][q]
    std::vector<size_t> psi_h_dev;                 // its slab in the CPML operator's device slabs

    // Swaps the H-side ψ buffers after a step that wrote the other ones,
    // and points the per-operator kernels' slabs at the current ones.
    void swap_psi_h() {
        std::vector<SlabDev>* dev = nullptr;
        for (auto& op : ops)
            if (op.kind == EMS_OP_CPML) dev = &op.cpml;
        for (size_t q = 0; q < psi_h.size(); ++q) {
            std::swap(psi_h[q].first, psi_h[q].second);
            if (dev) (*dev)[psi_h_dev[q]].psi = psi_h[q].first;
        }
    }
    // The split schedule: CPML layer shell segments per side (0 H, 1 E).
    ShellDev shell[2] = {};
    // The split schedule's row CPML (split.cuh row_cpml): every slab's
    // correction inside the update kernels' CPML variant over the quads that
    // hold layer nodes, no shell kernel; used when switched on
    // (ems_gpu_set_row_cpml) and the plan applies.
    RowCpml rowc;
    bool row_cpml_on = false;
    // The sweep schedule: x chunks of sweep_planes planes, each chunk's
    // shell boxes (first box, first node) and pole edges (first edge) per
    // side; entry [chunks] closes the last range.
    uint32_t sweep_planes = 0;
    bool sweep_ok = false;
    // The interior schedule (6): the box the one-pass kernel updates, and
    // why the schedule is unavailable ("" if it is not).
    InteriorBox ibox{};
    std::string interior_why = "no tables";
    uint32_t interior_planes = kInPlanes;  // planes a block of the interior kernel marches through
    // The marching schedule (7): why it is unavailable ("" if it is not),
    // its tile shape (kMarchShapes), planes per block, and the tensor maps
    // of the old fields of each buffer (keyed by the buffer's u_x and shape).
    std::string march_why = "no tables";
    int march_shape = 0;
    uint32_t march_planes = kMarchPlanes;
    struct MarchMapSet {
        const float* key = nullptr;
        int shape = -1;
        MarchMaps m{};
    } march_maps[2];
    std::vector<uint32_t> chunk_box[2], chunk_node[2], chunk_edge[2];
    std::vector<SlabGeo> slab_geo;       // to re-cut the shell for another chunk size
    // The chunk loop of a sweep step as a CUDA graph ([0] plain, [1] energy
    // step), captured on first use; rebuilt when the chunks change.
    cudaGraphExec_t sweep_graph[2] = {nullptr, nullptr};
    uint64_t sweep_graph_launches[2] = {0, 0};
    int nslab[2][3] = {{0, 0, 0}, {0, 0, 0}};
    std::vector<uint32_t> pole_plane[2]; // plane of every pole edge: electric, magnetic
    const uint32_t* run_of[2] = {nullptr, nullptr};  // per pole edge its run: electric, magnetic
    // The split schedule's pole kernels store the corrected value as the
    // saved value of the side (electric, magnetic) instead of a capture
    // kernel (pole_prev_fold); the electric one is current only after a split
    // step with no field upload since.
    bool fold_prev[2] = {false, false};
    bool prev_e_valid = false;
    double* qpartials = nullptr;    // energy shares of the split H update
    size_t n_qpartials = 0;
    uint32_t* counter = nullptr;
    int* status = nullptr;
    double* fpartials = nullptr;
    // Kernel timing (ems_gpu_profile): event pairs recorded around the
    // field-update kernels, per kernel id.
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pairs[3];
    std::vector<cudaEvent_t> ev_free;
    double prof_ms[3] = {0, 0, 0};
    uint64_t prof_n[3] = {0, 0, 0};

    cudaEvent_t take_event() {
        if (!ev_free.empty()) {
            cudaEvent_t e = ev_free.back();
            ev_free.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    // Records the start event of a timed kernel; returns it (or null).
    cudaEvent_t prof_begin() {
        if (!profiling) return nullptr;
        cudaEvent_t a = take_event();
        cudaEventRecord(a, stream);
        return a;
    }
    void prof_end(int kernel, cudaEvent_t a) {
        if (!a) return;
        cudaEvent_t b = take_event();
        cudaEventRecord(b, stream);
        ev_pairs[kernel].push_back({a, b});
        if (ev_pairs[kernel].size() >= 4096) prof_collect();
    }
    void prof_collect() {
        cudaStreamSynchronize(stream);
        for (int k = 0; k < 3; ++k) {
            for (auto& pr : ev_pairs[k]) {
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, pr.first, pr.second);
                prof_ms[k] += ms;
                prof_n[k] += 1;
                ev_free.push_back(pr.first);
                ev_free.push_back(pr.second);
            }
            ev_pairs[k].clear();
        }
    }

    // Small tables come out of 4 MiB arena chunks (256-byte aligned), so an
    // engine of a batch costs a few cudaMalloc calls rather than a hundred;
    // arrays of 1 MiB and more get their own allocation. Everything is
    // zeroed and lives until ems_gpu_destroy.
    static constexpr size_t kArenaChunk = 4u << 20, kArenaMax = 1u << 20;
    char* arena = nullptr;
    size_t arena_used = 0;

    template <class T>
    T* alloc(size_t n) {
        const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
        if (bytes < kArenaMax) {
            const size_t need = (bytes + 255) & ~(size_t)255;
            if (!arena || arena_used + need > kArenaChunk) {
                auto b = std::make_unique<DevBuf>();
                if (cudaMalloc(&b->p, kArenaChunk) != cudaSuccess) return nullptr;
                cudaMemsetAsync(b->p, 0, kArenaChunk, stream);
                b->bytes = kArenaChunk;
                b->chunk = true;
                arena = (char*)b->p;
                arena_used = 0;
                bufs.push_back(std::move(b));
            }
            T* p = (T*)(arena + arena_used);
            arena_used += need;
            return p;
        }
        auto b = std::make_unique<DevBuf>();
        if (cudaMalloc(&b->p, bytes) != cudaSuccess) return nullptr;
        cudaMemsetAsync(b->p, 0, bytes, stream);
        b->bytes = bytes;
        T* p = (T*)b->p;
        bufs.push_back(std::move(b));
        return p;
    }
    template <class T>
    T* upload(const T* h, size_t n) {
        T* d = alloc<T>(n);
        if (d && n && h) cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, stream);
        return d;
    }
    void release(void* p) {
        for (size_t k = 0; k < bufs.size(); ++k)
            if (bufs[k]->p == p && !bufs[k]->chunk) {
                bufs.erase(bufs.begin() + k);
                return;
            }
    }
};

namespace {

ems_status fail(ems_gpu* h, ems_status s, const std::string& m) {
    if (h) h->err = m;
    return s;
}

ems_status check(ems_gpu* h, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return EMS_OK;
    return fail(h, EMS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Remaps a reference node index (i*ny + j)*nz + k to the padded device index.
inline uint32_t dev_index(const Grid& g, uint64_t idx) {
    uint64_t k = idx % g.nz;
    uint64_t r = idx / g.nz;
    return (uint32_t)(r * g.pitch + k);
}

// Grows a sample buffer to hold `need` values (copying what it holds).
ems_status grow(ems_gpu* h, double** buf, size_t count, size_t* cap, size_t need) {
    if (need <= *cap) return EMS_OK;
    size_t nc = std::max<size_t>(need, std::max<size_t>(1024, *cap * 2));
    double* nb = h->alloc<double>(nc);
    if (!nb) return fail(h, EMS_ERR_NOMEM, "sample buffer");
    if (*buf && count) cudaMemcpyAsync(nb, *buf, count * sizeof(double), cudaMemcpyDeviceToDevice, h->stream);
    if (*buf) {
        cudaStreamSynchronize(h->stream);
        h->release(*buf);
    }
    *buf = nb;
    *cap = nc;
    return EMS_OK;
}

ems_status make_side(ems_gpu* h, const ems_pole_side& t, PoleSideDev& d) {
    d.n_edges = t.n_edges;
    d.n_poles = t.n_poles;
    if (!t.n_edges) return EMS_OK;
    if (!t.axis || !t.node || !t.sum_inv_z || !t.pole_end || (t.n_poles && (!t.kind || !t.a || !t.inv_c || !t.inv_z || !t.half_l)))
        return fail(h, EMS_ERR_INVALID, "pole table: missing array");
    std::vector<uint32_t> node(t.n_edges);
    uint32_t prev = 0;
    for (size_t e = 0; e < t.n_edges; ++e) {
        if (t.node[e] >= h->g.n || t.axis[e] > 2) return fail(h, EMS_ERR_INVALID, "pole table: edge outside the grid");
        if (t.pole_end[e] < prev || t.pole_end[e] - prev > kMaxPoles)
            return fail(h, EMS_ERR_INVALID, "pole table: bad pole_end (at most 16 poles per edge)");
        prev = t.pole_end[e];
        node[e] = dev_index(h->g, t.node[e]);
    }
    if (prev != t.n_poles) return fail(h, EMS_ERR_INVALID, "pole table: pole_end does not end at n_poles");
    d.axis = h->upload(t.axis, t.n_edges);
    d.node = h->upload(node.data(), t.n_edges);
    d.sum_inv_z = h->upload(t.sum_inv_z, t.n_edges);
    d.pole_end = h->upload(t.pole_end, t.n_edges);
    d.kind = h->upload(t.kind, t.n_poles);
    d.a = h->upload(t.a, t.n_poles);
    d.inv_c = h->upload(t.inv_c, t.n_poles);
    d.inv_z = h->upload(t.inv_z, t.n_poles);
    d.half_l = h->upload(t.half_l, t.n_poles);
    d.prev = h->alloc<float>(t.n_edges);
    d.j = h->alloc<double>(t.n_poles);
    d.q = h->alloc<double>(t.n_poles);
    if (!d.axis || !d.node || !d.sum_inv_z || !d.pole_end || !d.kind || !d.a || !d.inv_c || !d.inv_z || !d.half_l ||
        !d.prev || !d.j || !d.q)
        return fail(h, EMS_ERR_NOMEM, "pole table");
    return EMS_OK;
}

unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// Fused kernel instances: rows per tile × the thread bound of the launch.
template <int TJ, int MAXT>
void launch_fused(const FusedParams& P, unsigned grid, unsigned threads, size_t smem, cudaStream_t s) {
    k_fused<TJ, MAXT><<<grid, threads, smem, s>>>(P);
}

using FusedLaunch = void (*)(const FusedParams&, unsigned, unsigned, size_t, cudaStream_t);

template <int TJ, int MAXT>
bool try_tj(ems_gpu* h, int max_smem) {
    if (h->g.pitch > (uint32_t)MAXT) return false;
    const size_t bytes = fused_smem_bytes<TJ>(h->g.pitch);
    if (bytes > (size_t)max_smem) return false;
    if (cudaFuncSetAttribute(k_fused<TJ, MAXT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
        return false;
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_fused<TJ, MAXT>, (int)h->g.pitch, bytes) != cudaSuccess ||
        bps < 1)
        return false;
    h->fused_launch = launch_fused<TJ, MAXT>;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    h->fused_tj = TJ;
    h->fused_smem = bytes;
    h->fused_grid = (unsigned)(sms * bps);
    return true;
}

// The sweep schedule's chunks of S planes: the CPML shell of each side cut
// into boxes that never straddle a chunk (the split schedule uses the same
// boxes), each chunk's box and node range, and its pole edges.
ems_status build_chunks(ems_gpu* h, uint32_t S) {
    const Grid& g = h->g;
    const uint64_t nodes[3] = {g.nx, g.ny, g.nz};
    h->sweep_planes = S;
    for (auto& gx : h->sweep_graph)
        if (gx) {
            cudaGraphExecDestroy(gx);
            gx = nullptr;
        }
    std::vector<uint32_t> cuts;
    for (uint32_t x = S; x < g.nx; x += S) cuts.push_back(x);
    for (int side = 0; side < 2; ++side) {
        uint32_t total = 0;
        const std::vector<ShellBox> boxes = shell_boxes(h->slab_geo, h->nslab[side], nodes, side, &total, cuts);
        ShellDev& Sd = h->shell[side];
        Sd = ShellDev{};
        Sd.n_box = (uint32_t)boxes.size();
        Sd.total = total;
        if (Sd.n_box) {
            Sd.box = h->upload(boxes.data(), boxes.size());
            const std::vector<uint32_t> win = shell_windows(boxes, total);
            Sd.first_box = h->upload(win.data(), win.size());
            if (!Sd.box || !Sd.first_box) return fail(h, EMS_ERR_NOMEM, "CPML shell");
        }
        auto& cb = h->chunk_box[side];
        auto& cn = h->chunk_node[side];
        cb.clear();
        cn.clear();
        size_t q = 0;
        for (uint32_t a0 = 0; a0 < g.nx; a0 += S) {
            while (q < boxes.size() && boxes[q].lo[0] < a0) ++q;
            cb.push_back((uint32_t)q);
            cn.push_back(q < boxes.size() ? boxes[q].start : total);
        }
        cb.push_back((uint32_t)boxes.size());
        cn.push_back(total);
        auto& ce = h->chunk_edge[side];
        ce.clear();
        const auto& pl = h->pole_plane[side];
        size_t e = 0;
        for (uint32_t a0 = 0; a0 < g.nx; a0 += S) {
            while (e < pl.size() && pl[e] < a0) ++e;
            ce.push_back((uint32_t)e);
        }
        ce.push_back((uint32_t)pl.size());
    }
    return EMS_OK;
}

// Builds the tables of the table-driven schedules (fused_tables.h) and
// uploads them: the two-kernel schedule runs every model whose CPML and
// dispersive operators are single; the fused kernel in addition needs no
// magnetic poles, no magnetic sources and shared memory for its tile.
ems_status setup_fused(ems_gpu* h, const ems_engine_desc* d) {
    const Grid& g = h->g;
    FusedTables T = build_fused_tables(d, g.pitch);
    h->tables_why = T.why;
    h->fused_why = T.why.empty() ? T.fused_why : T.why;
    if (!T.why.empty()) return EMS_OK;
    FusedParams& P = h->fp;
    P = FusedParams{};
    P.g = g;
    P.dt = h->dt;
    for (int l = 0; l < 12; ++l) {
        if (T.lane[l].pooled) {
            P.lane[l].dense = nullptr;
            P.lane[l].rid = h->upload(T.lane[l].rid.data(), T.lane[l].rid.size());
            P.lane[l].rows = h->upload(T.lane[l].rows.data(), T.lane[l].rows.size());
            P.lane[l].bg = T.lane[l].bg;
            if (!P.lane[l].rid || !P.lane[l].rows) return fail(h, EMS_ERR_NOMEM, "pooled coefficients");
        } else {
            P.lane[l].dense = h->co[l];
        }
    }
    // CPML slabs: the engine's device copies (b, a, k, ψ), in the tables' order
    // (both keep the non-empty slabs of the table in order).
    const std::vector<SlabDev>* dev_slabs = nullptr;
    for (auto& op : h->ops)
        if (op.kind == EMS_OP_CPML) dev_slabs = &op.cpml;
    for (int side = 0; side < 2; ++side)
        for (int c = 0; c < 3; ++c) P.nslab[side][c] = T.nslab[side][c];
    size_t q_dev = 0;
    for (const FusedSlabSpec& sp : T.slabs) {
        const SlabDev& sd = (*dev_slabs)[q_dev++];
        FSlab& f = P.slab[sp.side][sp.comp][sp.q];
        for (int a = 0; a < 3; ++a) {
            f.lo[a] = sd.lo[a];
            f.hi[a] = sd.hi[a];
        }
        f.normal = (uint32_t)sd.normal;
        f.b = sd.b;
        f.a = sd.a;
        f.k = sd.k;
        f.psi_old = sd.psi;
        f.psi_new = sd.psi;
        if (!sp.side) {
            h->psi_h.push_back({sd.psi, nullptr});
            h->psi_h_at.push_back({sp.comp, sp.q});
            h->psi_h_dev.push_back(q_dev - 1);
        }
    }
    for (int a = 0; a < 3; ++a) {
        P.cmask[a] = h->upload(T.cmask[a].data(), T.cmask[a].size());
        if (!P.cmask[a]) return fail(h, EMS_ERR_NOMEM, "CPML masks");
    }
    P.poles_first = T.poles_first ? 1 : 0;
    PoleSideDev* pe_dev = nullptr;
    PoleSideDev* ph_dev = nullptr;
    for (auto& op : h->ops)
        if (op.kind == EMS_OP_POLES) {
            pe_dev = &op.poles.e;
            ph_dev = &op.poles.h;
        }
    if (T.has_poles) {
        P.has_poles = 1;
        P.runs = h->upload(T.runs.data(), T.runs.size());
        P.sets = h->upload(T.sets.data(), T.sets.size());
        P.row_runs = h->upload(T.row_runs.data(), T.row_runs.size());
        P.pj = pe_dev->j;
        P.pq = pe_dev->q;
        h->run_of[0] = h->upload(T.run_of.data(), T.run_of.size());
        if (!P.runs || !P.sets || !P.row_runs || !h->run_of[0]) return fail(h, EMS_ERR_NOMEM, "pole runs");
    }
    if (T.has_poles_h) {
        P.has_poles_h = 1;
        P.runs_h = h->upload(T.h.runs.data(), T.h.runs.size());
        P.sets_h = h->upload(T.h.sets.data(), T.h.sets.size());
        P.row_runs_h = h->upload(T.h.row_runs.data(), T.h.row_runs.size());
        P.pj_h = ph_dev->j;
        P.pq_h = ph_dev->q;
        P.prev_h = ph_dev->prev;
        h->run_of[1] = h->upload(T.h.run_of.data(), T.h.run_of.size());
        if (!P.runs_h || !P.sets_h || !P.row_runs_h || !h->run_of[1]) return fail(h, EMS_ERR_NOMEM, "pole runs");
    }
    if (g.nz >= (1u << 24)) {
        h->tables_why = h->fused_why = "z rows of 2^24 nodes or more";
        return EMS_OK;
    }
    h->slab_geo = slab_geometry(T);
    for (int sd = 0; sd < 2; ++sd)
        for (int c = 0; c < 3; ++c) h->nslab[sd][c] = T.nslab[sd][c];
    // The plane of every pole edge (a side's edges are in plane order).
    for (int side = 0; side < 2; ++side) {
        h->pole_plane[side].clear();
        for (size_t k = 0; k < d->n_ops; ++k)
            if (d->ops[k].kind == EMS_OP_POLES) {
                const auto* pp = (const ems_poles*)d->ops[k].table;
                const ems_pole_side* ps = side ? &pp->magnetic : &pp->electric;
                const uint64_t per_plane = (uint64_t)g.ny * g.nz;
                for (size_t e = 0; e < ps->n_edges; ++e) h->pole_plane[side].push_back((uint32_t)(ps->node[e] / per_plane));
            }
    }
    {
        int l2 = 0;
        cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, h->device);
        const double plane = 6.0 * g.ny * g.pitch * 4.0;
        const uint32_t S = (uint32_t)std::max(2.0, std::min(64.0, std::floor(0.45 * (l2 > 0 ? l2 : 50 << 20) / plane)));
        ems_status st = build_chunks(h, S);
        if (st) return st;
    }
    // Row CPML: with the CPML registered before every other slab operator
    // (its corrections then come first after each update) and no openEMS
    // PML layers.
    {
        bool cpml_first = true, seen_cpml = false;
        for (size_t k = 0; k < d->n_ops; ++k) {
            const int kind = d->ops[k].kind;
            if (kind == EMS_OP_CPML) seen_cpml = true;
            if ((kind == EMS_OP_POLES || kind == EMS_OP_UPML) && !seen_cpml) cpml_first = false;
            if (kind == EMS_OP_UPML) cpml_first = false;
        }
        const uint64_t nodes3[3] = {g.nx, g.ny, g.nz};
        h->rowc = (seen_cpml && cpml_first) ? row_cpml_plan(h->slab_geo, nodes3) : RowCpml{};
    }
    // The sweep needs no magnetic sources or conducting sheets (their serial
    // post_h hooks would sit between a chunk's H and E updates) and no
    // openEMS PML layers (their hooks are not cut into chunks).
    h->sweep_ok = true;
    for (size_t k = 0; k < d->n_ops; ++k) {
        if (d->ops[k].kind == EMS_OP_SOURCE) {
            const auto* sr = (const ems_source*)d->ops[k].table;
            if (sr->kind == EMS_SOFT_H || sr->kind == EMS_HARD_H) h->sweep_ok = false;
        }
        if (d->ops[k].kind == EMS_OP_SHEET) h->sweep_ok = false;
        if (d->ops[k].kind == EMS_OP_UPML) {
            h->sweep_ok = false;
            if (h->fused_why.empty()) h->fused_why = "openEMS PML layers";
        }
    }
    h->interior_why = interior_box(d, g, h->ibox);
    h->march_why = march_why(d);
    h->fold_prev[0] = T.has_poles && pole_prev_fold(d, true, T.poles_first);
    h->fold_prev[1] = T.has_poles_h && pole_prev_fold(d, false, T.poles_first);
    h->n_qpartials = (size_t)split_blocks_x(g) * g.nx;
    h->qpartials = h->alloc<double>(h->n_qpartials);
    if (!h->qpartials) return fail(h, EMS_ERR_NOMEM, "energy shares");
    h->n_spartials = (size_t)blocks_for(g.nz, kSepJ * kSeg) * blocks_for(g.ny, kSepK) * g.nx;
    h->spartials = h->alloc<double>(h->n_spartials);
    if (!h->spartials) return fail(h, EMS_ERR_NOMEM, "energy shares");
    h->tables_ok = true;
    // The fused kernel.
    if (!h->fused_why.empty()) return EMS_OK;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
    if (!(try_tj<6, 576>(h, max_smem) || try_tj<4, 576>(h, max_smem) || try_tj<2, 576>(h, max_smem) ||
          try_tj<4, 1024>(h, max_smem) || try_tj<2, 1024>(h, max_smem))) {
        h->fused_why = "shared memory";
        return EMS_OK;
    }
    for (size_t q = 0; q < T.slabs.size(); ++q) (void)q;
    size_t qh = 0;
    for (const FusedSlabSpec& sp : T.slabs) {
        if (sp.side) continue;
        float* other = h->alloc<float>(sp.len);
        if (!other) return fail(h, EMS_ERR_NOMEM, "CPML state");
        h->psi_h[qh++].second = other;
    }
    fused_work(P, g.nx, g.ny, h->fused_tj, h->fused_grid);
    h->counter = h->alloc<uint32_t>(1);
    h->status = h->alloc<int>(1);
    h->fpartials = h->alloc<double>(h->fused_grid);
    for (int a = 0; a < 3; ++a) {
        h->u2[a] = h->alloc<float>(g.np);
        h->i2[a] = h->alloc<float>(g.np);
        if (!h->u2[a] || !h->i2[a]) return fail(h, EMS_ERR_NOMEM, "second field buffers");
    }
    if (!h->counter || !h->status || !h->fpartials) return fail(h, EMS_ERR_NOMEM, "fused schedule");
    P.counter = h->counter;
    P.status = h->status;
    P.partials = h->fpartials;
    h->fused_ok = true;
    return EMS_OK;
}

// The schedule a step runs: 1 the per-operator kernels, 2 fused, 3 two
// kernels, 4 split. Automatic: split, which measures fastest on B200, where
// the tables allow it.
int active_schedule(const ems_gpu* h) {
    switch (h->schedule) {
    case 1: return 1;
    case 2: return h->fused_ok ? 2 : (h->tables_ok ? 3 : 1);
    case 3: return h->tables_ok ? 3 : 1;
    case 4: return h->tables_ok ? 4 : 1;
    case 5: return h->tables_ok ? (h->sweep_ok ? 5 : 4) : 1;
    case 6: return h->tables_ok ? (h->interior_why.empty() ? 6 : 4) : 1;
    case 7: return h->tables_ok ? (h->march_why.empty() ? 7 : 4) : 1;
    default: return h->tables_ok ? 4 : 1;
    }
}

bool use_fused(const ems_gpu* h) { return active_schedule(h) == 2; }

ems_status serial_post_h(ems_gpu* h, const Fields& f);
ems_status serial_pre_e(ems_gpu* h, const Fields& f);
ems_status serial_post_e(ems_gpu* h, const Fields& f);

// One step through the fused kernel: lumped pre_e hooks on u^n, the fused
// H + E pass into the other buffers, then the serial hooks on the new fields.
ems_status run_step_fused(ems_gpu* h, bool energy) {
    cudaStream_t s = h->stream;
    // The fused step swaps the field and ψ buffers: a captured sweep graph
    // would point at the old ones.
    for (auto& gx : h->sweep_graph)
        if (gx) {
            cudaGraphExecDestroy(gx);
            gx = nullptr;
        }
    Fields f{{h->u[0], h->u[1], h->u[2]}, {h->i[0], h->i[1], h->i[2]}};
    ems_status st = serial_pre_e(h, f);
    if (st) return st;
    FusedParams P = h->fp;
    for (int a = 0; a < 3; ++a) {
        P.uo[a] = h->u[a];
        P.io[a] = h->i[a];
        P.un[a] = h->u2[a];
        P.in[a] = h->i2[a];
    }
    for (size_t q = 0; q < h->psi_h.size(); ++q) {
        FSlab& fs = P.slab[0][h->psi_h_at[q].first][h->psi_h_at[q].second];
        fs.psi_old = h->psi_h[q].first;
        fs.psi_new = h->psi_h[q].second;
    }
    P.energy = energy ? 1 : 0;
    cudaMemsetAsync(h->counter, 0, sizeof(uint32_t), s);
    cudaEvent_t ev = h->prof_begin();
    h->fused_launch(P, h->fused_grid, h->g.pitch, h->fused_smem, s);
    h->prof_end(2, ev);
    h->launches += 2;
    if (energy) {
        k_reduce_partials<<<1, 1024, 0, s>>>(h->fpartials, h->fused_grid, h->d_energy);
        ++h->launches;
    }
    for (int a = 0; a < 3; ++a) {
        std::swap(h->u[a], h->u2[a]);
        std::swap(h->i[a], h->i2[a]);
    }
    h->swap_psi_h();
    Fields nf{{h->u[0], h->u[1], h->u[2]}, {h->i[0], h->i[1], h->i[2]}};
    st = serial_post_h(h, nf);
    if (st) return st;
    st = serial_post_e(h, nf);
    if (st) return st;
    ++h->step;
    return EMS_OK;
}

// One step through the two-kernel schedule (separate.cuh), in place.
ems_status run_step_two(ems_gpu* h, bool energy) {
    cudaStream_t s = h->stream;
    const Grid& g = h->g;
    Fields f{{h->u[0], h->u[1], h->u[2]}, {h->i[0], h->i[1], h->i[2]}};
    FusedParams P = h->fp;
    for (int a = 0; a < 3; ++a) {
        P.uo[a] = P.un[a] = h->u[a];
        P.io[a] = P.in[a] = h->i[a];
    }
    for (size_t q = 0; q < h->psi_h.size(); ++q) {
        FSlab& fs = P.slab[0][h->psi_h_at[q].first][h->psi_h_at[q].second];
        fs.psi_old = fs.psi_new = h->psi_h[q].first;
    }
    P.partials = h->spartials;
    dim3 blk(kSepK, kSepJ, 1);
    dim3 grd(blocks_for(g.nz, kSepJ * kSeg), blocks_for(g.ny, kSepK), g.nx);
    cudaEvent_t ev = h->prof_begin();
    if (energy) {
        k_step_h<true><<<grd, blk, 0, s>>>(P);
    } else {
        k_step_h<false><<<grd, blk, 0, s>>>(P);
    }
    h->prof_end(0, ev);
    ++h->launches;
    if (energy) {
        k_reduce_partials<<<1, 1024, 0, s>>>(h->spartials, h->n_spartials, h->d_energy);
        ++h->launches;
    }
    ems_status st = serial_post_h(h, f);
    if (st) return st;
    st = serial_pre_e(h, f);
    if (st) return st;
    ev = h->prof_begin();
    k_step_e<<<grd, blk, 0, s>>>(P);
    h->prof_end(1, ev);
    ++h->launches;
    // Magnetic-pole edges save i^{n+1/2} after the E update (src/engine/dispersive.rs:1730-1744).
    for (auto& op : h->ops)
        if (op.kind == EMS_OP_POLES && op.poles.h.n_edges) {
            k_poles_capture<<<blocks_for(op.poles.h.n_edges, 256), 256, 0, s>>>(f, op.poles.h, false);
            ++h->launches;
        }
    st = serial_post_e(h, f);
    if (st) return st;
    ++h->step;
    return EMS_OK;
}

// One step through the sweep schedule: the split kernels run chunk by
// chunk along x (H update, its slab hooks, E update, its slab hooks for the
// chunk's planes), so the fields a chunk's E update reads were just touched
// by its H update and come from L2. Order is the reference's per node: the E
// update of plane i needs H of planes i and i − 1 (this chunk and the last,
// both final) and changes only u of its own planes, which no later H update
// reads. Lumped elements save u^n before the first chunk (u is unchanged
// until the E updates); current probes sample after the last chunk (nothing
// changes i after its slab hooks); magnetic sources are excluded (sweep_ok).
ems_status run_step_sweep(ems_gpu* h, bool energy) {
    const Grid& g = h->g;
    cudaStream_t s = h->stream;
    Fields f{{h->u[0], h->u[1], h->u[2]}, {h->i[0], h->i[1], h->i[2]}};
    Coeffs c;
    for (int l = 0; l < 12; ++l) c.c[l] = h->co[l];
    FusedParams P = h->fp;
    for (int a = 0; a < 3; ++a) {
        P.uo[a] = P.un[a] = h->u[a];
        P.io[a] = P.in[a] = h->i[a];
    }
    for (size_t q = 0; q < h->psi_h.size(); ++q) {
        FSlab& fs = P.slab[0][h->psi_h_at[q].first][h->psi_h_at[q].second];
        fs.psi_old = fs.psi_new = h->psi_h[q].first;
    }
    P.partials = h->qpartials;
    ems_status st = serial_pre_e(h, f);
    if (st) return st;
    const ems_gpu::Op* cpml = nullptr;
    const ems_gpu::Op* poles = nullptr;
    for (auto& op : h->ops) {
        if (op.kind == EMS_OP_CPML) cpml = &op;
        if (op.kind == EMS_OP_POLES) poles = &op;
    }
    const bool pf = h->fp.poles_first != 0;
    // The electric saved values u^n, unless the pole kernel kept them.
    if (poles && poles->poles.e.n_edges && !(h->fold_prev[0] && h->prev_e_valid)) {
        k_poles_capture<<<blocks_for(poles->poles.e.n_edges, 256), 256, 0, s>>>(f, poles->poles.e, true);
        ++h->launches;
    }
    const uint32_t bx = split_blocks_x(g), S = h->sweep_planes;
    auto shell = [&](int side, size_t ch) {
        const uint32_t n0 = h->chunk_node[side][ch], n1 = h->chunk_node[side][ch + 1];
        if (!cpml || n1 == n0) return;
        ShellDev sd = h->shell[side];
        sd.total = n1 - n0;
        sd.base = n0;
        const uint32_t nb = (sd.total + 32 * kShellWarps - 1) / (32 * kShellWarps);
        if (side) k_shell<1><<<nb, 32 * kShellWarps, 0, s>>>(P, sd);
        else k_shell<0><<<nb, 32 * kShellWarps, 0, s>>>(P, sd);
        ++h->launches;
    };
    auto pole = [&](int side, size_t ch) {  // side 0 electric, 1 magnetic
        if (!poles) return;
        const PoleSideDev& ps = side ? poles->poles.h : poles->poles.e;
        const uint32_t e0 = h->chunk_edge[side][ch], e1 = h->chunk_edge[side][ch + 1];
        if (!ps.n_edges || e1 == e0) return;
        k_poles_blocks<<<blocks_for(e1 - e0, kPoleBlock), kPoleBlock, 0, s>>>(f, c, ps, side ? P.runs_h : P.runs, side ? P.sets_h : P.sets,
                                                             h->run_of[side], side ? 0 : 1, h->dt,
                                                             h->fold_prev[side] ? 1 : 0, e0, e1);
        ++h->launches;
    };
    // The chunk loop (and the energy sum) depends on nothing the host
    // changes between steps: it is captured once as a CUDA graph, so its
    // hundreds of small launches cost one graph launch per step.
    const int gi = energy ? 1 : 0;
    if (!h->sweep_graph[gi]) {
        const uint64_t before = h->launches;
        cudaGraph_t graph = nullptr;
        if (check(h, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "sweep capture")) return EMS_ERR_CUDA;
        size_t ch = 0;
        for (uint32_t a0 = 0; a0 < g.nx; a0 += S, ++ch) {
            const uint32_t np = std::min(S, g.nx - a0);
            const dim3 grd(bx, np, 1);
            if (h->oe_curl) {
                if (energy) k_split_h<true, true><<<grd, kSplitThreads, 0, s>>>(P, a0);
                else k_split_h<false, true><<<grd, kSplitThreads, 0, s>>>(P, a0);
            } else if (energy) {
                k_split_h<true><<<grd, kSplitThreads, 0, s>>>(P, a0);
            } else {
                k_split_h<false><<<grd, kSplitThreads, 0, s>>>(P, a0);
            }
            ++h->launches;
            if (pf) { pole(1, ch); shell(0, ch); } else { shell(0, ch); pole(1, ch); }
            if (h->oe_curl) k_split_e<true><<<grd, kSplitThreads, 0, s>>>(P, a0);
            else k_split_e<<<grd, kSplitThreads, 0, s>>>(P, a0);
            ++h->launches;
            if (pf) { pole(0, ch); shell(1, ch); } else { shell(1, ch); pole(0, ch); }
        }
        if (energy) {
            k_reduce_partials<<<1, 1024, 0, s>>>(h->qpartials, h->n_qpartials, h->d_energy);
            ++h->launches;
        }
        if (check(h, cudaStreamEndCapture(s, &graph), "sweep capture")) return EMS_ERR_CUDA;
        const cudaError_t e = cudaGraphInstantiate(&h->sweep_graph[gi], graph, 0);
        cudaGraphDestroy(graph);
        if (check(h, e, "sweep graph")) return EMS_ERR_CUDA;
        h->sweep_graph_launches[gi] = h->launches - before;
        h->launches = before;
    }
    cudaEvent_t ev = h->prof_begin();
    if (check(h, cudaGraphLaunch(h->sweep_graph[gi], s), "sweep graph launch")) return EMS_ERR_CUDA;
    h->launches += h->sweep_graph_launches[gi];
    h->prof_end(0, ev);
    // The magnetic saved values (i after the E update), unless kept.
    if (poles && poles->poles.h.n_edges && !h->fold_prev[1]) {
        k_poles_capture<<<blocks_for(poles->poles.h.n_edges, 256), 256, 0, s>>>(f, poles->poles.h, false);
        ++h->launches;
    }
    st = serial_post_h(h, f);
    if (st) return st;
    st = serial_post_e(h, f);
    if (st) return st;
    h->prev_e_valid = h->fold_prev[0];
    ++h->step;
    return EMS_OK;
}

// One step through the interior schedule (interior.cuh): the old fields in
// one buffer, the new ones written into the other, which becomes the
// current one. The split H update and its CPML correction over the nodes
// outside the interior box, the one-pass kernel over the box, the split E
// update and its CPML correction outside it, then the electric poles and the
// serial hooks on the new fields. Steps that record the energy run the
// split schedule in place.
ems_status run_step_interior(ems_gpu* h) {
    const Grid& g = h->g;
    cudaStream_t s = h->stream;
    if (!h->u2[0]) {
        // The second buffers start as copies: the entries no kernel writes
        // (edges that do not exist, row padding) then agree in both.
        for (int a = 0; a < 3; ++a) {
            h->u2[a] = h->alloc<float>(g.np);
            h->i2[a] = h->alloc<float>(g.np);
            if (!h->u2[a] || !h->i2[a]) return fail(h, EMS_ERR_NOMEM, "second field buffers");
            if (check(h, cudaMemcpyAsync(h->u2[a], h->u[a], g.np * sizeof(float), cudaMemcpyDeviceToDevice, s),
                      "second field buffers") ||
                check(h, cudaMemcpyAsync(h->i2[a], h->i[a], g.np * sizeof(float), cudaMemcpyDeviceToDevice, s),
                      "second field buffers"))
                return EMS_ERR_CUDA;
        }
    }
    // A captured sweep step holds the buffers it was captured with.
    for (auto& gx : h->sweep_graph)
        if (gx) {
            cudaGraphExecDestroy(gx);
            gx = nullptr;
        }
    const Fields fa{{h->u[0], h->u[1], h->u[2]}, {h->i[0], h->i[1], h->i[2]}};
    const Fields fb{{h->u2[0], h->u2[1], h->u2[2]}, {h->i2[0], h->i2[1], h->i2[2]}};
    Coeffs c;
    for (int l = 0; l < 12; ++l) c.c[l] = h->co[l];
    ems_status st = serial_pre_e(h, fa);
    if (st) return st;
    FusedParams P = h->fp;
    for (int a = 0; a < 3; ++a) {
        P.uo[a] = fa.u[a];
        P.io[a] = fa.i[a];
        P.un[a] = fb.u[a];
        P.in[a] = fb.i[a];
    }
    for (size_t q = 0; q < h->psi_h.size(); ++q) {
        FSlab& fs = P.slab[0][h->psi_h_at[q].first][h->psi_h_at[q].second];
        fs.psi_old = fs.psi_new = h->psi_h[q].first;
    }
    P.partials = h->qpartials;
    P.skip = h->ibox;
    const bool oe = h->oe_curl;
    // The split kernels over the nodes outside the box only: the planes
    // before and after it, then in its planes the rows before and after it
    // and the quads of its rows before and after it.
    const InteriorBox& B = h->ibox;
    const uint32_t qpr = g.pitch >> 2, zl = B.lo[2] / 4u, zr = B.hi[2] / 4u, nzl = zl + (qpr - zr);
    auto outer = [&](auto launch) {
        const uint32_t bx = split_blocks_x(g);
        P.qmap = QuadMap{};
        if (B.lo[0]) launch(dim3(bx, B.lo[0], 1), 0u);
        if (g.nx > B.hi[0]) launch(dim3(bx, g.nx - B.hi[0], 1), B.hi[0]);
        const uint32_t xn = B.hi[0] - B.lo[0];
        P.qmap = QuadMap{0u, 0u, 0u, 1u, 0u, 0u, B.lo[1] * qpr};
        if (P.qmap.count) launch(dim3(blocks_for(P.qmap.count, kSplitThreads), xn, 1), B.lo[0]);
        P.qmap = QuadMap{0u, B.hi[1] * qpr, 0u, 1u, 0u, 0u, (g.ny - B.hi[1]) * qpr};
        if (P.qmap.count) launch(dim3(blocks_for(P.qmap.count, kSplitThreads), xn, 1), B.lo[0]);
        P.qmap = QuadMap{1u, 0u, B.lo[1], nzl, zl, zr, (B.hi[1] - B.lo[1]) * nzl};
        if (P.qmap.count) launch(dim3(blocks_for(P.qmap.count, kSplitThreads), xn, 1), B.lo[0]);
        P.qmap = QuadMap{};
    };
    // The electric saved values u^n, unless the pole kernel kept them.
    for (auto& op : h->ops)
        if (op.kind == EMS_OP_POLES && op.poles.e.n_edges && !(h->fold_prev[0] && h->prev_e_valid)) {
            k_poles_capture<<<blocks_for(op.poles.e.n_edges, 256), 256, 0, s>>>(fa, op.poles.e, true);
            ++h->launches;
        }
    cudaEvent_t ev = h->prof_begin();
    outer([&](dim3 grd, uint32_t i0) {
        if (oe) k_split_h<false, true><<<grd, kSplitThreads, 0, s>>>(P, i0);
        else k_split_h<false><<<grd, kSplitThreads, 0, s>>>(P, i0);
        ++h->launches;
    });
    h->prof_end(0, ev);
    for (auto& op : h->ops)
        if (op.kind == EMS_OP_CPML)
            if (const uint32_t nb = shell_blocks(h->shell[0])) {
                k_shell<0><<<nb, 32 * kShellWarps, 0, s>>>(P, h->shell[0]);
                ++h->launches;
            }
    uint32_t ib[3];
    interior_blocks(h->ibox, h->interior_planes, ib);
    const dim3 igrd(ib[0], ib[1], ib[2]);
    ev = h->prof_begin();
    if (oe) k_interior<true><<<igrd, 32 * kInWarps, 0, s>>>(P, h->ibox, h->interior_planes);
    else k_interior<false><<<igrd, 32 * kInWarps, 0, s>>>(P, h->ibox, h->interior_planes);
    h->prof_end(2, ev);
    ++h->launches;
    ev = h->prof_begin();
    outer([&](dim3 grd, uint32_t i0) {
        if (oe) k_split_e<true><<<grd, kSplitThreads, 0, s>>>(P, i0);
        else k_split_e<<<grd, kSplitThreads, 0, s>>>(P, i0);
        ++h->launches;
    });
    h->prof_end(1, ev);
    for (auto& op : h->ops) {
        if (op.kind == EMS_OP_CPML) {
            if (const uint32_t nb = shell_blocks(h->shell[1])) {
                k_shell<1><<<nb, 32 * kShellWarps, 0, s>>>(P, h->shell[1]);
                ++h->launches;
            }
        } else if (op.kind == EMS_OP_POLES && op.poles.e.n_edges) {
            k_poles_blocks<<<blocks_for(op.poles.e.n_edges, kPoleBlock), kPoleBlock, 0, s>>>(
                fb, c, op.poles.e, P.runs, P.sets, h->run_of[0], 1, h->dt, h->fold_prev[0] ? 1 : 0, 0u,
                (uint32_t)op.poles.e.n_edges);
            ++h->launches;
        }
    }
    h->prev_e_valid = h->fold_prev[0];
    for (int a = 0; a < 3; ++a) {
        std::swap(h->u[a], h->u2[a]);
        std::swap(h->i[a], h->i2[a]);
    }
    st = serial_post_h(h, fb);
    if (st) return st;
    st = serial_post_e(h, fb);
    if (st) return st;
    ++h->step;
    return EMS_OK;
}

// The tile shapes of the marching kernel: rows per block and ring stages.
struct MarchShape {
    uint32_t rows, stages;
};
constexpr MarchShape kMarchShapes[] = {{7, 3}, {15, 3}, {8, 4}, {3, 4}};
constexpr int kNumMarchShapes = (int)(sizeof(kMarchShapes) / sizeof(kMarchShapes[0]));

// cuTensorMapEncodeTiled from the driver (through the runtime, so the
// library needs no link to libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// The six tensor maps of the old fields of buffer (u, i) for tiles of R rows:
// extents (pitch, ny, nx), boxes (kMW, R + 2, 1) and (kMW, R + 1, 1),
// out-of-grid entries read as zero.
static ems_status encode_march_maps(ems_gpu* h, float* const u[3], float* const i[3], uint32_t R, MarchMaps& M) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return fail(h, EMS_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const Grid& g = h->g;
    const cuuint64_t dims[3] = {g.pitch, g.ny, g.nx};
    const cuuint64_t strides[2] = {(cuuint64_t)g.pitch * 4, (cuuint64_t)g.ny * g.pitch * 4};
    const cuuint32_t ubox[3] = {kMW, R + 2, 1}, ibox[3] = {kMW, R + 1, 1}, es[3] = {1, 1, 1};
    for (int c = 0; c < 3; ++c) {
        for (int side = 0; side < 2; ++side) {
            CUresult r = enc(side ? &M.i[c] : &M.u[c], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, side ? (void*)i[c] : (void*)u[c],
                             dims, strides, side ? ibox : ubox, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return fail(h, EMS_ERR_CUDA, "cuTensorMapEncodeTiled failed");
        }
    }
    return EMS_OK;
}

template <uint32_t R, uint32_t S>
static ems_status launch_march(ems_gpu* h, const FusedParams& P, const MarchMaps& M, bool oe) {
    const size_t smem = MarchLayout<R>::bytes(S);
    uint32_t nb[3];
    march_blocks(h->g, R, h->march_planes, nb);
    const dim3 grd(nb[0], nb[1], nb[2]);
    if (oe) {
        cudaFuncSetAttribute(k_march<R, S, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_march<R, S, true><<<grd, 32 * (R + 1), smem, h->stream>>>(P, M, h->march_planes);
    } else {
        cudaFuncSetAttribute(k_march<R, S, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_march<R, S, false><<<grd, 32 * (R + 1), smem, h->stream>>>(P, M, h->march_planes);
    }
    return check(h, cudaGetLastError(), "marching kernel");
}

// One step through the marching schedule (march.cuh): the old fields in one
// buffer, the one-pass kernel (both updates and both CPML corrections over
// the whole grid) writing the new ones into the other, the electric poles on
// the new fields (u^n from the old buffer), then the serial hooks on the new
// fields. Steps that record the energy run the split schedule in place.
ems_status run_step_march(ems_gpu* h) {
    const Grid& g = h->g;
    cudaStream_t s = h->stream;
    if (!h->u2[0]) {
        // The second buffers start as copies: entries no kernel writes
        // (row padding) then agree in both.
        for (int a = 0; a < 3; ++a) {
            h->u2[a] = h->alloc<float>(g.np);
            h->i2[a] = h->alloc<float>(g.np);
            if (!h->u2[a] || !h->i2[a]) return fail(h, EMS_ERR_NOMEM, "second field buffers");
            if (check(h, cudaMemcpyAsync(h->u2[a], h->u[a], g.np * sizeof(float), cudaMemcpyDeviceToDevice, s),
                      "second field buffers") ||
                check(h, cudaMemcpyAsync(h->i2[a], h->i[a], g.np * sizeof(float), cudaMemcpyDeviceToDevice, s),
                      "second field buffers"))
                return EMS_ERR_CUDA;
        }
    }
    // The H-side ψ in two buffers: a node's H value is computed again by the
    // blocks next to its own, which must read the old ψ.
    for (size_t q = 0; q < h->psi_h.size(); ++q) {
        if (h->psi_h[q].second) continue;
        const FSlab& fs = h->fp.slab[0][h->psi_h_at[q].first][h->psi_h_at[q].second];
        const size_t len = (size_t)(fs.hi[0] - fs.lo[0]) * (fs.hi[1] - fs.lo[1]) * (fs.hi[2] - fs.lo[2]);
        float* other = h->alloc<float>(len);
        if (!other) return fail(h, EMS_ERR_NOMEM, "CPML state");
        if (check(h, cudaMemcpyAsync(other, h->psi_h[q].first, len * sizeof(float), cudaMemcpyDeviceToDevice, s),
                  "CPML state"))
            return EMS_ERR_CUDA;
        h->psi_h[q].second = other;
    }
    if (!h->status) {
        h->status = h->alloc<int>(1);
        if (!h->status) return fail(h, EMS_ERR_NOMEM, "status flag");
    }
    for (auto& gx : h->sweep_graph)
        if (gx) {
            cudaGraphExecDestroy(gx);
            gx = nullptr;
        }
    const Fields fa{{h->u[0], h->u[1], h->u[2]}, {h->i[0], h->i[1], h->i[2]}};
    const Fields fb{{h->u2[0], h->u2[1], h->u2[2]}, {h->i2[0], h->i2[1], h->i2[2]}};
    Coeffs c;
    for (int l = 0; l < 12; ++l) c.c[l] = h->co[l];
    ems_status st = serial_pre_e(h, fa);
    if (st) return st;
    FusedParams P = h->fp;
    for (int a = 0; a < 3; ++a) {
        P.uo[a] = fa.u[a];
        P.io[a] = fa.i[a];
        P.un[a] = fb.u[a];
        P.in[a] = fb.i[a];
    }
    for (size_t q = 0; q < h->psi_h.size(); ++q) {
        FSlab& fs = P.slab[0][h->psi_h_at[q].first][h->psi_h_at[q].second];
        fs.psi_old = h->psi_h[q].first;
        fs.psi_new = h->psi_h[q].second;
    }
    P.status = h->status;
    P.diverged = h->diverged;
    P.wait_ns = h->test_wait_ns;
    P.test_extra_tx = h->test_wait_ns ? 16u : 0u;
    h->test_wait_ns = 0;
    const int shape = h->march_shape;
    const uint32_t R = kMarchShapes[shape].rows;
    auto& ms = h->march_maps[h->u[0] == h->march_maps[0].key ? 0 : 1];
    if (ms.key != h->u[0] || ms.shape != shape) {
        st = encode_march_maps(h, h->u, h->i, R, ms.m);
        if (st) return st;
        ms.key = h->u[0];
        ms.shape = shape;
    }
    cudaEvent_t ev = h->prof_begin();
    const bool oe = h->oe_curl;
    switch (shape) {
    case 0: st = launch_march<7, 3>(h, P, ms.m, oe); break;
    case 1: st = launch_march<15, 3>(h, P, ms.m, oe); break;
    case 2: st = launch_march<8, 4>(h, P, ms.m, oe); break;
    default: st = launch_march<3, 4>(h, P, ms.m, oe); break;
    }
    h->prof_end(2, ev);
    ++h->launches;
    if (st) return st;
    // The electric poles on the new fields, u^n read from the old buffer.
    for (auto& op : h->ops)
        if (op.kind == EMS_OP_POLES && op.poles.e.n_edges) {
            k_poles_blocks<true><<<blocks_for(op.poles.e.n_edges, kPoleBlock), kPoleBlock, 0, s>>>(
                fb, c, op.poles.e, P.runs, P.sets, h->run_of[0], 1, h->dt, 0, 0u, (uint32_t)op.poles.e.n_edges, fa);
            ++h->launches;
        }
    // The saved values the split schedule keeps are not current after it.
    h->prev_e_valid = false;
    for (int a = 0; a < 3; ++a) {
        std::swap(h->u[a], h->u2[a]);
        std::swap(h->i[a], h->i2[a]);
    }
    h->swap_psi_h();
    st = serial_post_h(h, fb);
    if (st) return st;
    st = serial_post_e(h, fb);
    if (st) return st;
    ++h->step;
    return EMS_OK;
}

// One step through the per-operator kernels; energy: record the
// invariant's field part into d_energy[0].
// One update of the split schedule with the row CPML (h->rowc): the CPML
// variant of the update kernel over every quad that holds a layer node of
// the side (the x-layer planes whole; in the other planes the y-layer rows
// whole and, of the rows between, the quads at both ends that reach into
// the z layers), the plain kernel over the rest. Quads are numbered row by
// row within a plane: QuadMap mode 0 takes a range of a plane's quads, mode
// 1 the quads [0, zl) and [zr, ...) of each of a range of rows (zl = 0: the
// quads from zr on).
template <int SIDE>
void launch_split_rows(ems_gpu* h, const FusedParams& P0, bool oe, cudaStream_t s) {
    const Grid& g = h->g;
    const RowCpml& R = h->rowc;
    const uint32_t qpr = g.pitch >> 2, qrow = (g.nz + 3u) / 4u;
    const uint32_t xl = R.lo[SIDE][0], xh = R.hi[SIDE][0], yl = R.lo[SIDE][1], yh = R.hi[SIDE][1];
    const uint32_t zl = (R.lo[SIDE][2] + 3u) / 4u, zr = std::max(zl, R.hi[SIDE][2] / 4u);
    auto go = [&](bool cpml, uint32_t i0, uint32_t planes, const QuadMap& M) {
        if (!planes || !M.count) return;
        FusedParams P = P0;
        P.qmap = M;
        const dim3 grd(blocks_for(M.count, kSplitThreads), planes, 1);
        if (SIDE == 0) {
            if (cpml && oe) k_split_h<false, true, true><<<grd, kSplitThreads, 0, s>>>(P, i0);
            else if (cpml) k_split_h<false, false, true><<<grd, kSplitThreads, 0, s>>>(P, i0);
            else if (oe) k_split_h<false, true><<<grd, kSplitThreads, 0, s>>>(P, i0);
            else k_split_h<false><<<grd, kSplitThreads, 0, s>>>(P, i0);
        } else {
            if (cpml && oe) k_split_e<true, true><<<grd, kSplitThreads, 0, s>>>(P, i0);
            else if (cpml) k_split_e<false, true><<<grd, kSplitThreads, 0, s>>>(P, i0);
            else if (oe) k_split_e<true><<<grd, kSplitThreads, 0, s>>>(P, i0);
            else k_split_e<<<grd, kSplitThreads, 0, s>>>(P, i0);
        }
        ++h->launches;
    };
    const uint32_t mid = xh > xl ? xh - xl : 0u, rows = yh > yl ? yh - yl : 0u;
    const uint32_t ends = zl + (qrow > zr ? qrow - zr : 0u), inner = zr - zl;
    go(true, 0u, xl, QuadMap{0u, 0u, 0u, 0u, 0u, 0u, g.ny * qpr});
    go(true, xh, g.nx - xh, QuadMap{0u, 0u, 0u, 0u, 0u, 0u, g.ny * qpr});
    go(true, xl, mid, QuadMap{0u, 0u, 0u, 0u, 0u, 0u, yl * qpr});
    go(true, xl, mid, QuadMap{0u, yh * qpr, 0u, 0u, 0u, 0u, (g.ny - yh) * qpr});
    go(true, xl, mid, QuadMap{1u, 0u, yl, ends, zl, zr, rows * ends});
    go(false, xl, mid, QuadMap{1u, 0u, yl, inner, 0u, zl, rows * inner});
}

ems_status run_step(ems_gpu* h, bool energy) {
    const int sch = active_schedule(h);
    // Only the per-operator, split and sweep steps keep the electric saved values.
    if (sch != 4 && sch != 5 && sch != 6 && sch != 7) h->prev_e_valid = false;
    if (sch == 6 && !energy) return run_step_interior(h);
    if (sch == 7 && !energy) return run_step_march(h);
    if (sch == 2) return run_step_fused(h, energy);
    if (sch == 3) return run_step_two(h, energy);
    if (sch == 5) return run_step_sweep(h, energy);
    // Schedules 1 and 4 share the hook sequence; split (4) runs the table
    // kernels of split.cuh for the updates and one shell kernel per CPML side.
    const bool split = sch == 4 || sch == 6 || sch == 7;
    const Grid& g = h->g;
    cudaStream_t s = h->stream;
    Fields f{{h->u[0], h->u[1], h->u[2]}, {h->i[0], h->i[1], h->i[2]}};
    Coeffs c;
    for (int l = 0; l < 12; ++l) c.c[l] = h->co[l];
    FusedParams P;
    if (split) {
        P = h->fp;
        for (int a = 0; a < 3; ++a) {
            P.uo[a] = P.un[a] = h->u[a];
            P.io[a] = P.in[a] = h->i[a];
        }
        for (size_t q = 0; q < h->psi_h.size(); ++q) {
            FSlab& fs = P.slab[0][h->psi_h_at[q].first][h->psi_h_at[q].second];
            fs.psi_old = fs.psi_new = h->psi_h[q].first;
        }
        P.partials = h->qpartials;
    }
    dim3 blk(kRowThreads, 1, 1);
    dim3 grd(blocks_for(g.nz, kRowThreads), (unsigned)g.ny, (unsigned)g.nx);
    const dim3 qgrd(split_blocks_x(g), g.nx, 1);
    cudaEvent_t ev = h->prof_begin();
    const bool oe = h->oe_curl;
    // The row CPML: split schedule, steps without energy.
    const bool rows = sch == 4 && !energy && h->rowc.ok && h->row_cpml_on;
    if (rows) {
        launch_split_rows<0>(h, P, oe, s);
        --h->launches;  // counted per launch inside; one is added below
    } else if (split) {
        if (energy) {
            if (oe) k_split_h<true, true><<<qgrd, kSplitThreads, 0, s>>>(P, 0u);
            else k_split_h<true><<<qgrd, kSplitThreads, 0, s>>>(P, 0u);
        } else {
            if (oe) k_split_h<false, true><<<qgrd, kSplitThreads, 0, s>>>(P, 0u);
            else k_split_h<false><<<qgrd, kSplitThreads, 0, s>>>(P, 0u);
        }
    } else if (energy) {
        if (oe) k_update_h<true, true><<<grd, blk, 0, s>>>(g, f, c, h->partials);
        else k_update_h<true><<<grd, blk, 0, s>>>(g, f, c, h->partials);
    } else {
        if (oe) k_update_h<false, true><<<grd, blk, 0, s>>>(g, f, c, nullptr);
        else k_update_h<false><<<grd, blk, 0, s>>>(g, f, c, nullptr);
    }
    h->prof_end(0, ev);
    ++h->launches;
    if (energy) {
        if (split) {
            k_reduce_partials<<<1, 1024, 0, s>>>(h->qpartials, h->n_qpartials, h->d_energy);
        } else {
            k_reduce_partials<<<1, 1024, 0, s>>>(h->partials, h->n_partials, h->d_energy);
        }
        ++h->launches;
    }
    // Slab hooks after the H update, in registration order.
    for (auto& op : h->ops) {
        if (op.kind == EMS_OP_CPML && split) {
            if (const uint32_t nb = rows ? 0u : shell_blocks(h->shell[0])) {
                k_shell<0><<<nb, 32 * kShellWarps, 0, s>>>(P, h->shell[0]);
                ++h->launches;
            }
        } else if (op.kind == EMS_OP_CPML) {
            for (const SlabDev& sd : op.cpml) {
                if (sd.e_side) continue;
                dim3 sg(blocks_for(sd.hi[2] - sd.lo[2], 64), (unsigned)(sd.hi[1] - sd.lo[1]), (unsigned)(sd.hi[0] - sd.lo[0]));
                k_cpml<false><<<sg, 64, 0, s>>>(g, f, c, sd);
                ++h->launches;
            }
        } else if (op.kind == EMS_OP_POLES) {
            if (op.poles.h.n_edges && split) {
                k_poles_blocks<<<blocks_for(op.poles.h.n_edges, kPoleBlock), kPoleBlock, 0, s>>>(
                    f, c, op.poles.h, P.runs_h, P.sets_h, h->run_of[1], 0, h->dt, h->fold_prev[1] ? 1 : 0, 0u,
                    (uint32_t)op.poles.h.n_edges);
                ++h->launches;
            } else if (op.poles.h.n_edges) {
                k_poles_correct<<<blocks_for(op.poles.h.n_edges, 256), 256, 0, s>>>(g, f, c, op.poles.h, false, h->dt);
                ++h->launches;
            }
            if (op.poles.e.n_edges && !(split && h->fold_prev[0] && h->prev_e_valid)) {
                k_poles_capture<<<blocks_for(op.poles.e.n_edges, 256), 256, 0, s>>>(f, op.poles.e, true);
                ++h->launches;
            }
        } else if (op.kind == EMS_OP_UPML) {
            // upml.rs:443-454: E start values from u, then the H layer update.
            if (const uint32_t n = op.upml[0].n + op.upml[1].n) {
                k_upml_hook<<<blocks_for(n, 256), 256, 0, s>>>(f.u[0], f.u[1], f.u[2], op.upml[0], f.i[0], f.i[1],
                                                              f.i[2], op.upml[1]);
                ++h->launches;
            }
        }
    }
    ems_status st = serial_post_h(h, f);
    if (st) return st;
    st = serial_pre_e(h, f);
    if (st) return st;
    ev = h->prof_begin();
    if (rows) {
        launch_split_rows<1>(h, P, oe, s);
        --h->launches;
    } else if (split) {
        if (oe) k_split_e<true><<<qgrd, kSplitThreads, 0, s>>>(P, 0u);
        else k_split_e<<<qgrd, kSplitThreads, 0, s>>>(P, 0u);
    } else {
        if (oe) k_update_e<true><<<grd, blk, 0, s>>>(g, f, c);
        else k_update_e<<<grd, blk, 0, s>>>(g, f, c);
    }
    h->prof_end(1, ev);
    ++h->launches;
    for (auto& op : h->ops) {
        if (op.kind == EMS_OP_CPML && split) {
            if (const uint32_t nb = rows ? 0u : shell_blocks(h->shell[1])) {
                k_shell<1><<<nb, 32 * kShellWarps, 0, s>>>(P, h->shell[1]);
                ++h->launches;
            }
        } else if (op.kind == EMS_OP_CPML) {
            for (const SlabDev& sd : op.cpml) {
                if (!sd.e_side) continue;
                dim3 sg(blocks_for(sd.hi[2] - sd.lo[2], 64), (unsigned)(sd.hi[1] - sd.lo[1]), (unsigned)(sd.hi[0] - sd.lo[0]));
                k_cpml<true><<<sg, 64, 0, s>>>(g, f, c, sd);
                ++h->launches;
            }
        } else if (op.kind == EMS_OP_POLES) {
            if (op.poles.e.n_edges && split) {
                k_poles_blocks<<<blocks_for(op.poles.e.n_edges, kPoleBlock), kPoleBlock, 0, s>>>(
                    f, c, op.poles.e, P.runs, P.sets, h->run_of[0], 1, h->dt, h->fold_prev[0] ? 1 : 0, 0u,
                    (uint32_t)op.poles.e.n_edges);
                ++h->launches;
            } else if (op.poles.e.n_edges) {
                k_poles_correct<<<blocks_for(op.poles.e.n_edges, 256), 256, 0, s>>>(g, f, c, op.poles.e, true, h->dt);
                ++h->launches;
            }
            if (op.poles.h.n_edges && !(split && h->fold_prev[1])) {
                k_poles_capture<<<blocks_for(op.poles.h.n_edges, 256), 256, 0, s>>>(f, op.poles.h, false);
                ++h->launches;
            }
        } else if (op.kind == EMS_OP_UPML) {
            // upml.rs:456-464: H start values from i, then the E layer update.
            if (const uint32_t n = op.upml[0].n + op.upml[1].n) {
                k_upml_hook<<<blocks_for(n, 256), 256, 0, s>>>(f.i[0], f.i[1], f.i[2], op.upml[1], f.u[0], f.u[1],
                                                              f.u[2], op.upml[0]);
                ++h->launches;
            }
        }
    }
    st = serial_post_e(h, f);
    if (st) return st;
    if (split) h->prev_e_valid = h->fold_prev[0];
    ++h->step;
    return EMS_OK;
}

// Uploads a conducting-sheet table (include/ems_gpu.h, ems_sheet) after
// checking every index it holds, and builds the post_h table: per dual
// edge with a nonzero correction, the (edge, corr) pairs in edge order.
ems_status setup_sheet(ems_gpu* h, const ems_sheet* t, ems_gpu::Op& op) {
    auto fail = [](const char* why) {
        std::fprintf(stderr, "ems_gpu: conducting sheet: %s\n", why);
        return EMS_ERR_INVALID;
    };
    const Grid& g = h->g;
    const size_t ne = t->n_edges, nc = t->n_couplings;
    if (ne >= (1ull << 31) || nc >= (1ull << 31) || t->n_konst >= (1ull << 31) || t->n_a >= (1ull << 31))
        return fail("table too large");
    if (ne && (!t->axis || !t->node || !t->nn || !t->konst0 || !t->a0 || !t->coupling_end || !t->c_edge))
        return fail("missing arrays");
    if (nc && (!t->c_axis || !t->c_node || !t->w_up || !t->w_dn || !t->corr || !t->ecorr)) return fail("missing arrays");
    if ((t->n_konst && (!t->two_c || !t->cp || !t->inv_den)) || (t->n_a && !t->a)) return fail("missing arrays");
    std::vector<uint32_t> node(ne), n0(ne), l0(ne), c0(ne + 1, 0), cnode(nc);
    std::vector<uint64_t> keys(ne);
    uint64_t nodes_total = 0, layers_total = 0;
    uint32_t c = 0;
    for (size_t e = 0; e < ne; ++e) {
        const uint32_t nn = t->nn[e], end = t->coupling_end[e];
        if (t->axis[e] > 2 || t->node[e] >= g.n || nn < 2 || end < c || end > nc ||
            (uint64_t)t->konst0[e] + nn > t->n_konst || (uint64_t)t->a0[e] + nn - 1 > t->n_a)
            return fail("edge entry out of range");
        node[e] = dev_index(g, t->node[e]);
        keys[e] = t->node[e] * 3 + t->axis[e];
        n0[e] = (uint32_t)nodes_total;
        l0[e] = (uint32_t)layers_total;
        nodes_total += nn;
        layers_total += nn - 1;
        if (nodes_total >= (1ull << 31)) return fail("ladders too large");
        c = end;
        c0[e + 1] = end;
    }
    if (c != nc) return fail("couplings not covered by the edges");
    // Each sheet edge is written by one thread of post_e: no edge twice.
    std::sort(keys.begin(), keys.end());
    if (std::adjacent_find(keys.begin(), keys.end()) != keys.end()) return fail("an edge listed twice");
    std::unordered_map<uint64_t, uint32_t> tix;
    std::vector<std::vector<std::pair<uint32_t, double>>> tlist;
    std::vector<uint8_t> taxis;
    std::vector<uint32_t> tnode;
    for (size_t e = 0; e < ne; ++e)
        for (uint32_t q = c0[e]; q < c0[e + 1]; ++q) {
            if (t->c_axis[q] > 2 || t->c_node[q] >= g.n) return fail("coupling out of range");
            cnode[q] = dev_index(g, t->c_node[q]);
            if (t->corr[q] == 0.0) continue;
            const uint64_t key = t->c_node[q] * 3 + t->c_axis[q];
            auto it = tix.find(key);
            if (it == tix.end()) {
                it = tix.emplace(key, (uint32_t)tlist.size()).first;
                tlist.emplace_back();
                taxis.push_back(t->c_axis[q]);
                tnode.push_back(cnode[q]);
            }
            tlist[it->second].emplace_back((uint32_t)e, t->corr[q]);
        }
    std::vector<uint32_t> t0(1, 0), tedge;
    std::vector<double> tcorr;
    for (const auto& l : tlist) {
        for (const auto& [e, k] : l) {
            tedge.push_back(e);
            tcorr.push_back(k);
        }
        t0.push_back((uint32_t)tedge.size());
    }
    SheetDevT& D = op.sheet;
    D.n_edges = (uint32_t)ne;
    D.n_targets = (uint32_t)tlist.size();
    op.sheet_nodes = nodes_total;
    op.sheet_layers = layers_total;
    if (!ne) return EMS_OK;
    D.axis = h->upload(t->axis, ne);
    D.node = h->upload(node.data(), ne);
    D.nn = h->upload(t->nn, ne);
    D.k0 = h->upload(t->konst0, ne);
    D.a0 = h->upload(t->a0, ne);
    D.n0 = h->upload(n0.data(), ne);
    D.l0 = h->upload(l0.data(), ne);
    D.c0 = h->upload(c0.data(), ne + 1);
    D.c_edge = h->upload(t->c_edge, ne);
    D.c_axis = h->upload(t->c_axis, nc);
    D.c_node = h->upload(cnode.data(), nc);
    D.w_up = h->upload(t->w_up, nc);
    D.w_dn = h->upload(t->w_dn, nc);
    D.ecorr = h->upload(t->ecorr, nc);
    D.two_c = h->upload(t->two_c, t->n_konst);
    D.cp = h->upload(t->cp, t->n_konst);
    D.inv_den = h->upload(t->inv_den, t->n_konst);
    D.a = h->upload(t->a, t->n_a);
    D.u = h->alloc<double>(nodes_total);
    D.h = h->alloc<double>(layers_total);
    D.x = h->alloc<double>(nodes_total);
    D.wcorr = h->alloc<double>(ne);
    D.t_axis = h->upload(taxis.data(), taxis.size());
    D.t_node = h->upload(tnode.data(), tnode.size());
    D.t0 = h->upload(t0.data(), t0.size());
    D.t_edge = h->upload(tedge.data(), tedge.size());
    D.t_corr = h->upload(tcorr.data(), tcorr.size());
    if (!D.axis || !D.node || !D.nn || !D.k0 || !D.a0 || !D.n0 || !D.l0 || !D.c0 || !D.c_edge || !D.c_axis ||
        !D.c_node || !D.w_up || !D.w_dn || !D.ecorr || !D.two_c || !D.cp || !D.inv_den || !D.a || !D.u || !D.h ||
        !D.x || !D.wcorr || !D.t_axis || !D.t_node || !D.t0 || !D.t_edge || !D.t_corr)
        return EMS_ERR_NOMEM;
    return EMS_OK;
}

// Serial post_h hooks in registration order: magnetic sources, conducting
// sheets, current probes.
ems_status serial_post_h(ems_gpu* h, const Fields& f) {
    cudaStream_t s = h->stream;
    for (auto& op : h->ops) {
        if (op.kind == EMS_OP_SOURCE && (op.source.kind == EMS_SOFT_H || op.source.kind == EMS_HARD_H)) {
            const ems_gpu::SourceDev& sd = op.source;
            float a = h->step < sd.amp.size() ? sd.amp[h->step] : 0.0f;
            bool hard = sd.kind == EMS_HARD_H;
            if (!hard && a == 0.0f) continue;
            k_source<<<blocks_for(sd.n, 256), 256, 0, s>>>(f.i[0], f.i[1], f.i[2], sd.axis, sd.node, sd.weight, sd.n, a, hard);
            ++h->launches;
        } else if (op.kind == EMS_OP_SHEET && op.sheet.n_edges) {
            const SheetDevT& sd = op.sheet;
            k_sheet_post_h<<<blocks_for(sd.n_targets + sd.n_edges, 256), 256, 0, s>>>(f.u[0], f.u[1], f.u[2], f.i[0],
                                                                                      f.i[1], f.i[2], sd);
            ++h->launches;
        } else if (op.kind == EMS_OP_PROBE && op.probe.quantity == EMS_PROBE_CURRENT && h->step % op.probe.interval == 0) {
            ems_gpu::ProbeDev& p = op.probe;
            ems_status st = grow(h, &p.values, p.count, &p.cap, p.count + 1);
            if (st) return st;
            k_probe<<<1, 32, 0, s>>>(f.i[0], f.i[1], f.i[2], p.d, p.values + p.count);
            ++h->launches;
            ++p.count;
        }
    }
    return EMS_OK;
}

// pre_e: lumped elements and Mur boundaries save u^n.
ems_status serial_pre_e(ems_gpu* h, const Fields& f) {
    for (auto& op : h->ops) {
        if (op.kind == EMS_OP_LUMPED && (op.lumped.record || op.lumped.has_branch)) {
            k_lumped_pre_e<<<blocks_for(op.lumped.n_edges, 128), 128, 0, h->stream>>>(f.u[op.lumped.axis], op.lumped.d);
            ++h->launches;
        } else if (op.kind == EMS_OP_MUR && op.mur.n) {
            k_mur_save<<<blocks_for(op.mur.n, 256), 256, 0, h->stream>>>(f.u[0], f.u[1], f.u[2], op.mur);
            ++h->launches;
        }
    }
    return EMS_OK;
}

// Serial post_e hooks in registration order: lumped elements, Mur
// boundaries, electric sources, conducting sheets, voltage probes.
ems_status serial_post_e(ems_gpu* h, const Fields& f) {
    cudaStream_t s = h->stream;
    for (auto& op : h->ops) {
        if (op.kind == EMS_OP_MUR) {
            const MurDevT& m = op.mur;
            if (m.n_edges) {
                k_mur_update<<<blocks_for(m.n_edges, 256), 256, 0, s>>>(f.u[0], f.u[1], f.u[2], m, h->step, 0u, m.n_edges);
                ++h->launches;
            }
            if (m.n > m.n_edges) {
                k_mur_update<<<blocks_for(m.n - m.n_edges, 256), 256, 0, s>>>(f.u[0], f.u[1], f.u[2], m, h->step,
                                                                               m.n_edges, m.n);
                ++h->launches;
            }
        } else if (op.kind == EMS_OP_LUMPED) {
            ems_gpu::LumpedDev& L = op.lumped;
            double val = (L.has_src && h->step < L.amp.size()) ? L.amp[h->step] : 0.0;
            bool active = L.has_src && val != 0.0;
            size_t idx = L.count;
            if (L.record) {
                ems_status st = grow(h, &L.rec, L.count, &L.cap, L.count + 1);
                if (st) return st;
                if (L.columns) {
                    st = grow(h, &L.pv, L.count, &L.vcap, L.count + 1);
                    if (st) return st;
                    st = grow(h, &L.pi, L.count, &L.icap, L.count + 1);
                    if (st) return st;
                }
            }
            k_lumped_post_e<<<1, 256, 0, s>>>(f.u[L.axis], L.d, val, active ? 1 : 0, h->dt,
                                              L.record ? L.rec + idx : nullptr, L.columns ? L.pv + idx : nullptr,
                                              L.columns ? L.pi + idx : nullptr);
            ++h->launches;
            if (L.record) ++L.count;
        } else if (op.kind == EMS_OP_SOURCE && (op.source.kind == EMS_SOFT_E || op.source.kind == EMS_HARD_E)) {
            const ems_gpu::SourceDev& sd = op.source;
            float a = h->step < sd.amp.size() ? sd.amp[h->step] : 0.0f;
            bool hard = sd.kind == EMS_HARD_E;
            if (!hard && a == 0.0f) continue;
            k_source<<<blocks_for(sd.n, 256), 256, 0, s>>>(f.u[0], f.u[1], f.u[2], sd.axis, sd.node, sd.weight, sd.n, a, hard);
            ++h->launches;
        } else if (op.kind == EMS_OP_SHEET && op.sheet.n_edges) {
            const SheetDevT& sd = op.sheet;
            k_sheet_post_e<<<blocks_for(sd.n_edges, 128), 128, 0, s>>>(f.u[0], f.u[1], f.u[2], f.i[0], f.i[1], f.i[2], sd);
            ++h->launches;
        } else if (op.kind == EMS_OP_PROBE && op.probe.quantity == EMS_PROBE_VOLTAGE && h->step % op.probe.interval == 0) {
            ems_gpu::ProbeDev& p = op.probe;
            ems_status st = grow(h, &p.values, p.count, &p.cap, p.count + 1);
            if (st) return st;
            k_probe<<<1, 32, 0, s>>>(f.u[0], f.u[1], f.u[2], p.d, p.values + p.count);
            ++h->launches;
            ++p.count;
        }
    }
    return EMS_OK;
}

}  // namespace

extern "C" {

ems_status ems_gpu_create(const ems_engine_desc* d, int device, ems_gpu** out) {
    if (!d || !out) return EMS_ERR_INVALID;
    *out = nullptr;
    if (d->nodes[0] < 2 || d->nodes[1] < 2 || d->nodes[2] < 2 || !(d->dt > 0.0)) return EMS_ERR_INVALID;
    for (int l = 0; l < 12; ++l)
        if (!d->coeff[l]) return EMS_ERR_INVALID;
    auto h = std::make_unique<ems_gpu>();
    h->device = device;
    if (check(h.get(), cudaSetDevice(device), "cudaSetDevice")) return EMS_ERR_CUDA;
    if (check(h.get(), cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream")) return EMS_ERR_CUDA;
    Grid& g = h->g;
    g.nx = (uint32_t)d->nodes[0];
    g.ny = (uint32_t)d->nodes[1];
    g.nz = (uint32_t)d->nodes[2];
    g.pitch = (g.nz + 31u) & ~31u;
    g.n = (uint64_t)g.nx * g.ny * g.nz;
    g.np = (uint64_t)g.nx * g.ny * g.pitch;
    if (g.np >= (1ull << 32) - 1) return EMS_ERR_INVALID;  // 32-bit device indices
    h->dt = d->dt;
    const size_t np = g.np;
    for (int a = 0; a < 3; ++a) {
        h->u[a] = h->alloc<float>(np);
        h->i[a] = h->alloc<float>(np);
        if (!h->u[a] || !h->i[a]) return EMS_ERR_NOMEM;
    }
    // Coefficients: reference rows copied into padded rows (padding zero).
    for (int l = 0; l < 12; ++l) {
        h->co[l] = h->alloc<float>(np);
        if (!h->co[l]) return EMS_ERR_NOMEM;
        if (check(h.get(), cudaMemcpy2DAsync(h->co[l], g.pitch * sizeof(float), d->coeff[l], g.nz * sizeof(float),
                                             g.nz * sizeof(float), (size_t)g.nx * g.ny, cudaMemcpyHostToDevice, h->stream),
                  "coefficient upload"))
            return EMS_ERR_CUDA;
    }
    h->n_partials = (size_t)blocks_for(g.nz, kRowThreads) * g.ny * g.nx;
    h->partials = h->alloc<double>(h->n_partials);
    h->d_energy = h->alloc<double>(2);
    h->diverged = h->alloc<int>(1);
    if (!h->partials || !h->d_energy || !h->diverged) return EMS_ERR_NOMEM;
    if (check(h.get(), cudaMemsetAsync(h->diverged, 0, sizeof(int), h->stream), "divergence flag")) return EMS_ERR_CUDA;
    for (size_t k = 0; k < d->n_ops; ++k) {
        ems_gpu::Op op;
        op.kind = d->ops[k].kind;
        const void* t = d->ops[k].table;
        if (!t) return EMS_ERR_INVALID;
        switch (op.kind) {
        case EMS_OP_CPML: {
            const auto* c = (const ems_cpml*)t;
            for (size_t q = 0; q < c->n_slabs; ++q) {
                const ems_cpml_slab& s = c->slabs[q];
                SlabDev sd{};
                bool ok = s.comp >= 0 && s.comp < 3 && s.normal >= 0 && s.normal < 3 && s.other >= 0 && s.other < 3;
                for (int a = 0; ok && a < 3; ++a) ok = s.lo[a] <= s.hi[a] && s.hi[a] <= d->nodes[a];
                if (ok && !s.e_side) ok = s.hi[s.normal] < d->nodes[s.normal];  // reads node + 1 along normal
                if (!ok || !s.b || !s.a || !s.k) return EMS_ERR_INVALID;
                sd.e_side = s.e_side;
                sd.comp = s.comp;
                sd.normal = s.normal;
                sd.other = s.other;
                sd.sign = s.sign;
                for (int a = 0; a < 3; ++a) {
                    sd.lo[a] = (uint32_t)s.lo[a];
                    sd.hi[a] = (uint32_t)s.hi[a];
                }
                size_t depth = s.hi[s.normal] - s.lo[s.normal];
                size_t len = (size_t)(s.hi[0] - s.lo[0]) * (s.hi[1] - s.lo[1]) * (s.hi[2] - s.lo[2]);
                if (!len) continue;
                sd.b = h->upload(s.b, depth);
                sd.a = h->upload(s.a, depth);
                sd.k = h->upload(s.k, depth);
                sd.psi = h->alloc<float>(len);
                if (!sd.b || !sd.a || !sd.k || !sd.psi) return EMS_ERR_NOMEM;
                op.cpml.push_back(sd);
            }
            break;
        }
        case EMS_OP_POLES: {
            const auto* p = (const ems_poles*)t;
            ems_status st = make_side(h.get(), p->electric, op.poles.e);
            if (st) { std::fprintf(stderr, "ems_gpu: %s\n", h->err.c_str()); return st; }
            st = make_side(h.get(), p->magnetic, op.poles.h);
            if (st) { std::fprintf(stderr, "ems_gpu: %s\n", h->err.c_str()); return st; }
            break;
        }
        case EMS_OP_LUMPED: {
            const auto* l = (const ems_lumped*)t;
            auto& L = op.lumped;
            size_t ne = l->n_edges;
            if (l->axis < 0 || l->axis > 2 || !ne || !l->node || !l->cb || !l->g_src || ne > 4096) return EMS_ERR_INVALID;
            std::vector<uint32_t> node(ne);
            for (size_t e = 0; e < ne; ++e) {
                if (l->node[e] >= g.n) return EMS_ERR_INVALID;
                node[e] = dev_index(g, l->node[e]);
            }
            L.axis = l->axis;
            L.n_edges = ne;
            L.has_src = l->src_w != nullptr;
            L.has_branch = l->has_branch != 0;
            L.record = l->record != 0;
            L.columns = l->port_columns;
            if (L.columns && !L.record) return EMS_ERR_INVALID;
            if (L.has_src) L.amp.assign(l->src_amp, l->src_amp + l->n_src_amp);
            LumpedDevT& D = L.d;
            D.n = (uint32_t)ne;
            D.series = (double)(l->series ? l->series : 1);
            D.columns = (double)l->port_columns;
            D.src_in_branch = l->src_in_branch;
            D.has_branch = l->has_branch;
            D.record = l->record;
            D.node = h->upload(node.data(), ne);
            D.cb = h->upload(l->cb, ne);
            D.g_src = h->upload(l->g_src, ne);
            D.src_w = L.has_src ? h->upload(l->src_w, ne) : nullptr;
            if (L.has_branch) {
                if (!l->two_l_dt || !l->inv_c || !l->z) return EMS_ERR_INVALID;
                D.two_l_dt = h->upload(l->two_l_dt, ne);
                D.inv_c = h->upload(l->inv_c, ne);
                D.z = h->upload(l->z, ne);
            }
            if (L.record) {
                if (!l->rec_g || !l->rec_c) return EMS_ERR_INVALID;
                D.rec_g = h->upload(l->rec_g, ne);
                D.rec_c = h->upload(l->rec_c, ne);
            }
            D.openems_order = l->openems_order;
            if (l->oe_k) {
                if (!L.has_branch || !l->oe_vi || !l->openems_order) return EMS_ERR_INVALID;
                D.oe_k = h->upload(l->oe_k, ne);
                D.oe_vi = h->upload(l->oe_vi, ne);
                D.oe_s = h->alloc<float>(ne);
                if (!D.oe_k || !D.oe_vi || !D.oe_s) return EMS_ERR_NOMEM;
            }
            D.v = h->alloc<double>(ne);
            D.bj = h->alloc<double>(ne);
            D.bq = h->alloc<double>(ne);
            D.bu_prev = h->alloc<double>(ne);
            D.j_avg = h->alloc<double>(ne);
            D.ru_prev = h->alloc<double>(ne);
            if (!D.node || !D.cb || !D.g_src || !D.v || !D.bj || !D.bq || !D.bu_prev || !D.j_avg || !D.ru_prev)
                return EMS_ERR_NOMEM;
            break;
        }
        case EMS_OP_SOURCE: {
            const auto* sr = (const ems_source*)t;
            auto& S = op.source;
            if (sr->kind < 0 || sr->kind > 3) return EMS_ERR_INVALID;
            S.kind = sr->kind;
            S.n = sr->n_edges;
            std::vector<uint32_t> node(S.n);
            for (size_t e = 0; e < S.n; ++e) {
                if (sr->node[e] >= g.n || sr->axis[e] > 2) return EMS_ERR_INVALID;
                node[e] = dev_index(g, sr->node[e]);
            }
            // Edges must be distinct: the kernel updates them in parallel.
            std::vector<uint64_t> key(S.n);
            for (size_t e = 0; e < S.n; ++e) key[e] = sr->node[e] * 3 + sr->axis[e];
            std::sort(key.begin(), key.end());
            if (std::adjacent_find(key.begin(), key.end()) != key.end()) return EMS_ERR_INVALID;
            S.node = h->upload(node.data(), S.n);
            S.axis = h->upload(sr->axis, S.n);
            S.weight = h->upload(sr->weight, S.n);
            S.amp.assign(sr->amp, sr->amp + sr->n_amp);
            if (S.n && (!S.node || !S.axis || !S.weight)) return EMS_ERR_NOMEM;
            break;
        }
        case EMS_OP_PROBE: {
            const auto* pr = (const ems_probe*)t;
            auto& P = op.probe;
            if (pr->quantity < 0 || pr->quantity > 1) return EMS_ERR_INVALID;
            P.quantity = pr->quantity;
            P.interval = pr->interval ? pr->interval : 1;
            std::vector<uint32_t> node(pr->n_entries);
            for (size_t e = 0; e < pr->n_entries; ++e) {
                if (pr->node[e] >= g.n || pr->axis[e] > 2) return EMS_ERR_INVALID;
                node[e] = dev_index(g, pr->node[e]);
            }
            P.d.n = (uint32_t)pr->n_entries;
            P.d.f32_sum = pr->f32_sum;
            P.d.node = h->upload(node.data(), pr->n_entries);
            P.d.axis = h->upload(pr->axis, pr->n_entries);
            P.d.weight = h->upload(pr->weight, pr->n_entries);
            break;
        }
        case EMS_OP_UPML: {
            const auto* pm = (const ems_upml*)t;
            for (int sd = 0; sd < 2; ++sd) {
                const size_t n = pm->n[sd];
                UpmlSideDev& D = op.upml[sd];
                if (n >= (1ull << 31) || (n && (!pm->axis[sd] || !pm->node[sd] || !pm->co[sd]))) return EMS_ERR_INVALID;
                if (!n) continue;
                std::vector<uint32_t> node(n);
                for (size_t e = 0; e < n; ++e) {
                    if (pm->axis[sd][e] > 2 || pm->node[sd][e] >= g.n) return EMS_ERR_INVALID;
                    node[e] = dev_index(g, pm->node[sd][e]);
                }
                D.n = (uint32_t)n;
                D.axis = h->upload(pm->axis[sd], n);
                D.node = h->upload(node.data(), n);
                D.co = (const float4*)h->upload(pm->co[sd], 4 * n);
                D.f = h->alloc<float>(n);
                D.v = h->alloc<float>(n);
                if (!D.axis || !D.node || !D.co || !D.f || !D.v) return EMS_ERR_NOMEM;
            }
            h->has_upml = true;
            break;
        }
        case EMS_OP_MUR: {
            const auto* m = (const ems_mur*)t;
            MurDevT& M = op.mur;
            const size_t n = m->n;
            auto fail = [](ems_gpu*, ems_status st, const char* why) {
                std::fprintf(stderr, "ems_gpu: %s\n", why);
                return st;
            };
            if (m->n_edges > n || n >= (1ull << 31) || (n && (!m->axis || !m->node || !m->inner || !m->k)) ||
                (m->count_energy && n && !m->cap))
                return fail(h.get(), EMS_ERR_INVALID, "Mur boundary: inconsistent table");
            std::vector<uint32_t> node(n), inner(2 * n, 0);
            for (size_t e = 0; e < n; ++e) {
                const size_t nb = e < m->n_edges ? 1 : 2;
                if (m->axis[e] > 2 || m->node[e] >= g.n) return fail(h.get(), EMS_ERR_INVALID, "Mur boundary: entry out of range");
                node[e] = dev_index(g, m->node[e]);
                for (size_t q = 0; q < nb; ++q) {
                    if (m->inner[2 * e + q] >= g.n) return fail(h.get(), EMS_ERR_INVALID, "Mur boundary: entry out of range");
                    inner[2 * e + q] = dev_index(g, m->inner[2 * e + q]);
                }
            }
            // The entries of one launch run in parallel: within the face
            // edges (and within the shared edges) every entry is distinct
            // and none reads another's edge.
            for (int phase = 0; phase < 2; ++phase) {
                const size_t a0 = phase ? m->n_edges : 0, a1 = phase ? n : m->n_edges, nb = phase ? 2 : 1;
                std::vector<uint64_t> w, r;
                for (size_t e = a0; e < a1; ++e) {
                    w.push_back(m->node[e] * 3 + m->axis[e]);
                    for (size_t q = 0; q < nb; ++q) r.push_back(m->inner[2 * e + q] * 3 + m->axis[e]);
                }
                std::sort(w.begin(), w.end());
                if (std::adjacent_find(w.begin(), w.end()) != w.end())
                    return fail(h.get(), EMS_ERR_INVALID, "Mur boundary: an edge listed twice");
                for (uint64_t x : r)
                    if (std::binary_search(w.begin(), w.end(), x))
                        return fail(h.get(), EMS_ERR_INVALID, "Mur boundary: an edge reads another edge of its launch");
            }
            M.n = (uint32_t)n;
            M.n_edges = (uint32_t)m->n_edges;
            M.openems_order = m->openems_order != 0;
            M.openems_corners = m->openems_corners != 0;
            op.mur_energy = m->count_energy != 0 && n;
            if (n) {
                M.axis = h->upload(m->axis, n);
                M.node = h->upload(node.data(), n);
                M.inner = h->upload(inner.data(), 2 * n);
                M.k = h->upload(m->k, 2 * n);
                M.hold = m->hold ? h->upload(m->hold, n) : nullptr;
                M.cap = op.mur_energy ? h->upload(m->cap, n) : nullptr;
                M.saved = h->alloc<float>(3 * n);
                M.last = h->alloc<float>(n);
                if (!M.axis || !M.node || !M.inner || !M.k || !M.saved || !M.last || (m->hold && !M.hold) ||
                    (op.mur_energy && !M.cap))
                    return EMS_ERR_NOMEM;
            }
            break;
        }
        case EMS_OP_SHEET: {
            ems_status st = setup_sheet(h.get(), (const ems_sheet*)t, op);
            if (st) return st;
            break;
        }
        default:
            return EMS_ERR_INVALID;
        }
        h->ops.push_back(std::move(op));
    }
    {
        ems_status st = setup_fused(h.get(), d);
        if (st) return st;
    }
    if (check(h.get(), cudaStreamSynchronize(h->stream), "create")) return EMS_ERR_CUDA;
    *out = h.release();
    return EMS_OK;
}

ems_status ems_gpu_destroy(ems_gpu* h) {
    if (!h) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    for (auto& gx : h->sweep_graph)
        if (gx) cudaGraphExecDestroy(gx);
    h->prof_collect();
    for (cudaEvent_t e : h->ev_free) cudaEventDestroy(e);
    h->bufs.clear();
    cudaStreamDestroy(h->stream);
    delete h;
    return EMS_OK;
}

// Autotune cache: text lines "<key> <value> <ms>"; the last line of a key wins.
static bool tune_lookup(const std::string& path, const std::string& key, int* value) {
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return false;
    char line[512];
    bool found = false;
    while (std::fgets(line, sizeof line, f)) {
        std::string l(line);
        while (!l.empty() && (l.back() == '\n' || l.back() == ' ')) l.pop_back();
        const size_t p2 = l.rfind(' ');                                   // before <ms>
        if (p2 == std::string::npos || p2 == 0) continue;
        const size_t p1 = l.rfind(' ', p2 - 1);                           // before <value>
        if (p1 == std::string::npos || p1 != key.size() || l.compare(0, p1, key) != 0) continue;
        *value = std::atoi(l.c_str() + p1 + 1);
        found = true;
    }
    std::fclose(f);
    return found;
}

static void tune_record(const std::string& path, const std::string& key, int value, double ms) {
    FILE* f = std::fopen(path.c_str(), "a");
    if (!f) return;
    std::fprintf(f, "%s %d %.6f\n", key.c_str(), value, ms);
    std::fclose(f);
}

constexpr int kTuneSteps = 4;  // per candidate: one warm-up step and three timed

// One step of a tuning engine: the current candidate's schedule, timed.
static ems_status tune_step(ems_gpu* h) {
    auto& T = h->tune;
    h->schedule = T.cand[T.at];
    const bool timed = T.done > 0;
    if (timed) cudaEventRecord(T.e0, h->stream);
    ems_status st = run_step(h, false);
    if (st) return st;
    if (timed) {
        cudaEventRecord(T.e1, h->stream);
        cudaEventSynchronize(T.e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, T.e0, T.e1);
        T.ms[T.at] += ms;
    }
    if (++T.done == kTuneSteps) {
        T.done = 0;
        if (++T.at == T.cand.size()) {
            size_t best = 0;
            for (size_t q = 1; q < T.cand.size(); ++q)
                if (T.ms[q] < T.ms[best]) best = q;
            h->schedule = T.cand[best];
            tune_record(T.cache, T.key, T.cand[best], T.ms[best] / (kTuneSteps - 1));
            T.active = false;
            cudaEventDestroy(T.e0);
            cudaEventDestroy(T.e1);
        }
    }
    return EMS_OK;
}

// Samples state m (the state after m steps) into every dump that is due.
static ems_status dumps_sample(ems_gpu* h, uint64_t m, bool first) {
    for (auto& T : h->tdumps) {
        if (first == T.started) continue;
        T.started = true;
        if (m % T.interval) continue;
        const size_t n = (size_t)T.d.npts * 3;
        ems_status st = grow(h, &T.buf, T.used, &T.cap, T.used + n);
        if (st) return st;
        DumpDev d = T.d;
        for (int a = 0; a < 3; ++a) d.f[a] = T.field ? h->i[a] : h->u[a];
        k_snapshot<<<blocks_for(d.npts, 256), 256, 0, h->stream>>>(d, T.buf + T.used);
        ++h->launches;
        T.used += n;
        T.states.push_back(m);
    }
    for (auto& D : h->dumps) {
        if (first == D.started) continue;
        D.started = true;
        if (m % D.interval) continue;
        DumpDev d = D.d;
        for (int a = 0; a < 3; ++a) d.f[a] = D.field ? h->i[a] : h->u[a];
        k_dump<<<blocks_for(d.npts, 256), 256, 0, h->stream>>>(d, (double)m);
        ++h->launches;
    }
    return EMS_OK;
}

// One step with the dumps: the first sample of a new dump is the state the
// step starts from (src/engine/dump.rs Cursor::pre_h), then the state after
// every step (Cursor::post_e).
static ems_status step_dumped(ems_gpu* h, bool energy) {
    const bool any = !h->dumps.empty() || !h->tdumps.empty();
    ems_status st = any ? dumps_sample(h, h->step, true) : EMS_OK;
    if (st) return st;
    st = (!energy && h->tune.active) ? tune_step(h) : run_step(h, energy);
    if (st) return st;
    return any ? dumps_sample(h, h->step, false) : EMS_OK;
}

ems_status ems_gpu_run(ems_gpu* h, uint64_t n) {
    if (!h) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    for (uint64_t s = 0; s < n; ++s) {
        ems_status st = step_dumped(h, false);
        if (st) return st;
    }
    return check(h, cudaGetLastError(), "run");
}

// A sampler's table into a dump (include/ems_gpu.h, ems_sampler): every tap
// of nonzero weight must lie in the grid and in the factor box, the factor
// box in the grid. Sets the dump's points and field (1: i, 0: u).
static ems_status dump_sampler(ems_gpu* h, const ems_sampler* sp, DumpDev& d, int* field, uint64_t* npts) {
    const Grid& g = h->g;
    const uint64_t nn[3] = {g.nx, g.ny, g.nz};
    if (sp->quantity < EMS_DUMP_E || sp->quantity > EMS_DUMP_B || !sp->tap_idx || !sp->tap_w)
        return fail(h, EMS_ERR_INVALID, "sampler: invalid table");
    uint64_t n = 1;
    for (int a = 0; a < 3; ++a) {
        if (!sp->dims[a] || sp->dims[a] >= (1u << 30)) return fail(h, EMS_ERR_INVALID, "sampler: invalid dims");
        n *= sp->dims[a];
        if (n >= (1ull << 31)) return fail(h, EMS_ERR_INVALID, "sampler: too many points");
        if (sp->factors && (!sp->fac_dims[a] || sp->fac_lo[a] + sp->fac_dims[a] > nn[a]))
            return fail(h, EMS_ERR_INVALID, "sampler: factor box outside the grid");
    }
    const uint64_t off[3] = {0, 3 * sp->dims[0], 3 * (sp->dims[0] + sp->dims[1])};
    const uint64_t taps = 2 * 3 * (sp->dims[0] + sp->dims[1] + sp->dims[2]);
    for (int a = 0; a < 3; ++a)
        for (uint64_t q = 2 * off[a]; q < 2 * (off[a] + 3 * sp->dims[a]); ++q) {
            if (sp->tap_w[q] == 0.0) continue;
            const uint64_t x = sp->tap_idx[q];
            if (x >= nn[a] || (sp->factors && (x < sp->fac_lo[a] || x >= sp->fac_lo[a] + sp->fac_dims[a])))
                return fail(h, EMS_ERR_INVALID, "sampler: a tap outside the grid or the factor box");
        }
    const uint64_t vol = sp->factors ? sp->fac_dims[0] * sp->fac_dims[1] * sp->fac_dims[2] : 0;
    if (vol >= (1ull << 31)) return fail(h, EMS_ERR_INVALID, "sampler: factor box too large");
    d.samp = 1;
    d.roth = sp->quantity == EMS_DUMP_ROTH;
    for (int a = 0; a < 3; ++a) {
        d.n[a] = (uint32_t)sp->dims[a];
        d.off[a] = (uint32_t)off[a];
        d.flo[a] = (uint32_t)sp->fac_lo[a];
        d.fdim[a] = (uint32_t)sp->fac_dims[a];
        d.lo[a] = 0;
        d.st[a] = 1;
        d.inv_len[a] = nullptr;
    }
    d.tidx = h->upload(sp->tap_idx, taps);
    d.tw = h->upload(sp->tap_w, taps);
    d.fac = sp->factors ? h->upload(sp->factors, 3 * vol) : nullptr;
    if (!d.tidx || !d.tw || (sp->factors && !d.fac)) return fail(h, EMS_ERR_NOMEM, "sampler");
    *field = (sp->quantity == EMS_DUMP_H || sp->quantity == EMS_DUMP_B || sp->quantity == EMS_DUMP_ROTH) ? 1 : 0;
    *npts = n;
    return EMS_OK;
}

ems_status ems_gpu_freq_dump_add(ems_gpu* h, const ems_freq_dump* spec, size_t* id) {
    if (!h || !spec || !id || !spec->freqs || !spec->n_freqs) return EMS_ERR_INVALID;
    if (!spec->sampler && (spec->field < 0 || spec->field > 1)) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    const Grid& g = h->g;
    const uint32_t nn[3] = {g.nx, g.ny, g.nz};
    ems_gpu::FreqDump D;
    DumpDev& d = D.d;
    d = DumpDev{};
    uint64_t npts = 1;
    int field = spec->field;
    if (spec->sampler) {
        ems_status st = dump_sampler(h, spec->sampler, d, &field, &npts);
        if (st) return st;
    }
    for (int a = 0; a < 3 && !spec->sampler; ++a) {
        const uint64_t st = spec->stride[a] ? spec->stride[a] : 1;
        if (spec->lo[a] > spec->hi[a] || spec->hi[a] >= nn[a] || !spec->inv_len[a]) return EMS_ERR_INVALID;
        d.lo[a] = (uint32_t)spec->lo[a];
        d.st[a] = (uint32_t)st;
        d.n[a] = (uint32_t)((spec->hi[a] - spec->lo[a]) / st + 1);
        npts *= d.n[a];
        d.inv_len[a] = h->upload(spec->inv_len[a], nn[a]);
        if (!d.inv_len[a]) return fail(h, EMS_ERR_NOMEM, "dump");
    }
    if (npts * spec->n_freqs * 6 >= (1ull << 34)) return fail(h, EMS_ERR_INVALID, "dump too large");
    d.pitch = g.pitch;
    d.ny = g.ny;
    d.npts = (uint32_t)npts;
    d.nf = (uint32_t)spec->n_freqs;
    d.freqs = h->upload(spec->freqs, spec->n_freqs);
    d.dt = h->dt;
    d.t0 = field ? -0.5 * h->dt : 0.0;
    d.acc = h->alloc<double>(npts * spec->n_freqs * 6);
    if (!d.freqs || !d.acc) return fail(h, EMS_ERR_NOMEM, "dump");
    D.field = field;
    D.interval = spec->interval ? spec->interval : 1;
    h->dumps.push_back(D);
    *id = h->dumps.size() - 1;
    return check(h, cudaStreamSynchronize(h->stream), "dump");
}

ems_status ems_gpu_time_dump_add(ems_gpu* h, const ems_time_dump* spec, size_t* id) {
    if (!h || !spec || !id) return EMS_ERR_INVALID;
    if (!spec->sampler && (spec->field < 0 || spec->field > 1)) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    const Grid& g = h->g;
    const uint32_t nn[3] = {g.nx, g.ny, g.nz};
    ems_gpu::TimeDump T;
    DumpDev& d = T.d;
    d = DumpDev{};
    uint64_t npts = 1;
    int field = spec->field;
    if (spec->sampler) {
        ems_status st = dump_sampler(h, spec->sampler, d, &field, &npts);
        if (st) return st;
    }
    for (int a = 0; a < 3 && !spec->sampler; ++a) {
        const uint64_t st = spec->stride[a] ? spec->stride[a] : 1;
        if (spec->lo[a] > spec->hi[a] || spec->hi[a] >= nn[a] || !spec->inv_len[a]) return EMS_ERR_INVALID;
        d.lo[a] = (uint32_t)spec->lo[a];
        d.st[a] = (uint32_t)st;
        d.n[a] = (uint32_t)((spec->hi[a] - spec->lo[a]) / st + 1);
        npts *= d.n[a];
        d.inv_len[a] = h->upload(spec->inv_len[a], nn[a]);
        if (!d.inv_len[a]) return fail(h, EMS_ERR_NOMEM, "time dump");
    }
    if (npts >= (1ull << 31)) return fail(h, EMS_ERR_INVALID, "time dump too large");
    d.pitch = g.pitch;
    d.ny = g.ny;
    d.npts = (uint32_t)npts;
    T.field = field;
    T.interval = spec->interval ? spec->interval : 1;
    h->tdumps.push_back(std::move(T));
    *id = h->tdumps.size() - 1;
    return check(h, cudaStreamSynchronize(h->stream), "time dump");
}

ems_status ems_gpu_upml_state(ems_gpu* h, size_t op, int side, float* f, float* v, size_t cap) {
    if (!h || op >= h->ops.size() || h->ops[op].kind != EMS_OP_UPML || side < 0 || side > 1 || !f || !v)
        return EMS_ERR_INVALID;
    const UpmlSideDev& D = h->ops[op].upml[side];
    if (cap < D.n) return EMS_ERR_INVALID;
    if (!D.n) return EMS_OK;
    cudaSetDevice(h->device);
    if (check(h, cudaMemcpyAsync(f, D.f, D.n * sizeof(float), cudaMemcpyDeviceToHost, h->stream), "PML state") ||
        check(h, cudaMemcpyAsync(v, D.v, D.n * sizeof(float), cudaMemcpyDeviceToHost, h->stream), "PML state") ||
        check(h, cudaStreamSynchronize(h->stream), "PML state"))
        return EMS_ERR_CUDA;
    return EMS_OK;
}

ems_status ems_gpu_time_dump_count(const ems_gpu* h, size_t id, size_t* n) {
    if (!h || !n || id >= h->tdumps.size()) return EMS_ERR_INVALID;
    *n = h->tdumps[id].states.size();
    return EMS_OK;
}

ems_status ems_gpu_time_dump_read(ems_gpu* h, size_t id, size_t k, double* out, size_t cap, uint64_t* state) {
    if (!h || !out || id >= h->tdumps.size()) return EMS_ERR_INVALID;
    const auto& T = h->tdumps[id];
    const size_t n = (size_t)T.d.npts * 3;
    if (k >= T.states.size() || cap < n) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    if (check(h, cudaMemcpyAsync(out, T.buf + k * n, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
              "time dump read") ||
        check(h, cudaStreamSynchronize(h->stream), "time dump read"))
        return EMS_ERR_CUDA;
    if (state) *state = T.states[k];
    return EMS_OK;
}

ems_status ems_gpu_freq_dump_read(ems_gpu* h, size_t id, size_t k, double* out, size_t cap) {
    if (!h || !out || id >= h->dumps.size()) return EMS_ERR_INVALID;
    const auto& D = h->dumps[id];
    if (k >= D.d.nf || cap < (size_t)D.d.npts * 6) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    if (check(h, cudaMemcpyAsync(out, D.d.acc + (size_t)k * D.d.npts * 6, (size_t)D.d.npts * 6 * sizeof(double),
                                 cudaMemcpyDeviceToHost, h->stream), "dump read") ||
        check(h, cudaStreamSynchronize(h->stream), "dump read"))
        return EMS_ERR_CUDA;
    const double s = (double)D.interval * h->dt;
    for (size_t q = 0; q < (size_t)D.d.npts * 6; ++q) out[q] *= s;
    return EMS_OK;
}

ems_status ems_gpu_autotune(ems_gpu* h, const char* cache_path) {
    if (!h || !cache_path) return EMS_ERR_INVALID;
    auto& T = h->tune;
    char key[256];
    std::snprintf(key, sizeof key, "engine %ux%ux%u ops=%zu tables=%d curl=%d", h->g.nx, h->g.ny, h->g.nz,
                  h->ops.size(), h->tables_ok ? 1 : 0, h->oe_curl ? 1 : 0);
    std::string k(key);
    for (auto& op : h->ops) k += "," + std::to_string(op.kind);
    T.key = k;
    T.cache = cache_path;
    int v = 0;
    if (tune_lookup(T.cache, T.key, &v) &&
        (v == 1 || ((v == 4 || (v == 3 && !h->oe_curl && !h->has_upml)) && h->tables_ok) ||
         (v == 5 && h->tables_ok && h->sweep_ok))) {
        h->schedule = v;
        return EMS_OK;
    }
    // In-place schedules only (the per-operator, two-kernel and split ones
    // share the CPML state buffers).
    T.cand.clear();
    if (h->tables_ok) T.cand = (h->oe_curl || h->has_upml) ? std::vector<int>{4} : std::vector<int>{4, 3};
    if (h->tables_ok && h->sweep_ok) T.cand.push_back(5);
    if (h->tables_ok && h->interior_why.empty()) T.cand.push_back(6);
    if (h->tables_ok && h->march_why.empty()) T.cand.push_back(7);
    T.cand.push_back(1);
    T.ms.assign(T.cand.size(), 0.0);
    T.at = 0;
    T.done = 0;
    if (check(h, cudaEventCreate(&T.e0), "autotune") || check(h, cudaEventCreate(&T.e1), "autotune"))
        return EMS_ERR_CUDA;
    T.active = true;
    return EMS_OK;
}

// Reads (and clears) the device flags: a bounded wait of the fused or
// marching kernel that ran out (EMS_ERR_TIMEOUT), a non-finite field value a
// marching step wrote (EMS_ERR_DIVERGED). The errors surface here, at the
// host's next check, as the reference's stepping itself never fails
// (src/engine/mod.rs:456-458).
static ems_status device_status(ems_gpu* h) {
    int st[2] = {0, 0};
    if (h->status &&
        check(h, cudaMemcpyAsync(&st[0], h->status, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "status"))
        return EMS_ERR_CUDA;
    if (check(h, cudaMemcpyAsync(&st[1], h->diverged, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "status"))
        return EMS_ERR_CUDA;
    if (check(h, cudaStreamSynchronize(h->stream), "status")) return EMS_ERR_CUDA;
    if (st[0] || st[1]) {
        if (h->status) cudaMemsetAsync(h->status, 0, sizeof(int), h->stream);
        cudaMemsetAsync(h->diverged, 0, sizeof(int), h->stream);
        if (check(h, cudaStreamSynchronize(h->stream), "status")) return EMS_ERR_CUDA;
    }
    if (st[0]) return fail(h, EMS_ERR_TIMEOUT, "a bounded wait of the fused or marching kernel ran out");
    if (st[1]) return fail(h, EMS_ERR_DIVERGED, "a marching step wrote a non-finite field value");
    return EMS_OK;
}

ems_status ems_gpu_step_with_energy(ems_gpu* h, double* energy) {
    if (!h || !energy) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    // Operator energies of the state before the step (src/engine/mod.rs:819-823).
    double w_ops = 0.0;
    for (auto& op : h->ops) {
        double x = 0.0;
        if (op.kind == EMS_OP_POLES) {
            k_pole_energy<<<1, 1024, 0, h->stream>>>(op.poles.e, op.poles.h, h->d_energy + 1);
            ++h->launches;
        } else if (op.kind == EMS_OP_LUMPED && op.lumped.has_branch) {
            k_branch_energy<<<1, 1, 0, h->stream>>>(op.lumped.d, h->dt, h->d_energy + 1);
            ++h->launches;
        } else if (op.kind == EMS_OP_MUR && op.mur_energy) {
            k_mur_energy<<<1, 1024, 0, h->stream>>>(op.mur, h->d_energy + 1);
            ++h->launches;
        } else if (op.kind == EMS_OP_SHEET && op.sheet.n_edges) {
            k_sheet_energy<<<1, 1024, 0, h->stream>>>(op.sheet, h->dt, h->d_energy + 1);
            ++h->launches;
        } else {
            continue;
        }
        if (check(h, cudaMemcpyAsync(&x, h->d_energy + 1, sizeof(double), cudaMemcpyDeviceToHost, h->stream), "energy"))
            return EMS_ERR_CUDA;
        if (check(h, cudaStreamSynchronize(h->stream), "energy")) return EMS_ERR_CUDA;
        w_ops += x;
    }
    ems_status st = step_dumped(h, true);
    if (st) return st;
    double w = 0.0;
    if (check(h, cudaMemcpyAsync(&w, h->d_energy, sizeof(double), cudaMemcpyDeviceToHost, h->stream), "energy"))
        return EMS_ERR_CUDA;
    if (check(h, cudaStreamSynchronize(h->stream), "energy")) return EMS_ERR_CUDA;
    *energy = 0.25 * h->dt * w + w_ops;
    return device_status(h);
}

ems_status ems_gpu_timestep(const ems_gpu* h, uint64_t* n) {
    if (!h || !n) return EMS_ERR_INVALID;
    *n = h->step;
    return EMS_OK;
}

ems_status ems_gpu_download_field(ems_gpu* h, int field, int axis, float* host) {
    if (!h || !host || field < 0 || field > 1 || axis < 0 || axis > 2) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    const Grid& g = h->g;
    float* src = field == 0 ? h->u[axis] : h->i[axis];
    if (check(h, cudaMemcpy2DAsync(host, g.nz * sizeof(float), src, g.pitch * sizeof(float), g.nz * sizeof(float),
                                   (size_t)g.nx * g.ny, cudaMemcpyDeviceToHost, h->stream),
              "download"))
        return EMS_ERR_CUDA;
    if (check(h, cudaStreamSynchronize(h->stream), "download")) return EMS_ERR_CUDA;
    return device_status(h);
}

ems_status ems_gpu_upload_field(ems_gpu* h, int field, int axis, const float* host) {
    if (!h || !host || field < 0 || field > 1 || axis < 0 || axis > 2) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    const Grid& g = h->g;
    if (field == 0) h->prev_e_valid = false;  // the saved electric values are captured again
    // Both buffers of a double-buffered field get the values (the padding
    // entries the kernels read as zero stay equal in both).
    float* dsts[2] = {field == 0 ? h->u[axis] : h->i[axis], field == 0 ? h->u2[axis] : h->i2[axis]};
    for (float* dst : dsts) {
        if (!dst) continue;
        if (check(h, cudaMemcpy2DAsync(dst, g.pitch * sizeof(float), host, g.nz * sizeof(float), g.nz * sizeof(float),
                                       (size_t)g.nx * g.ny, cudaMemcpyHostToDevice, h->stream),
                  "upload"))
            return EMS_ERR_CUDA;
    }
    return check(h, cudaStreamSynchronize(h->stream), "upload");
}

ems_status ems_gpu_samples(ems_gpu* h, size_t op, int which, double* out, size_t cap, size_t* n) {
    if (!h || !n || op >= h->ops.size()) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    auto& o = h->ops[op];
    const double* src = nullptr;
    size_t cnt = 0;
    if (o.kind == EMS_OP_PROBE && which == 0) {
        src = o.probe.values;
        cnt = o.probe.count;
    } else if (o.kind == EMS_OP_LUMPED && o.lumped.record && which >= 0 && which <= 2) {
        if (which > 0 && !o.lumped.columns) return EMS_ERR_INVALID;
        src = which == 0 ? o.lumped.rec : (which == 1 ? o.lumped.pv : o.lumped.pi);
        cnt = o.lumped.count;
    } else if (o.kind == EMS_OP_SHEET && (which == 0 || which == 1)) {
        src = which == 0 ? o.sheet.u : o.sheet.h;
        cnt = which == 0 ? o.sheet_nodes : o.sheet_layers;
    } else {
        return fail(h, EMS_ERR_INVALID, "no such series");
    }
    *n = cnt;
    if (out && cnt && cap) {
        size_t m = std::min(cap, cnt);
        if (check(h, cudaMemcpyAsync(out, src, m * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "samples"))
            return EMS_ERR_CUDA;
    }
    if (check(h, cudaStreamSynchronize(h->stream), "samples")) return EMS_ERR_CUDA;
    return device_status(h);
}

ems_status ems_gpu_last_sample(ems_gpu* h, size_t op, int which, double* out) {
    if (!h || !out || op >= h->ops.size()) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    auto& o = h->ops[op];
    const double* src = nullptr;
    size_t cnt = 0;
    if (o.kind == EMS_OP_PROBE && which == 0) {
        src = o.probe.values;
        cnt = o.probe.count;
    } else if (o.kind == EMS_OP_LUMPED && o.lumped.record && which >= 0 && which <= 2 && (which == 0 || o.lumped.columns)) {
        src = which == 0 ? o.lumped.rec : (which == 1 ? o.lumped.pv : o.lumped.pi);
        cnt = o.lumped.count;
    }
    if (!src || !cnt) return fail(h, EMS_ERR_INVALID, "no sample");
    if (check(h, cudaMemcpyAsync(out, src + cnt - 1, sizeof(double), cudaMemcpyDeviceToHost, h->stream), "sample"))
        return EMS_ERR_CUDA;
    return check(h, cudaStreamSynchronize(h->stream), "sample");
}

ems_status ems_gpu_source_amplitude(ems_gpu* h, size_t op, uint64_t first, const double* values, size_t n) {
    if (!h || (!values && n) || op >= h->ops.size()) return EMS_ERR_INVALID;
    auto& o = h->ops[op];
    if (o.kind == EMS_OP_SOURCE) {
        if (o.source.amp.size() < first + n) o.source.amp.resize(first + n, 0.0f);
        for (size_t q = 0; q < n; ++q) o.source.amp[first + q] = (float)values[q];
    } else if (o.kind == EMS_OP_LUMPED && o.lumped.has_src) {
        if (o.lumped.amp.size() < first + n) o.lumped.amp.resize(first + n, 0.0);
        for (size_t q = 0; q < n; ++q) o.lumped.amp[first + q] = values[q];
    } else {
        return fail(h, EMS_ERR_INVALID, "not a source");
    }
    return EMS_OK;
}

const char* ems_gpu_last_error(const ems_gpu* h) { return h ? h->err.c_str() : "null handle"; }

ems_status ems_gpu_launch_count(const ems_gpu* h, uint64_t* n) {
    if (!h || !n) return EMS_ERR_INVALID;
    *n = h->launches;
    return EMS_OK;
}

ems_status ems_gpu_stream(const ems_gpu* h, void** stream) {
    if (!h || !stream) return EMS_ERR_INVALID;
    *stream = (void*)h->stream;
    return EMS_OK;
}

ems_status ems_gpu_profile(ems_gpu* h, int enable) {
    if (!h) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    h->prof_collect();
    h->profiling = enable != 0;
    return EMS_OK;
}

ems_status ems_gpu_profile_read(ems_gpu* h, int kernel, double* ms, uint64_t* launches) {
    if (!h || !ms || !launches || kernel < 0 || kernel > 2) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    h->prof_collect();
    *ms = h->prof_ms[kernel];
    *launches = h->prof_n[kernel];
    h->prof_ms[kernel] = 0.0;
    h->prof_n[kernel] = 0;
    return check(h, cudaGetLastError(), "profile");
}

ems_status ems_gpu_set_schedule(ems_gpu* h, int schedule) {
    if (!h || schedule < 0 || schedule > 7) return EMS_ERR_INVALID;
    if (h->oe_curl && (schedule == 2 || schedule == 3))
        return fail(h, EMS_ERR_INVALID, "the fused and two-kernel schedules sum the curl in the default order only");
    if (h->has_upml && (schedule == 2 || schedule == 3 || schedule == 5))
        return fail(h, EMS_ERR_INVALID, "openEMS PML layers run on the per-operator and split schedules only");
    if (schedule == 2 && !h->fused_ok) return fail(h, EMS_ERR_INVALID, "fused schedule unavailable: " + h->fused_why);
    if (schedule == 3 && !h->tables_ok) return fail(h, EMS_ERR_INVALID, "two-kernel schedule unavailable: " + h->tables_why);
    if (schedule == 4 && !h->tables_ok) return fail(h, EMS_ERR_INVALID, "split schedule unavailable: " + h->tables_why);
    if (schedule == 5 && !(h->tables_ok && h->sweep_ok))
        return fail(h, EMS_ERR_INVALID, "sweep schedule unavailable: " + (h->tables_ok ? std::string("magnetic sources, conducting sheets or openEMS PML layers") : h->tables_why));
    if (schedule == 6 && !(h->tables_ok && h->interior_why.empty()))
        return fail(h, EMS_ERR_INVALID, "interior schedule unavailable: " + (h->tables_ok ? h->interior_why : h->tables_why));
    if (schedule == 7 && !(h->tables_ok && h->march_why.empty()))
        return fail(h, EMS_ERR_INVALID, "marching schedule unavailable: " + (h->tables_ok ? h->march_why : h->tables_why));
    h->schedule = schedule;
    return EMS_OK;
}

ems_status ems_gpu_set_curl_order(ems_gpu* h, int order) {
    if (!h || order < 0 || order > 1) return EMS_ERR_INVALID;
    if (order == 1 && (h->schedule == 2 || h->schedule == 3))
        return fail(h, EMS_ERR_INVALID, "the fused and two-kernel schedules sum the curl in the default order only");
    h->oe_curl = order == 1;
    // A captured sweep step holds the other kernels.
    for (auto& gx : h->sweep_graph)
        if (gx) {
            cudaGraphExecDestroy(gx);
            gx = nullptr;
        }
    return EMS_OK;
}

ems_status ems_gpu_set_interior_planes(ems_gpu* h, uint32_t planes) {
    if (!h || planes < 1 || planes > 4096) return EMS_ERR_INVALID;
    h->interior_planes = planes;
    return EMS_OK;
}

ems_status ems_gpu_check(ems_gpu* h) {
    if (!h) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    if (check(h, cudaGetLastError(), "check")) return EMS_ERR_CUDA;
    return device_status(h);
}

ems_status ems_gpu_test_wait_timeout(ems_gpu* h, uint64_t limit_ns) {
    if (!h || !limit_ns || limit_ns > 10000000000ull) return EMS_ERR_INVALID;
    h->test_wait_ns = limit_ns;
    return EMS_OK;
}

ems_status ems_gpu_set_march(ems_gpu* h, int shape, uint32_t planes) {
    if (!h || shape < 0 || shape >= kNumMarchShapes || planes < 1 || planes > 4096) return EMS_ERR_INVALID;
    h->march_shape = shape;
    h->march_planes = planes;
    return EMS_OK;
}

ems_status ems_gpu_set_sweep_planes(ems_gpu* h, uint32_t planes) {
    if (!h || !planes || !h->tables_ok) return EMS_ERR_INVALID;
    cudaSetDevice(h->device);
    if (check(h, cudaStreamSynchronize(h->stream), "sweep planes")) return EMS_ERR_CUDA;
    ems_status st = build_chunks(h, std::min(planes, h->g.nx));
    if (st) return st;
    return check(h, cudaStreamSynchronize(h->stream), "sweep planes");
}

ems_status ems_gpu_schedule(const ems_gpu* h, int* active) {
    if (!h || !active) return EMS_ERR_INVALID;
    *active = active_schedule(h);
    return EMS_OK;
}

ems_status ems_gpu_row_cpml(const ems_gpu* h, int* on) {
    if (!h || !on) return EMS_ERR_INVALID;
    *on = h->tables_ok && h->rowc.ok && h->row_cpml_on ? 1 : 0;
    return EMS_OK;
}

ems_status ems_gpu_set_row_cpml(ems_gpu* h, int on) {
    if (!h) return EMS_ERR_INVALID;
    if (on && !(h->tables_ok && h->rowc.ok))
        return fail(h, EMS_ERR_INVALID, "row CPML unavailable (no CPML, a slab operator registered before it, "
                                        "openEMS PML layers, or a slab off the faces)");
    h->row_cpml_on = on != 0;
    return EMS_OK;
}

ems_status ems_gpu_interior_box(ems_gpu* h, uint32_t box[6]) {
    if (!h || !box) return EMS_ERR_INVALID;
    if (!(h->tables_ok && h->interior_why.empty()))
        return fail(h, EMS_ERR_INVALID, "interior schedule unavailable: " + (h->tables_ok ? h->interior_why : h->tables_why));
    for (int a = 0; a < 3; ++a) {
        box[a] = h->ibox.lo[a];
        box[3 + a] = h->ibox.hi[a];
    }
    return EMS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches (batch.cuh): many models stepping together, one CUDA graph per step.

struct ems_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    std::vector<ems_gpu*> models;            // owned
    std::vector<std::unique_ptr<DevBuf>> bufs;
    uint64_t max_steps = 0;
    std::vector<uint32_t> start[BK_KINDS];   // host copies of the prefix sums (frozen models count 0)
    std::vector<std::array<uint32_t, BK_KINDS>> blocks;  // each model's blocks per kernel kind
    BatchTable T{};
    std::vector<int> active;
    int* d_active = nullptr;
    uint32_t* d_steps = nullptr;
    BatchSource* d_src[2] = {nullptr, nullptr};  // [0] H sources, [1] E sources
    uint32_t n_src[2] = {0, 0};
    BatchProbe* d_probe[2] = {nullptr, nullptr}; // [0] current, [1] voltage
    uint32_t n_probe[2] = {0, 0};
    BatchLumped* d_lumped = nullptr;
    uint32_t n_lumped = 0;
    bool any_cpml = false, any_poles_e = false, any_poles_h = false, poles_first = false;
    double* partials = nullptr;
    double* ops_energy = nullptr;
    double* energies = nullptr;
    // Sample series: (model, op) → device buffer, interval (0: per step), which.
    struct Series {
        size_t model, op;
        int which;
        uint32_t interval, cap;
        double* dev;
    };
    std::vector<Series> series;
    unsigned grid[BK_KINDS] = {0, 0, 0, 0, 0};  // persistent grid per kind
    uint64_t resident[BK_KINDS] = {0, 0, 0, 0, 0};  // blocks resident at once per kind
    cudaGraphExec_t step_graph = nullptr, energy_graph = nullptr;
    // Autotuning of the persistent grids (ems_batch_autotune): code 0 one
    // block per work item, 1 the resident blocks, 2 half of them.
    struct Tune {
        bool active = false;
        std::string cache, key;
        std::vector<int> cand;
        std::vector<double> ms;
        size_t at = 0;
        int done = 0;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
    } tune;
    int grid_code = 1;

    template <class T_>
    T_* alloc(size_t n) {
        auto b = std::make_unique<DevBuf>();
        size_t bytes = std::max<size_t>(n, 1) * sizeof(T_);
        if (cudaMalloc(&b->p, bytes) != cudaSuccess) return nullptr;
        cudaMemsetAsync(b->p, 0, bytes, stream);
        b->bytes = bytes;
        T_* p = (T_*)b->p;
        bufs.push_back(std::move(b));
        return p;
    }
    template <class T_>
    T_* upload(const T_* h, size_t n) {
        T_* d = alloc<T_>(n);
        if (d && n && h) cudaMemcpyAsync(d, h, n * sizeof(T_), cudaMemcpyHostToDevice, stream);
        return d;
    }
};

namespace {

ems_status bfail(ems_batch* b, ems_status s, const std::string& m) {
    if (b) b->err = m;
    return s;
}

// The whole step of every active model, in the hook order of the split
// schedule (run_step), each kernel over all models at once.
void batch_enqueue_step(ems_batch* b, bool energy) {
    cudaStream_t s = b->stream;
    const BatchTable& T = b->T;
    const uint32_t nm = T.n;
    if (energy) k_batch_ops_energy<<<nm, 1024, 0, s>>>(T, b->d_lumped, b->n_lumped, b->ops_energy);
    if (b->grid[BK_SPLIT]) {
        if (energy) k_batch_h<true><<<b->grid[BK_SPLIT], kSplitThreads, 0, s>>>(T, b->partials);
        else k_batch_h<false><<<b->grid[BK_SPLIT], kSplitThreads, 0, s>>>(T, nullptr);
    }
    auto shell = [&](int side) {
        if (!b->grid[BK_SHELL_H + side]) return;
        if (side) k_batch_shell<1><<<b->grid[BK_SHELL_E], 32 * kShellWarps, 0, s>>>(T);
        else k_batch_shell<0><<<b->grid[BK_SHELL_H], 32 * kShellWarps, 0, s>>>(T);
    };
    auto poles_h = [&] {
        if (b->grid[BK_POLES_H]) k_batch_poles<0><<<b->grid[BK_POLES_H], 256, 0, s>>>(T);
        if (b->grid[BK_POLES_E]) k_batch_capture<1><<<b->grid[BK_POLES_E], 256, 0, s>>>(T);
    };
    auto poles_e = [&] {
        if (b->grid[BK_POLES_E]) k_batch_poles<1><<<b->grid[BK_POLES_E], 256, 0, s>>>(T);
        if (b->grid[BK_POLES_H]) k_batch_capture<0><<<b->grid[BK_POLES_H], 256, 0, s>>>(T);
    };
    // Slab hooks after H, in registration order; then serial post_h.
    if (b->poles_first) { poles_h(); shell(0); } else { shell(0); poles_h(); }
    if (b->n_src[0]) k_batch_sources<0><<<blocks_for(b->n_src[0], 256), 256, 0, s>>>(T, b->d_src[0], b->n_src[0]);
    if (b->n_probe[0]) k_batch_probes<0><<<blocks_for(b->n_probe[0], 128), 128, 0, s>>>(T, b->d_probe[0], b->n_probe[0]);
    if (b->n_lumped) k_batch_lumped_pre<<<b->n_lumped, 128, 0, s>>>(T, b->d_lumped, b->n_lumped);
    if (b->grid[BK_SPLIT]) k_batch_e<<<b->grid[BK_SPLIT], kSplitThreads, 0, s>>>(T);
    if (b->poles_first) { poles_e(); shell(1); } else { shell(1); poles_e(); }
    if (b->n_lumped) k_batch_lumped_post<<<b->n_lumped, 256, 0, s>>>(T, b->d_lumped, b->n_lumped);
    if (b->n_src[1]) k_batch_sources<1><<<blocks_for(b->n_src[1], 256), 256, 0, s>>>(T, b->d_src[1], b->n_src[1]);
    if (b->n_probe[1]) k_batch_probes<1><<<blocks_for(b->n_probe[1], 128), 128, 0, s>>>(T, b->d_probe[1], b->n_probe[1]);
    if (energy) k_batch_energy<<<nm, 1024, 0, s>>>(T, b->partials, b->ops_energy, b->energies);
    k_batch_advance<<<blocks_for(nm, 128), 128, 0, s>>>(T, b->d_steps);
}

// The persistent grid of each kernel kind for grid code `code`.
void batch_grids(ems_batch* b, int code) {
    for (int k = 0; k < BK_KINDS; ++k) {
        // All models' work, frozen or not: a graph keeps every kernel a
        // model may need when it is resumed.
        uint64_t work = 0;
        for (const auto& mb : b->blocks) work += mb[k];
        uint64_t g = work;
        if (code == 1) g = std::min<uint64_t>(work, b->resident[k]);
        if (code == 2) g = std::min<uint64_t>(work, std::max<uint64_t>(1, b->resident[k] / 2));
        b->grid[k] = (unsigned)g;
    }
    b->grid_code = code;
}

ems_status batch_capture(ems_batch* b, bool energy, cudaGraphExec_t* out);

// Captures the step and energy-step graphs for the current grids.
ems_status batch_graphs(ems_batch* b) {
    if (b->step_graph) cudaGraphExecDestroy(b->step_graph);
    if (b->energy_graph) cudaGraphExecDestroy(b->energy_graph);
    b->step_graph = b->energy_graph = nullptr;
    ems_status st = batch_capture(b, false, &b->step_graph);
    if (st) return st;
    return batch_capture(b, true, &b->energy_graph);
}

ems_status batch_capture(ems_batch* b, bool energy, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return bfail(b, EMS_ERR_CUDA, "graph capture");
    batch_enqueue_step(b, energy);
    if (cudaStreamEndCapture(b->stream, &g) != cudaSuccess || !g) return bfail(b, EMS_ERR_CUDA, "graph capture");
    cudaError_t e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return bfail(b, EMS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return EMS_OK;
}

// Checks the operator order a batch can run: per model, the serial post_h
// hooks are H sources then current probes, the serial post_e hooks lumped
// elements then E sources then voltage probes (the order the batched
// kernels run them in), and no two sources (or lumped elements) of a model
// share an edge (they are applied in parallel).
std::string batch_ineligible(const ems_engine_desc* d) {
    int phase_e = 0, phase_h = 0;
    std::vector<uint64_t> ke, kh, kl;
    for (size_t k = 0; k < d->n_ops; ++k) {
        const int kind = d->ops[k].kind;
        int pe = -1, ph = -1;
        if (kind == EMS_OP_LUMPED) {
            pe = 0;
            const auto* l = (const ems_lumped*)d->ops[k].table;
            for (size_t e = 0; e < l->n_edges; ++e) kl.push_back(l->node[e]);
        } else if (kind == EMS_OP_SOURCE) {
            const auto* sr = (const ems_source*)d->ops[k].table;
            const bool e_side = sr->kind == EMS_SOFT_E || sr->kind == EMS_HARD_E;
            (e_side ? pe : ph) = e_side ? 1 : 0;
            for (size_t e = 0; e < sr->n_edges; ++e) (e_side ? ke : kh).push_back(sr->node[e] * 3 + sr->axis[e]);
        } else if (kind == EMS_OP_PROBE) {
            const auto* pr = (const ems_probe*)d->ops[k].table;
            if (pr->quantity == EMS_PROBE_VOLTAGE) pe = 2;
            else ph = 1;
        }
        if (kind == EMS_OP_MUR) return "Mur boundaries";
        if (kind == EMS_OP_SHEET) return "conducting sheets";
        if (kind == EMS_OP_UPML) return "openEMS PML layers";
        if (pe >= 0) {
            if (pe < phase_e) return "post_e hooks not in the order lumped, E sources, voltage probes";
            phase_e = pe;
        }
        if (ph >= 0) {
            if (ph < phase_h) return "post_h hooks not in the order H sources, current probes";
            phase_h = ph;
        }
    }
    for (auto* v : {&ke, &kh, &kl}) {
        std::sort(v->begin(), v->end());
        if (std::adjacent_find(v->begin(), v->end()) != v->end()) return "two sources or lumped elements share an edge";
    }
    return "";
}

}  // namespace

extern "C" {

ems_status ems_batch_create(const ems_engine_desc* const* descs, size_t n_models, int device, uint64_t max_steps,
                            ems_batch** out) {
    if (!descs || !out || !n_models || n_models > kMaxBatch || max_steps == 0 || max_steps >= (1ull << 31))
        return EMS_ERR_INVALID;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return EMS_ERR_CUDA;
    // Everything made so far is released on every early return.
    struct Guard {
        ems_batch* b;
        ~Guard() {
            if (b) ems_batch_destroy(b);
        }
    } guard{new ems_batch};
    ems_batch* b = guard.b;
    b->device = device;
    b->max_steps = max_steps;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return EMS_ERR_CUDA;
    std::vector<BatchModel> hm(n_models);
    std::vector<BatchSource> src[2];
    std::vector<BatchProbe> prb[2];
    std::vector<BatchLumped> lum;
    for (int k = 0; k < BK_KINDS; ++k) b->start[k].assign(1, 0u);
    int pf = -1;
    for (size_t m = 0; m < n_models; ++m) {
        const ems_engine_desc* d = descs[m];
        if (!d) return EMS_ERR_INVALID;
        std::string why = batch_ineligible(d);
        if (!why.empty()) {
            std::fprintf(stderr, "ems_batch: model %zu: %s\n", m, why.c_str());
            return EMS_ERR_INVALID;
        }
        ems_gpu* h = nullptr;
        ems_status st = ems_gpu_create(d, device, &h);
        if (st) return st;
        b->models.push_back(h);
        if (!h->tables_ok) {
            std::fprintf(stderr, "ems_batch: model %zu: %s\n", m, h->tables_why.c_str());
            return EMS_ERR_INVALID;
        }
        const Grid& g = h->g;
        BatchModel& M = hm[m];
        M = BatchModel{};
        M.P = h->fp;
        for (int a = 0; a < 3; ++a) {
            M.P.uo[a] = M.P.un[a] = h->u[a];
            M.P.io[a] = M.P.in[a] = h->i[a];
            M.f.u[a] = h->u[a];
            M.f.i[a] = h->i[a];
        }
        for (size_t q = 0; q < h->psi_h.size(); ++q) {
            FSlab& fs = M.P.slab[0][h->psi_h_at[q].first][h->psi_h_at[q].second];
            fs.psi_old = fs.psi_new = h->psi_h[q].first;
        }
        for (int l = 0; l < 12; ++l) M.c.c[l] = h->co[l];
        M.shell[0] = h->shell[0];
        M.shell[1] = h->shell[1];
        M.run_of[0] = h->run_of[0];
        M.run_of[1] = h->run_of[1];
        M.dt = h->dt;
        M.bx = split_blocks_x(g);
        bool has_cpml = false, has_poles = false;
        for (auto& op : h->ops) {
            if (op.kind == EMS_OP_CPML) has_cpml = true;
            if (op.kind == EMS_OP_POLES) {
                has_poles = true;
                M.pe = op.poles.e;
                M.ph = op.poles.h;
            }
        }
        if (has_cpml && has_poles) {
            if (pf >= 0 && pf != h->fp.poles_first) return EMS_ERR_INVALID;
            pf = h->fp.poles_first;
        }
        b->any_cpml |= has_cpml;
        b->any_poles_e |= M.pe.n_edges > 0;
        b->any_poles_h |= M.ph.n_edges > 0;
        const uint32_t blocks[BK_KINDS] = {M.bx * g.nx, shell_blocks(M.shell[0]), shell_blocks(M.shell[1]),
                                           (uint32_t)blocks_for(M.pe.n_edges, 256),
                                           (uint32_t)blocks_for(M.ph.n_edges, 256)};
        for (int k = 0; k < BK_KINDS; ++k) {
            const uint64_t next = (uint64_t)b->start[k].back() + blocks[k];
            if (next >= (1ull << 32)) return EMS_ERR_INVALID;
            b->start[k].push_back((uint32_t)next);
        }
        b->blocks.push_back({blocks[0], blocks[1], blocks[2], blocks[3], blocks[4]});
        // Serial hooks: sources, probes, lumped elements (device tables).
        size_t op_i = 0;
        for (auto& op : h->ops) {
            const size_t op_index = op_i++;
            if (op.kind == EMS_OP_SOURCE) {
                const auto* sr = (const ems_source*)d->ops[op_index].table;
                const bool e_side = sr->kind == EMS_SOFT_E || sr->kind == EMS_HARD_E;
                const bool hard = sr->kind == EMS_HARD_E || sr->kind == EMS_HARD_H;
                const float* amp = op.source.amp.empty() ? nullptr : b->upload(op.source.amp.data(), op.source.amp.size());
                for (size_t e = 0; e < sr->n_edges; ++e)
                    src[e_side ? 1 : 0].push_back(BatchSource{(uint32_t)m, dev_index(g, sr->node[e]), sr->axis[e],
                                                              hard ? 1u : 0u, sr->weight[e],
                                                              (uint32_t)op.source.amp.size(), amp});
            } else if (op.kind == EMS_OP_PROBE) {
                const ems_gpu::ProbeDev& P = op.probe;
                const uint32_t interval = (uint32_t)std::min<uint64_t>(P.interval, max_steps);
                const uint32_t cap = (uint32_t)((max_steps - 1) / interval + 1);
                double* v = b->alloc<double>(cap);
                if (!v) return EMS_ERR_NOMEM;
                prb[P.quantity == EMS_PROBE_VOLTAGE ? 1 : 0].push_back(BatchProbe{(uint32_t)m, interval, cap, P.d, v});
                b->series.push_back({m, op_index, 0, interval, cap, v});
            } else if (op.kind == EMS_OP_LUMPED) {
                const ems_gpu::LumpedDev& L = op.lumped;
                BatchLumped bl{};
                bl.model = (uint32_t)m;
                bl.axis = (uint32_t)L.axis;
                bl.cap = (uint32_t)max_steps;
                bl.has_src = L.has_src ? 1u : 0u;
                bl.d = L.d;
                bl.n_amp = (uint32_t)L.amp.size();
                bl.amp = L.amp.empty() ? nullptr : b->upload(L.amp.data(), L.amp.size());
                if (L.record) {
                    bl.rec = b->alloc<double>(max_steps);
                    if (!bl.rec) return EMS_ERR_NOMEM;
                    b->series.push_back({m, op_index, 0, 1, (uint32_t)max_steps, bl.rec});
                }
                if (L.columns) {
                    bl.pv = b->alloc<double>(max_steps);
                    bl.pi = b->alloc<double>(max_steps);
                    if (!bl.pv || !bl.pi) return EMS_ERR_NOMEM;
                    b->series.push_back({m, op_index, 1, 1, (uint32_t)max_steps, bl.pv});
                    b->series.push_back({m, op_index, 2, 1, (uint32_t)max_steps, bl.pi});
                }
                lum.push_back(bl);
            }
        }
    }
    b->poles_first = pf == 1;
    b->active.assign(n_models, 1);
    BatchTable& T = b->T;
    T.n = (uint32_t)n_models;
    T.models = b->upload(hm.data(), n_models);
    for (int k = 0; k < BK_KINDS; ++k) T.start[k] = b->upload(b->start[k].data(), b->start[k].size());
    b->d_active = b->upload(b->active.data(), n_models);
    b->d_steps = b->alloc<uint32_t>(n_models);
    T.active = b->d_active;
    T.steps = b->d_steps;
    for (int sd = 0; sd < 2; ++sd) {
        b->n_src[sd] = (uint32_t)src[sd].size();
        b->d_src[sd] = b->upload(src[sd].data(), src[sd].size());
        b->n_probe[sd] = (uint32_t)prb[sd].size();
        b->d_probe[sd] = b->upload(prb[sd].data(), prb[sd].size());
    }
    b->n_lumped = (uint32_t)lum.size();
    b->d_lumped = b->upload(lum.data(), lum.size());
    b->partials = b->alloc<double>(b->start[BK_SPLIT].back());
    b->ops_energy = b->alloc<double>(n_models);
    b->energies = b->alloc<double>(n_models);
    if (!T.models || !b->d_active || !b->d_steps || !b->partials || !b->ops_energy || !b->energies)
        return EMS_ERR_NOMEM;
    // Persistent grids: as many blocks as are resident at once (at most the
    // work), so each block walks the packed index with a stride.
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    int occ[BK_KINDS] = {8, 6, 6, 8, 8};
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[BK_SPLIT], k_batch_e, kSplitThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[BK_SHELL_H], k_batch_shell<0>, 32 * kShellWarps, 0);
    occ[BK_SHELL_E] = occ[BK_SHELL_H];
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[BK_POLES_E], k_batch_poles<1>, 256, 0);
    occ[BK_POLES_H] = occ[BK_POLES_E];
    for (int k = 0; k < BK_KINDS; ++k) b->resident[k] = (uint64_t)sms * std::max(1, occ[k]);
    batch_grids(b, 1);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return EMS_ERR_CUDA;
    ems_status st = batch_graphs(b);
    if (st) return st;
    guard.b = nullptr;
    *out = b;
    return EMS_OK;
}

ems_status ems_batch_destroy(ems_batch* b) {
    if (!b) return EMS_ERR_INVALID;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->step_graph) cudaGraphExecDestroy(b->step_graph);
    if (b->energy_graph) cudaGraphExecDestroy(b->energy_graph);
    b->bufs.clear();
    for (ems_gpu* h : b->models) ems_gpu_destroy(h);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return EMS_OK;
}

// One step of a tuning batch: the current candidate's graph, timed.
static ems_status batch_tune_step(ems_batch* b) {
    auto& T = b->tune;
    if (b->grid_code != T.cand[T.at]) {
        batch_grids(b, T.cand[T.at]);
        ems_status st = batch_graphs(b);
        if (st) return st;
    }
    const bool timed = T.done > 0;
    if (timed) cudaEventRecord(T.e0, b->stream);
    if (cudaGraphLaunch(b->step_graph, b->stream) != cudaSuccess) return bfail(b, EMS_ERR_CUDA, "graph launch");
    if (timed) {
        cudaEventRecord(T.e1, b->stream);
        cudaEventSynchronize(T.e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, T.e0, T.e1);
        T.ms[T.at] += ms;
    }
    if (++T.done == kTuneSteps) {
        T.done = 0;
        if (++T.at == T.cand.size()) {
            size_t best = 0;
            for (size_t q = 1; q < T.cand.size(); ++q)
                if (T.ms[q] < T.ms[best]) best = q;
            tune_record(T.cache, T.key, T.cand[best], T.ms[best] / (kTuneSteps - 1));
            T.active = false;
            cudaEventDestroy(T.e0);
            cudaEventDestroy(T.e1);
            if (b->grid_code != T.cand[best]) {
                batch_grids(b, T.cand[best]);
                return batch_graphs(b);
            }
        }
    }
    return EMS_OK;
}

ems_status ems_batch_run(ems_batch* b, uint64_t n) {
    if (!b) return EMS_ERR_INVALID;
    cudaSetDevice(b->device);
    for (uint64_t q = 0; q < n; ++q) {
        if (b->tune.active) {
            ems_status st = batch_tune_step(b);
            if (st) return st;
        } else if (cudaGraphLaunch(b->step_graph, b->stream) != cudaSuccess) {
            return bfail(b, EMS_ERR_CUDA, "graph launch");
        }
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? EMS_OK : bfail(b, EMS_ERR_CUDA, cudaGetErrorString(e));
}

ems_status ems_batch_autotune(ems_batch* b, const char* cache_path) {
    if (!b || !cache_path) return EMS_ERR_INVALID;
    cudaSetDevice(b->device);
    auto& T = b->tune;
    char key[256];
    std::snprintf(key, sizeof key, "batch n=%zu blocks=%u,%u,%u,%u,%u", b->models.size(), b->start[0].back(),
                  b->start[1].back(), b->start[2].back(), b->start[3].back(), b->start[4].back());
    T.key = key;
    T.cache = cache_path;
    int v = 0;
    if (tune_lookup(T.cache, T.key, &v) && v >= 0 && v <= 2) {
        if (v != b->grid_code) {
            batch_grids(b, v);
            return batch_graphs(b);
        }
        return EMS_OK;
    }
    T.cand = {1, 0, 2};
    T.ms.assign(T.cand.size(), 0.0);
    T.at = 0;
    T.done = 0;
    if (cudaEventCreate(&T.e0) != cudaSuccess || cudaEventCreate(&T.e1) != cudaSuccess)
        return bfail(b, EMS_ERR_CUDA, "autotune");
    T.active = true;
    return EMS_OK;
}

ems_status ems_batch_step_with_energy(ems_batch* b, double* energies) {
    if (!b || !energies) return EMS_ERR_INVALID;
    cudaSetDevice(b->device);
    const size_t n = b->models.size();
    if (cudaMemsetAsync(b->energies, 0, n * sizeof(double), b->stream) != cudaSuccess ||
        cudaGraphLaunch(b->energy_graph, b->stream) != cudaSuccess ||
        cudaMemcpyAsync(energies, b->energies, n * sizeof(double), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess)
        return bfail(b, EMS_ERR_CUDA, "energy step");
    return EMS_OK;
}

ems_status ems_batch_set_active(ems_batch* b, size_t model, int active) {
    if (!b || model >= b->models.size()) return EMS_ERR_INVALID;
    cudaSetDevice(b->device);
    b->active[model] = active ? 1 : 0;
    // The packed block table shrinks to the active models (a frozen model's
    // range becomes empty), so the persistent grids walk only live work;
    // the graphs read the table from device memory and need no re-capture.
    const size_t n = b->models.size();
    for (int k = 0; k < BK_KINDS; ++k) {
        auto& st = b->start[k];
        for (size_t m = 0; m < n; ++m) st[m + 1] = st[m] + (b->active[m] ? b->blocks[m][k] : 0u);
    }
    // Ordered with the graph launches on the batch's stream.
    bool ok = cudaMemcpyAsync(b->d_active + model, &b->active[model], sizeof(int), cudaMemcpyHostToDevice,
                              b->stream) == cudaSuccess;
    for (int k = 0; ok && k < BK_KINDS; ++k)
        ok = cudaMemcpyAsync((void*)b->T.start[k], b->start[k].data(), (n + 1) * sizeof(uint32_t),
                             cudaMemcpyHostToDevice, b->stream) == cudaSuccess;
    if (!ok || cudaStreamSynchronize(b->stream) != cudaSuccess) return bfail(b, EMS_ERR_CUDA, "set active");
    return EMS_OK;
}

ems_status ems_batch_timestep(ems_batch* b, size_t model, uint64_t* n) {
    if (!b || !n || model >= b->models.size()) return EMS_ERR_INVALID;
    cudaSetDevice(b->device);
    uint32_t v = 0;
    if (cudaMemcpyAsync(&v, b->d_steps + model, sizeof(v), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess)
        return bfail(b, EMS_ERR_CUDA, "timestep");
    *n = v;
    return EMS_OK;
}

ems_status ems_batch_samples(ems_batch* b, size_t model, size_t op, int which, double* out, size_t cap, size_t* n) {
    if (!b || !n || model >= b->models.size()) return EMS_ERR_INVALID;
    uint64_t steps = 0;
    ems_status st = ems_batch_timestep(b, model, &steps);
    if (st) return st;
    for (const auto& sr : b->series) {
        if (sr.model != model || sr.op != op || sr.which != which) continue;
        const uint64_t count = std::min<uint64_t>(steps ? (steps - 1) / sr.interval + 1 : 0, sr.cap);
        *n = (size_t)count;
        if (!out) return EMS_OK;
        const size_t k = std::min<size_t>(cap, (size_t)count);
        if (k && (cudaMemcpyAsync(out, sr.dev, k * sizeof(double), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess ||
                  cudaStreamSynchronize(b->stream) != cudaSuccess))
            return bfail(b, EMS_ERR_CUDA, "samples");
        return EMS_OK;
    }
    return bfail(b, EMS_ERR_INVALID, "no such series");
}

ems_status ems_batch_download_field(ems_batch* b, size_t model, int field, int axis, float* host) {
    if (!b || model >= b->models.size()) return EMS_ERR_INVALID;
    cudaSetDevice(b->device);
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return bfail(b, EMS_ERR_CUDA, "download");
    return ems_gpu_download_field(b->models[model], field, axis, host);
}

ems_status ems_batch_stream(const ems_batch* b, void** stream) {
    if (!b || !stream) return EMS_ERR_INVALID;
    *stream = (void*)b->stream;
    return EMS_OK;
}

const char* ems_batch_last_error(const ems_batch* b) { return b ? b->err.c_str() : "null batch"; }

}  // extern "C"
