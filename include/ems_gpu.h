/*
 * ems_gpu.h — C ABI of the B200 FDTD time-stepping engine.
 *
 * This is the drop-in boundary for the time stepping of the ems FDTD
 * solver: it replaces `pool::drive` and the per-step work of the operators
 * that run inside it (src/engine/pool.rs:884-940, src/engine/mod.rs:833-992).
 * The host keeps everything above it (mesh compilation, coefficient and
 * operator set-up, ports, post-processing) and hands the engine, once, the
 * tables those steps produce; the engine then advances the fields on one
 * GPU and returns probe samples, port series and energies.
 *
 * Conventions (those of the reference engine, src/engine/mod.rs:21-62):
 *  - a node [i, j, k] has the linear index (i*ny + j)*nz + k (z fastest);
 *    every field and coefficient array has one entry per node;
 *  - u[a] are the E edge voltages, i[a] the H dual-edge currents of axis a;
 *  - one step: i^{n-1/2} -> i^{n+1/2} (H), then u^n -> u^{n+1} (E);
 *  - coefficient lanes: ca 0-2, cb 3-5, da 6-8, db 9-11 (src/engine/coeffs.rs:327-391).
 *
 * All tables are copied at ems_gpu_create; the caller keeps ownership of
 * its buffers. One handle = one CUDA stream; a handle is not thread-safe.
 * Every call returns an ems_status; the text of the last error of a handle
 * is ems_gpu_last_error(h).
 */
#ifndef EMS_GPU_H
#define EMS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
typedef enum {
    EMS_OK = 0,
    EMS_ERR_INVALID = 1,  /* invalid argument or table                 */
    EMS_ERR_CUDA = 2,     /* a CUDA call failed                          */
    EMS_ERR_DIVERGED = 3, /* NaN/Inf found in a checked quantity         */
    EMS_ERR_TIMEOUT = 4,  /* a bounded device wait ran out               */
    EMS_ERR_NOMEM = 5     /* device or host allocation failed            */
} ems_status;

/* Operator kinds, in the order the engine runs their hooks within a
 * half-step (the registration order of the descriptor decides between
 * operators of the same hook). */
typedef enum {
    EMS_OP_CPML = 1,   /* slab hooks post_h / post_e   (src/engine/boundary/cpml.rs:816-883) */
    EMS_OP_POLES = 2,  /* slab hooks post_h / post_e   (src/engine/dispersive.rs:1687-1744)  */
    EMS_OP_LUMPED = 3, /* serial pre_e / post_e        (src/engine/lumped.rs:1123-1236)      */
    EMS_OP_SOURCE = 4, /* serial post_h or post_e      (src/engine/excite.rs:104-173)        */
    EMS_OP_PROBE = 5,  /* serial post_h or post_e      (src/engine/probe.rs:480-510)         */
    EMS_OP_MUR = 6,    /* serial pre_e / post_e        (src/engine/boundary/mur.rs:781-843)  */
    EMS_OP_UPML = 7,   /* slab hooks post_h / post_e   (src/engine/boundary/upml.rs:443-470) */
    EMS_OP_SHEET = 8   /* serial post_h / post_e       (src/engine/sheet.rs:941-1050)        */
} ems_op_kind;

/* One CPML slab: the correction of one field component in one face layer
 * (src/engine/boundary/cpml.rs:392-520, Slab). For every node of the box
 * lo..hi (half-open, node indices):
 *   s = sign*(h - l)         (derivative of component `other` along `normal`)
 *   psi = flush(b*psi + a*s)
 *   t = flush(t + scale*coef*(k*s + psi))
 * with t = u[comp] (E side, coef = cb, scale = +1, h/l = i[other] at the
 * node and one node below, zero outside) or t = i[comp] (H side, coef = db,
 * scale = -1, h/l = u[other] one node above and at the node). b, a, k are
 * per depth index node[normal] - lo[normal]; psi starts at zero. */
typedef struct {
    int32_t e_side;  /* 1: corrects u (after the E update); 0: corrects i   */
    int32_t comp;    /* corrected component axis (0 x, 1 y, 2 z)            */
    int32_t normal;  /* layer normal axis                                   */
    int32_t other;   /* differentiated component axis                       */
    float sign;      /* +1 if normal == next(comp), else -1                 */
    uint64_t lo[3];
    uint64_t hi[3];
    const float* b;  /* hi[normal]-lo[normal] values each */
    const float* a;
    const float* k;  /* 1/kappa - 1 (less a1/b for the linear rule) */
} ems_cpml_slab;

typedef struct {
    size_t n_slabs;
    const ems_cpml_slab* slabs; /* E and H slabs, in layer order */
} ems_cpml;

/* Pole kinds of one dispersive branch (src/engine/dispersive.rs:961-971):
 * trapezoidal, leapfrog, openEMS's f32 leapfrog of a Lorentz/Drude pole
 * (OpenEmsPole, dispersive.rs:846-899: a = A, inv_c = K, inv_z = B, state
 * j = V, q = W; applied before the edge's other poles) and openEMS's f32
 * Debye update of an edge whose poles are all of that kind
 * (with_openems_debye, dispersive.rs:1824-1857: a = F, inv_c = 1 - g,
 * inv_z = b, state j = Q). The two openEMS kinds hold f32 values in the f64
 * arrays, carry no energy (half_l = 0) and add nothing to sum_inv_z. */
typedef enum {
    EMS_POLE_TRAPEZOIDAL = 0,
    EMS_POLE_LEAPFROG = 1,
    EMS_POLE_OPENEMS = 2,
    EMS_POLE_OPENEMS_DEBYE = 3
} ems_pole_kind;

/* The poles of one field type (electric: E edges; magnetic: H dual edges)
 * of a dispersive medium (src/engine/dispersive.rs:973-1041, Side). Edges
 * are in the reference order (plane, axis, offset); an edge's poles are
 * [pole_end[e-1], pole_end[e]) in insertion order. Per pole: trapezoidal
 * (a = 2L/dt, inv_c = 1/C_p, inv_z = 1/z) or leapfrog (a = k_a, inv_c,
 * inv_z = k_b), half_l = L/2 for the energy. sum_inv_z is the sum of
 * inv_z over the edge's trapezoidal poles. */
typedef struct {
    size_t n_edges;
    const uint8_t* axis;
    const uint64_t* node;      /* node index (i*ny+j)*nz+k */
    const double* sum_inv_z;
    const uint32_t* pole_end;
    size_t n_poles;
    const uint8_t* kind;       /* ems_pole_kind per pole */
    const double* a;
    const double* inv_c;
    const double* inv_z;
    const double* half_l;
} ems_pole_side;

typedef struct {
    ems_pole_side electric;
    ems_pole_side magnetic;
} ems_poles;

/* A lumped element on E edges along `axis` (src/engine/lumped.rs:880-1013
 * install, 1123-1236 post_e). Its resistor and parallel capacitor are
 * already folded into the uploaded ca/cb. Per edge: cb (the folded edge
 * coefficient), g_src (conductance in series with the source), src_w
 * (source weight, V_s share), and with a branch 2L/dt, 1/C, z; with a
 * current record g and c. src_amp[n] is the source value at (n+1/2)*dt
 * for step n (n < n_src_amp; 0 beyond). A port (port_columns > 0) also
 * records V = sum(u)/columns after each step and I = -record.
 * openems_order (openEMS files, LumpedElement::openems_order): the branch
 * is driven by the voltage its own update left the step before (not u^n
 * saved in pre_e) and the source is added after the branch; with oe_k
 * (parallel inductor, openEMS's explicit update in f32): per edge the f32
 * state s <- f32(s + f32(oe_k*f32(u_prev))), u <- f32(u - s), the branch
 * current s/oe_vi. NULL oe_k: the trapezoidal branch. */
typedef struct {
    int32_t axis;
    size_t n_edges;
    const uint64_t* node;
    const double* cb;
    const double* g_src;
    uint64_t series;            /* M: edges in series */
    int32_t src_in_branch;      /* series topology: source sits in the branch */
    const double* src_w;        /* NULL: no source */
    size_t n_src_amp;
    const double* src_amp;
    int32_t has_branch;
    const double* two_l_dt;
    const double* inv_c;
    const double* z;
    int32_t record;             /* record the terminal current */
    const double* rec_g;
    const double* rec_c;
    uint64_t port_columns;      /* > 0: a lumped port (src/engine/port.rs:262-290) */
    int32_t openems_order;      /* openEMS's operation order around the branch */
    const float* oe_k;          /* NULL, or per edge f32(dt/L)*f32(dt/(C + G dt/2)) */
    const double* oe_vi;        /* with oe_k: per edge dt/(C + G dt/2) */
} ems_lumped;

/* Edge source kinds (src/engine/excite.rs:13-40). */
typedef enum { EMS_SOFT_E = 0, EMS_HARD_E = 1, EMS_SOFT_H = 2, EMS_HARD_H = 3 } ems_source_kind;

/* An edge source: amp[n] = f32(amplitude(t_n)) for step n with t_n the
 * kind's sample time ((n+1/2)dt soft E, (n+1)dt hard E, n dt soft H,
 * (n+1/2)dt hard H); 0 for n >= n_amp. */
typedef struct {
    int32_t kind;
    size_t n_edges;
    const uint8_t* axis;
    const uint64_t* node;
    const float* weight;
    size_t n_amp;
    const float* amp;
} ems_source;

/* Probe quantities (src/engine/probe.rs:12-19). */
typedef enum { EMS_PROBE_VOLTAGE = 0, EMS_PROBE_CURRENT = 1 } ems_probe_quantity;

/* A probe: the weighted sum of field entries, in entry order, every
 * `interval` steps (steps with n % interval == 0); voltage after the E
 * update at (n+1)dt, current after the H update at (n+1/2)dt. */
typedef struct {
    int32_t quantity;
    size_t n_entries;
    const uint8_t* axis;
    const uint64_t* node;
    const double* weight;
    uint64_t interval;
    int32_t f32_sum;            /* accumulate in f32 (openEMS current probes) */
} ems_probe;

/* A first-order Mur absorbing boundary (src/engine/boundary/mur.rs:103-139
 * Edge and Corner, 249-299 the update). Entries [0, n_edges) are face
 * edges with one 1-D update, entries [n_edges, n) edges shared by two Mur
 * faces, updated after every face edge as the mean of two 1-D updates.
 * Per entry: the E edge along axis[e] at node[e], its interior neighbours
 * inner[2e] (and inner[2e+1] for a shared edge) and coefficients k[2e]
 * (k[2e+1]), hold[e] (no update before that step; NULL: none) and cap[e]
 * (capacitance counted by the energy with count_energy).
 *   pre_e:  b = u[node], i0 = u[inner0] (i1 = u[inner1])  (u^n)
 *   post_e: face edge   u[node] = i0 + k0*(u[inner0] - b)
 *                       (openems_order: (i0 - k0*b) + k0*u[inner0])
 *           shared edge u[node] = 0.5*(v0 + v1), each v the face update
 *                       along its own normal (openems_corners: i0 - k0*b)
 * All in f32. No face edge may be another face edge's neighbour, no
 * shared edge another shared edge's (the updates run in parallel). */
typedef struct {
    size_t n;
    size_t n_edges;
    const uint8_t* axis;
    const uint64_t* node;
    const uint64_t* inner;     /* 2 per entry (the second unused for face edges) */
    const float* k;            /* 2 per entry */
    const uint64_t* hold;      /* NULL: every entry updates from step 0 */
    const double* cap;         /* NULL unless count_energy */
    int32_t openems_order;
    int32_t openems_corners;
    int32_t count_energy;      /* energy: sum of 1/2 cap u^2 over the last written values */
} ems_mur;

/* openEMS's uniaxial PML layers (src/engine/boundary/upml.rs:1-140): the
 * layer edges of side 0 (E edges) and 1 (H dual edges), whose coefficients
 * the host already rewrote to (0, dt/((A/l)(1 + a_p))) so that the update
 * kernel leaves the flux increment t in the field. Per edge: axis, node and
 * the f32 coefficients co[4e..4e+3] = (1 - a_p)/(1 + a_p), (1 - a_q)/(1 + a_q),
 * (1 + a_a)/((1 + a_q) m), (1 - a_a)/((1 + a_q) m). Each edge keeps its flux
 * F and start value v (zero at first). After the H update: v of every E
 * edge = u (refresh), then every H edge: F' = flush(flush(co0*F) + t),
 * x = flush(flush(flush(co1*v) - flush(co3*F)) + flush(co2*F')), F = F',
 * v = x, field = x (apply); after the E update the same with the sides
 * swapped. */
typedef struct {
    size_t n[2];
    const uint8_t* axis[2];
    const uint64_t* node[2];
    const float* co[2];
} ems_upml;

/* Conducting sheets (src/engine/sheet.rs:403-1090, ConductingSheet): thin
 * lossy conductors on mesh planes. Sheet edge e (the E edge along axis[e]
 * at node[e]) carries a ladder across the sheet's thickness: nn[e] node
 * voltages u_0..u_{nn-1} (u_0 the face on the + side along the normal,
 * which the field array holds; u_{nn-1} the - face) and nn[e] - 1 layer
 * currents h_j, all f64 and zero at first. Its constants: per node
 * two_c = 2C_k/dt, cp = Thomas c'_k, inv_den = 1/den_k from konst0[e]; per
 * layer a = dt/(2L_j) from a0[e] (edges with equal ladders share them);
 * c_edge the edge capacitance dt(1 + ca)/(2cb). Couplings
 * [coupling_end[e-1], coupling_end[e]) are the dual edges around its dual
 * face: the H entry (c_axis, c_node), its signed weights w_up, w_dn in
 * Ampere's law of the two faces, corr and ecorr = L·corr/2 with
 * L = dt(1 + da)/(2db) the dual edge's inductance.
 *   post_h, per edge: u_0 = u[edge]; per coupling with corr != 0, in edge
 *     then coupling order: i = flush(i + f32(corr·(u_{nn-1} - u_0)));
 *   post_e, per edge: s_up = sum w_up·i, s_dn = sum w_dn·i (from 0, in
 *     coupling order), one tridiagonal solve for the mean voltages x_k,
 *     h_j += 2a_j(x_j - x_{j+1}), u_k = 2x_k - u_k, u[edge] = flush(f32(u_0)).
 * Energy: sum_k two_c·dt·u_k^2/4 - c_edge·u[edge]^2/2 + sum_j L_j·h_j^2/2
 * (L_j = dt/(2a_j)) plus sum ecorr·i·(u_{nn-1} - u[edge]) taken at the
 * end of the last post_e. */
typedef struct {
    size_t n_edges;
    const uint8_t* axis;
    const uint64_t* node;
    const uint32_t* nn;
    const uint32_t* konst0;
    const uint32_t* a0;
    const uint32_t* coupling_end;
    const double* c_edge;
    size_t n_couplings;
    const uint8_t* c_axis;
    const uint64_t* c_node;
    const double* w_up;
    const double* w_dn;
    const double* corr;
    const double* ecorr;
    size_t n_konst;
    const double* two_c;
    const double* cp;
    const double* inv_den;
    size_t n_a;
    const double* a;
} ems_sheet;

typedef struct {
    int32_t kind; /* ems_op_kind */
    const void* table; /* ems_cpml*, ems_poles*, ems_lumped*, ems_source*, ems_probe*, ems_mur*, ems_upml*, ems_sheet* */
} ems_op;

/* Everything an engine is built from: the grid size, the time step, the
 * twelve coefficient arrays (reference layout) and the operators in
 * registration order. */
typedef struct {
    uint64_t nodes[3];
    double dt;
    const float* coeff[12];
    size_t n_ops;
    const ems_op* ops;
} ems_engine_desc;

typedef struct ems_gpu ems_gpu;

/* Builds an engine on CUDA device `device` (replaces EngineBuilder::build_from
 * + Engine::add_operator, src/engine/mod.rs:325-381, 549-572). */
ems_status ems_gpu_create(const ems_engine_desc* desc, int device, ems_gpu** out);

/* Releases all device memory of the engine. */
ems_status ems_gpu_destroy(ems_gpu* h);

/* Advances n steps (Engine::run, src/engine/mod.rs:826). */
ems_status ems_gpu_run(ems_gpu* h, uint64_t n);

/* Advances one step and returns in *energy the energy invariant W^n of the
 * state before the step plus the operators' stored energy
 * (Engine::step_with_energy, src/engine/mod.rs:819). */
ems_status ems_gpu_step_with_energy(ems_gpu* h, double* energy);

/* Number of completed steps. */
ems_status ems_gpu_timestep(const ems_gpu* h, uint64_t* n);

/* Copies component `axis` of u (field 0) or i (field 1) to/from `host`
 * (nx*ny*nz floats, reference layout; Engine::u_component / fields_mut). */
ems_status ems_gpu_download_field(ems_gpu* h, int field, int axis, float* host);
ems_status ems_gpu_upload_field(ems_gpu* h, int field, int axis, const float* host);

/* Samples of operator `op` (index into desc->ops): a probe's values
 * (which = 0), a lumped element's current record (which = 0) or, for a
 * port, its voltage (which = 1) and current (which = 2), or a conducting
 * sheet's ladder state: every edge's node voltages (which = 0) or layer
 * currents (which = 1), edge after edge (ConductingSheet::lower_voltage,
 * src/engine/sheet.rs:628-633, is the last node of an edge). Writes up to
 * `cap` values into `out` (may be NULL) and the total count into *n. */
ems_status ems_gpu_samples(ems_gpu* h, size_t op, int which, double* out, size_t cap, size_t* n);

/* The latest sample of a series of ems_gpu_samples (EMS_ERR_INVALID if the
 * series is empty): one device-to-host read of 8 bytes. */
ems_status ems_gpu_last_sample(ems_gpu* h, size_t op, int which, double* out);

/* Overwrites amplitudes [first, first + n) of the source table of operator
 * `op` (an edge source: f32 values; a lumped element: f64 values given as
 * the doubles in `values`) from host memory, growing the table as needed:
 * a host may feed a source step by step instead of tabulating it at
 * creation. */
ems_status ems_gpu_source_amplitude(ems_gpu* h, size_t op, uint64_t first, const double* values, size_t n);

/* The energy invariant W^n of a field state, for callers that cannot
 * allocate device memory when they need it (a framework that owns all
 * device memory through its own pool, a real-time loop that must not
 * allocate after start-up). It has no counterpart in the reference.
 *
 * u, i: the six field arrays, i holding i^{n-1/2}; coeff: the twelve
 * coefficient arrays; all device arrays in the reference layout
 * ((i*ny + j)*nz + k, nx*ny*nz floats each). Writes
 * W^n = dt/4 * [sum (1+ca)/cb u^2 + sum (1+da)/db i^{n-1/2} i^{n+1/2}]
 * (i^{n+1/2} the H update's value, not stored; no operator energies) to the
 * device double `energy`, in stream `stream` (a cudaStream_t; NULL: the
 * legacy default stream), asynchronously. It calls no allocator: its working
 * memory is a file-scope device array of 2048 doubles (16 KiB) that every
 * GPU which loads the library holds until the process exits. At most
 * 2^31 - 1 nodes (EMS_ERR_INVALID beyond). The first call on a device looks
 * up that array's address (cudaGetSymbolAddress, with the device current)
 * and should come before any stream capture; device ordinals 0..63 only
 * (EMS_ERR_INVALID beyond), and an address looked up before a
 * cudaDeviceReset of its device is kept and no longer valid after it. All
 * calls share the array: calls that overlap on the GPU (other streams, other
 * host threads) race. */
ems_status ems_energy_noalloc(const uint64_t nodes[3], double dt, const float* const u[3], const float* const i[3],
                              const float* const coeff[12], double* energy, void* stream);

/* Text of the last error of handle `h` ("" if none; a static text if h is NULL). */
const char* ems_gpu_last_error(const ems_gpu* h);

/* Device kernels launched since creation (for bookkeeping). */
ems_status ems_gpu_launch_count(const ems_gpu* h, uint64_t* n);

/* The CUDA stream (cudaStream_t) all work of the handle runs on, so a host
 * can order its own work after it or time it with events. */
ems_status ems_gpu_stream(const ems_gpu* h, void** stream);

/* Kernel timing: with enable != 0 the engine records CUDA events around its
 * field-update kernels (kernel 0: H update, 1: E update, 2: fused step);
 * ems_gpu_profile_read returns their summed device time [ms] and launch
 * count since the last read, and resets them. */
ems_status ems_gpu_profile(ems_gpu* h, int enable);
ems_status ems_gpu_profile_read(ems_gpu* h, int kernel, double* ms, uint64_t* launches);

/* Selects the step schedule: 0 = automatic (the fastest one the model
 * allows), 1 = one kernel per field update and operator, 2 = the fused
 * single-pass kernel, 3 = two kernels (H with its slab hooks, E with its
 * slab hooks), 4 = split (streaming H and E updates, one CPML shell kernel
 * per side, the other hooks per operator), 5 = sweep (the split kernels
 * chunk by chunk along x, so each chunk's E update reads what its H update
 * left in L2; not with magnetic sources), 6 = interior (one pass of both
 * updates over the box inside the CPML layers, the split kernels around it,
 * old and new fields in two buffers; CPML, electric poles, E sources and
 * probes only; energy steps run the split kernels), 7 = marching (one pass
 * of both updates and both CPML corrections over the whole grid, plane
 * windows staged in shared memory by TMA, old and new fields in two
 * buffers, then the electric poles and the hooks; the same operators as 6;
 * energy steps run the split kernels). Results are identical bit for bit.
 * Asking for a schedule the model cannot run returns EMS_ERR_INVALID. */
ems_status ems_gpu_set_schedule(ems_gpu* h, int schedule);

/* The schedule steps run with (1 to 7 as above). */
ems_status ems_gpu_schedule(const ems_gpu* h, int* active);

/* The interior schedule's box, nodes [box[0..2], box[3..5]) along x, y, z;
 * EMS_ERR_INVALID (and why, in ems_gpu_last_error) if the model cannot run
 * that schedule. */
ems_status ems_gpu_interior_box(ems_gpu* h, uint32_t box[6]);

/* The row CPML of the split schedule: steps without energy apply the CPML
 * corrections inside the update kernels (a CPML variant of each update over
 * the quads that hold layer nodes, no shell kernel) instead of the shell
 * kernels; identical results. Off by default (on B200 it measures slower
 * than the shells on the 512^3 dispersive box). ems_gpu_set_row_cpml
 * returns EMS_ERR_INVALID for on = 1 where it does not apply (no CPML, a
 * slab operator registered before the CPML, openEMS PML layers, a slab off
 * the faces); ems_gpu_row_cpml reports whether steps use it. */
ems_status ems_gpu_set_row_cpml(ems_gpu* h, int on);
ems_status ems_gpu_row_cpml(const ems_gpu* h, int* on);

/* The order in which the H and E updates sum the four terms of an edge's
 * circulation (CurlOrder, src/engine/kernel.rs:81-108): 0 the reference's
 * default (a - b) - (c - d); 1 openEMS's, ((a - b) + d) - c for H and
 * ((a - b) - c) + d for E with every operation's subnormal result flushed,
 * which openEMS files use (their fields then equal openEMS's where the
 * coefficients do). Order 1 runs on the per-operator, split and sweep
 * schedules; it is refused while the fused or two-kernel schedule is set,
 * and those are refused while it is on. */
ems_status ems_gpu_set_curl_order(ems_gpu* h, int order);

/* The sweep schedule's chunk size in x-planes (set at creation so that a
 * chunk's fields take under half of L2; larger than nx: one chunk). */
ems_status ems_gpu_set_sweep_planes(ems_gpu* h, uint32_t planes);

/* Planes a block of the interior schedule's one-pass kernel marches through
 * (1 to 4096; default 32): a block first computes the H values of the plane
 * before its chunk again, so short chunks add work and long ones fewer,
 * longer-lived blocks. */
ems_status ems_gpu_set_interior_planes(ems_gpu* h, uint32_t planes);

/* Synchronises the handle's stream and reports what its device flags hold
 * since the last check (and clears them): EMS_ERR_TIMEOUT if a bounded wait
 * of the fused or marching kernel ran out, EMS_ERR_DIVERGED if a marching
 * step wrote a non-finite field value (NaN or Inf). Field downloads, sample
 * reads and step_with_energy report the same at their end. This is the
 * check at which device errors surface: stepping itself never fails, as in
 * the reference (src/engine/mod.rs:456-458; the run loop's Diverged outcome,
 * src/engine/run.rs:156-161). */
ems_status ems_gpu_check(ems_gpu* h);

/* Test hook of the bounded waits: the next marching step's first block
 * expects 16 more bytes on its first ring barrier than its copies deliver
 * (every copy lands; the phase never completes) and its waits give up after
 * `limit_ns` nanoseconds (1 .. 10^10). That block then sets the timeout flag
 * and returns; the step's result is not defined, and the next check returns
 * EMS_ERR_TIMEOUT. The handle and the device context stay usable. */
ems_status ems_gpu_test_wait_timeout(ems_gpu* h, uint64_t limit_ns);

/* The marching schedule's tile shape (0: 7 rows, 3 stages, two blocks per
 * SM; 1: 15 rows, 3 stages, one block; 2: 8 rows, 4 stages, one block; 3: 3
 * rows, 4 stages, three blocks) and the planes a block marches through (1
 * to 4096; default 32). */
ems_status ems_gpu_set_march(ems_gpu* h, int shape, uint32_t planes);

/* Picks the fastest in-place schedule (4, 3, 5 or 1) for this model's grid
 * shape and operators: from `cache_path` (a text file of earlier picks,
 * lines "<key> <schedule> <ms>") if it holds the key, else by timing each
 * candidate over the next steps ems_gpu_run takes (four steps each, the
 * first untimed; the results do not depend on the schedule, so these are
 * ordinary steps) and appending the pick to the file. No counterpart in
 * the reference, whose CPU engine has a single code path. */
ems_status ems_gpu_autotune(ems_gpu* h, const char* cache_path);

/* ---- Field samplers (FieldSampler, src/engine/dump.rs:487-940): one
 * quantity converted to field units and interpolated at a set of sample
 * points, dims[0] x dims[1] x dims[2] points, z fastest. Built on the host
 * (ems_sampler_new, include/ems_host.h).
 *
 * Every value is a tensor product of 1-D rules: component c at sample
 * (p, q, r) is the sum, in the order x tap, y tap, z tap, skipping taps of
 * weight 0, of wx*wy*wz*m*x with x the unknown of component c at the tap
 * node (u for E, J, D; i for H, B; for rot H the circulation of i around
 * the primary edge c, i_b(p) - i_a(p) - i_b(p - a) + i_a(p - b) with (a, b)
 * the axes after c) and m the factor of component c at that node (1 when
 * `factors` is NULL). Along axis a, component c's two taps of sample s are
 * entries 2*(off[a] + c*dims[a] + s) + t, t = 0, 1, of tap_idx (the node
 * index along a) and tap_w, with off = {0, 3*dims[0], 3*(dims[0] + dims[1])}.
 * The factors cover the node box fac_lo + [0, fac_dims) (every node any
 * tap of weight != 0 reads), z fastest, component c at
 * c * fac_dims[0]*fac_dims[1]*fac_dims[2]. */
typedef enum {
    EMS_DUMP_E = 0, EMS_DUMP_H = 1, EMS_DUMP_J = 2, EMS_DUMP_ROTH = 3, EMS_DUMP_D = 4, EMS_DUMP_B = 5
} ems_dump_quantity;

typedef struct {
    int32_t quantity;   /* ems_dump_quantity */
    uint64_t dims[3];
    const uint32_t* tap_idx;
    const double* tap_w;
    uint64_t fac_lo[3];
    uint64_t fac_dims[3];
    const double* factors;
} ems_sampler;

/* ---- Frequency-domain field dumps (src/engine/dump.rs:1420-1700,
 * FreqDump with DumpPosition::Native and DumpTiming::State): a running DFT
 * on the device of one field over a box of nodes.
 *
 * field 0 samples E = u/len (primary edge length), field 1 H = i/len (dual
 * edge length), each component at the edge that starts at the node (raw,
 * not interpolated); inv_len[c] holds 1/len of the component-c edges per
 * node index along axis c (nodes[c] values, 0 where no edge). Points are
 * the nodes lo + q*stride <= hi of the box (inclusive), z fastest. The
 * states m = 0, 1, 2, ... (the state after m steps; the first sampled is
 * the state when the dump is added) with m % interval == 0 are accumulated
 * as X(f) = sum x(t_m) e^{-j 2 pi f t_m} * interval*dt, t_m = m*dt (E) or
 * (m - 1/2)*dt (H), the phase reduced exactly (post/dft.rs phase_cycles). */
typedef struct {
    int32_t field;
    uint64_t lo[3], hi[3], stride[3];
    const double* inv_len[3];
    size_t n_freqs;
    const double* freqs;
    uint64_t interval;
    const ems_sampler* sampler; /* not NULL: its points and quantity (field, box and inv_len unused);
                                   H, B and rot H at (m - 1/2)*dt */
} ems_freq_dump;

/* Adds a dump (before or between runs); *id is its index. */
ems_status ems_gpu_freq_dump_add(ems_gpu* h, const ems_freq_dump* spec, size_t* id);

/* A time-domain dump (TimeDump with native positions, src/engine/dump.rs:
 * 1-80, Schedule::Every): snapshots of E = u/len or H = i/len* (f64, len
 * from inv_len as in ems_freq_dump) at the nodes lo + q*stride <= hi of the
 * box, z fastest, of the states m (the state after m steps: E at m*dt, H
 * at (m - 1/2)*dt; the first sampled is the state when the dump is added)
 * with m % interval == 0, kept on the device until read. */
typedef struct {
    int32_t field;
    uint64_t lo[3], hi[3], stride[3];
    const double* inv_len[3];
    uint64_t interval;
    const ems_sampler* sampler; /* as in ems_freq_dump */
} ems_time_dump;

ems_status ems_gpu_time_dump_add(ems_gpu* h, const ems_time_dump* spec, size_t* id);
/* The flux F and start value v of every edge of side `side` (0 E, 1 H) of the
 * EMS_OP_UPML operator `op`, in table order (cap >= the side's edges). */
ems_status ems_gpu_upml_state(ems_gpu* h, size_t op, int side, float* f, float* v, size_t cap);
/* Number of snapshots taken so far. */
ems_status ems_gpu_time_dump_count(const ems_gpu* h, size_t id, size_t* n);
/* Snapshot k: 3 values per point (x, y, z components) into out (cap >= 3 *
 * points); *state (if not NULL) the state m it shows. */
ems_status ems_gpu_time_dump_read(ems_gpu* h, size_t id, size_t k, double* out, size_t cap, uint64_t* state);

/* The transform at frequency index k: 3 complex values (re, im
 * interleaved: 6 doubles) per point, z fastest; cap in doubles. */
ems_status ems_gpu_freq_dump_read(ems_gpu* h, size_t id, size_t k, double* out, size_t cap);

/* ---- Batches: many models stepping together.
 *
 * No counterpart in the reference, where a parameter sweep runs
 * Simulation::run (src/sim/mod.rs:1044) once per model. A batch builds
 * every model as ems_gpu_create does and steps them together on one device:
 * each kernel kind of the split schedule runs once per step over all models
 * (a packed per-model block table walked by a persistent grid), the serial
 * hooks run batched from device-side step counters, and a whole step is one
 * CUDA graph. Each model's fields, probe and port series equal those of the
 * same model run alone bit for bit. A model needs the split schedule's
 * tables, its post_e hooks in the order lumped elements, E sources, voltage
 * probes and its post_h hooks in the order H sources, current probes, and
 * no two sources (or lumped elements) on one edge; otherwise creation
 * returns EMS_ERR_INVALID. max_steps (< 2^31) bounds the recorded series. */
typedef struct ems_batch ems_batch;

ems_status ems_batch_create(const ems_engine_desc* const* descs, size_t n_models, int device, uint64_t max_steps,
                            ems_batch** out);
ems_status ems_batch_destroy(ems_batch* b);

/* Advances every active model n steps. */
ems_status ems_batch_run(ems_batch* b, uint64_t n);

/* Advances every active model one step and writes each model's energy
 * invariant W^n of the state before the step (as ems_gpu_step_with_energy)
 * to energies[model]; 0 for inactive models. */
ems_status ems_batch_step_with_energy(ems_batch* b, double* energies);

/* Freezes (active = 0) or resumes a model: a frozen model keeps its state
 * and takes no steps (its end criterion has been met). */
ems_status ems_batch_set_active(ems_batch* b, size_t model, int active);

/* Completed steps of a model. */
ems_status ems_batch_timestep(ems_batch* b, size_t model, uint64_t* n);

/* A model's series as ems_gpu_samples (op: index into its descriptor's ops). */
ems_status ems_batch_samples(ems_batch* b, size_t model, size_t op, int which, double* out, size_t cap, size_t* n);

/* A model's field component in reference layout. */
ems_status ems_batch_download_field(ems_batch* b, size_t model, int field, int axis, float* host);

/* Picks the persistent grid of the batched kernels (one block per work
 * item, the resident blocks, or half of them) for this batch's shape: from
 * `cache_path` if it holds the key, else by timing each candidate over the
 * next steps ems_batch_run takes (results do not depend on the grid) and
 * appending the pick to the file. No counterpart in the reference. */
ems_status ems_batch_autotune(ems_batch* b, const char* cache_path);

/* The batch's CUDA stream (cudaStream_t). */
ems_status ems_batch_stream(const ems_batch* b, void** stream);

/* Text of the batch's last error. */
const char* ems_batch_last_error(const ems_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* EMS_GPU_H */
