/*
 * ems_host.h — host-side model set-up and run loop of the B200 engine.
 *
 * The host side of the drop-in: it restates, in C++, what the reference's
 * Rust host computes before and around the time stepping — the Cartesian
 * grid (src/engine/grid.rs), per-cell materials (src/engine/material.rs),
 * their per-edge averages and the update coefficients
 * (src/engine/edge_material.rs:376-425, src/engine/coeffs.rs:327-391,
 * 879-966), the CPML layers (src/engine/boundary/cpml.rs:979-1196), the
 * dispersive pole tables (src/engine/dispersive.rs:1896-1985, 2054-2470),
 * lumped ports (src/engine/lumped.rs:880-1013, src/engine/port.rs:102-160),
 * edge sources, probes, the Gaussian waveform (src/waveform.rs:442-470),
 * the end-criterion run loop (src/engine/run.rs:424-540) and the DFT /
 * port analysis (src/post/dft.rs, src/post/port.rs) — and hands the engine
 * its tables as an ems_engine_desc (include/ems_gpu.h).
 */
#ifndef EMS_HOST_H
#define EMS_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "ems_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ems_model ems_model;
typedef struct ems_cellset ems_cellset;
typedef struct ems_dispersive ems_dispersive;

/* Physical constants of the reference (src/constants.rs:9-18). */
double ems_const_eps0(void);
double ems_const_mu0(void);
double ems_const_c0(void);

/* A model on the rectilinear grid with the given mesh lines [m]
 * (Grid::new, src/engine/grid.rs:71-110). NULL on invalid lines. */
ems_model* ems_model_new(const double* x, size_t nx, const double* y, size_t ny, const double* z, size_t nz);
void ems_model_free(ems_model* m);
const char* ems_model_error(const ems_model* m);
void ems_model_nodes(const ems_model* m, uint64_t nodes[3]);

/* Adds a material (Material, src/engine/material.rs); returns its id (0 is
 * the vacuum background) or -1. */
int ems_model_material(ems_model* m, const double eps_r[3], const double mu_r[3], const double kappa[3],
                       const double sigma_m[3]);

/* Cell sets: a mask over the cells, filled by boxes (cell index ranges
 * lo..hi, half-open) and spheres (cells whose centre lies inside). */
ems_cellset* ems_cellset_new(const ems_model* m);
void ems_cellset_free(ems_cellset* s);
int ems_cellset_box(ems_cellset* s, const uint64_t lo[3], const uint64_t hi[3]);
int ems_cellset_sphere(ems_cellset* s, const double centre[3], double radius);
uint64_t ems_cellset_count(const ems_cellset* s);

/* Assigns material `mat` to the cells of `s` (CellMaterials::fill_box). */
int ems_model_fill(ems_model* m, const ems_cellset* s, int mat);

/* Marks the E edges along `axis` starting at the nodes of the box lo..hi
 * (inclusive node ranges) as PEC (CellMaterials PEC mask). */
int ems_model_pec_edges(ems_model* m, int axis, const uint64_t lo[3], const uint64_t hi[3]);

/* Face conditions in x_min, x_max, y_min, y_max, z_min, z_max order
 * (0 PEC, 1 PMC); default all PEC (FaceConditions, src/engine/coeffs.rs). */
int ems_model_faces(ems_model* m, const int faces[6]);

/* Phase velocities [m/s] of the edges along `axis` on Mur `face` (0 x_min,
 * 1 x_max, ... 5 z_max) for a face in local-medium mode, in place of the
 * medium of the edges next to it (MurMedia, src/engine/boundary/mur.rs:
 * 140-180): one value per node of the face plane, index p[u]·n[w] + p[w]
 * with u < w the two other axes; 0 keeps the local medium. Before
 * ems_model_add_mur. */
int ems_model_set_mur_media(ems_model* m, int face, int axis, const double* v);

/* Per-edge materials in place of the averages of the cells (EdgeMaterials,
 * src/engine/edge_material.rs:19-67, the form a sub-cell rasteriser such as
 * csx::discretize produces): for the E edges along `axis` (field 0: v0 =
 * eps_r, v1 = kappa) or the H dual edges (field 1: v0 = mu_r, v1 = sigma_m),
 * one value per node in reference layout. Before build. */
int ems_model_set_edge_materials(ems_model* m, int field, int axis, const double* v0, const double* v1);

/* Computes dt = courant * courant_limit (TimeStep::Courant, courant in
 * (0, 1]) or, with fixed_dt != 0, takes it (TimeStep::Fixed: finite, > 0
 * and at most the limit, src/engine/coeffs.rs:195-230), then the
 * coefficients (Coefficients::compute). Must precede the operators. */
int ems_model_build(ems_model* m, double courant, double fixed_dt);
/* Builds with the time step dt taken as given (TimeStep::Bound,
 * src/engine/coeffs.rs:233-236: a step established elsewhere, such as
 * openEMS's criterion below). flags: 1 openEMS's coefficient rounding (C,
 * G, L, R rounded to f32 and formed with openEMS's vacuum constants;
 * CoeffRounding, src/engine/coeffs.rs:705-760), 2 openEMS's average of the
 * magnetic conductivity over the two halves of a dual edge (openems_sigma_m,
 * src/compile/openems.rs:580-650). */
int ems_model_build_bound(ems_model* m, double dt, int flags);
/* openEMS's time step of the model's grid and materials by TimeStepMethod
 * `method` (3 Rennings, openEMS's default; 1 the Gershgorin "CFL" bound),
 * before any TimeStepFactor (openems_timestep, src/engine/timestep.rs:
 * 213-287). 0 for an unknown method. */
double ems_model_openems_timestep(const ems_model* m, int method);
/* openEMS's PML_n layers (OpenEmsPml::with_materials, src/engine/boundary/
 * upml.rs:560-724) of cells[f] cells on each face f with cells[f] > 0 (the
 * faces built PEC): rewrites the coefficients of the layer edges and adds
 * the EMS_OP_UPML operator with their tables. Returns the op index. */
int ems_model_add_openems_pml(ems_model* m, const uint64_t cells[6]);
/* Replaces the circuit of the E edge along `axis` at `node` after build: its
 * capacitance `cap` [F] and conductance `cond` [S] (a negative value keeps
 * the medium's), rounded like the model's circuit values, give its ca, cb
 * (replace_medium, src/sim/map.rs:1525-1606: how openEMS folds a parallel
 * R/C lumped element into its edges). */
int ems_model_set_edge_circuit(ems_model* m, int axis, const uint64_t node[3], double cap, double cond);
/* Zeroes the update coefficients of the E edges (field 0: ca, cb) or H
 * dual edges (field 1: da, db) along `axis` at the nodes of the inclusive
 * box lo..hi, after build (openEMS's PMC half cell, pmc_half_cell,
 * src/compile/mod.rs:1556-1626, is made of such boxes). */
int ems_model_zero_edges(ems_model* m, int field, int axis, const uint64_t lo[3], const uint64_t hi[3]);
double ems_model_dt(const ems_model* m);
double ems_model_courant_limit(const ems_model* m);
/* Coefficient lane `lane` (0..11) in reference layout (valid after build). */
const float* ems_model_coeff(const ems_model* m, int lane);

/* CPML layers (CpmlBoundary::new): cells[f] > 0 puts a layer of that many
 * cells on face f with grading order m, sigma_factor, kappa_max, alpha_max
 * and the linear (1) or constant (0) convolution. Returns the op index. */
int ems_model_add_cpml(ems_model* m, const uint64_t cells[6], double grading, double sigma_factor,
                       double kappa_max, double alpha_max, int linear);
/* The refractive index the layer on `face` is tuned for (after add_cpml). */
double ems_model_cpml_index(const ems_model* m, int face);

/* Dispersive media (Dispersive, src/engine/dispersive.rs). Pole kinds:
 * 0 Lorentz (omega_p, omega_0, gamma), 1 Drude (omega_p, gamma, -),
 * 2 Debye (delta_eps, tau, -); frequencies in rad/s. */
ems_dispersive* ems_dispersive_new(void);
void ems_dispersive_free(ems_dispersive* d);
/* Fills the cells of `s` with the poles for `field` (0 electric, 1
 * magnetic): every edge touching them gets each pole scaled by the share
 * of its averaging volume inside (Dispersive::fill_cells). */
int ems_dispersive_fill(ems_dispersive* d, const ems_model* m, const ems_cellset* s, int field, size_t n_poles,
                        const int* kind, const double* p1, const double* p2, const double* p3);
/* Adds one pole of `kind` (parameters as for ems_dispersive_fill), unscaled,
 * to the E edge (field 0) or H dual edge (field 1) along `axis` at `node`
 * (Dispersive::push of an EdgePole, src/engine/dispersive.rs:474-507): the
 * openEMS files' rule of full poles per edge. Kind 3, E edges and the
 * openEMS pole scheme only: a branch of openEMS's conducting-sheet model,
 * p1 = L [H], p2 = R [Ohm] (OpenEmsSheetBranches::push,
 * src/engine/openems_sheet.rs:56-80), installed with the edge's coefficient
 * as it is when ems_model_add_dispersive runs. */
int ems_dispersive_add_edge(ems_dispersive* d, int field, int axis, const uint64_t node[3], int kind, double p1,
                            double p2, double p3);
/* The averaged static material of the E edge (field 0: eps_r, kappa) or H
 * dual edge (field 1: mu_r, sigma_m) along `axis` at `node`
 * (EdgeMaterials::from_cells, src/engine/edge_material.rs:376-413). */
int ems_model_edge_material(const ems_model* m, int field, int axis, const uint64_t node[3], double out[2]);
/* Installs the medium with scheme 0 trapezoidal / 1 leapfrog / 2 openEMS's
 * f32 arithmetic (OpenEmsPole for Lorentz and Drude poles, given the
 * material's own omega_p, applied first on their edge; openEMS's Debye
 * update on electric edges whose poles are all Debye poles; other Debye
 * poles trapezoidal; src/engine/dispersive.rs:846-960); op index. */
int ems_model_add_dispersive(ems_model* m, ems_dispersive* d, int scheme);

/* Waveforms: 0 Gaussian (f0, fc; src/waveform.rs Waveform::Gaussian). */
double ems_waveform_value(int kind, double f0, double fc, double t, double dt);
double ems_waveform_duration(int kind, double f0, double fc);

/* A lumped port (LumpedPort::new(region, r).excite_waveform(w, amplitude))
 * along `axis` over the node box lo..hi (inclusive); the source table is
 * sampled for n_steps steps. Returns the op index. */
int ems_model_add_lumped_port(ems_model* m, int axis, const uint64_t lo[3], const uint64_t hi[3], double r,
                              int wave, double f0, double fc, double amplitude, uint64_t n_steps);

/* A lumped element over the node box lo..hi along `axis`
 * (LumpedElement::new(region).r(r).l(l).c(c).topology(t), src/engine/
 * lumped.rs:380-1013): r [ohm], l [H], c [F], each absent when <= 0;
 * series_topology 0 parallel (R and C folded into the edges, L as a branch),
 * 1 series (R + L + C as a branch, a lone R folded). record: record the
 * terminal current (record_current). port: a LumpedPort (a resistor that
 * also records V and I, src/engine/port.rs:102-290). amp[n]: the Thevenin
 * source value at (n + 1/2)*dt for step n < n_amp, 0 beyond (amp NULL: no
 * source); a source on a parallel element needs r. Returns the op index. */
int ems_model_add_lumped(ems_model* m, int axis, const uint64_t lo[3], const uint64_t hi[3], double r, double l,
                         double c, int series_topology, int record, int port, const double* amp, uint64_t n_amp);
/* A lumped element with an inductor or in series the way an openEMS file
 * has it (src/sim/map.rs:820-1000, 1525-1632; model built with openEMS's
 * rounding): R, L, C spread in csx's equal parts (R·p/s, L·p/s, C·s/p), the
 * element's C and 1/R replacing the medium's on its edges, the edge
 * capacitance limited at omega (> 0: 1/(20·omega·R_e), 1/(20·omega²·L_e)
 * of a parallel element, 1/(20·omega·|Z_e|) of a series branch), openEMS's
 * order around the branch, and for a parallel inductor with
 * explicit_inductor openEMS's explicit f32 update. src_w (per edge) and
 * amp[n] (the source at (n + 1/2)·dt): the element's Thevenin source of a
 * parallel element with a resistor, or NULL. Returns the op index. */
int ems_model_add_lumped_openems(ems_model* m, int axis, const uint64_t lo[3], const uint64_t hi[3], double r,
                                 double l, double c, int series_topology, double omega, int explicit_inductor,
                                 const double* src_w, const double* amp, uint64_t n_amp);

/* An edge source of `kind` (ems_source_kind) on n edges with the waveform
 * sampled for n_steps steps. nodes: 3*n indices. Returns the op index. */
int ems_model_add_source(ems_model* m, int kind, size_t n, const int* axis, const uint64_t* nodes,
                         const double* weight, int wave, double f0, double fc, uint64_t n_steps);

/* An edge source whose amplitude the caller has sampled: amp[n] is the
 * amplitude at the kind's sample time of step n (f64, rounded to f32 as
 * the reference does). Returns the op index. */
int ems_model_add_source_table(ems_model* m, int kind, size_t n, const int* axis, const uint64_t* nodes,
                               const double* weight, const double* amp, uint64_t n_steps);

/* A probe (Probe) on n entries; returns the op index. */
int ems_model_add_probe(ems_model* m, int quantity, size_t n, const int* axis, const uint64_t* nodes,
                        const double* weight, uint64_t interval);

/* A first-order Mur absorbing boundary (MurBoundary::with_faces /
 * with_faces_in, src/engine/boundary/mur.rs:355-604) on the faces f with
 * mode[f] = 1 (phase velocity velocity[f] m/s) or 2 (each edge's local
 * medium speed c0/sqrt(eps_r mu_r)); 0 leaves the face alone. Mur faces
 * must be PEC. hold_until (NULL: none): no update of the edges at face f
 * before step hold_until[f] (MurBoundary::hold_faces). flags: 1 openEMS
 * operation order, 2 openEMS shared-edge update, 4 count the boundary
 * edges' energy. Edges on two Mur faces take the mean of both updates.
 * Returns the op index or -1. */
int ems_model_add_mur(ems_model* m, const int mode[6], const double velocity[6], const uint64_t hold_until[6],
                      int flags);

/* An absorbing sheet inside the domain (csx AbsorbingBC, AbsorbingSheet::new,
 * src/engine/boundary/abc.rs:131-240): first-order Mur on the tangential E
 * edges of the rectangle start..stop (inclusive nodes; the normal entry
 * ignored) on mesh plane `plane` normal to `normal`, absorbing waves that
 * travel along +normal (positive) or -normal, at phase velocity `velocity`
 * [m/s] or, for velocity <= 0, the local c0/sqrt(eps_r mu_r) per edge;
 * openems_order: openEMS's order of the update and its f32 v·dt. Installed
 * as an EMS_OP_MUR table of face edges. Returns the op index or -1. */
int ems_model_add_absorbing_sheet(ems_model* m, int normal, uint64_t plane, int positive, const uint64_t start[3],
                                  const uint64_t stop[3], double velocity, int openems_order);

/* Conducting sheets (ConductingSheet::new(f_max), push, add_to;
 * src/engine/sheet.rs:529-935) on the built model, Cartesian, outlines on
 * mesh lines: n sheet edges, edge e the E edge along axis[e] at node
 * nodes[3e..3e+2] on a sheet normal to normal[e], of conductivity sigma[e]
 * [S/m] and thickness thickness[e] [m]; share_c/share_g (NULL, or < 0 for
 * an edge: the default) the shares of the edge's capacitance and
 * conductance on the + side. f_max: the highest frequency the layers
 * resolve (0: 1/(10 dt)). Edges are installed in node order; PEC edges and
 * duplicates are skipped. Writes the installed and skipped counts (either
 * may be NULL) and returns the op index, or -1 for an invalid edge or
 * f_max (nothing added). */
int ems_model_add_sheet(ems_model* m, size_t n, const int* axis, const uint64_t* nodes, const int* normal,
                        const double* sigma, const double* thickness, const double* share_c, const double* share_g,
                        double f_max, uint64_t* installed, uint64_t* skipped);

/* Layer thicknesses of a sheet (sigma, thickness) resolved up to f_max
 * (layer_profile, src/engine/sheet.rs:244-271): writes up to `cap` values
 * and returns their number. */
size_t ems_sheet_layer_profile(double sigma, double thickness, double f_max, double* out, size_t cap);

/* Field samplers (FieldSampler::new, src/engine/dump.rs:508-528): the
 * table (include/ems_gpu.h, ems_sampler) of `quantity` (ems_dump_quantity)
 * over the node box between corners a and b (any order, inclusive) with
 * `stride` (0 counts as 1; NULL: 1) at `position` 0 nodes, 1 cell centres
 * (the node along a degenerate axis), 2 native (raw edge values, no
 * interpolation). J, D and B take their factors from the built model's
 * coefficients. NULL for a box outside the grid (the model's error says
 * why). Cartesian grids. */
typedef struct ems_sampler_host ems_sampler_host;
ems_sampler_host* ems_sampler_new(ems_model* m, int quantity, int position, const uint64_t a[3], const uint64_t b[3],
                                  const uint64_t stride[3]);
/* FieldSampler::openems (src/engine/dump.rs:530-571): explicit increasing
 * sample indices per axis (node indices; cell indices for cell centres,
 * n - 1 the virtual cell beyond the last node, value 0) with openEMS's
 * rules: H at a node is the plain mean of its dual edges (0 on the outer
 * nodes), H along its axis at a cell centre interpolated between the dual
 * edges' midpoints, rot H over dual faces with full outer cells. */
ems_sampler_host* ems_sampler_new_indices(ems_model* m, int quantity, int position, const uint64_t* const idx[3],
                                          const size_t n[3]);
const ems_sampler* ems_sampler_table(const ems_sampler_host* s);
/* Coordinates [m] of the sample points along `axis` (*n of them). */
const double* ems_sampler_coords(const ems_sampler_host* s, int axis, size_t* n);
void ems_sampler_free(ems_sampler_host* s);

/* Sums probe `op`'s entries in f32 (openEMS's current probes, the
 * `f32_sum` of Probe, src/engine/probe.rs:381-392) when `on`. */
int ems_model_probe_f32(ems_model* m, int op, int on);

/* The engine descriptor (valid until the model changes or is freed). */
const ems_engine_desc* ems_model_desc(ems_model* m);

/* DFT X(f) = sum x(t0 + n dt) e^{-j 2 pi f t_n} dt (src/post/dft.rs:218). */
void ems_dft(double t0, double dt, const double* x, size_t n, const double* freqs, size_t nf, double* re,
             double* im);

/* The end-criterion run loop (src/engine/run.rs:424-540) over a stepper
 * given as callbacks. */
typedef struct {
    void* ctx;
    int (*run)(void* ctx, uint64_t n);
    int (*step_with_energy)(void* ctx, double* energy);
} ems_stepper;

typedef struct {
    uint64_t max_timesteps;
    int has_end_criteria;
    double energy_ratio;      /* stop when W/W_max < ratio (10^(dB/10)) */
    uint64_t check_interval;  /* K, default 50 */
    int has_excitation_end;
    double excitation_end;    /* checks count only for t > end */
    double dt;
} ems_run_limits;

typedef struct {
    int reason;               /* 0 energy decay, 1 max timesteps, 2 diverged, 3 stepper error */
    uint64_t steps;
    double energy;
    double max_energy;
    double ratio_db;
    uint64_t checks;
} ems_run_outcome;

int ems_drive(const ems_stepper* s, const ems_run_limits* limits, ems_run_outcome* out);

/* The same run loop for n models stepping together (an ems_batch): each
 * model gets exactly the checks, stop reason and step count ems_drive gives
 * it alone; a model that stops is frozen (set_active 0) while the others go
 * on. All limits must share check_interval. No counterpart in the
 * reference, which drives one engine at a time. */
typedef struct {
    void* ctx;
    size_t n_models;
    int (*run)(void* ctx, uint64_t n);
    int (*step_with_energy)(void* ctx, double* energies); /* n_models values */
    int (*set_active)(void* ctx, size_t model, int active);
} ems_batch_stepper;

int ems_batch_drive(const ems_batch_stepper* s, const ems_run_limits* limits, ems_run_outcome* out);

#ifdef __cplusplus
}
#endif

#endif
