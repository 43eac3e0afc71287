/*
 * oracle.h — CPU restatement of the ems engine's time stepping.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the CUDA engine is compared
 * with, and the timed CPU baseline; nothing in the product (ems_b200/) may
 * call it. It restates, in plain C++ with one thread per x-slab, the
 * reference engine's step (src/engine/pool.rs, kernel.rs, boundary/cpml.rs,
 * dispersive.rs, lumped.rs, excite.rs, probe.rs) and consumes the same
 * engine descriptor as the CUDA engine (include/ems_gpu.h).
 *
 * Pinning: the restatement follows the cited reference sources expression
 * by expression; it is checked against the reference's own analytic and
 * known-answer tests restated in tests/ (cavity modes, invariant energy,
 * CPML reflection levels, discrete dispersive susceptibility, lumped-port
 * matched line) and against the openEMS fixture series the reference
 * ships (tests/golden/).
 */
#ifndef EMS_ORACLE_H
#define EMS_ORACLE_H

#include "../include/ems_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_engine oracle_engine;

/* threads = 0: one per available core, capped like the reference's
 * default_threads_for (src/engine/mod.rs:404-428). */
int oracle_create(const ems_engine_desc* desc, int threads, oracle_engine** out);
int oracle_destroy(oracle_engine* e);
int oracle_threads(const oracle_engine* e);
/* 0: the reference's default curl order (a - b) - (c - d); 1: openEMS's
 * order with every operation flushed (CurlOrder, src/engine/kernel.rs:81-108). */
int oracle_set_curl_order(oracle_engine* e, int order);
/* The flux F and start value v of every edge of side `side` (0 E, 1 H) of
 * the EMS_OP_UPML operator `op`, in table order (cap >= the side's edges). */
int oracle_upml_state(oracle_engine* e, size_t op, int side, float* f, float* v, size_t cap);
int oracle_run(oracle_engine* e, uint64_t n);
int oracle_step_with_energy(oracle_engine* e, double* energy);
int oracle_download_field(oracle_engine* e, int field, int axis, float* host);
int oracle_upload_field(oracle_engine* e, int field, int axis, const float* host);
int oracle_samples(oracle_engine* e, size_t op, int which, double* out, size_t cap, size_t* n);
/* The current state sampled by `s` (FieldSampler::sample_with,
 * src/engine/dump.rs:836-906): 3 values per point, z fastest. */
int oracle_sample(oracle_engine* e, const ems_sampler* s, double* out);

#ifdef __cplusplus
}
#endif

#endif
