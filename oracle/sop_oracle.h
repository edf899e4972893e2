/*
 * sop_oracle.h — CPU restatement of SOP-GPU's Langevin step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: the parity tests, the
 * smoke check and the CPU baseline leg of the benchmark call it.  The product
 * library never links, loads or calls anything here.
 *
 * Every function restates one reference kernel or updater in plain C with
 * IEEE FP32 arithmetic in the reference's expression order (no fused
 * multiply-add, no fast math), plus an FP64 mirror of the force terms for
 * error statements.  File:line citations refer to the SOP-GPU source tree.
 */
#ifndef SOP_ORACLE_H
#define SOP_ORACLE_H

#include <stdint.h>
#include "../include/sopb.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_job orc_job;

/* The reference's PARAMETER() defaults (mandatory keys zero), written from
 * the headers under src/ for the oracle's own use, so that the CPU baseline
 * fills a job description without the product library. */
void orc_default_params(sopb_params* p);

/* ran2 as seen by a fresh process (src/Integrators/ran2.cpp:51-89). */
double orc_ran2(int32_t* idum, int32_t* state /* [34]: idum2, iy, iv[32] */);
void orc_ran2_state_init(int32_t* state);
/* generateSeeds (src/Integrators/ht.cu:40-56). */
void orc_generate_seeds(int32_t seed, int64_t count, uint32_t* out4);
/* One rforce() call (src/Integrators/ht.cu:93-106) for n beads: advances
 * seeds[4n] and writes 4 Gaussians per bead into out[4n]. */
void orc_rforce_n(int32_t n, uint32_t* seeds, float* out);
/* The HT integer stream: `draws` HybridTaus() outputs of one state. */
void orc_hybrid_taus(uint32_t* seed4, int32_t draws, uint32_t* out);

orc_job* orc_job_create(const sopb_job_desc* desc);
void orc_job_destroy(orc_job* job);
int orc_job_status(const orc_job* job);
int64_t orc_job_step(const orc_job* job);
/* runGPU's loop for nsteps steps (src/gsop.cu:129-148). */
int orc_job_advance(orc_job* job, int64_t nsteps);
/* Advances many jobs on `nthreads` OpenMP threads (one job per thread). */
int orc_jobs_advance(orc_job** jobs, int32_t njobs, int64_t nsteps, int32_t nthreads);
/* Potential forces at the current coordinates, FP32 (out4) and FP64 (out4d),
 * plus per component the FP32 rounding scale (abs4d): the magnitudes of the
 * quantities each term subtracts, for a condition-aware relative error.
 * Any output may be NULL. */
void orc_job_forces(orc_job* job, float* out4, double* out4d, double* abs4d);
void orc_job_read(const orc_job* job, int32_t what, void* out);
void orc_job_write(orc_job* job, int32_t what, const void* in);
void orc_job_rebuild(orc_job* job, int32_t possible, int32_t verlet);
void orc_job_pairlist(const orc_job* job, int32_t possible, int32_t* counts, int32_t* rows, int32_t cap);
/* The output manager's .dat quantities at the current coordinates
 * (src/Updaters/output_manager.cu:73-222, the energy kernels and
 * SOPPotential::sumEnergies): T, E_fene, E_native, E_pairs, E_total,
 * intact native contacts, Rg, TEA epsilon (0 without TEA). */
void orc_job_observables(const orc_job* job, double* out8);
/* Drains the pulling / indentation event log (sopb_log_row rows). */
int32_t orc_job_log(orc_job* job, sopb_log_row* rows, int32_t max_rows);

/* Exact-HI helpers (src/Integrators/bdhitea_kernel.cu:89-190). */
/* Normalised RPY tensor D (3n x 3n, row-major) at coords xyz[3n]. */
void orc_rpy_tensor(int32_t n, const float* xyz, float a, double* D);
/* The reference's in-place decomposition of a float matrix (stride m):
 * lower triangle = L, upper triangle = L^T. */
void orc_cholesky_ref(int32_t m, float* M);
/* B' of integrateCholesky_L: the symmetrised upper 3x3 blocks of M. */
void orc_ref_b_matrix(int32_t n, const float* M, double* B);

#ifdef __cplusplus
}
#endif

#endif
