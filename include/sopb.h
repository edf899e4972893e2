/*
 * sopb.h — C ABI of the B200-native SOP Langevin step.
 *
 * This is the drop-in boundary for SOP-GPU's hot path: the overdamped
 * Langevin step of the SOP C-alpha model (FENE bonds, native LJ 12-6,
 * repulsive r^-6 pairs, possible-pairs and Verlet pairlist rebuilds, the
 * Ermak-McCammon integrator with Hybrid Taus noise, force-ramp/force-clamp
 * pulling, continuous-surface nanoindentation and RPY hydrodynamic noise by
 * TEA or Cholesky).  Every entry point is plain C: pointers, sizes and int
 * status codes; no CUDA or torch types appear in any signature.  A CUDA
 * stream may be passed as an opaque pointer.
 *
 * Reference interfaces replaced (paths inside the SOP-GPU source tree):
 *   - SOPPotential / SOPUpdater / SOPIntegrator and the time loop
 *       src/gsop.h:69-105, src/gsop.cu:111-163
 *   - per-plugin device maps uploaded by constructors
 *       src/Potentials/covalent.cu:86-121, src/Potentials/native.cu:73-110,
 *       src/Updaters/pairlist.cu:60-128, src/Integrators/ht.cu:29-56
 *   - DIE()/exit(-1) error handling (src/Util/wrapper.cpp:28-42) becomes
 *     status codes; nothing in the library exits the process.
 *
 * Threading: a context is used from one host thread at a time.  All work on
 * a context is ordered on the context's stream.
 */
#ifndef SOPB_H
#define SOPB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SOPB_ABI_VERSION 1

/* Status codes.  The reference DIE()s on each of these conditions. */
enum {
    SOPB_OK = 0,
    SOPB_ERR_INVALID = 1,     /* bad argument or configuration               */
    SOPB_ERR_CAPACITY = 2,    /* a neighbour list outgrew its capacity        */
    SOPB_ERR_NONFINITE = 3,   /* a coordinate became NaN or Inf               */
    SOPB_ERR_CUDA = 4,        /* CUDA runtime error                           */
    SOPB_ERR_TIMEOUT = 5,     /* a bounded device wait ran out                */
    SOPB_ERR_NOMEM = 6,       /* device arena exhausted                       */
    SOPB_ERR_UNSUPPORTED = 7, /* feature combination not supported            */
    SOPB_ERR_HI = 8,          /* TEA "capricious" abort (epsilon > 1 etc.)    */
    SOPB_ERR_NODEVICE = 9     /* no CUDA device or library built without one  */
};

/* Pull direction (src/Potentials/pulling.h:21). */
enum { SOPB_PULL_END_TO_END = 0, SOPB_PULL_VECTOR = 1 };

/* HI noise treatment for hi_exact (src/Integrators/bdhitea_kernel.cu:303-361). */
enum {
    SOPB_HI_B_CHOLESKY = 0,   /* B = L, the true Cholesky factor of D         */
    SOPB_HI_B_REFCOMPAT = 1   /* the reference's symmetrised upper 3x3 blocks */
};

/*
 * Simulation parameters of one job.  Field names are the reference's config
 * keys (same meaning, same units: A, kcal/mol, tau_H).  sopb_default_params()
 * fills the reference defaults; mandatory keys without a default are zero.
 */
typedef struct sopb_params {
    /* Integrators/langevin.h:12-23 */
    float timestep;            /* h (mandatory)                               */
    float zeta;                /* 50                                           */
    float temperature;         /* 0.6                                          */
    int32_t minimization;      /* 0: no random force when 1                    */
    int32_t heating;           /* TemperatureUpdater on/off                    */
    float initialT;
    float deltaT;
    int32_t tempFreq;
    /* Potentials/covalent.h:12-14 */
    float kspring_cov;         /* 20                                           */
    float R_limit;             /* 2                                            */
    /* Potentials/pairs.h:12-15 */
    float a;                   /* 3.8                                          */
    float el;                  /* 1                                            */
    float pairs_cutoff;        /* 20: force cutoff                             */
    /* Updaters/pairlist.h:12-14, Updaters/possiblepairlist.h:12-13 */
    float pairlist_cutoff;     /* 20: Verlet list cutoff                       */
    int32_t pairs_freq;        /* 1000                                         */
    float pairs_threshold;     /* 200: possible-pairs cutoff                   */
    int32_t possiblepairs_freq;/* 100000                                       */
    int32_t max_pairs;         /* capacity of a bead's Verlet row (512)        */
    int32_t max_possiblePairs; /* capacity of a bead's possible-pairs row      */
    /* loop: gsop.h:34, gsop.cu:117-122 */
    int32_t nav;               /* 1000                                         */
    int32_t stride;            /* updater period; 0 = min(nav, frequencies)    */
    /* Potentials/pulling.h:15-26 */
    int32_t pulling;
    float deltax;              /* cantilever speed per pullFreq steps          */
    float k_trans;             /* 0.05                                         */
    float fconst;              /* force-clamp magnitude                        */
    int32_t pullFreq;          /* defaults to nav                              */
    int32_t pull_direction;    /* SOPB_PULL_*                                  */
    float pullVector[3];
    int32_t fixedEnd;
    int32_t pulledEnd;
    /* Potentials/indentation.h:12-38 (continuous surface) */
    int32_t indentation;
    float indentationChip[3];
    float indentationTip[3];
    float indentationDirection[3];
    float indentationSurfaceR0[3];
    float indentationSurfaceN[3];
    float indentationTipR;
    float indentationKs;
    float indentationDeltaX;
    int32_t indentationMoveSurface;
    int32_t indentationFixTrans;
    float indentationTipSigma, indentationTipEl, indentationTipA, indentationTipB;
    float indentationSurfSigma, indentationSurfEl, indentationSurfA, indentationSurfB;
    float indentationTipZeta;  /* 5000                                         */
    int64_t indentationRetractionStep; /* -1                                   */
    /* Integrators/bdhitea.h:15-21 */
    int32_t hi_on;
    int32_t hi_exact;
    float hi_a;                /* 1.8                                          */
    int32_t hi_epsilon_freq;
    int32_t hi_capricious;     /* 1                                            */
    int32_t hi_unlisted;       /* 1                                            */
    float hi_epsmax;           /* 999                                          */
    /* keys added by this library (do not change the meaning of old ones) */
    int32_t hi_b_mode;         /* SOPB_HI_B_*; default SOPB_HI_B_CHOLESKY      */
    int32_t hi_refresh;        /* refactor D every k steps (reference: 1)      */
    int32_t lanes_per_bead;    /* 0 = autotuned                                */
    int32_t cell_list;         /* possible pairs by cell list: 0 auto, 1 on, 2 off */
    int32_t grid_path;         /* 0 auto (resident kernel when it fits), 1 grid */
    float R_limit_bond;        /* 8: a native contact within it counts intact   */
    int32_t log_rows;          /* event-log ring of a pulling (deltax != 0),    */
                               /* indentation or pulling-plane job, rows; a   */
                               /* power of two, 0 = 1024                      */
    /* Potentials/indentation.h:39-47 (discrete surface) */
    int32_t indentationDiscreteSurf; /* surface as a square of beads           */
    int32_t indentationSurfaceSize;  /* 51: beads per side                     */
    float indentationSurfaceStep;    /* 1.4: bead spacing                      */
    float indentationPairsCutoff;    /* 40: surface-bead list cutoff           */
    /* Potentials/pulling_plane.h:12-27 */
    int32_t pullingPlane;
    float pullingPlaneDeltax;        /* cantilever displacement per update     */
    float pullingPlaneKs;            /* 0.05: bead-plane spring                */
    float pullingPlaneKsCant;        /* 0.05: plane-cantilever spring          */
    float pullingPlaneZeta;          /* 200: plane friction                    */
    float pullingPlaneDir[3];        /* plane normal (normalised on use)       */
    float pullingPlanePos[3];        /* a point of both planes at step 0       */
    int32_t pullingPlaneUpdateFreq;  /* defaults to nav                        */
    int32_t pullingPlaneOutputFreq;  /* defaults to nav                        */
    /* key added by this library */
    float verlet_skin;               /* near list kept between Verlet         */
                                     /* rebuilds: the possible pairs within   */
                                     /* pairlist_cutoff + skin, re-filtered   */
                                     /* until a bead moved skin/2; the Verlet */
                                     /* rows are those of a full filter.      */
                                     /* A; 0 = 4, < 0 = no near list          */
    int32_t reserved2[3];
} sopb_params;

/*
 * One job: a single SOP chain system (one "trajectory" of the reference).
 * Indices are 0-based bead numbers local to the job, as in the .top file.
 */
typedef struct sopb_job_desc {
    int32_t n;                         /* beads                               */
    const float* xyz;                  /* [3n] coordinates, A                 */
    int32_t nbonds;
    const int32_t* bonds;              /* [2*nbonds] (i, j) in .top order     */
    const float* bonds_r0;             /* [nbonds]                            */
    int32_t nnatives;
    const int32_t* natives;            /* [2*nnatives] (i, j)                 */
    const float* natives_r0;           /* [nnatives]                          */
    const float* natives_eh;           /* [nnatives]                          */
    int32_t nfixed;
    const int32_t* fixed;              /* pulling 'fixed' bead list           */
    int32_t npulled;
    const int32_t* pulled;             /* pulling 'pulled' bead list          */
    const uint32_t* seeds;             /* [4n] Hybrid Taus states, or NULL    */
    int32_t seed;                      /* used when seeds == NULL             */
    int32_t reserved;
    sopb_params params;
    int32_t nplane_fixed;
    const int32_t* plane_fixed;        /* pulling plane 'plane_fixed' beads   */
    int32_t nplane_pulled;
    const int32_t* plane_pulled;       /* pulling plane 'plane_pulled' beads  */
} sopb_job_desc;

typedef struct sopb_context sopb_context;
typedef struct sopb_job sopb_job;

/* Quantities readable from / writable to a job (sopb_job_read/_write). */
enum {
    SOPB_COORDS = 0,   /* float[4n]  x y z w, w = 0 (gsop.d_coord)           */
    SOPB_SEEDS = 1,    /* uint32[4n] Hybrid Taus states (ht.d_seeds)         */
    SOPB_TEMP = 2,     /* float[n]   kinetic temperature accumulator (d_T)    */
    SOPB_FORCES = 3,   /* float[4n]  potential forces at the current coords,  */
                       /*            computed on demand (read only)           */
    SOPB_TIPFORCES = 4,/* float[4n]  per-bead tip force accumulator           */
    SOPB_PULLSTATE = 5,/* float[12]  extForce[3] cant[3] cant0[3] vec[3]      */
    SOPB_TIPSTATE = 6, /* float[16]  tip[3] chip[3] micaR[3] V dx fav[4] pad  */
    SOPB_HISTATE = 7,  /* float[4]   TEA beta', epsilon (computeTEAeps), 0, 0 */
    SOPB_HIFACTOR = 8, /* float[9n^2] exact HI: the (3n)^2 tensor, row-major, */
                       /*            its lower triangle the Cholesky factor L */
                       /*            of D at the last refresh (read only);    */
                       /*            the upper triangle is unspecified (the   */
                       /*            reference-compatible noise mode keeps    */
                       /*            the reference's mirrored factor there)   */
    SOPB_OBSERVABLES = 9 /* double[8] the .dat columns of the output manager,  */
                       /* computed on the device at the current coordinates: */
                       /* T (averaged over beads and the nav window), FENE,  */
                       /* native and repulsive energies, their total, intact */
                       /* native contacts, Rg, TEA epsilon (0 without TEA)   */
                       /* (src/Updaters/output_manager.cu:73-222) (read only) */
};

/* ---- host utilities ---------------------------------------------------- */

/* ABI version (SOPB_ABI_VERSION). */
int sopb_version(void);

/* Human-readable text for a status code. */
const char* sopb_status_string(int status);

/* Fills *p with the reference defaults: the PARAMETER() defaults of the
 * integrator, potential and updater headers under src/ (langevin.h,
 * covalent.h, pairs.h, pairlist.h, possiblepairlist.h, pulling.h,
 * indentation.h, bdhitea.h). */
void sopb_default_params(sopb_params* p);

/* Hybrid Taus seeding: replaces initRand/generateSeeds
 * (src/Integrators/ht.cu:29-56) with ran2 (src/Integrators/ran2.cpp:51-89) as
 * seen by a fresh process.  Writes count uint4 states (4*count uint32) drawn
 * from one ran2 stream started at `seed` (the reference passes seed+firstrun
 * and draws all Ntr*N states of a multi-run job from that one stream). */
int sopb_generate_seeds(int32_t seed, int64_t count, uint32_t* out4);

/* ---- device context ------------------------------------------------------ */

/* Opens a context on `device`; work is ordered on `stream` (a cudaStream_t,
 * NULL = a new non-blocking stream owned by the context).  Replaces
 * initGPU() (src/gsop.cu:45-64). */
int sopb_context_create(int32_t device, void* stream, sopb_context** out);
int sopb_context_destroy(sopb_context* ctx);
/* Shape policy of the resident kernel for jobs created from now on: lanes
 * cooperating on one bead's force sum (a power of two up to 32, default
 * 4), and beads per lane group (default 1; the CTA holds about
 * n / beads_per_group groups, between 64 threads and max_block (default
 * 1024); <= 0 means one bead per group).  The defaults are the fastest
 * shape measured on a batch of 60-600-bead systems.  The autotuner's knob; a job keeps the shape it was
 * created with, so its result is the same alone and in any mix.  No
 * reference counterpart (the reference runs one thread per bead,
 * src/gsop.cuh:13). */
int sopb_context_set_shape_policy(sopb_context* ctx, int32_t lanes_per_bead, float beads_per_group, int32_t max_block);

/* Launch policy of grid-path HI jobs created from now on: the width of the
 * exact-HI factorisation's outer panels, in 128-column tiles (default 4:
 * each trailing tile is updated once per 512 columns), and the CTAs per SM
 * that the O(N^2) TEA and D F sums are sliced for (default 8).  Both change
 * only the order of floating-point sums; a job keeps the policy it was
 * created with.  The autotuner's knob for HI jobs; no reference counterpart
 * (the reference factorises unblocked, one CTA per trajectory,
 * src/Integrators/bdhitea_kernel.cu:154-190). */
int sopb_context_set_hi_policy(sopb_context* ctx, int32_t chol_panel_tiles, int32_t hi_ctas_per_sm);

/* Blocks until the context's stream and the streams its jobs last ran on
 * drain. */
int sopb_context_sync(sopb_context* ctx);

/* Device bytes a job needs (admission by HBM footprint): its maps and
 * lists, its share of the context's bead pools and, for a job on the grid
 * path (HI, above 2048 beads, or grid_path 1), its own buffers -- the HI
 * buffers and the exact-HI tensor included -- sized for the current
 * device.  Host arithmetic only; the reference has no counterpart (each of
 * its plugins allocates in its constructor). */
int sopb_job_footprint(const sopb_job_desc* desc, size_t* bytes);

/* Builds a job's device state: coordinates, covalent and native maps,
 * list storage, RNG states, pulling flags.  Replaces the constructors of
 * CovalentPotential, NativePotential, PairsPotential, PairList,
 * PossiblepairList, PullingPotential, IndentationPotential, LangevinIntegrator
 * and TeaIntegrator (src/gsop.cu:66-106). */
int sopb_job_create(sopb_context* ctx, const sopb_job_desc* desc, sopb_job** out);
int sopb_job_destroy(sopb_job* job);

/* Advances every job in `jobs` by `nsteps` Langevin steps.  For each job and
 * each step it does what one pass of runGPU's inner loop does
 * (src/gsop.cu:129-148): at step % stride == 0 the updaters run in the
 * reference order (indentation tip, pulling, possible pairs, temperature
 * reset, pairlist, heating, TEA), then all potentials are summed and the
 * integrator moves the beads.  Asynchronous on the context stream. */
int sopb_run(sopb_context* ctx, sopb_job* const* jobs, int32_t njobs, int64_t nsteps);

/* sopb_run ordered on `stream` (a cudaStream_t; NULL = the context stream)
 * instead of the context stream, so groups of jobs advance independently:
 * a serving loop gives each long job its own stream and polls for
 * completion instead of waiting for the slowest job of a batch.  A job's
 * work stays ordered across streams (a run starts after the job's previous
 * work, wherever it ran).  Reads, writes and sopb_job_destroy of a job are
 * ordered on the stream it last ran on; destroy does not wait: the job's
 * memory, bead range and slot are released once its last work finished.
 * No reference counterpart (the reference runs one job on the default
 * stream, src/gsop.cu:111-163). */
int sopb_run_on(sopb_context* ctx, sopb_job* const* jobs, int32_t njobs, int64_t nsteps, void* stream);

/* sopb_run_on with a step count per job (nsteps[k] >= 0 for jobs[k]): one
 * launch serves jobs that need different numbers of steps, each CTA of the
 * replica-resident kernel stopping at its own job's count.  No reference
 * counterpart. */
int sopb_run_ragged(sopb_context* ctx, sopb_job* const* jobs, int32_t njobs, const int64_t* nsteps, void* stream);

/* Device-reported status of a job (after sopb_context_sync). */
int sopb_job_status(sopb_job* job);
/* Current step counter of a job. */
int sopb_job_step(sopb_job* job, int64_t* step);
/* Bead count of a job. */
int sopb_job_size(sopb_job* job, int32_t* n);

/* Launch shape of a job's resident kernel: lanes cooperating on one bead
 * and the CTA size class.  A function of the job alone (not of the batch
 * it runs in); a job's launch class groups it with same-class jobs.  No
 * reference counterpart (the reference fixes one thread per bead,
 * src/gsop.cuh:13). */
int sopb_job_shape(sopb_job* job, int32_t* lanes_per_bead, int32_t* block);

/* Copies a quantity of one job to / from host memory (synchronous). */
int sopb_job_read(sopb_job* job, int32_t what, void* host_out);
int sopb_job_write(sopb_job* job, int32_t what, const void* host_in);

/* Reads the current Verlet pairlist (or possible-pairs list when
 * possible != 0) in the reference layout: counts[n] and a row of `cap`
 * entries per bead, -1 padded (d_pairs / d_pairsCount,
 * src/Updaters/pairlist_kernel.cu:33-76). */
int sopb_job_pairlist(sopb_job* job, int32_t possible, int32_t* counts, int32_t* rows, int32_t cap);

/* Rebuilds the possible-pairs list and/or the pairlist of a job now
 * (PossiblepairList::update / PairList::update without the step gate). */
int sopb_job_rebuild_lists(sopb_job* job, int32_t possible, int32_t verlet);

/* ---- event log --------------------------------------------------------
 * The reference's pulling and indentation updaters print one line per
 * update from the host (src/Potentials/pulling.cu:167-190,
 * src/Potentials/indentation.cu:440-534).  Here those updaters run inside
 * the step kernel, which appends the values to a per-job ring on the
 * device; the caller drains it at its output times.
 *
 * SOPB_LOG_PULL, at every step % pullFreq == 0 of a force-ramp job:
 *   v[0] |x[pulledEnd] - x[fixedEnd]|, v[1] that vector . pull vector,
 *   v[2] extForce . pull vector, v[3..5] extForce (the force applied from
 *   this step on).
 * SOPB_LOG_TIP, at every step % nav == 0 of an indentation job, after the
 *   tip's own step: v[0..2] the tip force averaged over nav, v[3] its norm,
 *   v[4] |chip - tip| before the tip moved, v[5] dx, v[6..8] the tip after
 *   the move, v[9..11] the cantilever base (chip).
 * SOPB_LOG_PLANE, at every step % pullingPlaneOutputFreq == 0 of a
 *   pulling-plane job, after the plane's own step
 *   (src/Potentials/pulling_plane.cu:183-258): v[0] the plane displacement,
 *   v[1] the cantilever displacement, v[2] the cantilever force on the
 *   plane, v[3] the beads' force on the plane, v[4] the distance between
 *   the centroids of the fixed and the pulled beads.
 */
typedef struct sopb_log_row {
    int32_t kind;                      /* SOPB_LOG_PULL or SOPB_LOG_TIP        */
    int32_t pad;
    int64_t step;
    float v[12];
} sopb_log_row;
enum { SOPB_LOG_PULL = 1, SOPB_LOG_TIP = 2, SOPB_LOG_PLANE = 3 };

/* Copies the rows appended since the last drain, oldest first, at most
 * max_rows of them, and sets *nrows.  Rows left over stay for the next
 * call.  Returns SOPB_ERR_CAPACITY (the rows still come back) when the
 * ring wrapped before the drain and the oldest rows were lost.  No
 * reference counterpart. */
int sopb_job_log(sopb_job* job, sopb_log_row* rows, int32_t max_rows, int32_t* nrows);

/* Bulk transfer of the coordinates of many jobs with one copy each way:
 * host_xyzw holds sum(n_j) float4 in the order of `jobs`. */
int sopb_jobs_upload_coords(sopb_context* ctx, sopb_job* const* jobs, int32_t njobs, const float* host_xyzw);
int sopb_jobs_download_coords(sopb_context* ctx, sopb_job* const* jobs, int32_t njobs, float* host_xyzw);

/* TEA coupling coefficients of one system, allocating no device memory.
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * programs that own all device memory through their own pool and do not let
 * a library allocate behind them, or code ordering work on a stream where an
 * allocation would stall or break it.  Runs the TEA updater's kernels (all
 * pairs, as hi_unlisted) on caller-owned device buffers:
 *   d_xyzw     in:  float[4n] coordinates (x y z w);
 *   d_ci4      out: float[4n] per bead, the squared row sums of the normalised
 *                   RPY blocks (x y z) and the sum of their entries (w), the
 *                   reference's d_ci / d_epsilon (bdhitea_kernel.cu:234-249);
 *   d_beta_eps out: float[2] beta' and epsilon (bdhitea.cu:143-169, as with
 *                   hi_capricious off: an epsilon above 1 is set to 1 without
 *                   an error, and hi_epsmax is not checked -- a caller that
 *                   needs either test compares epsilon with 1 or its limit).
 * d_xyzw and d_ci4 must be 16-byte aligned and d_beta_eps 4-byte aligned
 * (SOPB_ERR_INVALID otherwise).
 * Scratch is a 4 MiB array in the library image (held by every GPU that
 * loads the library until exit), shared by all calls: calls that overlap on
 * the GPU race and must be ordered by the caller.  n up to 262144 beads
 * (SOPB_ERR_CAPACITY above).  The first call in each CUDA context (the
 * device's primary context, one made with cuCtxCreate, or the new primary
 * context after a cudaDeviceReset) does a one-time set-up and should come
 * before any stream capture.  Work is queued on `stream` (a cudaStream_t,
 * NULL = the default stream); the call does not wait for it. */
int sopb_tea_coefficients_noalloc(const float* d_xyzw, int32_t n, float hi_a, float* d_ci4, float* d_beta_eps,
                                  void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SOPB_H */
