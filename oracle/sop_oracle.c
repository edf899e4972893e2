/*
 * sop_oracle.c — CPU restatement of SOP-GPU's Langevin step (test oracle).
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and the CPU
 * baseline leg of bench.py as the checker.  Never part of the product path.
 *
 * Arithmetic: IEEE binary32 in the reference's expression order, compiled
 * with -ffp-contract=off and without fast math, so integer outputs (seeds,
 * Hybrid Taus states, neighbour lists) are bit-exact restatements and float
 * outputs are the reference formulas evaluated in round-to-nearest.  FP64
 * mirrors of the force terms give error statements.  Citations are
 * path:line in the SOP-GPU source tree.
 */
#include "sop_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define F4(a, i) (&(a)[4 * (size_t)(i)])

/* ------------------------------------------------------------------------ */
/* PARAMETER() defaults of the reference headers; keys this library adds    */
/* take the values that keep the reference's behaviour.                     */
/* ------------------------------------------------------------------------ */
void orc_default_params(sopb_params* p) {
    memset(p, 0, sizeof(*p));
    p->zeta = 50.0f;                    /* Integrators/langevin.h:13 */
    p->temperature = 0.6f;              /* Integrators/langevin.h:14 */
    p->kspring_cov = 20.0f;             /* Potentials/covalent.h:12 */
    p->R_limit = 2.0f;                  /* Potentials/covalent.h:13 */
    p->R_limit_bond = 8.0f;             /* the output manager's intact-contact cutoff */
    p->pairs_cutoff = 20.0f;            /* Potentials/pairs.h:12 */
    p->el = 1.0f;                       /* Potentials/pairs.h:13 */
    p->a = 3.8f;                        /* Potentials/pairs.h:14 */
    p->max_pairs = 512;                 /* Potentials/pairs.h:15 */
    p->pairlist_cutoff = 20.0f;         /* Updaters/pairlist.h:12 */
    p->pairs_freq = 1000;               /* Updaters/pairlist.h:13 */
    p->max_possiblePairs = 4096;        /* Updaters/pairlist.h:14 */
    p->pairs_threshold = 200.0f;        /* Updaters/possiblepairlist.h:14 */
    p->possiblepairs_freq = 100000;     /* Updaters/possiblepairlist.h:15 */
    p->nav = 1000;                      /* gsop.h, nav */
    p->k_trans = 0.05f;                 /* Potentials/pulling.h:17 */
    p->pull_direction = SOPB_PULL_END_TO_END;   /* Potentials/pulling.h:21 */
    p->indentationTipSigma = 1.0f;      /* Potentials/indentation.h:24-25 */
    p->indentationSurfSigma = 1.0f;     /* Potentials/indentation.h:24,26 */
    p->indentationTipEl = 1.0f;         /* Potentials/indentation.h:27-28 */
    p->indentationSurfEl = 1.0f;        /* Potentials/indentation.h:27,29 */
    p->indentationTipA = 0.0f;          /* Potentials/indentation.h:30 */
    p->indentationTipB = 1.0f;          /* Potentials/indentation.h:31 */
    p->indentationSurfA = 0.0f;         /* Potentials/indentation.h:32 */
    p->indentationSurfB = 1.0f;         /* Potentials/indentation.h:33 */
    p->indentationTipZeta = 5000.0f;    /* Potentials/indentation.h:35 */
    p->indentationRetractionStep = -1;  /* Potentials/indentation.h:37 */
    p->indentationPairsCutoff = 40.0f;  /* Potentials/indentation.h:41 */
    p->indentationSurfaceSize = 51;     /* Potentials/indentation.h:45 */
    p->indentationSurfaceStep = 1.4f;   /* Potentials/indentation.h:46 */
    p->pullingPlaneKs = 0.05f;          /* Potentials/pulling_plane.h:15 */
    p->pullingPlaneKsCant = 0.05f;      /* Potentials/pulling_plane.h:16 */
    p->pullingPlaneZeta = 200.0f;       /* Potentials/pulling_plane.h:17 */
    p->hi_a = 1.8f;                     /* Integrators/bdhitea.h:17 */
    p->hi_capricious = 1;               /* Integrators/bdhitea.h:19 */
    p->hi_unlisted = 1;                 /* Integrators/bdhitea.h:20 */
    p->hi_epsmax = 999.0f;              /* Integrators/bdhitea.h:21 */
    p->hi_b_mode = SOPB_HI_B_CHOLESKY;
    p->hi_refresh = 1;                  /* the reference refactors D every step */
}

/* ------------------------------------------------------------------------ */
/* ran2: L'Ecuyer's combined LCG with a Bays-Durham shuffle, in the form of */
/* Numerical Recipes (src/Integrators/ran2.cpp:51-89).  The reference keeps */
/* idum2/iy/iv in static storage; a fresh process starts from idum2 =       */
/* 123456789, iy = 0, iv = {0}.  A positive seed skips the table warm-up.   */
/* ------------------------------------------------------------------------ */
enum { R2_IM1 = 2147483563, R2_IM2 = 2147483399, R2_IA1 = 40014, R2_IA2 = 40692,
       R2_IQ1 = 53668, R2_IQ2 = 52774, R2_IR1 = 12211, R2_IR2 = 3791, R2_NTAB = 32 };
#define R2_AM (1.0 / R2_IM1)
#define R2_IMM1 (R2_IM1 - 1)
#define R2_NDIV (1 + R2_IMM1 / R2_NTAB)
#define R2_RNMX (1.0 - 1.2e-7)

void orc_ran2_state_init(int32_t* st) {
    memset(st, 0, 34 * sizeof(int32_t));
    st[0] = 123456789;
}

double orc_ran2(int32_t* idum, int32_t* st) {
    int32_t* idum2 = &st[0];
    int32_t* iy = &st[1];
    int32_t* iv = &st[2];
    int32_t j, k;
    if (*idum <= 0) {
        if (-(*idum) < 1) *idum = 1;
        else *idum = -(*idum);
        *idum2 = *idum;
        for (j = R2_NTAB + 7; j >= 0; j--) {
            k = *idum / R2_IQ1;
            *idum = R2_IA1 * (*idum - k * R2_IQ1) - k * R2_IR1;
            if (*idum < 0) *idum += R2_IM1;
            if (j < R2_NTAB) iv[j] = *idum;
        }
        *iy = iv[0];
    }
    k = *idum / R2_IQ1;
    *idum = R2_IA1 * (*idum - k * R2_IQ1) - k * R2_IR1;
    if (*idum < 0) *idum += R2_IM1;
    k = *idum2 / R2_IQ2;
    *idum2 = R2_IA2 * (*idum2 - k * R2_IQ2) - k * R2_IR2;
    if (*idum2 < 0) *idum2 += R2_IM2;
    j = *iy / R2_NDIV;
    *iy = iv[j] - *idum2;
    iv[j] = *idum;
    if (*iy < 1) *iy += R2_IMM1;
    double t = R2_AM * (*iy);
    return t > R2_RNMX ? R2_RNMX : t;
}

/* generateSeeds (src/Integrators/ht.cu:40-56): each component is
 * (unsigned)(ran2*UINT_MAX), redrawn while < 128. */
void orc_generate_seeds(int32_t seed, int64_t count, uint32_t* out4) {
    int32_t st[34];
    orc_ran2_state_init(st);
    int32_t s = seed;
    for (int64_t i = 0; i < count; i++) {
        for (int c = 0; c < 4; c++) {
            uint32_t v;
            do {
                v = (uint32_t)(orc_ran2(&s, st) * (double)UINT_MAX);
            } while (v < 128u);
            out4[4 * i + c] = v;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Hybrid Taus (GPU Gems 3 ch. 37; src/Integrators/ht.cu:61-106).           */
/* ------------------------------------------------------------------------ */
static inline uint32_t taus_step(uint32_t* z, int s1, int s2, int s3, uint32_t m) {
    uint32_t b = (((*z << s1) ^ *z) >> s2);
    *z = (((*z & m) << s3) ^ b);
    return *z;
}
static inline uint32_t lcg_step(uint32_t* z, uint32_t a, uint32_t c) {
    *z = a * *z + c;
    return *z;
}
static inline uint32_t hybrid_taus(uint32_t* s) {
    uint32_t x = taus_step(&s[0], 13, 19, 12, 4294967294u);
    uint32_t y = taus_step(&s[1], 2, 25, 4, 4294967288u);
    uint32_t z = taus_step(&s[2], 3, 11, 17, 4294967280u);
    uint32_t w = lcg_step(&s[3], 1664525u, 1013904223u);
    return x ^ y ^ z ^ w;
}
static inline float uint_to_float(uint32_t u) {
    uint32_t bits = 0x3f800000u | (0x007fffffu & u);
    float f;
    memcpy(&f, &bits, 4);
    f = f - 1.0f;
    return f == 0.0f ? 1.0e-8f : f;
}
void orc_hybrid_taus(uint32_t* seed4, int32_t draws, uint32_t* out) {
    for (int32_t d = 0; d < draws; d++) out[d] = hybrid_taus(seed4);
}
/* rforce: Box-Muller on 4 draws; theta = 2*pi*u evaluated in double and
 * rounded to float as the reference's `2.0f*M_PI*u` is. */
static inline void rforce(uint32_t* s, float* g) {
    float r = sqrtf(-2.0f * logf(uint_to_float(hybrid_taus(s))));
    float theta = (float)(2.0 * M_PI * (double)uint_to_float(hybrid_taus(s)));
    g[0] = r * sinf(theta);
    g[1] = r * cosf(theta);
    r = sqrtf(-2.0f * logf(uint_to_float(hybrid_taus(s))));
    theta = (float)(2.0 * M_PI * (double)uint_to_float(hybrid_taus(s)));
    g[2] = r * sinf(theta);
    g[3] = r * cosf(theta);
}
void orc_rforce_n(int32_t n, uint32_t* seeds, float* out) {
    for (int32_t i = 0; i < n; i++) rforce(&seeds[4 * i], &out[4 * i]);
}

/* ------------------------------------------------------------------------ */
/* Job state                                                                 */
/* ------------------------------------------------------------------------ */
struct orc_job {
    int32_t n;
    sopb_params p;
    /* per-bead maps in the reference's slot order (covalent.cu:126-157,
     * native.cu:112-146): row-major here, [i*cap + k]. */
    int32_t cap_cov, cap_nat, cap_pp, cap_pl;
    int32_t *cov_cnt, *cov_j;
    float* cov_r0;
    int32_t *nat_cnt, *nat_j;
    float *nat_r02, *nat_m12;
    double *nat_r0d, *nat_ehd;
    int32_t *pp_cnt, *pp_j;
    int32_t *pl_cnt, *pl_j;
    float *x, *f, *T, *extF, *tipF;
    uint32_t* seeds;
    int64_t step;
    int32_t stride;
    /* Langevin constants (langevin.cu:17-62) */
    float var, hOverZeta, tempNorm, temp;
    /* FENE / LJ constants */
    float ks, R2, a2, m6, cut2;
    /* pulling (pulling.cu:36-214) */
    float pullvec[3], cant0[3], cant[3], extForce[3];
    int32_t npulled;
    int32_t* pulled;
    /* indentation (indentation.cu:75-207, 414-550) */
    float tip[3], chip[3], chip0[3], dir[3], micaR[3], micaR0[3], micaN[3];
    float tipR, tipAp, tipBp, surfAp, surfBp, cantKs, V, dx, tipZeta;
    float fav[4];
    /* HI (bdhitea.cu) */
    float *rf, *mf, *xc, *ci4, *eps;
    float beta, epsilon;
    float* tensor;
    int32_t status;
    int32_t refresh_due;   /* exact HI: refactorise D at the next step */
    /* the per-update lines of the pulling and indentation updaters */
    sopb_log_row* log;
    int32_t log_len, log_cap;
    /* discrete surface (indentation.cu:137-201, 311-362) */
    int32_t nsurf;
    float *surf0, *surf;     /* surface beads at dx = 0 and now, xyz */
    int32_t *mica_cnt, *mica_j, cap_mica;
    /* pulling plane (pulling_plane.cu:35-266) */
    uint8_t* plane_mask;     /* 1 fixed plane, 2 pulled plane */
    float *plane_r0, *plane_f;
    float plane_n[3], plane_p0[3], plane_displ, plane_cant;
};

static int32_t compute_stride(const sopb_params* p) {
    if (p->stride > 0) return p->stride;
    int32_t s = p->nav;
#define MINF(v) do { if ((v) > 0 && (v) < s) s = (v); } while (0)
    MINF(p->pairs_freq);
    MINF(p->possiblepairs_freq);
    if (p->pulling && p->deltax != 0.0f) MINF(p->pullFreq > 0 ? p->pullFreq : p->nav);
    if (p->heating) MINF(p->tempFreq);
    if (p->hi_on && !p->hi_exact) MINF(p->hi_epsilon_freq);
    if (p->hi_on && p->hi_exact && p->hi_refresh > 1) MINF(p->hi_refresh);   /* factor refresh updater */
    if (p->pullingPlane) MINF(p->pullingPlaneUpdateFreq > 0 ? p->pullingPlaneUpdateFreq : p->nav);
#undef MINF
    return s;
}

static void set_temperature(orc_job* j, float temp) {
    /* LangevinIntegrator::setTemperature (langevin.cu:44-48) */
    j->temp = temp;
    j->var = sqrtf(2.0f * temp * j->p.zeta / j->p.timestep);
}

orc_job* orc_job_create(const sopb_job_desc* d) {
    if (!d || d->n <= 0 || !d->xyz) return NULL;
    orc_job* j = (orc_job*)calloc(1, sizeof(orc_job));
    const int32_t n = d->n;
    j->n = n;
    j->p = d->params;
    const sopb_params* p = &j->p;
    /* covalent map (covalent.cu:65-109) */
    int32_t* cnt = (int32_t*)calloc(n, sizeof(int32_t));
    for (int32_t k = 0; k < d->nbonds; k++) { cnt[d->bonds[2 * k]]++; cnt[d->bonds[2 * k + 1]]++; }
    int32_t mx = 1;
    for (int32_t i = 0; i < n; i++) if (cnt[i] > mx) mx = cnt[i];
    j->cap_cov = mx;
    j->cov_cnt = (int32_t*)calloc(n, sizeof(int32_t));
    j->cov_j = (int32_t*)calloc((size_t)n * mx, sizeof(int32_t));
    j->cov_r0 = (float*)calloc((size_t)n * mx, sizeof(float));
    for (int32_t k = 0; k < d->nbonds; k++) {
        int32_t a = d->bonds[2 * k], b = d->bonds[2 * k + 1];
        j->cov_j[a * mx + j->cov_cnt[a]] = b;
        j->cov_r0[a * mx + j->cov_cnt[a]] = d->bonds_r0[k];
        j->cov_cnt[a]++;
        j->cov_j[b * mx + j->cov_cnt[b]] = a;
        j->cov_r0[b * mx + j->cov_cnt[b]] = d->bonds_r0[k];
        j->cov_cnt[b]++;
    }
    /* native map (native.cu:112-146) */
    memset(cnt, 0, n * sizeof(int32_t));
    for (int32_t k = 0; k < d->nnatives; k++) { cnt[d->natives[2 * k]]++; cnt[d->natives[2 * k + 1]]++; }
    mx = 1;
    for (int32_t i = 0; i < n; i++) if (cnt[i] > mx) mx = cnt[i];
    j->cap_nat = mx;
    j->nat_cnt = (int32_t*)calloc(n, sizeof(int32_t));
    j->nat_j = (int32_t*)calloc((size_t)n * mx, sizeof(int32_t));
    j->nat_r02 = (float*)calloc((size_t)n * mx, sizeof(float));
    j->nat_m12 = (float*)calloc((size_t)n * mx, sizeof(float));
    j->nat_r0d = (double*)calloc((size_t)n * mx, sizeof(double));
    j->nat_ehd = (double*)calloc((size_t)n * mx, sizeof(double));
    for (int32_t k = 0; k < d->nnatives; k++) {
        int32_t ab[2] = {d->natives[2 * k], d->natives[2 * k + 1]};
        float r0 = d->natives_r0[k], eh = d->natives_eh[k];
        for (int s = 0; s < 2; s++) {
            int32_t a = ab[s], b = ab[1 - s];
            int32_t slot = a * mx + j->nat_cnt[a];
            j->nat_j[slot] = b;
            j->nat_r02[slot] = r0 * r0;
            j->nat_m12[slot] = (float)(-12.0 * (double)eh / (double)(r0 * r0));
            j->nat_r0d[slot] = r0;
            j->nat_ehd[slot] = eh;
            j->nat_cnt[a]++;
        }
    }
    free(cnt);
    j->cap_pp = p->max_possiblePairs > 0 ? p->max_possiblePairs : 4096;
    j->cap_pl = p->max_pairs > 0 ? p->max_pairs : 512;
    j->pp_cnt = (int32_t*)calloc(n, sizeof(int32_t));
    j->pp_j = (int32_t*)malloc((size_t)n * j->cap_pp * sizeof(int32_t));
    j->pl_cnt = (int32_t*)calloc(n, sizeof(int32_t));
    j->pl_j = (int32_t*)malloc((size_t)n * j->cap_pl * sizeof(int32_t));
    for (size_t q = 0; q < (size_t)n * j->cap_pl; q++) j->pl_j[q] = -1;
    /* coordinates: gsop.cu:185-199 (w = 0) */
    j->x = (float*)calloc(4 * (size_t)n, sizeof(float));
    for (int32_t i = 0; i < n; i++) {
        j->x[4 * i] = d->xyz[3 * i];
        j->x[4 * i + 1] = d->xyz[3 * i + 1];
        j->x[4 * i + 2] = d->xyz[3 * i + 2];
    }
    j->f = (float*)calloc(4 * (size_t)n, sizeof(float));
    j->T = (float*)calloc(n, sizeof(float));
    j->extF = (float*)calloc(4 * (size_t)n, sizeof(float));
    j->tipF = (float*)calloc(4 * (size_t)n, sizeof(float));
    j->seeds = (uint32_t*)malloc(16 * (size_t)n);
    if (d->seeds) memcpy(j->seeds, d->seeds, 16 * (size_t)n);
    else orc_generate_seeds(d->seed, n, j->seeds);
    /* constants */
    j->stride = compute_stride(p);
    j->hOverZeta = p->timestep / p->zeta;
    j->tempNorm = (float)(p->zeta / (6.0 * p->timestep));
    set_temperature(j, p->heating ? p->initialT : p->temperature);
    j->ks = p->kspring_cov;
    j->R2 = p->R_limit * p->R_limit;
    j->a2 = p->a * p->a;
    j->m6 = -6.0f * p->el / j->a2;
    j->cut2 = p->pairs_cutoff * p->pairs_cutoff;
    /* pulling (pulling.cu:36-146) */
    if (p->pulling) {
        const float* xp = F4(j->x, p->pulledEnd);
        const float* xf = F4(j->x, p->fixedEnd);
        if (p->pull_direction == SOPB_PULL_VECTOR) {
            memcpy(j->pullvec, p->pullVector, 12);
        } else {
            float v[3] = {xp[0] - xf[0], xp[1] - xf[1], xp[2] - xf[2]};
            float len = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            for (int c = 0; c < 3; c++) j->pullvec[c] = v[c] / len;
        }
        for (int c = 0; c < 3; c++) j->cant0[c] = j->cant[c] = xp[c];
        j->npulled = d->npulled;
        j->pulled = (int32_t*)malloc((d->npulled + 1) * sizeof(int32_t));
        for (int32_t k = 0; k < d->npulled; k++) {
            int32_t i = d->pulled[k];
            j->pulled[k] = i;
            float* e = F4(j->extF, i);
            for (int c = 0; c < 3; c++) e[c] = j->pullvec[c] * p->fconst;
            e[3] = 2.0f;
        }
        for (int32_t k = 0; k < d->nfixed; k++) {
            float* e = F4(j->extF, d->fixed[k]);
            e[0] = e[1] = e[2] = 0.0f;
            e[3] = 1.0f;
        }
    }
    /* indentation (indentation.cu:75-137) */
    if (p->indentation) {
        for (int c = 0; c < 3; c++) {
            j->chip[c] = j->chip0[c] = p->indentationChip[c];
            j->tip[c] = p->indentationTip[c];
            j->dir[c] = p->indentationDirection[c];
            j->micaR[c] = j->micaR0[c] = p->indentationSurfaceR0[c];
            j->micaN[c] = p->indentationSurfaceN[c];
        }
        j->tipR = p->indentationTipR;
        j->cantKs = p->indentationKs;
        j->V = p->indentationDeltaX;
        j->dx = 0.0f;
        j->tipZeta = p->indentationTipZeta;
        j->tipAp = 12.0f * p->indentationTipEl * powf(p->indentationTipSigma, 12.0f) * p->indentationTipA;
        j->tipBp = 6.0f * p->indentationTipEl * powf(p->indentationTipSigma, 6.0f) * p->indentationTipB;
        j->surfAp = 12.0f * p->indentationSurfEl * powf(p->indentationSurfSigma, 12.0f) * p->indentationSurfA;
        j->surfBp = 6.0f * p->indentationSurfEl * powf(p->indentationSurfSigma, 6.0f) * p->indentationSurfB;
        float nrm = sqrtf(j->dir[0] * j->dir[0] + j->dir[1] * j->dir[1] + j->dir[2] * j->dir[2]);
        for (int c = 0; c < 3; c++) j->dir[c] /= nrm;
        nrm = sqrtf(j->micaN[0] * j->micaN[0] + j->micaN[1] * j->micaN[1] + j->micaN[2] * j->micaN[2]);
        for (int c = 0; c < 3; c++) j->micaN[c] /= nrm;
        if (p->indentationDiscreteSurf) {
            /* the square of surface beads of IndentationAminoUpdater
             * (indentation.cu:311-362), from the configured, unnormalised
             * surface normal */
            const int32_t S = p->indentationSurfaceSize;
            const float* nn = p->indentationSurfaceN;
            const float* r0 = p->indentationSurfaceR0;
            float r1[3];
            if (nn[0] == 0) { r1[0] = 1.0f; r1[1] = 0; r1[2] = 0; }
            else if (nn[1] == 0) { r1[0] = 0; r1[1] = 1.0f; r1[2] = 0; }
            else if (nn[2] == 0) { r1[0] = 0; r1[1] = 0; r1[2] = 1.0f; }
            else { r1[0] = 0; r1[1] = 1.0f; r1[2] = -(nn[1] / nn[2]) * r1[1]; }
            float norm = sqrtf(r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2]);
            for (int c = 0; c < 3; c++) r1[c] /= norm;
            float r2[3] = {nn[1] * r1[2] - nn[2] * r1[1], nn[2] * r1[0] - nn[0] * r1[2], nn[0] * r1[1] - nn[1] * r1[0]};
            j->nsurf = S * S;
            j->surf0 = (float*)malloc(3 * sizeof(float) * (size_t)j->nsurf);
            j->surf = (float*)malloc(3 * sizeof(float) * (size_t)j->nsurf);
            const float displ = p->indentationSurfaceStep;
            for (int32_t a = 0; a < S; a++)
                for (int32_t b = 0; b < S; b++) {
                    const int32_t i1 = a - S / 2, i2 = b - S / 2;
                    float* q = j->surf0 + 3 * (a * S + b);
                    for (int c = 0; c < 3; c++) q[c] = r0[c] + i1 * displ * r1[c] + i2 * displ * r2[c];
                }
            memcpy(j->surf, j->surf0, 3 * sizeof(float) * (size_t)j->nsurf);
            j->cap_mica = j->nsurf;
            j->mica_cnt = (int32_t*)calloc(n, sizeof(int32_t));
            j->mica_j = (int32_t*)malloc(sizeof(int32_t) * (size_t)n * j->cap_mica);
        }
    }
    /* pulling plane (pulling_plane.cu:35-135) */
    if (p->pullingPlane) {
        float v[3] = {p->pullingPlaneDir[0], p->pullingPlaneDir[1], p->pullingPlaneDir[2]};
        const float t = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int c = 0; c < 3; c++) { j->plane_n[c] = v[c] / t; j->plane_p0[c] = p->pullingPlanePos[c]; }
        j->plane_mask = (uint8_t*)calloc(n, 1);
        j->plane_r0 = (float*)calloc(n, sizeof(float));
        j->plane_f = (float*)calloc(n, sizeof(float));
        for (int32_t i = 0; i < n; i++) {
            const float* xi = F4(j->x, i);
            float dr[3] = {xi[0] - j->plane_p0[0], xi[1] - j->plane_p0[1], xi[2] - j->plane_p0[2]};
            j->plane_r0[i] = dr[0] * j->plane_n[0] + dr[1] * j->plane_n[1] + dr[2] * j->plane_n[2];
        }
        for (int32_t k = 0; k < d->nplane_pulled; k++) j->plane_mask[d->plane_pulled[k]] = 2;
        for (int32_t k = 0; k < d->nplane_fixed; k++) j->plane_mask[d->plane_fixed[k]] = 1;
    }
    if (p->hi_on) {
        j->rf = (float*)calloc(4 * (size_t)n, sizeof(float));
        j->mf = (float*)calloc(4 * (size_t)n, sizeof(float));
        j->xc = (float*)calloc(4 * (size_t)n, sizeof(float));
        j->ci4 = (float*)calloc(4 * (size_t)n, sizeof(float));
        j->eps = (float*)calloc(n, sizeof(float));
        if (p->hi_exact) j->tensor = (float*)calloc((size_t)9 * n * n, sizeof(float));
    }
    return j;
}

void orc_job_destroy(orc_job* j) {
    if (!j) return;
    void* ptrs[] = {j->cov_cnt, j->cov_j, j->cov_r0, j->nat_cnt, j->nat_j, j->nat_r02, j->nat_m12,
                    j->nat_r0d, j->nat_ehd, j->pp_cnt, j->pp_j, j->pl_cnt, j->pl_j, j->x, j->f, j->T,
                    j->extF, j->tipF, j->seeds, j->pulled, j->rf, j->mf, j->xc, j->ci4, j->eps, j->tensor,
                    j->log, j->surf0, j->surf, j->mica_cnt, j->mica_j, j->plane_mask, j->plane_r0, j->plane_f};
    for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); k++) free(ptrs[k]);
    free(j);
}

int orc_job_status(const orc_job* j) { return j->status; }
int64_t orc_job_step(const orc_job* j) { return j->step; }

/* ------------------------------------------------------------------------ */
/* Force terms                                                               */
/* ------------------------------------------------------------------------ */
/* covalent_kernel (src/Potentials/covalent_kernel.cu:28-51) */
static inline void covalent_bead(const orc_job* j, int32_t i, float* f) {
    const float* xi = F4(j->x, i);
    for (int32_t k = 0; k < j->cov_cnt[i]; k++) {
        int32_t s = i * j->cap_cov + k;
        const float* xj = F4(j->x, j->cov_j[s]);
        float r0 = j->cov_r0[s];
        float dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
        float w = sqrtf(dx * dx + dy * dy + dz * dz);
        w -= r0;
        w = j->ks * w / ((w + r0) * (1.0f - w * w / j->R2));
        f[0] += w * dx;
        f[1] += w * dy;
        f[2] += w * dz;
    }
}
/* native_kernel (src/Potentials/native_kernel.cu:27-52) */
static inline void native_bead(const orc_job* j, int32_t i, float* f) {
    const float* xi = F4(j->x, i);
    for (int32_t k = 0; k < j->nat_cnt[i]; k++) {
        int32_t s = i * j->cap_nat + k;
        const float* xj = F4(j->x, j->nat_j[s]);
        float dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
        float w = j->nat_r02[s] / (dx * dx + dy * dy + dz * dz);
        float p6 = w * w * w;
        w = w * (p6 * p6 - p6) * j->nat_m12[s];
        f[0] += dx * w;
        f[1] += dy * w;
        f[2] += dz * w;
    }
}
/* pairs_kernel (src/Potentials/pairs_kernel.cu:33-59) */
static inline void pairs_bead(const orc_job* j, int32_t i, float* f) {
    const float* xi = F4(j->x, i);
    for (int32_t k = 0; k < j->pl_cnt[i]; k++) {
        const float* xj = F4(j->x, j->pl_j[(size_t)i * j->cap_pl + k]);
        float dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
        float w = dx * dx + dy * dy + dz * dz;
        if (w < j->cut2) {
            w = j->a2 / w;
            w = w * w;
            w = j->m6 * w * w;
            f[0] += dx * w;
            f[1] += dy * w;
            f[2] += dz * w;
        }
    }
}
/* indentation_kernel (src/Potentials/indentation_kernel.cu:71-128) */
static inline void indentation_bead(orc_job* j, int32_t i, float* f) {
    const float* xi = F4(j->x, i);
    float* fin = F4(j->tipF, i);
    float dx = xi[0] - j->tip[0], dy = xi[1] - j->tip[1], dz = xi[2] - j->tip[2];
    float dw = sqrtf(dx * dx + dy * dy + dz * dz);
    float r2 = dw - j->tipR;
    r2 = 1.0f / r2;
    r2 = r2 * r2;
    float r6 = r2 * r2 * r2;
    float w = j->tipAp * r6 + j->tipBp;
    w = w * r6 / (dw * (dw - j->tipR));
    float df[3] = {dx * w, dy * w, dz * w};
    fin[0] += df[0];
    fin[1] += df[1];
    fin[2] += df[2];
    if (j->p.indentationDiscreteSurf) {
        /* indentationDiscreteSurf_kernel (indentation_kernel.cu:130-180):
         * the beads of the surface in the bead's list, no cutoff */
        f[0] += df[0];
        f[1] += df[1];
        f[2] += df[2];
        for (int32_t k = 0; k < j->mica_cnt[i]; k++) {
            const float* q = j->surf + 3 * j->mica_j[(size_t)i * j->cap_mica + k];
            float e[3] = {xi[0] - q[0], xi[1] - q[1], xi[2] - q[2]};
            float w2 = 1.0f / (e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            float s6 = w2 * w2 * w2;
            float c = (j->surfAp * s6 + j->surfBp) * s6 * w2;
            f[0] += e[0] * c;
            f[1] += e[1] * c;
            f[2] += e[2] * c;
        }
        return;
    }
    float mx = xi[0] - j->micaR[0], my = xi[1] - j->micaR[1], mz = xi[2] - j->micaR[2];
    float d = mx * j->micaN[0] + my * j->micaN[1] + mz * j->micaN[2];
    d = 1.0f / d;
    d = d * d;
    r6 = d * d * d;
    w = j->surfAp * r6 + j->surfBp;
    w = w * r6 * d;
    f[0] += j->micaN[0] * w + df[0];
    f[1] += j->micaN[1] * w + df[1];
    f[2] += j->micaN[2] * w + df[2];
}

/* pullingPlane_kernel (src/Potentials/pulling_plane_kernel.cu:25-52): a
 * spring along the plane normal to the fixed plane or the moving one. */
static inline void plane_bead(orc_job* j, int32_t i, float* f) {
    const int mask = j->plane_mask[i];
    if (!mask) return;
    const float* xi = F4(j->x, i);
    float pc[3] = {j->plane_p0[0], j->plane_p0[1], j->plane_p0[2]};
    if (mask == 2)
        for (int c = 0; c < 3; c++) pc[c] += j->plane_displ * j->plane_n[c];
    float dr = (xi[0] - pc[0]) * j->plane_n[0] + (xi[1] - pc[1]) * j->plane_n[1] + (xi[2] - pc[2]) * j->plane_n[2];
    float df = -j->p.pullingPlaneKs * (dr - j->plane_r0[i]);
    for (int c = 0; c < 3; c++) f[c] += df * j->plane_n[c];
    j->plane_f[i] = df;
}

/* All potentials of one bead in registration order (gsop.cu:80-85). */
static inline void potentials_bead(orc_job* j, int32_t i, float* f) {
    covalent_bead(j, i, f);
    native_bead(j, i, f);
    pairs_bead(j, i, f);
    if (j->p.indentation) indentation_bead(j, i, f);
    if (j->p.pullingPlane) plane_bead(j, i, f);
}

void orc_job_forces(orc_job* j, float* out4, double* out4d, double* abs4d) {
    const int32_t n = j->n;
    float* save = NULL;
    float* save_plane = NULL;
    if (j->p.indentation) { /* do not disturb the tip-force accumulator */
        save = (float*)malloc(16 * (size_t)n);
        memcpy(save, j->tipF, 16 * (size_t)n);
    }
    if (j->p.pullingPlane) {
        save_plane = (float*)malloc(4 * (size_t)n);
        memcpy(save_plane, j->plane_f, 4 * (size_t)n);
    }
    for (int32_t i = 0; i < n; i++) {
        if (out4) {
            float f[4] = {0, 0, 0, 0};
            potentials_bead(j, i, f);
            memcpy(F4(out4, i), f, 16);
        }
        if (out4d || abs4d) {
            /* FP64 mirror of the same terms */
            double fd[3] = {0, 0, 0}, fa[3] = {0, 0, 0};
            const float* xi = F4(j->x, i);
            for (int32_t k = 0; k < j->cov_cnt[i]; k++) {
                int32_t s = i * j->cap_cov + k;
                const float* xj = F4(j->x, j->cov_j[s]);
                double d[3] = {(double)xj[0] - xi[0], (double)xj[1] - xi[1], (double)xj[2] - xi[2]};
                double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                double dl = r - j->cov_r0[s];
                double R2 = (double)j->p.R_limit * j->p.R_limit, q = 1.0 - dl * dl / R2;
                double w = (double)j->ks * dl / (r * q);
                /* rounding scale: r - r0 cancels (|r| + |r0|) and so does q */
                double sc = fabs((double)j->ks * (r + j->cov_r0[s]) / (r * q)) + fabs(w) * (1.0 + dl * dl / R2) / fabs(q);
                for (int c = 0; c < 3; c++) { fd[c] += w * d[c]; fa[c] += sc * fabs(d[c]); }
            }
            for (int32_t k = 0; k < j->nat_cnt[i]; k++) {
                int32_t s = i * j->cap_nat + k;
                const float* xj = F4(j->x, j->nat_j[s]);
                double d[3] = {(double)xj[0] - xi[0], (double)xj[1] - xi[1], (double)xj[2] - xi[2]};
                double r0 = j->nat_r0d[s];
                double q = r0 * r0 / (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                double p6 = q * q * q;
                double m12 = -12.0 * j->nat_ehd[s] / (r0 * r0);
                double w = q * (p6 * p6 - p6) * m12;
                /* p6^2 - p6 cancels at r = r0: scale by |p6^2| + |p6| */
                double sc = q * (p6 * p6 + p6) * fabs(m12);
                for (int c = 0; c < 3; c++) { fd[c] += w * d[c]; fa[c] += sc * fabs(d[c]); }
            }
            for (int32_t k = 0; k < j->pl_cnt[i]; k++) {
                const float* xj = F4(j->x, j->pl_j[(size_t)i * j->cap_pl + k]);
                double d[3] = {(double)xj[0] - xi[0], (double)xj[1] - xi[1], (double)xj[2] - xi[2]};
                double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                if (r2 < (double)j->p.pairs_cutoff * j->p.pairs_cutoff) {
                    double q = (double)j->p.a * j->p.a / r2;
                    double w = -6.0 * j->p.el / ((double)j->p.a * j->p.a) * q * q * q * q;
                    for (int c = 0; c < 3; c++) { fd[c] += w * d[c]; fa[c] += fabs(w * d[c]); }
                }
            }
            if (j->p.indentation) {
                double d[3] = {(double)xi[0] - j->tip[0], (double)xi[1] - j->tip[1], (double)xi[2] - j->tip[2]};
                double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                double rho = r - j->tipR, r6 = 1.0 / (rho * rho * rho * rho * rho * rho);
                double w = ((double)j->tipAp * r6 + j->tipBp) * r6 / (r * rho);
                /* r - R_tip and the surface distance cancel: scale by the
                 * magnitudes that are subtracted */
                double stip = fabs(w) * 7.0 * (r + j->tipR) / fabs(rho);
                if (j->p.indentationDiscreteSurf) {
                    for (int c = 0; c < 3; c++) { fd[c] += w * d[c]; fa[c] += stip * fabs(d[c]); }
                    for (int32_t k = 0; k < j->mica_cnt[i]; k++) {
                        const float* q = j->surf + 3 * j->mica_j[(size_t)i * j->cap_mica + k];
                        double e[3] = {(double)xi[0] - q[0], (double)xi[1] - q[1], (double)xi[2] - q[2]};
                        double w2 = 1.0 / (e[0] * e[0] + e[1] * e[1] + e[2] * e[2]), s6 = w2 * w2 * w2;
                        double cw = ((double)j->surfAp * s6 + j->surfBp) * s6 * w2;
                        /* the difference cancels |x| + |q|; the A/B terms may cancel too */
                        double sc = (fabs((double)j->surfAp * s6) + fabs((double)j->surfBp)) * s6 * w2 * 16.0;
                        for (int c = 0; c < 3; c++) {
                            fd[c] += cw * e[c];
                            fa[c] += sc * (fabs((double)xi[c]) + fabs((double)q[c]));
                        }
                    }
                } else {
                    double m[3] = {(double)xi[0] - j->micaR[0], (double)xi[1] - j->micaR[1], (double)xi[2] - j->micaR[2]};
                    double dd = m[0] * j->micaN[0] + m[1] * j->micaN[1] + m[2] * j->micaN[2];
                    double s6 = 1.0 / (dd * dd * dd * dd * dd * dd);
                    double ws = ((double)j->surfAp * s6 + j->surfBp) * s6 / (dd * dd);
                    double mabs = fabs((double)xi[0] * j->micaN[0]) + fabs((double)xi[1] * j->micaN[1]) + fabs((double)xi[2] * j->micaN[2])
                                + fabs((double)j->micaR[0] * j->micaN[0]) + fabs((double)j->micaR[1] * j->micaN[1]) + fabs((double)j->micaR[2] * j->micaN[2]);
                    double ssurf = fabs(ws) * 8.0 * mabs / fabs(dd);
                    for (int c = 0; c < 3; c++) {
                        double t = w * d[c] + ws * j->micaN[c];
                        fd[c] += t;
                        fa[c] += stip * fabs(d[c]) + ssurf * fabs(j->micaN[c]);
                    }
                }
            }
            if (j->p.pullingPlane && j->plane_mask[i]) {
                double pc[3] = {j->plane_p0[0], j->plane_p0[1], j->plane_p0[2]};
                if (j->plane_mask[i] == 2)
                    for (int c = 0; c < 3; c++) pc[c] += (double)j->plane_displ * j->plane_n[c];
                double dr = ((double)xi[0] - pc[0]) * j->plane_n[0] + ((double)xi[1] - pc[1]) * j->plane_n[1] +
                            ((double)xi[2] - pc[2]) * j->plane_n[2];
                double df = -(double)j->p.pullingPlaneKs * (dr - j->plane_r0[i]);
                /* dr - r0 cancels the plane distances */
                double mag = 0;
                for (int c = 0; c < 3; c++) mag += (fabs((double)xi[c]) + fabs(pc[c])) * fabs(j->plane_n[c]);
                double sc = fabs((double)j->p.pullingPlaneKs) * (mag + fabs((double)j->plane_r0[i])) * 4.0;
                for (int c = 0; c < 3; c++) { fd[c] += df * j->plane_n[c]; fa[c] += sc * fabs(j->plane_n[c]); }
            }
            if (out4d) { for (int c = 0; c < 3; c++) out4d[4 * i + c] = fd[c]; out4d[4 * i + 3] = 0; }
            if (abs4d) { for (int c = 0; c < 3; c++) abs4d[4 * i + c] = fa[c]; abs4d[4 * i + 3] = 0; }
        }
    }
    if (save) {
        memcpy(j->tipF, save, 16 * (size_t)n);
        free(save);
    }
    if (save_plane) {
        memcpy(j->plane_f, save_plane, 4 * (size_t)n);
        free(save_plane);
    }
}

/* ------------------------------------------------------------------------ */
/* Neighbour lists                                                           */
/* ------------------------------------------------------------------------ */
/* generate_possiblepairs (src/Updaters/possiblepairlist_kernel.cu:18-71) */
static void possiblepairs(orc_job* j) {
    const int32_t n = j->n;
    for (int32_t i = 0; i < n; i++) {
        const float* xi = F4(j->x, i);
        int32_t c = 0;
        for (int32_t q = 0; q < n; q++) {
            if (q == i) continue;
            const float* xq = F4(j->x, q);
            float dx = xq[0] - xi[0], dy = xq[1] - xi[1], dz = xq[2] - xi[2];
            float r = sqrtf(dx * dx + dy * dy + dz * dz);
            if (r < j->p.pairs_threshold) {
                int add = 1;
                for (int32_t k = 0; k < j->cov_cnt[i]; k++) if (q == j->cov_j[i * j->cap_cov + k]) add = 0;
                if (add) for (int32_t k = 0; k < j->nat_cnt[i]; k++) if (q == j->nat_j[i * j->cap_nat + k]) add = 0;
                if (add) {
                    if (c < j->cap_pp) j->pp_j[(size_t)i * j->cap_pp + c] = q;
                    else j->status = SOPB_ERR_CAPACITY;
                    c++;
                }
            }
        }
        j->pp_cnt[i] = c < j->cap_pp ? c : j->cap_pp;
    }
}
/* generate_pairs (src/Updaters/pairlist_kernel.cu:33-76) */
static void pairlist(orc_job* j) {
    const int32_t n = j->n;
    for (int32_t i = 0; i < n; i++) {
        const float* xi = F4(j->x, i);
        int32_t c = 0;
        for (int32_t k = 0; k < j->pp_cnt[i]; k++) {
            int32_t q = j->pp_j[(size_t)i * j->cap_pp + k];
            const float* xq = F4(j->x, q);
            float dx = xq[0] - xi[0], dy = xq[1] - xi[1], dz = xq[2] - xi[2];
            float r = sqrtf(dx * dx + dy * dy + dz * dz);
            if (r < j->p.pairlist_cutoff) {
                if (c < j->cap_pl) j->pl_j[(size_t)i * j->cap_pl + c] = q;
                else j->status = SOPB_ERR_CAPACITY;
                c++;
            }
        }
        if (c > j->cap_pl) c = j->cap_pl;
        for (int32_t k = c; k < j->cap_pl; k++) j->pl_j[(size_t)i * j->cap_pl + k] = -1;
        j->pl_cnt[i] = c;
    }
}
void orc_job_rebuild(orc_job* j, int32_t possible, int32_t verlet) {
    if (possible) possiblepairs(j);
    if (verlet) pairlist(j);
}

/* ------------------------------------------------------------------------ */
/* Updaters                                                                  */
/* ------------------------------------------------------------------------ */
static void log_append(orc_job* j, int32_t kind, const float* v) {
    if (j->log_len == j->log_cap) {
        j->log_cap = j->log_cap ? 2 * j->log_cap : 64;
        j->log = (sopb_log_row*)realloc(j->log, (size_t)j->log_cap * sizeof(sopb_log_row));
    }
    sopb_log_row* r = &j->log[j->log_len++];
    memset(r, 0, sizeof(*r));
    r->kind = kind;
    r->step = j->step;
    memcpy(r->v, v, 12 * sizeof(float));
}

/* Drains the rows appended since the last call (oldest first). */
int32_t orc_job_log(orc_job* j, sopb_log_row* rows, int32_t max_rows) {
    int32_t take = j->log_len < max_rows ? j->log_len : max_rows;
    memcpy(rows, j->log, (size_t)take * sizeof(sopb_log_row));
    memmove(j->log, j->log + take, (size_t)(j->log_len - take) * sizeof(sopb_log_row));
    j->log_len -= take;
    return take;
}

/* PullingUpdater::update -> PullingPotential::updateForces
 * (src/Potentials/pulling.cu:152-165, 198-214) */
static void pulling_update(orc_job* j) {
    const sopb_params* p = &j->p;
    int32_t freq = p->pullFreq > 0 ? p->pullFreq : p->nav;
    float xt = p->deltax * (float)(j->step / freq);
    const float* xe = F4(j->x, p->pulledEnd);
    for (int c = 0; c < 3; c++) j->extForce[c] = p->k_trans * (j->cant[c] - xe[c]);
    for (int c = 0; c < 3; c++) j->cant[c] = j->cant0[c] + xt * j->pullvec[c];
    if (j->step % freq == 0) {
        /* savePullingData (src/Potentials/pulling.cu:167-190) */
        const float* xf = F4(j->x, p->fixedEnd);
        float e[3] = {xe[0] - xf[0], xe[1] - xf[1], xe[2] - xf[2]};
        float v[12] = {0};
        v[0] = sqrtf(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        v[1] = e[0] * j->pullvec[0] + e[1] * j->pullvec[1] + e[2] * j->pullvec[2];
        v[2] = j->extForce[0] * j->pullvec[0] + j->extForce[1] * j->pullvec[1] + j->extForce[2] * j->pullvec[2];
        v[3] = j->extForce[0];
        v[4] = j->extForce[1];
        v[5] = j->extForce[2];
        log_append(j, SOPB_LOG_PULL, v);
    }
    for (int32_t k = 0; k < j->npulled; k++) {
        float* e = F4(j->extF, j->pulled[k]);
        e[0] = j->extForce[0];
        e[1] = j->extForce[1];
        e[2] = j->extForce[2];
        e[3] = 2.0f;
    }
}

/* generateMicaList_kernel (src/Potentials/indentation_kernel.cu:182-201):
 * the surface beads within indentationPairsCutoff of each bead, in surface
 * order. */
static void mica_list(orc_job* j) {
    const float cut2 = j->p.indentationPairsCutoff * j->p.indentationPairsCutoff;
    for (int32_t i = 0; i < j->n; i++) {
        const float* xi = F4(j->x, i);
        int32_t cnt = 0;
        for (int32_t q = 0; q < j->nsurf; q++) {
            const float* s = j->surf + 3 * q;
            float e[3] = {xi[0] - s[0], xi[1] - s[1], xi[2] - s[2]};
            if (e[0] * e[0] + e[1] * e[1] + e[2] * e[2] < cut2) j->mica_j[(size_t)i * j->cap_mica + cnt++] = q;
        }
        j->mica_cnt[i] = cnt;
    }
}

/* IndentationTipUpdater::update (src/Potentials/indentation.cu:414-550),
 * continuous surface. */
static void indentation_update(orc_job* j) {
    const sopb_params* p = &j->p;
    if (j->step == p->indentationRetractionStep) j->V = -j->V;
    if (j->step % p->nav != 0) return;
    float f[4] = {0, 0, 0, 0};
    for (int32_t i = 0; i < j->n; i++) {
        float* t = F4(j->tipF, i);
        f[0] += t[0];
        f[1] += t[1];
        f[2] += t[2];
        t[0] = t[1] = t[2] = 0.0f;
    }
    for (int c = 0; c < 3; c++) f[c] /= (float)p->nav;
    f[3] = sqrtf(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    j->dx = (float)(j->step / p->nav) * j->V;
    if (p->indentationMoveSurface) {
        if (p->indentationDiscreteSurf) {
            for (int32_t q = 0; q < j->nsurf; q++)
                for (int c = 0; c < 3; c++) j->surf[3 * q + c] = j->surf0[3 * q + c] + j->dir[c] * j->dx;
        } else {
            for (int c = 0; c < 3; c++) j->micaR[c] = j->micaR0[c] + j->dir[c] * j->dx;
        }
    } else {
        for (int c = 0; c < 3; c++) j->chip[c] = j->chip0[c] + j->dir[c] * j->dx;
    }
    if (p->indentationDiscreteSurf) mica_list(j);
    float dr[3] = {j->chip[0] - j->tip[0], j->chip[1] - j->tip[1], j->chip[2] - j->tip[2]};
    float df[3];
    for (int c = 0; c < 3; c++) df[c] = -f[c] + dr[c] * j->cantKs;
    float mult = (p->timestep * (float)p->nav) / j->tipZeta;
    if (p->indentationFixTrans) {
        float ct = mult * df[0] * j->dir[0] + mult * df[1] * j->dir[1] + mult * df[2] * j->dir[2];
        for (int c = 0; c < 3; c++) j->tip[c] += ct * j->dir[c];
    } else {
        for (int c = 0; c < 3; c++) j->tip[c] += mult * df[c];
    }
    memcpy(j->fav, f, 16);
    const float v[12] = {f[0], f[1], f[2], f[3], sqrtf(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]), j->dx,
                         j->tip[0], j->tip[1], j->tip[2], j->chip[0], j->chip[1], j->chip[2]};
    log_append(j, SOPB_LOG_TIP, v);
}

/* PullingPlaneUpdater::update (src/Potentials/pulling_plane.cu:183-258),
 * every stride: the cantilever moves by deltax per update period, the plane
 * follows it by one overdamped step of update-period length against the
 * beads' pull, summed in bead order from the last forces. */
static void plane_update(orc_job* j) {
    const sopb_params* p = &j->p;
    const int32_t freq = p->pullingPlaneUpdateFreq > 0 ? p->pullingPlaneUpdateFreq : p->nav;
    const int32_t ofreq = p->pullingPlaneOutputFreq > 0 ? p->pullingPlaneOutputFreq : p->nav;
    const float xt = p->pullingPlaneDeltax * (float)j->step / (float)freq;
    j->plane_cant = xt;
    float ext = 0.0f;
    for (int32_t i = 0; i < j->n; i++)
        if (j->plane_mask[i] == 2) ext += j->plane_f[i];
    const float cant = (xt - j->plane_displ) * p->pullingPlaneKsCant;
    j->plane_displ += ((float)freq * p->timestep / p->pullingPlaneZeta) * (cant - ext);
    if (j->step % ofreq == 0) {
        float cf[3] = {0, 0, 0}, cp[3] = {0, 0, 0};
        int32_t nf = 0, np = 0;
        for (int32_t i = 0; i < j->n; i++) {
            const float* xi = F4(j->x, i);
            if (j->plane_mask[i] == 1) { for (int c = 0; c < 3; c++) cf[c] += xi[c]; nf++; }
            if (j->plane_mask[i] == 2) { for (int c = 0; c < 3; c++) cp[c] += xi[c]; np++; }
        }
        for (int c = 0; c < 3; c++) { cf[c] /= (float)nf; cp[c] /= (float)np; }
        float dx = cp[0] - cf[0], dy = cp[1] - cf[1], dz = cp[2] - cf[2];
        float v[12] = {0};
        v[0] = j->plane_displ;
        v[1] = j->plane_cant;
        v[2] = cant;
        v[3] = ext;
        v[4] = sqrtf(dx * dx + dy * dy + dz * dz);
        log_append(j, SOPB_LOG_PLANE, v);
    }
}

/* RPY block normalised by D_ii (src/Integrators/bdhitea_kernel.cu:67-87);
 * e is the unit vector, r the distance. */
static inline void rpy(float ex, float ey, float ez, float r, float a, float* D6) {
    float ra = r / a, crr, cii;
    if (ra > 2.f) {
        crr = 0.75f / ra * (1.f - 2.f / ra / ra);
        cii = 0.75f / ra * (1.f + 2.f / 3.f / ra / ra);
    } else {
        crr = 3.f * ra / 32.f;
        cii = 1.f - 9.f * ra / 32.f;
    }
    D6[0] = ex * ex * crr + cii; /* xx */
    D6[1] = ex * ey * crr;       /* xy */
    D6[2] = ex * ez * crr;       /* xz */
    D6[3] = ey * ey * crr + cii; /* yy */
    D6[4] = ey * ez * crr;       /* yz */
    D6[5] = ez * ez * crr + cii; /* zz */
}

/* integrateTea_epsilon[_unlisted] + TeaUpdater::update
 * (src/Integrators/bdhitea_kernel.cu:192-249, src/Integrators/bdhitea.cu:133-176) */
static void tea_epsilon_one(orc_job* j, int32_t i, int32_t q, float* sum) {
    const float* xi = F4(j->x, i);
    const float* xq = F4(j->x, q);
    float d[4] = {xq[0] - xi[0], xq[1] - xi[1], xq[2] - xi[2], 0};
    d[3] = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    d[0] /= d[3];
    d[1] /= d[3];
    d[2] /= d[3];
    float D[6];
    rpy(d[0], d[1], d[2], d[3], j->p.hi_a, D);
    sum[3] += D[0] + 2 * D[1] + 2 * D[2] + D[3] + 2 * D[4] + D[5];
    sum[0] += D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
    sum[1] += D[1] * D[1] + D[3] * D[3] + D[4] * D[4];
    sum[2] += D[2] * D[2] + D[4] * D[4] + D[5] * D[5];
}
static void tea_update(orc_job* j) {
    if (j->step % j->p.hi_epsilon_freq != 0) return;
    const int32_t n = j->n;
    for (int32_t i = 0; i < n; i++) {
        float s[4] = {0, 0, 0, 0};
        if (j->p.hi_unlisted) {
            for (int32_t q = 0; q < n; q++) if (q != i) tea_epsilon_one(j, i, q, s);
        } else {
            for (int32_t k = 0; k < j->cov_cnt[i]; k++) tea_epsilon_one(j, i, j->cov_j[i * j->cap_cov + k], s);
            for (int32_t k = 0; k < j->nat_cnt[i]; k++) tea_epsilon_one(j, i, j->nat_j[i * j->cap_nat + k], s);
            for (int32_t k = 0; k < j->pl_cnt[i]; k++) tea_epsilon_one(j, i, j->pl_j[(size_t)i * j->cap_pl + k], s);
        }
        memcpy(F4(j->ci4, i), s, 16);
        j->eps[i] = s[3];
    }
    double eps = 0.0;
    for (int32_t i = 0; i < n; i++) eps += j->eps[i];
    if (n > 1) eps /= 3. * n * (3. * n - 3.);
    if (eps > 1.0) {
        if (j->p.hi_capricious) j->status = SOPB_ERR_HI;
        eps = 1.0;
    }
    if (eps > j->p.hi_epsmax) j->status = SOPB_ERR_HI;
    double a = (3. * n - 1.) * eps * eps - (3. * n - 2.) * eps;
    j->epsilon = (float)eps;
    if (fabs(a) < 1e-7) {
        j->beta = .5f;
        if (j->p.hi_capricious && j->p.hi_a > 0.0f) j->status = SOPB_ERR_HI;
    } else {
        j->beta = (float)((1. - sqrt(1. - a)) / a);
    }
}

/* One pass of the updaters in the reference order (see gsop.cu:80-101 for
 * the creation order that fixes it). */
static void run_updaters(orc_job* j) {
    const sopb_params* p = &j->p;
    if (p->indentation) indentation_update(j);
    if (p->pulling && p->deltax != 0.0f) pulling_update(j);
    if (p->pullingPlane) plane_update(j);
    if (j->step % p->possiblepairs_freq == 0) possiblepairs(j);
    if (j->step % p->nav == 0) memset(j->T, 0, j->n * sizeof(float)); /* output_manager.cu:125-127 */
    if (j->step % p->pairs_freq == 0) pairlist(j);
    if (p->heating && j->step % p->tempFreq == 0) /* langevin.cu:129-135 */
        set_temperature(j, p->initialT + (float)(j->step / p->tempFreq) * p->deltaT);
    if (p->hi_on && !p->hi_exact) tea_update(j);
    if (p->hi_on && p->hi_exact && p->hi_refresh > 1 && j->step % p->hi_refresh == 0) j->refresh_due = 1;
}

/* ------------------------------------------------------------------------ */
/* Integrators                                                               */
/* ------------------------------------------------------------------------ */
/* integrateLangevin_kernel (src/Integrators/langevin_kernel.cu:17-58) */
static inline void langevin_bead(orc_job* j, int32_t i) {
    float* f = F4(j->f, i);
    float fx = f[0], fy = f[1], fz = f[2];
    f[0] = f[1] = f[2] = f[3] = 0.0f;
    if (!j->p.minimization) {
        float g[4];
        rforce(&j->seeds[4 * i], g);
        fx += g[0] * j->var;
        fy += g[1] * j->var;
        fz += g[2] * j->var;
    }
    if (j->p.pulling) {
        const float* e = F4(j->extF, i);
        if (e[3] == 1.0f) fx = fy = fz = 0.0f;
        if (e[3] == 2.0f) { fx += e[0]; fy += e[1]; fz += e[2]; }
    }
    float m = j->hOverZeta;
    float d0 = m * fx, d1 = m * fy, d2 = m * fz;
    float* x = F4(j->x, i);
    x[0] += d0;
    x[1] += d1;
    x[2] += d2;
    j->T[i] += j->tempNorm * (d0 * d0 + d1 * d1 + d2 * d2);
}

/* integrateTea_prepare (src/Integrators/bdhitea_kernel.cu:33-65) */
static void tea_prepare(orc_job* j) {
    for (int32_t i = 0; i < j->n; i++) {
        float g[4];
        rforce(&j->seeds[4 * i], g);
        g[0] *= j->var;
        g[1] *= j->var;
        g[2] *= j->var;
        memcpy(F4(j->rf, i), g, 16);
        float* f = F4(j->f, i);
        float m[4] = {f[0], f[1], f[2], f[3]};
        if (j->p.pulling) {
            const float* e = F4(j->extF, i);
            if (e[3] == 1.0f) m[0] = m[1] = m[2] = 0.0f;
            if (e[3] == 2.0f) { m[0] += e[0]; m[1] += e[1]; m[2] += e[2]; }
        }
        memcpy(F4(j->mf, i), m, 16);
        f[0] = f[1] = f[2] = f[3] = 0.0f;
        memcpy(F4(j->xc, i), F4(j->x, i), 16);
    }
}

static inline void integrate_final(orc_job* j, int32_t i, float fx, float fy, float fz) {
    if (j->p.pulling && F4(j->extF, i)[3] == 1.0f) fx = fy = fz = 0.0f;
    float m = j->hOverZeta;
    float d0 = m * fx, d1 = m * fy, d2 = m * fz;
    const float* xc = F4(j->xc, i);
    float* x = F4(j->x, i);
    x[0] = xc[0] + d0;
    x[1] = xc[1] + d1;
    x[2] = xc[2] + d2;
    x[3] = xc[3];
    j->T[i] = j->T[i] + j->tempNorm * (d0 * d0 + d1 * d1 + d2 * d2);
}

/* integrateTea_force (src/Integrators/bdhitea_kernel.cu:252-301), reading the
 * coordinate copy as the NOTEXTURE build does. */
static inline void tea_force(orc_job* j, const float* xi, int32_t q, const float* ci, float* out) {
    const float* xq = F4(j->xc, q);
    float d[4] = {xq[0] - xi[0], xq[1] - xi[1], xq[2] - xi[2], 0};
    d[3] = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    d[0] /= d[3];
    d[1] /= d[3];
    d[2] /= d[3];
    const float* mq = F4(j->mf, q);
    const float* rq = F4(j->rf, q);
    float f0 = mq[0] + rq[0] * ci[0], f1 = mq[1] + rq[1] * ci[1], f2 = mq[2] + rq[2] * ci[2];
    float D[6];
    rpy(d[0], d[1], d[2], d[3], j->p.hi_a, D);
    out[0] += D[0] * f0 + D[1] * f1 + D[2] * f2;
    out[1] += D[1] * f0 + D[3] * f1 + D[4] * f2;
    out[2] += D[2] * f0 + D[4] * f1 + D[5] * f2;
}
/* integrateTea_kernel[_unlisted] (src/Integrators/bdhitea_kernel.cu:364-515) */
static void tea_integrate(orc_job* j) {
    const int32_t n = j->n;
    float* newx = (float*)malloc(16 * (size_t)n);
    float* newT = (float*)malloc(4 * (size_t)n);
    for (int32_t i = 0; i < n; i++) {
        const float* c4 = F4(j->ci4, i);
        float b2 = j->beta * j->beta;
        float ci[3] = {1.f / sqrtf(1.f + b2 * c4[0]), 1.f / sqrtf(1.f + b2 * c4[1]), 1.f / sqrtf(1.f + b2 * c4[2])};
        const float* m = F4(j->mf, i);
        const float* r = F4(j->rf, i);
        float f[3] = {m[0] + r[0] * ci[0], m[1] + r[1] * ci[1], m[2] + r[2] * ci[2]};
        for (int c = 0; c < 3; c++) ci[c] *= j->beta;
        const float* xi = F4(j->xc, i);
        float df[3];
        if (j->p.hi_unlisted) {
            for (int32_t q = 0; q < n; q++) {
                if (q == i) continue;
                df[0] = df[1] = df[2] = 0.0f;
                tea_force(j, xi, q, ci, df);
                f[0] += df[0]; f[1] += df[1]; f[2] += df[2];
            }
        } else {
            for (int32_t k = 0; k < j->cov_cnt[i]; k++) {
                df[0] = df[1] = df[2] = 0.0f;
                tea_force(j, xi, j->cov_j[i * j->cap_cov + k], ci, df);
                f[0] += df[0]; f[1] += df[1]; f[2] += df[2];
            }
            for (int32_t k = 0; k < j->nat_cnt[i]; k++) {
                df[0] = df[1] = df[2] = 0.0f;
                tea_force(j, xi, j->nat_j[i * j->cap_nat + k], ci, df);
                f[0] += df[0]; f[1] += df[1]; f[2] += df[2];
            }
            for (int32_t k = 0; k < j->pl_cnt[i]; k++) {
                df[0] = df[1] = df[2] = 0.0f;
                tea_force(j, xi, j->pl_j[(size_t)i * j->cap_pl + k], ci, df);
                f[0] += df[0]; f[1] += df[1]; f[2] += df[2];
            }
        }
        /* integrate into temporaries: all beads read the copies */
        float fx = f[0], fy = f[1], fz = f[2];
        if (j->p.pulling && F4(j->extF, i)[3] == 1.0f) fx = fy = fz = 0.0f;
        float mlt = j->hOverZeta;
        float d0 = mlt * fx, d1 = mlt * fy, d2 = mlt * fz;
        newx[4 * i] = xi[0] + d0;
        newx[4 * i + 1] = xi[1] + d1;
        newx[4 * i + 2] = xi[2] + d2;
        newx[4 * i + 3] = xi[3];
        newT[i] = j->T[i] + j->tempNorm * (d0 * d0 + d1 * d1 + d2 * d2);
    }
    memcpy(j->x, newx, 16 * (size_t)n);
    memcpy(j->T, newT, 4 * (size_t)n);
    free(newx);
    free(newT);
}

/* integrateCholesky_D (src/Integrators/bdhitea_kernel.cu:89-152).  The
 * reference thread writes mforce[i] while others read mforce[j]; here every
 * bead reads the prepared forces (the race-free intent). */
static void chol_D(orc_job* j, int assemble) {
    const int32_t n = j->n, m = 3 * n;
    float* M = j->tensor;
    float* nm = (float*)malloc(16 * (size_t)n);
    /* bead i writes block column i of M and its own sum: no sharing */
#pragma omp parallel for schedule(static) if (n > 512)
    for (int32_t i = 0; i < n; i++) {
        const float* xi = F4(j->x, i);
        float f[4];
        memcpy(f, F4(j->mf, i), 16);
        for (int32_t q = 0; q < n; q++) {
            float* row0 = &M[(size_t)(3 * q) * m + 3 * i];
            float* row1 = row0 + m;
            float* row2 = row1 + m;
            if (q == i) {
                if (assemble) {
                    row0[0] = 1; row0[1] = 0; row0[2] = 0;
                    row1[0] = 0; row1[1] = 1; row1[2] = 0;
                    row2[0] = 0; row2[1] = 0; row2[2] = 1;
                }
                continue;
            }
            const float* xq = F4(j->x, q);
            float d[4] = {xq[0] - xi[0], xq[1] - xi[1], xq[2] - xi[2], 0};
            d[3] = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            d[0] /= d[3];
            d[1] /= d[3];
            d[2] /= d[3];
            float D[6];
            rpy(d[0], d[1], d[2], d[3], j->p.hi_a, D);
            if (assemble) {
                row0[0] = D[0]; row0[1] = D[1]; row0[2] = D[2];
                row1[0] = D[1]; row1[1] = D[3]; row1[2] = D[4];
                row2[0] = D[2]; row2[1] = D[4]; row2[2] = D[5];
            }
            const float* fq = F4(j->mf, q);
            f[0] += D[0] * fq[0] + D[1] * fq[1] + D[2] * fq[2];
            f[1] += D[1] * fq[0] + D[3] * fq[1] + D[4] * fq[2];
            f[2] += D[2] * fq[0] + D[4] * fq[1] + D[5] * fq[2];
        }
        memcpy(F4(nm, i), f, 16);
    }
    memcpy(j->mf, nm, 16 * (size_t)n);
    free(nm);
}

/* integrateCholesky_decompose (src/Integrators/bdhitea_kernel.cu:154-190):
 * column by column; afterwards M holds L below and L^T above the diagonal.
 * Column c starts from row c of M (D[c][t] for t >= c, and L[c][k] for
 * k < c written by the earlier columns), subtracts L[t][k] * L[c][k] for
 * k = 0, 1, ..., c-1 in that order, and divides by sqrtf of the diagonal.
 *
 * The columns are taken in panels of ORC_CHOL_PANEL: the subtractions of
 * the columns finished before a panel are applied to all of its columns
 * while each row k of M is in cache (OpenMP over t), then the panel's own
 * columns are finished one after the other.  Every entry still sees its
 * subtractions in increasing k, one rounding each (no contraction), so the
 * result is bit-identical to the column-at-a-time loop. */
#define ORC_CHOL_PANEL 64
void orc_cholesky_ref(int32_t m, float* M) {
    const int32_t P = ORC_CHOL_PANEL;
    float* V = (float*)malloc(sizeof(float) * (size_t)P * m);   /* V[(c - c0) * m + t] */
    for (int32_t c0 = 0; c0 < m; c0 += P) {
        const int32_t c1 = c0 + P < m ? c0 + P : m, w = c1 - c0;
        /* the panel's rows of D and the columns finished before it */
#pragma omp parallel for schedule(static)
        for (int32_t tb = c0; tb < m; tb += 256) {
            const int32_t te = tb + 256 < m ? tb + 256 : m;
            for (int32_t c = c0; c < c1; c++)
                for (int32_t t = tb; t < te; t++) V[(size_t)(c - c0) * m + t] = M[(size_t)c * m + t];
            for (int32_t k = 0; k < c0; k++) {
                const float* Mk = &M[(size_t)k * m];
                for (int32_t c = c0; c < c1; c++) {
                    const float lck = M[(size_t)c * m + k];
                    float* v = &V[(size_t)(c - c0) * m];
                    const int32_t t0 = tb > c ? tb : c;
#pragma omp simd
                    for (int32_t t = t0; t < te; t++) v[t] -= Mk[t] * lck;
                }
            }
        }
        /* the panel's own columns, in order */
        for (int32_t c = c0; c < c1; c++) {
            float* v = &V[(size_t)(c - c0) * m];
#pragma omp parallel for schedule(static) if (m - c > 2048)
            for (int32_t tb = c; tb < m; tb += 512) {
                const int32_t te = tb + 512 < m ? tb + 512 : m;
                for (int32_t k = c0; k < c; k++) {
                    const float* Mk = &M[(size_t)k * m];
                    const float lck = M[(size_t)c * m + k];
#pragma omp simd
                    for (int32_t t = tb; t < te; t++) v[t] -= Mk[t] * lck;
                }
            }
            const float diag = sqrtf(v[c]);
            for (int32_t t = c; t < m; t++) {
                const float q = v[t] / diag;
                M[(size_t)t * m + c] = q;
                M[(size_t)c * m + t] = q;
            }
        }
        (void)w;
    }
    free(V);
}

/* integrateCholesky_L (src/Integrators/bdhitea_kernel.cu:303-361): block
 * (i,q), q <= i, uses M[3q+r][3i+c] for r <= c as a symmetric 3x3. */
static inline void ref_b_block(int32_t m, const float* M, int32_t i, int32_t q, float* B6) {
    const float* L0 = &M[(size_t)(3 * q) * m + 3 * i];
    B6[0] = L0[0]; B6[1] = L0[1]; B6[2] = L0[2];
    B6[3] = L0[m + 1]; B6[4] = L0[m + 2];
    B6[5] = L0[2 * m + 2];
}
void orc_ref_b_matrix(int32_t n, const float* M, double* B) {
    const int32_t m = 3 * n;
    memset(B, 0, sizeof(double) * (size_t)m * m);
    for (int32_t i = 0; i < n; i++)
        for (int32_t q = 0; q <= i; q++) {
            float b[6];
            ref_b_block(m, M, i, q, b);
            double s[3][3] = {{b[0], b[1], b[2]}, {b[1], b[3], b[4]}, {b[2], b[4], b[5]}};
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) B[(size_t)(3 * i + r) * m + 3 * q + c] = s[r][c];
        }
}
static void chol_L(orc_job* j) {
    const int32_t n = j->n, m = 3 * n;
    const float* M = j->tensor;
    for (int32_t i = 0; i < n; i++) {
        float f[3];
        memcpy(f, F4(j->mf, i), 12);
        for (int32_t q = 0; q <= i; q++) {
            float b[6];
            if (j->p.hi_b_mode == SOPB_HI_B_REFCOMPAT) {
                ref_b_block(m, M, i, q, b);
                const float* g = F4(j->rf, q);
                f[0] += b[0] * g[0] + b[1] * g[1] + b[2] * g[2];
                f[1] += b[1] * g[0] + b[3] * g[1] + b[4] * g[2];
                f[2] += b[2] * g[0] + b[4] * g[1] + b[5] * g[2];
            } else {
                /* B = L: rows 3i..3i+2, columns 3q..3q+2 of the lower triangle */
                const float* g = F4(j->rf, q);
                for (int r = 0; r < 3; r++) {
                    float acc = 0.0f;
                    for (int c = 0; c < 3; c++) {
                        int32_t row = 3 * i + r, col = 3 * q + c;
                        if (col <= row) acc += M[(size_t)row * m + col] * g[c];
                    }
                    f[r] += acc;
                }
            }
        }
        integrate_final(j, i, f[0], f[1], f[2]);
    }
}

void orc_rpy_tensor(int32_t n, const float* xyz, float a, double* D) {
    const int32_t m = 3 * n;
    for (int32_t i = 0; i < n; i++)
        for (int32_t q = 0; q < n; q++) {
            double* b = &D[(size_t)(3 * i) * m + 3 * q];
            if (i == q) {
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) b[(size_t)r * m + c] = (r == c);
                continue;
            }
            double d[3] = {(double)xyz[3 * q] - xyz[3 * i], (double)xyz[3 * q + 1] - xyz[3 * i + 1],
                           (double)xyz[3 * q + 2] - xyz[3 * i + 2]};
            double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            double ra = r / a, crr, cii;
            if (ra > 2.0) {
                crr = 0.75 / ra * (1.0 - 2.0 / (ra * ra));
                cii = 0.75 / ra * (1.0 + 2.0 / 3.0 / (ra * ra));
            } else {
                crr = 3.0 * ra / 32.0;
                cii = 1.0 - 9.0 * ra / 32.0;
            }
            for (int rr = 0; rr < 3; rr++)
                for (int c = 0; c < 3; c++)
                    b[(size_t)rr * m + c] = d[rr] / r * d[c] / r * crr + (rr == c ? cii : 0.0);
        }
}

/* ------------------------------------------------------------------------ */
/* The loop                                                                  */
/* ------------------------------------------------------------------------ */
static int is_finite_coords(const orc_job* j) {
    for (int32_t i = 0; i < 4 * j->n; i++) if (!isfinite(j->x[i])) return 0;
    return 1;
}

/* One Langevin step: potentials in registration order, then the
 * integrator (gsop.cu:135-142). */
static void one_step(orc_job* j) {
    const int32_t n = j->n;
    for (int32_t i = 0; i < n; i++) potentials_bead(j, i, F4(j->f, i));
    if (!j->p.hi_on) {
        for (int32_t i = 0; i < n; i++) langevin_bead(j, i);
    } else {
        tea_prepare(j);
        if (!j->p.hi_exact) {
            tea_integrate(j);
        } else {
            /* the factor of D is refreshed every step (hi_refresh 1, the
             * reference) or at the updater boundaries due for it */
            const int refresh = j->p.hi_refresh <= 1 || j->refresh_due;
            chol_D(j, refresh);
            if (refresh) orc_cholesky_ref(3 * n, j->tensor);
            j->refresh_due = 0;
            chol_L(j);
        }
    }
}

int orc_job_advance(orc_job* j, int64_t nsteps) {
    for (int64_t s = 0; s < nsteps; s++) {
        if (j->status) return j->status;
        if (j->step % j->stride == 0) run_updaters(j);
        if (j->status) return j->status;
        one_step(j);
        j->step++;
    }
    if (!is_finite_coords(j)) j->status = SOPB_ERR_NONFINITE;
    return j->status;
}

int orc_jobs_advance(orc_job** jobs, int32_t njobs, int64_t nsteps, int32_t nthreads) {
    int rc = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) reduction(| : rc)
#endif
    for (int32_t k = 0; k < njobs; k++) rc |= orc_job_advance(jobs[k], nsteps);
    (void)nthreads;
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Accessors                                                                 */
/* ------------------------------------------------------------------------ */
void orc_job_read(const orc_job* j, int32_t what, void* out) {
    const size_t n = j->n;
    switch (what) {
    case SOPB_COORDS: memcpy(out, j->x, 16 * n); break;
    case SOPB_SEEDS: memcpy(out, j->seeds, 16 * n); break;
    case SOPB_TEMP: memcpy(out, j->T, 4 * n); break;
    case SOPB_FORCES: orc_job_forces((orc_job*)j, (float*)out, NULL, NULL); break;
    case SOPB_TIPFORCES: memcpy(out, j->tipF, 16 * n); break;
    case SOPB_PULLSTATE: {
        float* o = (float*)out;
        memcpy(o, j->extForce, 12);
        memcpy(o + 3, j->cant, 12);
        memcpy(o + 6, j->cant0, 12);
        memcpy(o + 9, j->pullvec, 12);
        break;
    }
    case SOPB_HISTATE: {
        float* o = (float*)out;
        o[0] = j->beta;
        o[1] = j->epsilon;
        o[2] = o[3] = 0.0f;
        break;
    }
    case SOPB_TIPSTATE: {
        float* o = (float*)out;
        memset(o, 0, 64);
        memcpy(o, j->tip, 12);
        memcpy(o + 3, j->chip, 12);
        memcpy(o + 6, j->micaR, 12);
        o[9] = j->V;
        o[10] = j->dx;
        memcpy(o + 11, j->fav, 16);
        break;
    }
    default: break;
    }
}

void orc_job_write(orc_job* j, int32_t what, const void* in) {
    const size_t n = j->n;
    switch (what) {
    case SOPB_COORDS: memcpy(j->x, in, 16 * n); break;
    case SOPB_SEEDS: memcpy(j->seeds, in, 16 * n); break;
    case SOPB_TEMP: memcpy(j->T, in, 4 * n); break;
    default: break;
    }
}

void orc_job_pairlist(const orc_job* j, int32_t possible, int32_t* counts, int32_t* rows, int32_t cap) {
    const int32_t* cnt = possible ? j->pp_cnt : j->pl_cnt;
    const int32_t* lst = possible ? j->pp_j : j->pl_j;
    const int32_t lcap = possible ? j->cap_pp : j->cap_pl;
    for (int32_t i = 0; i < j->n; i++) {
        counts[i] = cnt[i];
        for (int32_t k = 0; k < cap; k++)
            rows[(size_t)i * cap + k] = (k < cnt[i] && k < lcap) ? lst[(size_t)i * lcap + k] : -1;
    }
}

/* ------------------------------------------------------------------------ */
/* Observables (src/Updaters/output_manager.cu:73-222)                       */
/* ------------------------------------------------------------------------ */
void orc_job_observables(const orc_job* j, double* out) {
    const int32_t n = j->n;
    const float R_limit = sqrtf(j->R2);
    const float rlb = j->p.R_limit_bond > 0.0f ? j->p.R_limit_bond : 8.0f;
    double efene = 0.0, enat = 0.0, epair = 0.0, tsum = 0.0, rg = 0.0;
    int contacts = 0;
    for (int32_t i = 0; i < n; i++) {
        const float* xi = F4(j->x, i);
        /* covalentEnergy_kernel (covalent_kernel.cu:57-78) */
        float pot = 0.0f;
        for (int32_t k = 0; k < j->cov_cnt[i]; k++) {
            const size_t s = (size_t)i * j->cap_cov + k;
            const float* xj = F4(j->x, j->cov_j[s]);
            float dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
            float d = sqrtf(dx * dx + dy * dy + dz * dz) - j->cov_r0[s];
            pot -= 0.5f * j->ks * j->R2 * logf(1.0f - d * d / j->R2);
        }
        efene += pot;
        /* nativeEnergy_kernel (native_kernel.cu:57-82) */
        pot = 0.0f;
        for (int32_t k = 0; k < j->nat_cnt[i]; k++) {
            const size_t s = (size_t)i * j->cap_nat + k;
            const int32_t q = j->nat_j[s];
            const float* xj = F4(j->x, q);
            float dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
            float r2 = dx * dx + dy * dy + dz * dz;
            float w = j->nat_r02[s] / r2, p6 = w * w * w;
            pot += (-j->nat_m12[s] * j->nat_r02[s] / 12.0f) * (p6 * p6 - 2.0f * p6);
            /* computeNativeCounts (output_manager.cu:166-186): each contact once */
            if (q > i) {
                float dr = sqrtf(r2);
                if (dr < rlb || fabsf(sqrtf(j->nat_r02[s]) - dr) <= R_limit) contacts++;
            }
        }
        enat += pot;
        /* pairsEnergy_kernel (pairs_kernel.cu:69-91) */
        pot = 0.0f;
        for (int32_t k = 0; k < j->pl_cnt[i]; k++) {
            const float* xj = F4(j->x, j->pl_j[(size_t)i * j->cap_pl + k]);
            float dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
            float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < j->cut2) {
                float w = j->a2 / r2;
                pot += j->p.el * w * w * w;
            }
        }
        epair += pot;
        tsum += j->T[i];
        /* computeRg_kernel (output_manager_kernel.cu:14-31) */
        float g = 0.0f;
        for (int32_t q = 0; q < i; q++) {
            const float* xq = F4(j->x, q);
            float dx = xq[0] - xi[0], dy = xq[1] - xi[1], dz = xq[2] - xi[2];
            g += dx * dx + dy * dy + dz * dz;
        }
        rg += g;
    }
    out[0] = tsum / ((double)n * (double)j->p.nav);
    out[1] = efene * 0.5;
    out[2] = enat * 0.5;
    out[3] = epair * 0.5;
    out[4] = out[1] + out[2] + out[3];
    out[5] = contacts;
    out[6] = sqrt(rg / ((double)n * (double)n));
    out[7] = (j->p.hi_on && !j->p.hi_exact) ? (double)j->epsilon : 0.0;
}
