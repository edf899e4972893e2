// sopb_device.cuh — device-side job descriptor and per-bead math of the SOP
// Langevin step for sm_100a.
//
// One JobDev describes one independent SOP system (a "trajectory" of the
// reference).  Per-bead state lives in context-wide bead pools (coordinates,
// RNG states, temperature accumulator, flags) so a batch's coordinates move
// with one copy; the neighbour maps of a job are CSR (covalent, native) or
// either bitmasks over the job's beads or fixed-capacity index rows
// (possible pairs, Verlet pairs).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/sopb.h"

namespace sopb {

enum : int { FLAG_FREE = 0, FLAG_FIXED = 1, FLAG_PULLED = 2 };
constexpr int SOPB_STATUS_CAPACITY = SOPB_ERR_CAPACITY;
constexpr int SOPB_STATUS_NONFINITE = SOPB_ERR_NONFINITE;

struct JobDev {
    // ---- sizes and schedule ------------------------------------------------
    int32_t n;            // beads
    int32_t lpb;          // lanes cooperating on one bead's lists
    int32_t block;        // CTA size class of the resident kernel
    int32_t cap_pp;       // possible-pairs row capacity
    int32_t cap_pl;       // Verlet row capacity
    int32_t mask;         // 1: bitmask lists (shared-memory Verlet masks)
    int32_t W;            // words per bitmask row, ceil(n/32)
    int32_t max_pp;       // configured max_possiblePairs (overflow -> error)
    int32_t max_pl;       // configured max_pairs
    int32_t grid;         // 1: grid path (per-step kernels, CUDA graphs)
    int32_t lcache;       // shared-memory cache of the Verlet list, entries
    int32_t bsm;          // 1: bonded maps copied to shared memory for a launch
    int32_t ncov, nnat;   // covalent / native map entries (both directions)
    int32_t stride;       // updater period (gsop.cu:117-122)
    int32_t nav;
    int32_t pairs_freq;
    int32_t pp_freq;
    int32_t pull_freq;
    int32_t temp_freq;
    int32_t eps_freq;
    int64_t step;
    int64_t retraction_step;
    // ---- per-bead state (views into the context pools) ----------------------
    float4* x;            // coordinates, w = 0
    uint4* seeds;         // Hybrid Taus states
    float* T;             // kinetic temperature accumulator
    float4* tipF;         // per-bead tip force accumulator (indentation)
    uint8_t* flags;       // FLAG_*
    float4* xalt;         // second coordinate buffer (grid path ping-pong)
    float* log;           // [log_cap * 16] event-log ring (sopb_log_row), or null
    // ---- discrete surface and pulling plane (views into the job's memory) ------
    float4* surf;         // [nsurf] surface beads now
    float4* surf0;        // [nsurf] surface beads at dx = 0
    uint32_t* mica;       // [n * Wm] surface beads within the list cutoff, bitmask rows
    uint8_t* plane_mask;  // [n] 1: spring to the fixed plane, 2: to the pulled plane
    float* plane_r0;      // [n] distance from the plane at step 0
    float* plane_f;       // [n] last spring force along the normal
    int32_t* plane_idx;   // beads of the fixed plane, then of the pulled one, ascending
    // ---- maps ----------------------------------------------------------------
    int32_t* cov_off;     // [n+1]
    int32_t* cov_j;
    float* cov_r0;
    int32_t* nat_off;     // [n+1]
    int32_t* nat_j;
    float2* nat_par;      // (r0^2, -12 eh / r0^2)  (native.cu:112-146)
    int32_t* pp_cnt;      // [n]
    int32_t* pp_j;        // [n * cap_pp]
    int32_t* pl_cnt;      // [n]
    int32_t* pl_j;        // [n * cap_pl]
    uint32_t* ex_mask;    // [n * W] bonded + native partners and self
    uint32_t* pp_mask;    // [n * W] possible pairs (MASK mode)
    uint16_t* nr_j;       // [n * cap_nr] near list: possible pairs within pairlist_cutoff + skin
    int32_t* nr_cnt;      // [n]
    float4* x_ref;        // coordinates the near list was built at
    int32_t cap_nr;       // near-list row capacity
    int32_t nr_valid;     // 1: the near list holds every pair the next Verlet list can have
    float nr_t;           // r^2 threshold of the near list
    float drift2;         // squared displacement since x_ref that invalidates it
    float rlb;            // R_limit_bond: native contacts closer than it count intact
    // ---- force field ---------------------------------------------------------
    float ks, R2;         // FENE: kspring_cov, R_limit^2
    float c8, cut2;       // repulsive: -6 el a^6, pairs_cutoff^2
    float pl_cut;         // pairlist_cutoff
    float pp_thr;         // pairs_threshold
    float pl_t, pp_t;     // r^2 thresholds equivalent to sqrt(r^2) < pl_cut, < pp_thr
    // ---- integrator ------------------------------------------------------------
    float hOverZeta, tempNorm, var, zeta, h;
    int32_t minimization, heating;
    float initialT, deltaT;
    // ---- pulling ---------------------------------------------------------------
    int32_t pulling, ramp, pulledEnd, fixedEnd;
    float deltax, k_trans;
    float pullvec[3], cant0[3], cant[3], pullF[3];
    // ---- indentation (continuous surface) ------------------------------------
    int32_t indent, moveSurface, fixTrans, pad1;
    float tip[3], chip[3], chip0[3], dir[3], micaR[3], micaR0[3], micaN[3];
    float tipR, tipAp, tipBp, surfAp, surfBp, cantKs, V, dx, tipZeta;
    float fav[4];
    int32_t discrete;     // 1: the surface is a square of beads with per-bead lists
    int32_t nsurf, Wm;    // surface beads, words per bitmask row
    float mica_cut2;      // indentationPairsCutoff^2
    // ---- pulling plane (pulling_plane.cu) ----------------------------------------
    int32_t plane, plane_freq, plane_ofreq, nplane_fixed, nplane_pulled, pad3;
    float plane_n[3], plane_p0[3];
    float plane_ks, plane_kscant, plane_zeta, plane_deltax;
    float plane_displ, plane_cant;   // plane and cantilever displacement
    // ---- hydrodynamics (TEA / exact) ----------------------------------------------
    int32_t hi, hi_exact, hi_unlisted, hi_capricious, hi_bmode, hi_refresh;
    float hi_a, hi_epsmax;
    float beta;           // TEA beta' of the job (bdhitea.cu:158-169)
    float epsilon;        // last per-job epsilon (for output)
    // ---- status ---------------------------------------------------------------
    int32_t status;
    int32_t log_cap;      // rows of the event-log ring (a power of two), 0 = none
    uint32_t log_head;    // rows appended so far
    int32_t pad2;
};

// ---------------------------------------------------------------------------
// Hybrid Taus generator (L'Ecuyer's combined Tausworthe steps + an LCG,
// "GPU Gems 3" ch. 37), as used by the reference (src/Integrators/ht.cu:61-106).
// The integer stream is bit-exact; the Gaussians use the fast-math intrinsics
// the reference build uses (-use_fast_math, src/Makefile:14).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t taus_step(uint32_t& z, int s1, int s2, int s3, uint32_t m) {
    uint32_t b = (((z << s1) ^ z) >> s2);
    z = (((z & m) << s3) ^ b);
    return z;
}
__device__ __forceinline__ uint32_t hybrid_taus(uint4& s) {
    uint32_t a = taus_step(s.x, 13, 19, 12, 4294967294u);
    uint32_t b = taus_step(s.y, 2, 25, 4, 4294967288u);
    uint32_t c = taus_step(s.z, 3, 11, 17, 4294967280u);
    s.w = 1664525u * s.w + 1013904223u;
    return a ^ b ^ c ^ s.w;
}
// Mantissa fill to [1,2) minus one; exact zero maps to 1e-8 (ht.cu:61-69).
__device__ __forceinline__ float uint_to_unit(uint32_t u) {
    float f = __uint_as_float(0x3f800000u | (0x007fffffu & u)) - 1.0f;
    return f == 0.0f ? 1.0e-8f : f;
}
// Box-Muller on four draws.  The angle is 2*pi*u formed in double precision
// and rounded to float, as the reference's `2.0f*M_PI*u` is.
__device__ __forceinline__ float4 gaussian4(uint4& s) {
    float4 g;
    float r = sqrtf(-2.0f * __logf(uint_to_unit(hybrid_taus(s))));
    float th = __double2float_rn(6.283185307179586 * (double)uint_to_unit(hybrid_taus(s)));
    g.x = r * __sinf(th);
    g.y = r * __cosf(th);
    r = sqrtf(-2.0f * __logf(uint_to_unit(hybrid_taus(s))));
    th = __double2float_rn(6.283185307179586 * (double)uint_to_unit(hybrid_taus(s)));
    g.z = r * __sinf(th);
    g.w = r * __cosf(th);
    return g;
}

// List membership test sqrt(r^2) < cut of the reference
// (possiblepairlist_kernel.cu:45-46, pairlist_cutoff in pairlist_kernel.cu:57-63),
// with r^2 formed exactly as the CPU oracle forms it.  Because a correctly
// rounded square root is monotonic, sqrt(r^2) < cut holds exactly when
// r^2 < t for the threshold t = sqrt_threshold(cut) computed on the host,
// so the test needs no square root and list membership stays bit-exact.
__device__ __forceinline__ float dist2_rn(float4 xi, float4 xj) {
    const float dx = __fsub_rn(xj.x, xi.x), dy = __fsub_rn(xj.y, xi.y), dz = __fsub_rn(xj.z, xi.z);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}
__device__ __forceinline__ bool within_cutoff(float4 xi, float4 xj, float t) { return dist2_rn(xi, xj) < t; }

// FENE term (covalent_kernel.cu:28-51): Ks*(r-r0)/(r*(1-(r-r0)^2/R0^2)).
// r - r0 cancels for a near-relaxed bond, so r is formed with a correctly
// rounded square root (the reference's fast-math build uses the approximate
// one and loses ~1e-4 of the bond force there).
__device__ __forceinline__ void fene_term(float4 xi, float4 xj, float r0, float ks, float R2, float3& f) {
    float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    float w = __fsqrt_rn(dx * dx + dy * dy + dz * dz) - r0;
    w = __fdiv_rn(ks * w, (w + r0) * (1.0f - __fdiv_rn(w * w, R2)));
    f.x += w * dx;
    f.y += w * dy;
    f.z += w * dz;
}
// Native LJ 12-6 term (native_kernel.cu:27-52).
__device__ __forceinline__ void native_term(float4 xi, float4 xj, float2 par, float3& f) {
    float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    float w = par.x / (dx * dx + dy * dy + dz * dz);
    float p6 = w * w * w;
    w = w * (p6 * p6 - p6) * par.y;
    f.x += dx * w;
    f.y += dy * w;
    f.z += dz * w;
}
// Repulsive r^-6 term with the force cutoff (pairs_kernel.cu:33-59): the
// force on i is r_ij * (-6 el a^6 / r^8), formed as c8 * (1/r^2)^4 with
// c8 = -6 el a^6 precomputed, and zero beyond pairs_cutoff.
__device__ __forceinline__ void pair_term(float4 xi, float4 xj, float c8, float cut2, float3& f) {
    const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    const float r2 = dx * dx + dy * dy + dz * dz;
    float w = 1.0f / r2;
    w = w * w;
    w = c8 * (w * w);
    w = r2 < cut2 ? w : 0.0f;
    f.x += dx * w;
    f.y += dy * w;
    f.z += dz * w;
}

// Tip and continuous-surface terms (indentation_kernel.cu:71-128).  Returns
// the tip's share in tipf (accumulated per bead by the caller).
struct IndentGeom {
    float tip[3], micaR[3], micaN[3];
    float tipR, tipAp, tipBp, surfAp, surfBp;
};
// The tip alone (the first half of indentationDiscreteSurf_kernel,
// indentation_kernel.cu:130-157).
__device__ __forceinline__ void tip_term(float4 xi, const IndentGeom& g, float3& f, float3& tipf) {
    float dx = xi.x - g.tip[0], dy = xi.y - g.tip[1], dz = xi.z - g.tip[2];
    float dw = __fsqrt_rn(dx * dx + dy * dy + dz * dz);
    float r2 = __frcp_rn(dw - g.tipR);
    r2 = r2 * r2;
    float r6 = r2 * r2 * r2;
    float w = g.tipAp * r6 + g.tipBp;
    w = w * r6 / (dw * (dw - g.tipR));
    tipf = make_float3(dx * w, dy * w, dz * w);
    f.x += tipf.x;
    f.y += tipf.y;
    f.z += tipf.z;
}

// The surface beads of bead i's list, strided over the group's lanes
// (indentationDiscreteSurf_kernel's list loop, indentation_kernel.cu:159-177;
// no cutoff inside the list).
__device__ __forceinline__ void mica_partial(const JobDev& J, int i, float4 xi, int l, int lpb, float3& f) {
    const uint32_t* row = J.mica + (size_t)i * J.Wm;
    for (int w = l; w < J.Wm; w += lpb) {
        uint32_t bits = row[w];
        while (bits) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            const float4 q = J.surf[32 * w + b];
            const float ex = xi.x - q.x, ey = xi.y - q.y, ez = xi.z - q.z;
            const float w2 = 1.0f / (ex * ex + ey * ey + ez * ez);
            const float s6 = w2 * w2 * w2;
            const float c = (J.surfAp * s6 + J.surfBp) * s6 * w2;
            f.x += ex * c;
            f.y += ey * c;
            f.z += ez * c;
        }
    }
}

// pullingPlane_kernel (src/Potentials/pulling_plane_kernel.cu:25-52): a
// spring along the normal to the fixed plane (mask 1) or to the plane
// displaced by `displ` (mask 2).  Returns the spring force.
__device__ __forceinline__ float plane_term(const JobDev& J, float displ, int mask, float4 xi, float r0, float3& f) {
    float pc[3] = {J.plane_p0[0], J.plane_p0[1], J.plane_p0[2]};
    if (mask == 2)
        for (int c = 0; c < 3; ++c) pc[c] += displ * J.plane_n[c];
    const float dr = (xi.x - pc[0]) * J.plane_n[0] + (xi.y - pc[1]) * J.plane_n[1] + (xi.z - pc[2]) * J.plane_n[2];
    const float df = -J.plane_ks * (dr - r0);
    f.x += df * J.plane_n[0];
    f.y += df * J.plane_n[1];
    f.z += df * J.plane_n[2];
    return df;
}

__device__ __forceinline__ void indentation_term(float4 xi, const IndentGeom& g, float3& f, float3& tipf) {
    float dx = xi.x - g.tip[0], dy = xi.y - g.tip[1], dz = xi.z - g.tip[2];
    float dw = __fsqrt_rn(dx * dx + dy * dy + dz * dz);
    float r2 = __frcp_rn(dw - g.tipR);
    r2 = r2 * r2;
    float r6 = r2 * r2 * r2;
    float w = g.tipAp * r6 + g.tipBp;
    w = w * r6 / (dw * (dw - g.tipR));
    float3 df = make_float3(dx * w, dy * w, dz * w);
    tipf = df;
    float d = (xi.x - g.micaR[0]) * g.micaN[0] + (xi.y - g.micaR[1]) * g.micaN[1] + (xi.z - g.micaR[2]) * g.micaN[2];
    d = 1.0f / d;
    d = d * d;
    r6 = d * d * d;
    w = g.surfAp * r6 + g.surfBp;
    w = w * r6 * d;
    f.x += g.micaN[0] * w + df.x;
    f.y += g.micaN[1] * w + df.y;
    f.z += g.micaN[2] * w + df.z;
}

}  // namespace sopb
