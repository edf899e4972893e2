// sopb_hi.cuh — hydrodynamic interactions on the grid path.
//
// TEA (Geyer & Winter 2009, the reference's BDHI-TEA integrator,
// src/Integrators/bdhitea_kernel.cu:192-515): the O(N^2) sums over all bead
// pairs of a job run as tiles: a CTA takes 128 beads i and one slice of the
// j range, stages the slice's coordinates and forces in shared memory
// 128 at a time, and writes a partial sum per bead; a per-bead pass adds the
// slices in slice order, so the result does not depend on scheduling.  The
// per-job epsilon and beta' are reduced on the device in FP64, as the
// reference's host does (src/Integrators/bdhitea.cu:133-176).
//
// Exact HI for jobs up to 128 beads (3n <= 384, the reference's CHOLSIZE,
// src/Integrators/bdhitea.h:24): the normalised RPY tensor D is assembled
// every step, factorised in place by one CTA per job (L below, L^T above
// the diagonal, as integrateCholesky_decompose leaves it) and applied to the
// random forces with either the true factor (B = L) or, for parity with the
// reference, its symmetrised upper 3x3 blocks (integrateCholesky_L).
#pragma once

#include "sopb_grid.cuh"

namespace sopb {

constexpr int kHiTile = 128;

struct Blk6 {
    float xx, xy, xz, yy, yz, zz;
};

// RPY block normalised by D_ii (bdhitea_kernel.cu:67-87): (ex,ey,ez) unit
// vector from i to j, r the distance, a the hydrodynamic radius.
__device__ __forceinline__ Blk6 rpy_block(float ex, float ey, float ez, float r, float a) {
    const float ra = r / a;
    float crr, cii;
    if (ra > 2.f) {
        crr = 0.75f / ra * (1.f - 2.f / ra / ra);
        cii = 0.75f / ra * (1.f + 2.f / 3.f / ra / ra);
    } else {
        crr = 3.f * ra / 32.f;
        cii = 1.f - 9.f * ra / 32.f;
    }
    return {ex * ex * crr + cii, ex * ey * crr, ex * ez * crr, ey * ey * crr + cii, ey * ez * crr, ez * ez * crr + cii};
}

__device__ __forceinline__ Blk6 rpy_between(float4 xi, float4 xj, float a) {
    float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    const float r = sqrtf(dx * dx + dy * dy + dz * dz);
    dx /= r;
    dy /= r;
    dz /= r;
    return rpy_block(dx, dy, dz, r, a);
}

// The same block for the per-step O(n^2) sums, with one reciprocal square
// root per pair: e = d rsqrt(r^2), u = a / r = a rsqrt(r^2), and the far
// field (r > 2a) tested as r^2 > 4a^2; both branches are formed and one is
// selected, so a warp does not diverge on the pair distance.
__device__ __forceinline__ Blk6 rpy_fast(float4 xi, float4 xj, float a, float inv_a) {
    const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
    const float r2 = dx * dx + dy * dy + dz * dz;
    const float ir = rsqrtf(r2);
    const float ex = dx * ir, ey = dy * ir, ez = dz * ir;
    const float u = a * ir, u2 = u * u, ra = r2 * ir * inv_a;
    const bool far = r2 > 4.f * a * a;
    const float crr = far ? 0.75f * u * (1.f - 2.f * u2) : (3.f / 32.f) * ra;
    const float cii = far ? 0.75f * u * (1.f + (2.f / 3.f) * u2) : 1.f - (9.f / 32.f) * ra;
    return {ex * ex * crr + cii, ex * ey * crr, ex * ez * crr, ey * ey * crr + cii, ey * ez * crr, ez * ez * crr + cii};
}

// integrateTea_epsilon_local (bdhitea_kernel.cu:192-210): squared row sums
// (x, y, z) and the sum of all nine entries (w).
__device__ __forceinline__ void eps_stats(float4 xi, float4 xj, float a, float4& s) {
    const Blk6 d = rpy_between(xi, xj, a);
    s.w += d.xx + 2 * d.xy + 2 * d.xz + d.yy + 2 * d.yz + d.zz;
    s.x += d.xx * d.xx + d.xy * d.xy + d.xz * d.xz;
    s.y += d.xy * d.xy + d.yy * d.yy + d.yz * d.yz;
    s.z += d.xz * d.xz + d.yz * d.yz + d.zz * d.zz;
}

// integrateTea_force (bdhitea_kernel.cu:252-301): D_ij (F_j + beta C_i o g_j).
__device__ __forceinline__ void tea_pair(float4 xi, float4 xj, float4 mj, float4 rj, float3 bci, float a, float inv_a,
                                         float3& f) {
    const Blk6 d = rpy_fast(xi, xj, a, inv_a);
    const float f0 = mj.x + rj.x * bci.x, f1 = mj.y + rj.y * bci.y, f2 = mj.z + rj.z * bci.z;
    f.x += d.xx * f0 + d.xy * f1 + d.xz * f2;
    f.y += d.xy * f0 + d.yy * f1 + d.yz * f2;
    f.z += d.xz * f0 + d.yz * f1 + d.zz * f2;
}

__device__ __forceinline__ bool tea_eps_due(const JobDev& J, int64_t step) {
    return step % J.stride == 0 && step % J.eps_freq == 0;
}

// integrateTea_prepare (bdhitea_kernel.cu:33-65): random force rho*g,
// molecular force with pulling applied, coordinate copy.
__global__ void __launch_bounds__(kGridBlock)
k_hi_prepare(JobDev* __restrict__ Jp, GridAux aux) {
    __shared__ JobDev Js;
    load_job<kGridBlock>(Js, Jp);
    __syncthreads();
    const JobDev& J = Js;
    if (J.status) return;
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < J.n; i += gridDim.x * kGridBlock) {
        uint4 st = J.seeds[i];
        float4 g = gaussian4(st);
        J.seeds[i] = st;
        g.x *= J.var;
        g.y *= J.var;
        g.z *= J.var;
        aux.rf[i] = g;
        float4 f = aux.F[i];
        if (J.pulling) {
            const uint8_t fl = J.flags[i];
            if (fl == FLAG_FIXED) f.x = f.y = f.z = 0.f;
            if (fl == FLAG_PULLED) { f.x += J.pullF[0]; f.y += J.pullF[1]; f.z += J.pullF[2]; }
        }
        aux.mf[i] = f;
        aux.xc[i] = J.x[i];
    }
}

// ---- TEA epsilon (updater) --------------------------------------------------
__global__ void __launch_bounds__(kHiTile)
k_tea_eps_partial(JobDev* __restrict__ Jp, GridAux aux, int jsplit, int force) {
    __shared__ float4 xs[kHiTile];
    const JobDev& J = *Jp;
    const int64_t step = job_step(Jp);
    if (J.status || (!force && !tea_eps_due(J, step))) return;
    const int n = J.n, i = blockIdx.x * kHiTile + threadIdx.x, s = blockIdx.y;
    const float4 xi = J.x[i < n ? i : 0];
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    if (J.hi_unlisted) {
        const int span = ((n + jsplit - 1) / jsplit + kHiTile - 1) / kHiTile * kHiTile;
        const int j0 = s * span, j1 = min(n, j0 + span);
        for (int t0 = j0; t0 < j1; t0 += kHiTile) {
            __syncthreads();
            if (t0 + threadIdx.x < j1) xs[threadIdx.x] = J.x[t0 + threadIdx.x];
            __syncthreads();
            const int cnt = min(kHiTile, j1 - t0);
            if (i < n)
                for (int q = 0; q < cnt; ++q)
                    if (t0 + q != i) eps_stats(xi, xs[q], J.hi_a, acc);
        }
    } else if (s == 0 && i < n) {
        // integrateTea_epsilon: covalent, native and Verlet partners
        for (int k = J.cov_off[i]; k < J.cov_off[i + 1]; ++k) eps_stats(xi, J.x[J.cov_j[k]], J.hi_a, acc);
        for (int k = J.nat_off[i]; k < J.nat_off[i + 1]; ++k) eps_stats(xi, J.x[J.nat_j[k]], J.hi_a, acc);
        const int32_t* row = J.pl_j + (size_t)i * J.cap_pl;
        for (int k = 0; k < J.pl_cnt[i]; ++k) eps_stats(xi, J.x[row[k]], J.hi_a, acc);
    }
    if (i < n) aux.part[(size_t)s * n + i] = acc;
}

__global__ void __launch_bounds__(kGridBlock)
k_tea_eps_reduce(JobDev* __restrict__ Jp, GridAux aux, int jsplit, int force) {
    const JobDev& J = *Jp;
    const int64_t step = job_step(Jp);
    if (J.status || (!force && !tea_eps_due(J, step))) return;
    const int n = J.n;
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < n; i += gridDim.x * kGridBlock) {
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int s = 0; s < jsplit; ++s) {
            const float4 p = aux.part[(size_t)s * n + i];
            a.x += p.x; a.y += p.y; a.z += p.z; a.w += p.w;
        }
        aux.ci4[i] = a;
        aux.eps[i] = a.w;
    }
}

// TeaUpdater::update's host arithmetic (bdhitea.cu:143-169) in FP64: the
// average off-diagonal coupling epsilon, the capricious checks, and
// beta' = (1 - sqrt(1 - a)) / a with a = (3N-1) eps^2 - (3N-2) eps.
__global__ void __launch_bounds__(256)
k_tea_beta(JobDev* __restrict__ Jp, GridAux aux, int force) {
    __shared__ double red[256];
    JobDev& J = *Jp;
    const int64_t step = job_step(Jp);
    if (J.status || (!force && !tea_eps_due(J, step))) return;
    const int n = J.n;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) s += (double)aux.eps[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double eps = red[0];
        if (n > 1) eps /= 3. * n * (3. * n - 3.);
        int st = 0;
        if (eps > 1.0) {
            if (J.hi_capricious) st = SOPB_ERR_HI;
            eps = 1.0;
        }
        if (eps > J.hi_epsmax) st = SOPB_ERR_HI;
        const double a = (3. * n - 1.) * eps * eps - (3. * n - 2.) * eps;
        double beta;
        if (fabs(a) < 1e-7) {
            beta = 0.5;
            if (J.hi_capricious && J.hi_a > 0.0f) st = SOPB_ERR_HI;
        } else {
            beta = (1. - sqrt(1. - a)) / a;
        }
        J.beta = (float)beta;
        J.epsilon = (float)eps;
        if (st) J.status = st;
    }
}

// ---- TEA integration step ----------------------------------------------------
__device__ __forceinline__ float3 tea_bci(const JobDev& J, const GridAux& aux, int i, float3* ci_out) {
    const float4 c = aux.ci4[i];
    const float b2 = J.beta * J.beta;
    const float3 ci = make_float3(1.f / sqrtf(1.f + b2 * c.x), 1.f / sqrtf(1.f + b2 * c.y), 1.f / sqrtf(1.f + b2 * c.z));
    if (ci_out) *ci_out = ci;
    return make_float3(ci.x * J.beta, ci.y * J.beta, ci.z * J.beta);
}

__global__ void __launch_bounds__(kHiTile)
k_tea_force_partial(JobDev* __restrict__ Jp, GridAux aux, int jsplit) {
    __shared__ float4 xs[kHiTile], ms[kHiTile], rs[kHiTile];
    const JobDev& J = *Jp;
    if (J.status) return;
    const int n = J.n, i = blockIdx.x * kHiTile + threadIdx.x, s = blockIdx.y;
    const float4 xi = aux.xc[i < n ? i : 0];
    const float3 bci = tea_bci(J, aux, i < n ? i : 0, nullptr);
    const float a = J.hi_a, inv_a = 1.f / J.hi_a;
    float3 f = make_float3(0.f, 0.f, 0.f);
    if (J.hi_unlisted) {
        const int span = ((n + jsplit - 1) / jsplit + kHiTile - 1) / kHiTile * kHiTile;
        const int j0 = s * span, j1 = min(n, j0 + span);
        for (int t0 = j0; t0 < j1; t0 += kHiTile) {
            __syncthreads();
            const int q = t0 + threadIdx.x;
            if (q < j1) {
                xs[threadIdx.x] = aux.xc[q];
                ms[threadIdx.x] = aux.mf[q];
                rs[threadIdx.x] = aux.rf[q];
            }
            __syncthreads();
            const int cnt = min(kHiTile, j1 - t0);
            if (i < n) {
                if (t0 == blockIdx.x * kHiTile) {   // the tile of this CTA's own beads
                    for (int k = 0; k < cnt; ++k)
                        if (t0 + k != i) tea_pair(xi, xs[k], ms[k], rs[k], bci, a, inv_a, f);
                } else {
#pragma unroll 4
                    for (int k = 0; k < cnt; ++k) tea_pair(xi, xs[k], ms[k], rs[k], bci, a, inv_a, f);
                }
            }
        }
    } else if (s == 0 && i < n) {
        // integrateTea_kernel: covalent, native and Verlet partners
        for (int k = J.cov_off[i]; k < J.cov_off[i + 1]; ++k) {
            const int q = J.cov_j[k];
            tea_pair(xi, aux.xc[q], aux.mf[q], aux.rf[q], bci, a, inv_a, f);
        }
        for (int k = J.nat_off[i]; k < J.nat_off[i + 1]; ++k) {
            const int q = J.nat_j[k];
            tea_pair(xi, aux.xc[q], aux.mf[q], aux.rf[q], bci, a, inv_a, f);
        }
        const int32_t* row = J.pl_j + (size_t)i * J.cap_pl;
        for (int k = 0; k < J.pl_cnt[i]; ++k) {
            const int q = row[k];
            tea_pair(xi, aux.xc[q], aux.mf[q], aux.rf[q], bci, a, inv_a, f);
        }
    }
    if (i < n) aux.part[(size_t)s * n + i] = make_float4(f.x, f.y, f.z, 0.f);
}

__global__ void __launch_bounds__(kGridBlock)
k_tea_integrate(JobDev* __restrict__ Jp, GridAux aux, int jsplit) {
    __shared__ JobDev Js;
    load_job<kGridBlock>(Js, Jp);
    __syncthreads();
    const JobDev& J = Js;
    if (J.status) return;
    const int n = J.n;
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < n; i += gridDim.x * kGridBlock) {
        float3 ci;
        tea_bci(J, aux, i, &ci);
        const float4 m = aux.mf[i], r = aux.rf[i];
        float3 f = make_float3(m.x + r.x * ci.x, m.y + r.y * ci.y, m.z + r.z * ci.z);
        for (int s = 0; s < jsplit; ++s) {
            const float4 p = aux.part[(size_t)s * n + i];
            f.x += p.x; f.y += p.y; f.z += p.z;
        }
        if (J.pulling && J.flags[i] == FLAG_FIXED) f = make_float3(0.f, 0.f, 0.f);
        const float4 xc = aux.xc[i];
        const float dx = J.hOverZeta * f.x, dy = J.hOverZeta * f.y, dz = J.hOverZeta * f.z;
        J.x[i] = make_float4(xc.x + dx, xc.y + dy, xc.z + dz, xc.w);
        J.T[i] += J.tempNorm * (dx * dx + dy * dy + dz * dz);
    }
}

// ---- exact HI, n <= 128 ---------------------------------------------------------
// integrateCholesky_D (bdhitea_kernel.cu:89-152): bead i's block column of
// D (identity diagonal blocks; written when the factor is refreshed) and
// D F with every bead reading the prepared forces (the reference reads them
// while other threads overwrite them).
__global__ void __launch_bounds__(kGridBlock)
k_chol_D(JobDev* __restrict__ Jp, GridAux aux, int assemble) {
    const JobDev& J = *Jp;
    if (J.status) return;
    const int n = J.n, ld = aux.ld;
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < n; i += gridDim.x * kGridBlock) {
        const float4 xi = J.x[i];
        float4 f = aux.mf[i];
        for (int q = 0; q < n; ++q) {
            float* r0 = aux.tensor + (size_t)(3 * q) * ld + 3 * i;
            float* r1 = r0 + ld;
            float* r2 = r1 + ld;
            if (q == i) {
                if (assemble) {
                    r0[0] = 1.f; r0[1] = 0.f; r0[2] = 0.f;
                    r1[0] = 0.f; r1[1] = 1.f; r1[2] = 0.f;
                    r2[0] = 0.f; r2[1] = 0.f; r2[2] = 1.f;
                }
                continue;
            }
            const Blk6 d = rpy_between(xi, J.x[q], J.hi_a);
            if (assemble) {
                r0[0] = d.xx; r0[1] = d.xy; r0[2] = d.xz;
                r1[0] = d.xy; r1[1] = d.yy; r1[2] = d.yz;
                r2[0] = d.xz; r2[1] = d.yz; r2[2] = d.zz;
            }
            const float4 fq = aux.mf[q];
            f.x += d.xx * fq.x + d.xy * fq.y + d.xz * fq.z;
            f.y += d.xy * fq.x + d.yy * fq.y + d.yz * fq.z;
            f.z += d.xz * fq.x + d.yz * fq.y + d.zz * fq.z;
        }
        aux.F[i] = f;   // D F (the potential forces are no longer needed)
    }
}

// integrateCholesky_decompose (bdhitea_kernel.cu:154-190): one CTA of 3n
// threads, one column per round.
__global__ void __launch_bounds__(384)
k_chol_factor_small(JobDev* __restrict__ Jp, GridAux aux) {
    __shared__ float row[384];
    __shared__ float diag;
    const JobDev& J = *Jp;
    if (J.status) return;
    const int m = 3 * J.n, ld = aux.ld, t = threadIdx.x;
    float* M = aux.tensor;
    for (int j = 0; j < m; ++j) {
        if (t < m) row[t] = M[(size_t)j * ld + t];
        __syncthreads();
        float val = t < m ? row[t] : 0.f;
        if (t < m && t >= j)
            for (int k = 0; k < j; ++k) val -= M[(size_t)k * ld + t] * row[k];
        if (t == j) diag = sqrtf(val);
        __syncthreads();
        if (t < m && t >= j) {
            val = val / diag;
            M[(size_t)t * ld + j] = val;
            M[(size_t)j * ld + t] = val;
        }
        __syncthreads();
    }
}

// The true factor L of D at n <= 128 (B = L), the same factorisation as
// integrateCholesky_decompose (bdhitea_kernel.cu:154-190) in another order:
// right-looking in 32-column panels, in one CTA.  The panel (its rows from
// the diagonal down, at most 384 x 32) is factorised column by column with
// one thread per row holding the row in registers (IEEE square root and
// division, two barriers per column); it is written back, and the lower
// triangle of the trailing matrix takes the panel's rank-32 update from L2
// in 4 x 4 register tiles.  Only the lower triangle is written (the
// reference also mirrors the factor into the upper one, which its
// symmetrised noise matrix reads; that mode keeps k_chol_factor_small).
constexpr int kSmallPanel = 32;
constexpr int kSmallThreads = 512;                        // at least kSmallRows: one thread per panel row
constexpr int kSmallRows = 384;                            // 3n for n <= 128
constexpr int kSmallLd = kSmallPanel + 1;                  // floats per panel row in shared memory
constexpr size_t kSmallSmem = (size_t)kSmallRows * kSmallLd * sizeof(float);
static_assert(kSmallThreads >= kSmallRows, "one thread per panel row");

__global__ void __launch_bounds__(kSmallThreads)
k_chol_factor_panels(JobDev* __restrict__ Jp, GridAux aux) {
    extern __shared__ float P[];                           // [rows][kSmallLd]
    __shared__ float diag[kSmallPanel];
    __shared__ float col_s[kSmallRows];                    // the scaled column of the panel
    __shared__ float piv_s;
    if (Jp->status) return;
    const int m = 3 * Jp->n, ld = aux.ld, tid = threadIdx.x;
    float* M = aux.tensor;
    for (int p0 = 0; p0 < m; p0 += kSmallPanel) {
        const int pb = min(kSmallPanel, m - p0), rows = m - p0;
        for (int e = tid; e < rows * kSmallPanel; e += kSmallThreads) {
            const int r = e / kSmallPanel, c = e % kSmallPanel;
            P[r * kSmallLd + c] = c < pb && c <= r ? M[(size_t)(p0 + r) * ld + p0 + c] : 0.f;
        }
        __syncthreads();
        // the panel, column by column: thread r holds panel row r in
        // registers; per column the pivot's owner publishes it, every row
        // below scales its entry and publishes it, then updates its row
        {
            const int r = tid;
            const bool own = r < rows;
            float row[kSmallPanel];
#pragma unroll
            for (int k = 0; k < kSmallPanel; ++k) row[k] = own ? P[r * kSmallLd + k] : 0.f;
#pragma unroll
            for (int c = 0; c < kSmallPanel; ++c) {   // unrolled: row[] indices are constants
                if (c < pb) {                           // the same for the whole CTA
                    if (r == c) piv_s = row[c];
                    __syncthreads();
                    const float d = __fsqrt_rn(piv_s);
                    float lrc = 0.f;
                    if (r == c) diag[c] = d;
                    if (r > c && own) {
                        lrc = __fdiv_rn(row[c], d);
                        row[c] = lrc;
                        col_s[r] = lrc;
                    }
                    __syncthreads();
                    if (r > c && own) {
#pragma unroll
                        for (int k = c + 1; k < kSmallPanel; ++k)
                            if (k < pb && k <= r) row[k] -= lrc * col_s[k];
                    }
                }
            }
            __syncthreads();
            if (own) {
#pragma unroll
                for (int k = 0; k < kSmallPanel; ++k) P[r * kSmallLd + k] = row[k];
            }
            __syncthreads();
        }
        for (int e = tid; e < rows * kSmallPanel; e += kSmallThreads) {
            const int r = e / kSmallPanel, c = e % kSmallPanel;
            if (c < pb && c <= r) M[(size_t)(p0 + r) * ld + p0 + c] = r == c ? diag[c] : P[r * kSmallLd + c];
        }
        // trailing lower triangle: A22 -= L21 L21^T, 4 x 4 tiles (ti >= tj),
        // consecutive threads along a tile row
        const int n2 = rows - pb, nt = (n2 + 3) / 4, ntiles = nt * (nt + 1) / 2;
        for (int t = tid; t < ntiles; t += kSmallThreads) {
            int ti = (int)((sqrtf(8.f * (float)t + 1.f) - 1.f) * 0.5f);
            while (ti * (ti + 1) / 2 > t) --ti;
            while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
            const int tj = t - ti * (ti + 1) / 2;
            float acc[4][4] = {};
            const float* A = P + (size_t)(pb + 4 * ti) * kSmallLd;
            const float* B = P + (size_t)(pb + 4 * tj) * kSmallLd;
            for (int c = 0; c < pb; ++c) {
                float a[4], b[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    a[u] = 4 * ti + u < n2 ? A[u * kSmallLd + c] : 0.f;
                    b[u] = 4 * tj + u < n2 ? B[u * kSmallLd + c] : 0.f;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int v = 0; v < 4; ++v) acc[u][v] += a[u] * b[v];
            }
            // all sixteen entries loaded before any is stored (one L2 round trip)
            float mv[4][4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int row = 4 * ti + u, col = 4 * tj + v;
                    mv[u][v] = row < n2 && col <= row ? M[(size_t)(p0 + pb + row) * ld + p0 + pb + col] : 0.f;
                }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int row = 4 * ti + u, col = 4 * tj + v;
                    if (row < n2 && col <= row) M[(size_t)(p0 + pb + row) * ld + p0 + pb + col] = mv[u][v] - acc[u][v];
                }
        }
        __syncthreads();
    }
}

// integrateCholesky_L (bdhitea_kernel.cu:303-361): f_i = (D F)_i + sum_{q<=i}
// B_iq (rho g)_q, then the fixed beads and the Ermak-McCammon move.
__global__ void __launch_bounds__(kGridBlock)
k_chol_apply(JobDev* __restrict__ Jp, GridAux aux) {
    const JobDev& J = *Jp;
    if (J.status) return;
    const int n = J.n, ld = aux.ld;
    const float* M = aux.tensor;
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < n; i += gridDim.x * kGridBlock) {
        const float4 dfi = aux.F[i];
        float3 f = make_float3(dfi.x, dfi.y, dfi.z);
        for (int q = 0; q <= i; ++q) {
            const float4 g = aux.rf[q];
            if (J.hi_bmode == SOPB_HI_B_REFCOMPAT) {
                const float* L0 = M + (size_t)(3 * q) * ld + 3 * i;
                const float bxx = L0[0], bxy = L0[1], bxz = L0[2], byy = L0[ld + 1], byz = L0[ld + 2], bzz = L0[2 * ld + 2];
                f.x += bxx * g.x + bxy * g.y + bxz * g.z;
                f.y += bxy * g.x + byy * g.y + byz * g.z;
                f.z += bxz * g.x + byz * g.y + bzz * g.z;
            } else {
                const float gg[3] = {g.x, g.y, g.z};
                float acc[3];
                for (int r = 0; r < 3; ++r) {
                    acc[r] = 0.f;
                    for (int c = 0; c < 3; ++c)
                        if (3 * q + c <= 3 * i + r) acc[r] += M[(size_t)(3 * i + r) * ld + 3 * q + c] * gg[c];
                }
                f.x += acc[0];
                f.y += acc[1];
                f.z += acc[2];
            }
        }
        if (J.pulling && J.flags[i] == FLAG_FIXED) f = make_float3(0.f, 0.f, 0.f);
        const float4 xc = aux.xc[i];
        const float dx = J.hOverZeta * f.x, dy = J.hOverZeta * f.y, dz = J.hOverZeta * f.z;
        J.x[i] = make_float4(xc.x + dx, xc.y + dy, xc.z + dz, xc.w);
        J.T[i] = J.T[i] + J.tempNorm * (dx * dx + dy * dy + dz * dz);
    }
}

// integrateCholesky_L (bdhitea_kernel.cu:303-361) with the true factor at
// n <= 128: a warp per bead; the lanes split the columns of the bead's three
// rows of L (the noise vector rho g staged flat in shared memory), a fixed
// xor-shuffle tree sums them, then (D F)_i, the fixed beads and the
// Ermak-McCammon move as in k_chol_apply.
constexpr int kApplyWarps = 8;
__global__ void __launch_bounds__(32 * kApplyWarps)
k_chol_apply_warp(JobDev* __restrict__ Jp, GridAux aux) {
    __shared__ float gs[kSmallRows];
    const JobDev& J = *Jp;
    if (J.status) return;
    const int n = J.n, ld = aux.ld, lane = threadIdx.x & 31;
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        const float4 g = aux.rf[q];
        gs[3 * q] = g.x;
        gs[3 * q + 1] = g.y;
        gs[3 * q + 2] = g.z;
    }
    __syncthreads();
    const float* M = aux.tensor;
    const int i = blockIdx.x * kApplyWarps + (threadIdx.x >> 5);
    if (i >= n) return;
    float acc[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int row = 3 * i + r;
        const float* Lr = M + (size_t)row * ld;
        float a = 0.f;
        for (int c = lane; c <= row; c += 32) a += Lr[c] * gs[c];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        acc[r] = a;
    }
    if (lane == 0) {
        const float4 dfi = aux.F[i];
        float3 f = make_float3(dfi.x + acc[0], dfi.y + acc[1], dfi.z + acc[2]);
        if (J.pulling && J.flags[i] == FLAG_FIXED) f = make_float3(0.f, 0.f, 0.f);
        const float4 xc = aux.xc[i];
        const float dx = J.hOverZeta * f.x, dy = J.hOverZeta * f.y, dz = J.hOverZeta * f.z;
        J.x[i] = make_float4(xc.x + dx, xc.y + dy, xc.z + dz, xc.w);
        J.T[i] = J.T[i] + J.tempNorm * (dx * dx + dy * dy + dz * dz);
    }
}

}  // namespace sopb
