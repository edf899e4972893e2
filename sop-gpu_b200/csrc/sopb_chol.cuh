// sopb_chol.cuh — exact hydrodynamics (Ermak-McCammon with the Cholesky
// factor of the diffusion tensor) for jobs above 128 beads.
//
// The reference factorises the normalised RPY tensor D (3n x 3n, identity
// diagonal blocks) every step with one CTA and one thread per column, which
// limits it to n <= 128 (integrateCholesky_decompose,
// src/Integrators/bdhitea_kernel.cu:154-190).  Here D is assembled into a
// row-major matrix with a 32-float aligned leading dimension and factorised
// in place, lower triangle, by a right-looking blocked algorithm with 128-wide
// panels:
//   k_chol_potrf   the 128 x 128 diagonal block, one CTA in shared memory;
//   k_chol_trsm    the panel below it, L_ik = A_ik L_kk^-T, a warp per row;
//   k_chol_syrk    the trailing lower triangle, A_ij -= L_ik L_jk^T, in
//                  128 x 128 output tiles with 8 x 8 FP32 register tiles.
// The factor is refreshed every `hi_refresh` steps (an updater; 1 = every
// step, as the reference).  Every step applies it: (L g)_i by a warp per bead
// over the bead's three rows, D F by the TEA-style tiles, then the move
// (integrateCholesky_L, bdhitea_kernel.cu:303-361, with B = L).
// All reductions run in a fixed order, so results do not depend on scheduling.
#pragma once

#include "sopb_hi.cuh"

namespace sopb {

constexpr int kCholNB = 128;     // panel width
constexpr int kCholLdp = kCholNB + 1;
constexpr int kCholTile = 128;   // trailing-update output tile
constexpr int kCholKC = 8;       // K columns staged per round

__host__ __device__ inline int chol_ld(int n) { return (3 * n + 31) & ~31; }
constexpr size_t kCholPotrfSmem = (size_t)(kCholNB * kCholLdp + kCholNB) * 4;
constexpr size_t kCholTrsmSmem = (size_t)(kCholNB * kCholLdp + kCholNB) * 4;
constexpr int kCholMaxBeads = 16384;   // 3n floats of g in shared memory

// D, lower block triangle: block (i, q), q <= i, at rows 3i.., columns 3q..
// (integrateCholesky_D, bdhitea_kernel.cu:89-152, from the step's coordinates).
__global__ void __launch_bounds__(256)
k_hi_assemble(const JobDev* __restrict__ Jp, GridAux aux) {
    const JobDev& J = *Jp;
    if (J.status) return;
    const int i = blockIdx.y, ld = aux.ld;
    const float4 xi = aux.xc[i];
    for (int q = blockIdx.x * 256 + threadIdx.x; q <= i; q += gridDim.x * 256) {
        float* r0 = aux.tensor + (size_t)(3 * i) * ld + 3 * q;
        float* r1 = r0 + ld;
        float* r2 = r1 + ld;
        if (q == i) {
            r0[0] = 1.f; r0[1] = 0.f; r0[2] = 0.f;
            r1[0] = 0.f; r1[1] = 1.f; r1[2] = 0.f;
            r2[0] = 0.f; r2[1] = 0.f; r2[2] = 1.f;
            continue;
        }
        const Blk6 d = rpy_between(xi, aux.xc[q], J.hi_a);
        r0[0] = d.xx; r0[1] = d.xy; r0[2] = d.xz;
        r1[0] = d.xy; r1[1] = d.yy; r1[2] = d.yz;
        r2[0] = d.xz; r2[1] = d.yz; r2[2] = d.zz;
    }
}

// Cholesky of the diagonal block at (k, k), nb <= 128 rows, in shared memory.
// Column c: every thread reads the pivot d = A_cc and subtracts
// A_rc A_sc / d from the lower trailing entries it owns, while the scaled
// column A_rc / sqrt(d) is parked in the unused upper triangle; one barrier
// per column.  A pivot that is not positive sets the job's status.
__global__ void __launch_bounds__(256)
k_chol_potrf(JobDev* __restrict__ Jp, GridAux aux, int k) {
    extern __shared__ float A[];   // [kCholNB][kCholLdp], then the pivots' square roots
    if (Jp->status) return;
    const int m = 3 * Jp->n, ld = aux.ld, nb = min(kCholNB, m - k);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float* M = aux.tensor + (size_t)k * ld + k;
    for (int r = warp; r < nb; r += 8)
        for (int s = lane; s <= r; s += 32) A[r * kCholLdp + s] = M[(size_t)r * ld + s];
    __syncthreads();
    float* dg = A + kCholNB * kCholLdp;
    int bad = 0;
    for (int c = 0; c < nb; ++c) {
        const float d = A[c * kCholLdp + c];   // final: column c-1's updates are behind the barrier
        if (!(d > 0.f)) bad = 1;
        const float rs = rsqrtf(d), inv = 1.0f / d;
        for (int r = c + 1 + warp; r < nb; r += 8) {
            const float arc = A[r * kCholLdp + c];
            if (lane == 0) A[c * kCholLdp + r] = arc * rs;
            for (int s = c + 1 + lane; s <= r; s += 32) A[r * kCholLdp + s] -= arc * A[s * kCholLdp + c] * inv;
        }
        if (tid == 0) dg[c] = sqrtf(d);
        __syncthreads();
    }
    for (int r = warp; r < nb; r += 8)
        for (int s = lane; s <= r; s += 32) M[(size_t)r * ld + s] = s == r ? dg[r] : A[s * kCholLdp + r];
    if (bad && tid == 0) Jp->status = SOPB_ERR_HI;
}

// Panel solve below the diagonal block: row r of A[k+nb.., k..k+nb) becomes
// x with x L_kk^T = a, by forward substitution; a warp per row, lane l holds
// columns l, l+32, l+64, l+96.  L_kk and its reciprocal diagonal are staged
// in shared memory once per CTA.
__global__ void __launch_bounds__(256)
k_chol_trsm(JobDev* __restrict__ Jp, GridAux aux, int k) {
    extern __shared__ float L[];   // [kCholNB][kCholLdp] + inverse diagonal
    if (Jp->status) return;
    const int m = 3 * Jp->n, ld = aux.ld, nb = min(kCholNB, m - k);
    const int tid = threadIdx.x, lane = tid & 31;
    float* dinv = L + kCholNB * kCholLdp;
    const float* D = aux.tensor + (size_t)k * ld + k;
    for (int r = tid >> 5; r < nb; r += 8)
        for (int s = lane; s <= r; s += 32) L[r * kCholLdp + s] = D[(size_t)r * ld + s];
    __syncthreads();
    for (int c = tid; c < nb; c += 256) dinv[c] = 1.0f / L[c * kCholLdp + c];
    __syncthreads();
    const int warps = gridDim.x * 8;
    for (int r = k + nb + blockIdx.x * 8 + (tid >> 5); r < m; r += warps) {
        float* row = aux.tensor + (size_t)r * ld + k;
        float a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) a[u] = lane + 32 * u < nb ? row[lane + 32 * u] : 0.f;
        for (int c = 0; c < nb; ++c) {
            const int owner = c & 31, slot = c >> 5;
            float mine = slot == 0 ? a[0] : slot == 1 ? a[1] : slot == 2 ? a[2] : a[3];
            const float x = __shfl_sync(0xffffffffu, mine, owner) * dinv[c];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int cc = lane + 32 * u;
                if (cc == c) a[u] = x;
                else if (cc > c && cc < nb) a[u] -= x * L[cc * kCholLdp + c];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (lane + 32 * u < nb) row[lane + 32 * u] = a[u];
    }
}

// Trailing update of the lower triangle right of the panel:
// A[i][j] -= sum_c P[i][c] P[j][c] over the panel's columns, 128 x 128 output
// tiles (lower tiles only, blockIdx.x enumerates them row by row), 256
// threads with 8 x 8 outputs each, K staged 8 columns at a time.
__global__ void __launch_bounds__(256, 2)
k_chol_syrk(JobDev* __restrict__ Jp, GridAux aux, int k) {
    __shared__ __align__(16) float As[2][kCholKC][kCholTile + 4];
    __shared__ __align__(16) float Bs[2][kCholKC][kCholTile + 4];
    if (Jp->status) return;
    const int m = 3 * Jp->n, ld = aux.ld, nb = min(kCholNB, m - k), t0 = k + nb;
    // tile (I, J), I >= J, from the linear index
    const int b = blockIdx.x;
    int I = (int)((sqrtf(8.f * (float)b + 1.f) - 1.f) * 0.5f);
    while ((I + 1) * (I + 2) / 2 <= b) ++I;
    while (I * (I + 1) / 2 > b) --I;
    const int Jt = b - I * (I + 1) / 2;
    const int r0 = t0 + I * kCholTile, c0 = t0 + Jt * kCholTile;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const float* P = aux.tensor + k;
    // staging: thread loads row (tid >> 1) of the tile, 4 columns at (tid & 1) * 4
    const int lr = tid >> 1, lc = (tid & 1) * 4;
    auto fetch = [&](int row0, int kc) -> float4 {
        const int r = row0 + lr;
        if (r < m && kc + lc < nb) return *reinterpret_cast<const float4*>(P + (size_t)r * ld + kc + lc);
        return make_float4(0.f, 0.f, 0.f, 0.f);
    };
    float acc[8][8];
#pragma unroll
    for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[u][v] = 0.f;
    float4 pa = fetch(r0, 0), pb = fetch(c0, 0);
    int buf = 0;
    for (int kc = 0; kc < nb; kc += kCholKC) {
        As[buf][lc + 0][lr] = pa.x; As[buf][lc + 1][lr] = pa.y; As[buf][lc + 2][lr] = pa.z; As[buf][lc + 3][lr] = pa.w;
        Bs[buf][lc + 0][lr] = pb.x; Bs[buf][lc + 1][lr] = pb.y; Bs[buf][lc + 2][lr] = pb.z; Bs[buf][lc + 3][lr] = pb.w;
        __syncthreads();
        if (kc + kCholKC < nb) {
            pa = fetch(r0, kc + kCholKC);
            pb = fetch(c0, kc + kCholKC);
        }
#pragma unroll
        for (int kk = 0; kk < kCholKC; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][64 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][kk][64 + tx * 4]);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int v = 0; v < 8; ++v) acc[u][v] = fmaf(av[u], bv[v], acc[u][v]);
        }
        buf ^= 1;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int r = r0 + (u < 4 ? ty * 4 + u : 64 + ty * 4 + u - 4);
        if (r >= m) continue;
        float* crow = aux.tensor + (size_t)r * ld;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int c = c0 + h * 64 + tx * 4;
            if (c + 3 < m && c + 3 <= r) {
                float4 v = *reinterpret_cast<float4*>(crow + c);
                v.x -= acc[u][4 * h + 0]; v.y -= acc[u][4 * h + 1]; v.z -= acc[u][4 * h + 2]; v.w -= acc[u][4 * h + 3];
                *reinterpret_cast<float4*>(crow + c) = v;
            } else {
                for (int w = 0; w < 4; ++w)
                    if (c + w < m && c + w <= r) crow[c + w] -= acc[u][4 * h + w];
            }
        }
    }
}

// D F tiles: partial sums over one slice of j of D_ij F_j, j != i
// (integrateCholesky_D's product, bdhitea_kernel.cu:130-148).
__global__ void __launch_bounds__(kHiTile)
k_hi_df_partial(JobDev* __restrict__ Jp, GridAux aux, int jsplit) {
    __shared__ float4 xs[kHiTile], ms[kHiTile];
    const JobDev& J = *Jp;
    if (J.status) return;
    const int n = J.n, i = blockIdx.x * kHiTile + threadIdx.x, s = blockIdx.y;
    const float4 xi = aux.xc[i < n ? i : 0];
    float3 f = make_float3(0.f, 0.f, 0.f);
    const int span = ((n + jsplit - 1) / jsplit + kHiTile - 1) / kHiTile * kHiTile;
    const int j0 = s * span, j1 = min(n, j0 + span);
    for (int t0 = j0; t0 < j1; t0 += kHiTile) {
        __syncthreads();
        const int q = t0 + threadIdx.x;
        if (q < j1) {
            xs[threadIdx.x] = aux.xc[q];
            ms[threadIdx.x] = aux.mf[q];
        }
        __syncthreads();
        const int cnt = min(kHiTile, j1 - t0);
        if (i < n)
            for (int kk = 0; kk < cnt; ++kk) {
                if (t0 + kk == i) continue;
                const Blk6 d = rpy_between(xi, xs[kk], J.hi_a);
                const float4 fq = ms[kk];
                f.x += d.xx * fq.x + d.xy * fq.y + d.xz * fq.z;
                f.y += d.xy * fq.x + d.yy * fq.y + d.yz * fq.z;
                f.z += d.xz * fq.x + d.yz * fq.y + d.zz * fq.z;
            }
    }
    if (i < n) aux.part[(size_t)s * n + i] = make_float4(f.x, f.y, f.z, 0.f);
}

// The step with the factor: f_i = F_i + sum_s (D F partial)_s + (L g)_i, then
// the fixed beads, the move and the temperature (integrateCholesky_L with
// B = L).  A warp per bead: the bead's three rows of L against g (staged in
// shared memory as 3n floats), lanes strided over columns, a fixed shuffle
// tree per row.
__global__ void __launch_bounds__(256)
k_chol_apply_rows(JobDev* __restrict__ Jp, GridAux aux, int jsplit) {
    extern __shared__ float g[];   // [3n]
    const JobDev& J = *Jp;
    if (J.status) return;
    const int n = J.n, m = 3 * n, ld = aux.ld, tid = threadIdx.x, lane = tid & 31;
    for (int c = tid; c < n; c += 256) {
        const float4 r = aux.rf[c];
        g[3 * c] = r.x;
        g[3 * c + 1] = r.y;
        g[3 * c + 2] = r.z;
    }
    __syncthreads();
    for (int i = blockIdx.x * 8 + (tid >> 5); i < n; i += gridDim.x * 8) {
        float y[3];
#pragma unroll
        for (int rr = 0; rr < 3; ++rr) {
            const int r = 3 * i + rr;
            const float* row = aux.tensor + (size_t)r * ld;
            float s = 0.f;
            for (int c = lane; c <= r; c += 32) s = fmaf(row[c], g[c], s);
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            y[rr] = s;
        }
        if (lane == 0) {
            const float4 mi = aux.mf[i];
            float3 f = make_float3(mi.x, mi.y, mi.z);
            for (int s = 0; s < jsplit; ++s) {
                const float4 p = aux.part[(size_t)s * n + i];
                f.x += p.x; f.y += p.y; f.z += p.z;
            }
            f.x += y[0]; f.y += y[1]; f.z += y[2];
            if (J.pulling && J.flags[i] == FLAG_FIXED) f = make_float3(0.f, 0.f, 0.f);
            const float4 xc = aux.xc[i];
            const float dx = J.hOverZeta * f.x, dy = J.hOverZeta * f.y, dz = J.hOverZeta * f.z;
            J.x[i] = make_float4(xc.x + dx, xc.y + dy, xc.z + dz, xc.w);
            J.T[i] = J.T[i] + J.tempNorm * (dx * dx + dy * dy + dz * dz);
        }
    }
    (void)m;
}

}  // namespace sopb
