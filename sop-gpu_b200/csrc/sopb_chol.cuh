// sopb_chol.cuh — exact hydrodynamics (Ermak-McCammon with the Cholesky
// factor of the diffusion tensor) for jobs above 128 beads.
//
// The reference factorises the normalised RPY tensor D (3n x 3n, identity
// diagonal blocks) every step with one CTA and one thread per column, which
// limits it to n <= 128 (integrateCholesky_decompose,
// src/Integrators/bdhitea_kernel.cu:154-190).  Here D is assembled into a
// row-major matrix with a 32-float aligned leading dimension and factorised
// in place, lower triangle, by a right-looking blocked algorithm with 64-wide
// panels:
//   k_chol_potrf   the 64 x 64 diagonal block, one CTA, entries in registers;
//   k_chol_trsm    the panel below it, L_ik = A_ik L_kk^-T, a warp per row;
//   k_chol_syrk    the trailing lower triangle, A_ij -= L_ik L_jk^T, in
//                  128 x 128 output tiles with 8 x 8 FP32 register tiles.
// The trailing update does nearly all of the (3n)^3/3 flops; the panel
// kernels sit on the critical path, one panel after the other.
// The factor is refreshed every `hi_refresh` steps (an updater; 1 = every
// step, as the reference).  Every step applies it: (L g)_i by a warp per bead
// over the bead's three rows, D F by the TEA-style tiles, then the move
// (integrateCholesky_L, bdhitea_kernel.cu:303-361, with B = L).
// All reductions run in a fixed order, so results do not depend on scheduling.
#pragma once

#include "sopb_hi.cuh"

namespace sopb {

constexpr int kCholNB = 64;      // panel width
constexpr int kCholCPL = kCholNB / 32;   // panel columns per lane in the panel solve
constexpr int kCholLdp = kCholNB + 1;
constexpr int kCholTile = 128;   // trailing-update output tile
constexpr int kCholKC = 8;       // K columns staged per round

__host__ __device__ inline int chol_ld(int n) { return (3 * n + 31) & ~31; }
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

// Cholesky of the diagonal block at (k, k), nb <= 64 rows: 1024 threads,
// each holding up to 3 entries of the block's packed lower triangle in
// registers for the whole factorisation.  Column c: the owners of column c
// publish its entries (double-buffered), one barrier, then every thread
// finishes its column-c entries (L_cc = sqrt(a_cc), L_rc = a_rc / L_cc) and
// updates its entries right of c, a_rs -= a_rc a_sc / a_cc.  One barrier per
// column.  A pivot that is not positive sets the job's status.
constexpr int kPotrfThreads = 1024;
constexpr int kPotrfPer = (kCholNB * (kCholNB + 1) / 2 + kPotrfThreads - 1) / kPotrfThreads;

__global__ void __launch_bounds__(kPotrfThreads)
k_chol_potrf(JobDev* __restrict__ Jp, GridAux aux, int k) {
    __shared__ float col[2][kCholNB];
    if (Jp->status) return;
    const int m = 3 * Jp->n, ld = aux.ld, nb = min(kCholNB, m - k);
    const int tid = threadIdx.x, total = nb * (nb + 1) / 2;
    float* M = aux.tensor + (size_t)k * ld + k;
    float a[kPotrfPer];
    int rs[kPotrfPer];   // row << 8 | column
#pragma unroll
    for (int u = 0; u < kPotrfPer; ++u) {
        const int e = tid + u * kPotrfThreads;
        int r = (int)((sqrtf(8.f * (float)e + 1.f) - 1.f) * 0.5f);
        while ((r + 1) * (r + 2) / 2 <= e) ++r;
        while (r * (r + 1) / 2 > e) --r;
        const int c = e - r * (r + 1) / 2;
        rs[u] = e < total ? (r << 8 | c) : -1;
        a[u] = e < total ? M[(size_t)r * ld + c] : 0.f;
    }
    int bad = 0;
    for (int c = 0; c < nb; ++c) {
        float* cb = col[c & 1];
#pragma unroll
        for (int u = 0; u < kPotrfPer; ++u)
            if (rs[u] >= 0 && (rs[u] & 255) == c) cb[rs[u] >> 8] = a[u];
        __syncthreads();
        const float d = cb[c];
        if (!(d > 0.f)) bad = 1;
        const float inv = 1.0f / d, rsd = rsqrtf(d);
#pragma unroll
        for (int u = 0; u < kPotrfPer; ++u) {
            if (rs[u] < 0) continue;
            const int r = rs[u] >> 8, s = rs[u] & 255;
            if (s == c) a[u] = r == c ? sqrtf(d) : a[u] * rsd;
            else if (s > c) a[u] -= cb[r] * cb[s] * inv;
        }
    }
#pragma unroll
    for (int u = 0; u < kPotrfPer; ++u)
        if (rs[u] >= 0) M[(size_t)(rs[u] >> 8) * ld + (rs[u] & 255)] = a[u];
    if (bad && tid == 0) Jp->status = SOPB_ERR_HI;
}

// Panel solve below the diagonal block: row r of A[k+nb.., k..k+nb) becomes
// x with x L_kk^T = a, by forward substitution.  A warp takes four rows at
// once (independent chains, one shared read of L per column); lane l holds
// columns l and l+32 of each.  L_kk and its reciprocal diagonal are
// staged in shared memory once per CTA.
constexpr int kTrsmRows = 4;

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
    const int groups = gridDim.x * 8;
    for (int r0 = k + nb + (blockIdx.x * 8 + (tid >> 5)) * kTrsmRows; r0 < m; r0 += groups * kTrsmRows) {
        float a[kTrsmRows][kCholCPL];
#pragma unroll
        for (int q = 0; q < kTrsmRows; ++q)
#pragma unroll
            for (int u = 0; u < kCholCPL; ++u)
                a[q][u] = (r0 + q < m && lane + 32 * u < nb) ? aux.tensor[(size_t)(r0 + q) * ld + k + lane + 32 * u] : 0.f;
        for (int c = 0; c < nb; ++c) {
            const int owner = c & 31, slot = c >> 5;
            float lc[kCholCPL];
#pragma unroll
            for (int u = 0; u < kCholCPL; ++u) {
                const int cc = lane + 32 * u;
                lc[u] = (cc > c && cc < nb) ? L[cc * kCholLdp + c] : 0.f;
            }
            const float di = dinv[c];
#pragma unroll
            for (int q = 0; q < kTrsmRows; ++q) {
                float mine = a[q][0];
#pragma unroll
                for (int u = 1; u < kCholCPL; ++u)
                    if (slot == u) mine = a[q][u];
                const float x = __shfl_sync(0xffffffffu, mine, owner) * di;
#pragma unroll
                for (int u = 0; u < kCholCPL; ++u) {
                    if (lane + 32 * u == c) a[q][u] = x;
                    else a[q][u] -= x * lc[u];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kTrsmRows; ++q)
            if (r0 + q < m)
#pragma unroll
                for (int u = 0; u < kCholCPL; ++u)
                    if (lane + 32 * u < nb) aux.tensor[(size_t)(r0 + q) * ld + k + lane + 32 * u] = a[q][u];
    }
}

// Trailing update of the lower triangle right of the panel:
// A[i][j] -= sum_c P[i][c] P[j][c] over the panel's 64 columns, 128 x 128 output
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
