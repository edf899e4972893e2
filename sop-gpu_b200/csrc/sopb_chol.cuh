// sopb_chol.cuh — exact hydrodynamics (Ermak-McCammon with the Cholesky
// factor of the diffusion tensor) for jobs above 128 beads.
//
// The reference factorises the normalised RPY tensor D (3n x 3n, identity
// diagonal blocks) every step with one CTA and one thread per column, which
// limits it to n <= 128 (integrateCholesky_decompose,
// src/Integrators/bdhitea_kernel.cu:154-190).  Here D is assembled into a
// row-major matrix with a 32-float aligned leading dimension and factorised
// in place, lower triangle, in 128 x 128 tiles.  Tile columns are grouped in
// outer panels of W tile columns (W = 4 by default):
//   inside an outer panel, tile column J is brought up to date left-looking
//     (A_IJ -= sum over the panel's earlier columns, one long-K pass per
//     tile), then its diagonal tile is factorised in FP64 and the tiles
//     below it are solved;
//   after the outer panel, the trailing lower triangle is updated once with
//     K = the panel's 128 W columns: first the next outer panel's tile
//     columns (the critical path), then the rest on a second stream beside
//     the next outer panel's own work.
// Each C tile is read and written once per outer panel instead of once per
// 64 columns.  The products run on the 5th-generation tensor cores
// (tcgen05.mma kind::tf32, accumulator in TMEM) in a warp-specialised
// pipeline: eight warps load 32-column K chunks of both operands, split each
// FP32 value p into TF32 p_hi = rn(p) and p_lo = rn(p - p_hi), and store
// them in shared memory (three stages, mbarrier-tracked); one thread issues
// hi.hi + hi.lo + lo.hi per K step (the lo.lo term is below FP32 rounding),
// so the products keep FP32 accuracy; the same eight warps then read the
// accumulator from TMEM and update C in place.
// The factor is refreshed every `hi_refresh` steps (an updater; 1 = every
// step, as the reference).  Every step applies it: (L g)_i by a warp per bead
// over the bead's three rows, D F by the TEA-style tiles, then the move
// (integrateCholesky_L, bdhitea_kernel.cu:303-361, with B = L).
// All reductions run in a fixed order, so results do not depend on scheduling.
#pragma once

#include <cuda.h>

#include "sopb_hi.cuh"

namespace sopb {

constexpr int kCT = 128;                 // tile and panel width
constexpr int kCholPanelTiles = 4;       // default outer-panel width W, in tile columns

__host__ __device__ inline int chol_ld(int n) { return (3 * n + 31) & ~31; }
__host__ __device__ inline int chol_tiles(int m) { return (m + kCT - 1) / kCT; }
constexpr int kCholMaxBeads = 16384;     // 3n floats of g in shared memory

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

// Cholesky of the diagonal tile (J, J), nb <= 128 rows, and the inverse of
// its factor, in FP64 in shared memory, one CTA of 512 threads.
// Factor, by 8-wide sub-panels: every thread that solves a row factors the
// sub-panel's 8 x 8 diagonal block in registers (the same arithmetic in each
// thread, so nothing but a barrier sits between the pivots of a sub-panel;
// one FP64 rsqrt per pivot gives both L_cc = d rsqrt(d) and 1 / L_cc),
// solves its row of the sub-panel below the block (kept column-major beside
// the tile as well); then the trailing lower triangle is updated by warps in
// strips of 32 rows x 4 columns, a row per lane (eight terms per entry, in
// column order).
// Inverse X = L^-1 by recursive doubling: the sixteen 8 x 8 diagonal blocks
// by forward substitution (a thread per column), then four levels that
// merge pairs of diagonal blocks of size B = 8 .. 64, X_UT = -X_UU (L_UT
// X_TT), two triangular products per level with all 512 threads (its
// critical path is about 2B dependent FMAs per level instead of the 128 of
// a forward substitution).  X's strict lower triangle is kept transposed in
// the unused upper triangle of the tile, its diagonal beside it.  Tile loads
// are issued unconditionally (clamped addresses), 32 per thread in flight.
// Out: the factor (FP32) into the tensor's tile, X (FP32, zero above the
// diagonal and outside nb) into the inverse buffer of J's parity (aux.linv
// holds two) for the tile-column solves.  A
// pivot that is not positive sets the job's status.
constexpr int kPotrfThreads = 512;
constexpr int kPotrfW = 8;                    // sub-panel width
constexpr int kPotrfLd = kCT + 1;             // doubles
constexpr size_t kPotrfSmem = (size_t)(kCT * kPotrfLd + 2 * kCT + kPotrfW * kCT + kCT * kCT / 4) * sizeof(double);

// 1 / sqrt(d) in FP64 for d > 0: the FP32 estimate refined by two steps of
// the Newton-Raphson iteration y <- y (3 - d y^2) / 2, each of which roughly
// squares the relative error (2^-22 -> 2^-44 -> below FP64 rounding).
__device__ __forceinline__ double rsqrt_nr(double d) {
    double y = (double)rsqrtf((float)d);
    y = y * (1.5 - 0.5 * d * y * y);
    y = y * (1.5 - 0.5 * d * y * y);
    return y;
}

// rows c0 .. c0 + 7 of the sub-panel's diagonal block, factorised in registers
__device__ __forceinline__ void diag8_factor(const double* P, int c0, int w, double (&d8)[kPotrfW][kPotrfW],
                                             double (&rinv)[kPotrfW], int& bad) {
#pragma unroll
    for (int i = 0; i < kPotrfW; ++i)
#pragma unroll
        for (int jj = 0; jj < kPotrfW; ++jj)
            d8[i][jj] = (jj <= i && i < w) ? P[(c0 + i) * kPotrfLd + c0 + jj] : (i == jj ? 1.0 : 0.0);
#pragma unroll
    for (int c = 0; c < kPotrfW; ++c) {
        const double piv = d8[c][c];
        if (c < w && !(piv > 0.0)) bad = 1;
        const double rs = rsqrt_nr(piv);
        d8[c][c] = piv * rs;
        rinv[c] = rs;
#pragma unroll
        for (int i = c + 1; i < kPotrfW; ++i) d8[i][c] *= rs;
#pragma unroll
        for (int i = c + 1; i < kPotrfW; ++i)
#pragma unroll
            for (int jj = c + 1; jj <= i; ++jj) d8[i][jj] -= d8[i][c] * d8[jj][c];
    }
}

// One level of the recursive inverse: pairs of diagonal blocks of size B
// (top T, bottom U) merge as X_UT = -X_UU (L_UT X_TT), two triangular
// products.  Thread: row i of its pair's block, R = B / 8 consecutive
// columns j0 ..; the rows vary fastest within a warp, so the row-dependent
// operand is read row-parallel and the other one is a broadcast.  X[a][c],
// a > c, at P64[c][a]; X[a][a] at xd[a].  Ends with a barrier.
template <int B>
__device__ __forceinline__ void inv_level(double* P64, double* xd, double* ybuf) {
    constexpr int R = B / 8;
    const int tid = threadIdx.x, i = tid % B, j0 = ((tid / B) % 8) * R, pr = tid / (8 * B);
    const int i0 = 2 * B * pr;                 // the pair's first row / column
    double* Y = ybuf + pr * B * B;             // L_UT X_TT of this pair, row-major
    {
        double y[R];
#pragma unroll
        for (int t = 0; t < R; ++t) y[t] = 0.0;
        const double* Lr = P64 + (i0 + B + i) * kPotrfLd + i0;
        // X_TT[k][j] is zero for k < j: the first R values of k are triangular
#pragma unroll
        for (int dk = 0; dk < R; ++dk) {
            const int kk = j0 + dk;
            const double a = Lr[kk];
#pragma unroll
            for (int t = 0; t <= dk; ++t) {
                const int j = j0 + t;
                y[t] += a * (t == dk ? xd[i0 + j] : P64[(i0 + j) * kPotrfLd + i0 + kk]);
            }
        }
        for (int kk = j0 + R; kk < B; ++kk) {
            const double a = Lr[kk];
#pragma unroll
            for (int t = 0; t < R; ++t) y[t] += a * P64[(i0 + j0 + t) * kPotrfLd + i0 + kk];
        }
#pragma unroll
        for (int t = 0; t < R; ++t) Y[i * B + j0 + t] = y[t];
    }
    __syncthreads();
    {
        double x[R];
#pragma unroll
        for (int t = 0; t < R; ++t) x[t] = 0.0;
        const int a = i0 + B + i;
        for (int kk = 0; kk < i; ++kk) {
            const double xuu = P64[(i0 + B + kk) * kPotrfLd + a];
#pragma unroll
            for (int t = 0; t < R; ++t) x[t] -= xuu * Y[kk * B + j0 + t];
        }
        const double xaa = xd[a];
#pragma unroll
        for (int t = 0; t < R; ++t) P64[(i0 + j0 + t) * kPotrfLd + a] = x[t] - xaa * Y[i * B + j0 + t];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kPotrfThreads)
k_chol_potrf64(JobDev* __restrict__ Jp, GridAux aux, int J) {
    // [kCT][kPotrfLd] tile, the diagonal of X [kCT], 1 / L_cc [kCT], the
    // current sub-panel column-major [kPotrfW][kCT], inverse products
    extern __shared__ double P64[];
    __shared__ int stop;
    if (threadIdx.x == 0) stop = Jp->status;
    __syncthreads();
    if (stop) return;
    double* xd = P64 + kCT * kPotrfLd;
    double* rdiag = xd + kCT;
    double* panel = rdiag + kCT;
    double* ybuf = panel + kPotrfW * kCT;     // [kCT * kCT / 4]: the products of one inverse level
    const int m = 3 * Jp->n, ld = aux.ld, k = J * kCT, nb = min(kCT, m - k);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int kPer = kCT * kCT / kPotrfThreads;     // tile entries per thread
    float* M = aux.tensor + (size_t)k * ld + k;
    float* xout = aux.linv + (size_t)(J & 1) * kCT * kCT;   // two buffers: a solve may still read J - 1's
    {
        float v[kPer];
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int e = tid + u * kPotrfThreads, r = min(e >> 7, nb - 1), c = min(e & (kCT - 1), nb - 1);
            v[u] = M[(size_t)r * ld + c];
        }
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int e = tid + u * kPotrfThreads, r = e >> 7, c = e & (kCT - 1);
            if (r < nb && c <= r) P64[r * kPotrfLd + c] = (double)v[u];
        }
    }
    __syncthreads();
    int bad = 0;
    // ---- factor ----
    for (int c0 = 0; c0 < nb; c0 += kPotrfW) {
        const int w = min(kPotrfW, nb - c0), t0 = c0 + w;
        const int r = t0 + tid;              // this thread's row of the sub-panel below its block
        if (tid == 0 || r < nb) {
            double d8[kPotrfW][kPotrfW], rinv[kPotrfW];
            diag8_factor(P64, c0, w, d8, rinv, bad);
            if (tid == 0)
#pragma unroll
                for (int i = 0; i < kPotrfW; ++i) {
#pragma unroll
                    for (int jj = 0; jj <= i; ++jj)
                        if (i < w) P64[(c0 + i) * kPotrfLd + c0 + jj] = d8[i][jj];
                    if (i < w) rdiag[c0 + i] = rinv[i];
                }
            if (r < nb) {
                double x[kPotrfW];
#pragma unroll
                for (int c = 0; c < kPotrfW; ++c) x[c] = c < w ? P64[r * kPotrfLd + c0 + c] : 0.0;
#pragma unroll
                for (int c = 0; c < kPotrfW; ++c) {
                    double v = x[c];
#pragma unroll
                    for (int q = 0; q < c; ++q) v -= x[q] * d8[c][q];
                    x[c] = v * rinv[c];
                }
#pragma unroll
                for (int c = 0; c < kPotrfW; ++c)
                    if (c < w) {
                        P64[r * kPotrfLd + c0 + c] = x[c];
                        panel[c * kCT + r] = x[c];
                    }
            }
        }
        __syncthreads();
        // trailing lower triangle, rows and columns t0 .. nb - 1: a warp
        // takes a strip of 32 rows (a row per lane) by 4 columns at a time,
        // the sub-panel read column-major (each lane its row's value, the
        // four columns' values as broadcasts); eight terms per entry in
        // column order
        const int R = nb - t0, nstrips = (R + 31) >> 5;
        int ntasks = 0;
        for (int st = 0; st < nstrips; ++st) ntasks += (min(R, 32 * st + 32) + 3) >> 2;
        for (int task = warp; task < ntasks; task += kPotrfThreads / 32) {
            int st = 0, g = task;
            while (g >= ((min(R, 32 * st + 32) + 3) >> 2)) {
                g -= (min(R, 32 * st + 32) + 3) >> 2;
                ++st;
            }
            const int row = t0 + 32 * st + lane, q0 = t0 + 4 * g;
            double acc[4];
#pragma unroll
            for (int v = 0; v < 4; ++v)
                acc[v] = (row < nb && q0 + v <= row) ? P64[row * kPotrfLd + q0 + v] : 0.0;
#pragma unroll
            for (int c = 0; c < kPotrfW; ++c) {
                if (c < w) {
                    const double x = row < nb ? panel[c * kCT + row] : 0.0;
                    const double2 y01 = *reinterpret_cast<const double2*>(panel + c * kCT + q0);
                    const double2 y23 = *reinterpret_cast<const double2*>(panel + c * kCT + q0 + 2);
                    acc[0] -= x * y01.x;
                    acc[1] -= x * y01.y;
                    acc[2] -= x * y23.x;
                    acc[3] -= x * y23.y;
                }
            }
#pragma unroll
            for (int v = 0; v < 4; ++v)
                if (row < nb && q0 + v <= row) P64[row * kPotrfLd + q0 + v] = acc[v];
        }
        __syncthreads();
    }
    // ---- inverse X = L^-1 by recursive doubling of diagonal blocks ----
    // X[a][c], a > c, lives at P64[c][a]; X[a][a] at xd[a].  Rows and columns
    // from nb to 127 are made the identity first, so every level is full.
    for (int e = tid; e < (kCT - nb) * kCT; e += kPotrfThreads) {
        const int r = nb + e / kCT, c = e % kCT;
        if (c <= r) P64[r * kPotrfLd + c] = r == c ? 1.0 : 0.0;
        if (c == 0) rdiag[r] = 1.0;
    }
    __syncthreads();
    if (tid < kCT) {
        // the sixteen 8 x 8 diagonal blocks: thread (block, column cc)
        // solves L_bb x = e_cc by forward substitution
        const int b0 = tid & ~(kPotrfW - 1), cc = tid & (kPotrfW - 1);
        double x[kPotrfW];
#pragma unroll
        for (int r = 0; r < kPotrfW; ++r) {
            double v = r == cc ? 1.0 : 0.0;
#pragma unroll
            for (int q = 0; q < r; ++q)
                if (q >= cc) v -= P64[(b0 + r) * kPotrfLd + b0 + q] * x[q];
            x[r] = r < cc ? 0.0 : v * rdiag[b0 + r];
        }
#pragma unroll
        for (int r = 0; r < kPotrfW; ++r) {
            if (r == cc) xd[b0 + r] = x[r];
            else if (r > cc) P64[(b0 + cc) * kPotrfLd + b0 + r] = x[r];
        }
    }
    __syncthreads();
    // merge pairs of diagonal blocks of size B = 8, 16, 32, 64
    inv_level<8>(P64, xd, ybuf);
    inv_level<16>(P64, xd, ybuf);
    inv_level<32>(P64, xd, ybuf);
    inv_level<64>(P64, xd, ybuf);
    // out: the factor's rows (zero above the diagonal) and X, four columns
    // per store; a chunk that would pass column nb - 1 of the last tile
    // column (and reach the next row) is stored column by column
#pragma unroll 4
    for (int u = 0; u < kPer / 4; ++u) {
        const int e = tid + u * kPotrfThreads, r = e >> 5, c = (e & 31) * 4;
        float lv[4], xv[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int q = c + t;
            lv[t] = (r < nb && q <= r) ? (float)P64[r * kPotrfLd + q] : 0.f;
            xv[t] = (r < nb && q < nb) ? (r == q ? (float)xd[r] : (r > q ? (float)P64[q * kPotrfLd + r] : 0.f)) : 0.f;
        }
        *reinterpret_cast<float4*>(xout + r * kCT + c) = make_float4(xv[0], xv[1], xv[2], xv[3]);
        if (r < nb) {
            float* dst = M + (size_t)r * ld + c;
            if (c + 4 <= nb) {
                *reinterpret_cast<float4*>(dst) = make_float4(lv[0], lv[1], lv[2], lv[3]);
            } else {
#pragma unroll
                for (int t = 0; t < 4; ++t)
                    if (c + t < nb) dst[t] = lv[t];
            }
        }
    }
    if (bad) atomicMax(&Jp->status, SOPB_ERR_HI);
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
    const float a = J.hi_a, inv_a = 1.f / J.hi_a;
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
        auto term = [&](int kk) {
            const Blk6 d = rpy_fast(xi, xs[kk], a, inv_a);
            const float4 fq = ms[kk];
            f.x += d.xx * fq.x + d.xy * fq.y + d.xz * fq.z;
            f.y += d.xy * fq.x + d.yy * fq.y + d.yz * fq.z;
            f.z += d.xz * fq.x + d.yz * fq.y + d.zz * fq.z;
        };
        if (i < n) {
            if (t0 == blockIdx.x * kHiTile) {   // the tile of this CTA's own beads
                for (int kk = 0; kk < cnt; ++kk)
                    if (t0 + kk != i) term(kk);
            } else {
#pragma unroll 4
                for (int kk = 0; kk < cnt; ++kk) term(kk);
            }
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

// ---- tile products on the tensor cores (tcgen05, TF32 x3, TMA-fed) ---------
// One CTA per 128 x 128 output tile.  kTcUpdate: C_IJ -= sum over k in
// [k0, k1) of P_Ik P_Jk^T for lower tiles (I, J) in column order: column jc0
// from row tile i0 down, then the tile columns jc0 + 1, ... from their
// diagonal tiles down (gridDim.x tiles in all), P the factor's columns
// k0..k1 (one outer panel's, read from its TF32 hi and lo planes through
// tmap_a and tmap_b), lower entries of diagonal tiles only.  kTcSolve: C_IJ
// = A_IJ X^T for the tiles I = i0 + blockIdx.x of column J = jc0 (A from
// the tensor through tmap_a), X = L_JJ^-1 from the inverse buffer of J's
// parity (tmap_b) -- the tile-column solve as a product; the solved tile
// goes to the tensor and, split into TF32 hi and lo, to the planes of its
// outer panel (pw tile columns per panel) for the updates that read it.
// Pipeline over 32-column K chunks, three stages of 64 KB in shared memory:
//   warp 9 (one thread) loads the chunk onto the stage's "loaded" mbarrier:
//     an update four TMA tile loads (hi and lo of both operands), a solve
//     two (128 rows x 32 FP32 each, 128-byte swizzle);
//   for a solve, warps 0-7 split each value p into TF32 p_hi = rn(p),
//     written back in place, and p_lo = rn(p - p_hi), written beside it in
//     the same swizzled layout, then arrive on the stage's "converted"
//     mbarrier (an update's operands arrive split);
//   warp 8 (one thread) waits for the stage ("loaded" for an update,
//     "converted" for a solve) and issues 12 MMAs per chunk (4 K steps of 8; hi.hi into
//     one of three accumulator banks in turn, hi.lo + lo.hi into a fourth,
//     so that no bank accumulates a long K: the tensor cores' FP32
//     accumulation truncates) and commits them to the stage's "empty"
//     mbarrier, which releases it to the TMA thread; after the last chunk it
//     commits to the "done" mbarrier.
// Operands are K-major with 128-byte swizzle (descriptor layout type 2,
// 8-row groups 1024 B apart).  Every wait is bounded: on expiry the CTA stops
// loading and issuing, skips its C update and the job reports
// SOPB_ERR_TIMEOUT.  The epilogue: warp w reads TMEM lanes 32 (w mod 4),
// columns 64 (w / 4) onwards of every bank, sums the banks in FP32 and
// updates 64 consecutive entries of one C row, which an update loads into
// registers before it waits for the last MMAs.
enum { kTcUpdate = 0, kTcSolve = 1 };
constexpr int kTcKC = 32;                                 // K columns per stage (128 B of FP32)
constexpr int kTcStages = 3;
constexpr int kTcPart = kCT * kTcKC * 4;                  // 16 KB: one operand's chunk
constexpr int kTcStage = 4 * kTcPart;                     // A hi, B hi (TMA destinations), A lo, B lo
constexpr int kTcConverters = 256;                        // warps 0-7
constexpr int kTcThreads = kTcConverters + 64;            // + warp 8 (MMA) + warp 9 (TMA)
constexpr size_t kTcSmem = (size_t)kTcStages * kTcStage + 1024 + 256;
constexpr uint32_t kTcWaitLimit = 1u << 24;
constexpr uint32_t kTcTmemCols = 512;                     // four 128-column accumulator banks

__device__ __forceinline__ uint32_t tf32_rn(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// K-major shared-memory matrix descriptor, 128-byte swizzle: start address
// >> 4 [0,14), leading byte offset 16 >> 4 [16,30) (unused with swizzle),
// stride byte offset 1024 >> 4 [32,46) (8-row groups), version 1 [46,48),
// layout type 2 = SWIZZLE_128B [61,64).  K steps inside the 128-byte row
// advance the start address.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t smem_addr) {
    return (uint64_t)((smem_addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// kind::tf32, D = F32, A = B = TF32, both K-major, N = 128, M = 128
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, const volatile int* abort_flag) {
    for (uint32_t it = 0; it < kTcWaitLimit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (abort_flag && *abort_flag) return false;
    }
    return false;
}

// One TMA tile load (no multicast) of the box at column x, row y into
// shared memory, completing on mbarrier `bar`.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__global__ void __launch_bounds__(kTcThreads, 1)
k_chol_tc(const __grid_constant__ CUtensorMap tmap_a, const __grid_constant__ CUtensorMap tmap_b,
          JobDev* __restrict__ Jp, GridAux aux, int jc0, int i0, int k0, int k1, int mode, int pw) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ int stop;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) stop = Jp->status;
    __syncthreads();
    if (stop) return;
    const int m = 3 * Jp->n, ld = aux.ld, T = chol_tiles(m);
    int I, J;
    if (mode == kTcSolve) {
        J = jc0;
        I = i0 + blockIdx.x;
    } else {
        int b = blockIdx.x, top = i0;
        J = jc0;
        while (J < T - 1 && b >= T - top) {
            b -= T - top;
            ++J;
            top = J;
        }
        I = top + b;
    }
    const int r0 = I * kCT, c0 = J * kCT;
    // operand rows and the column of the first chunk: an update reads the
    // planes of the outer panel holding columns k0..k1 (rows by the panel's
    // parity, columns from the panel's first); a solve reads A_IJ from the
    // tensor and X from the inverse buffer of J's parity (rows 128 (J & 1))
    const int upan = (k0 / kCT) / pw, ubase = (upan & 1) * aux.plane_rows;
    const int a_row = mode == kTcSolve ? r0 : ubase + r0, a_col = mode == kTcSolve ? k0 : k0 - upan * pw * kCT;
    const int b_row = mode == kTcSolve ? (J & 1) * kCT : ubase + c0, b_col = mode == kTcSolve ? 0 : a_col;
    const int nk = (k1 - k0 + kTcKC - 1) / kTcKC;

    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(tc_smem);
    const uint32_t pad = (1024u - (sbase & 1023u)) & 1023u;
    unsigned char* buf = tc_smem + pad;
    const uint32_t sbuf = sbase + pad;
    const uint32_t bars = sbuf + kTcStages * kTcStage;   // loaded[s], converted[s], empty[s], done
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(buf + kTcStages * kTcStage + 8 * (3 * kTcStages + 1));
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    auto loaded = [&](int s) { return bars + 8u * (uint32_t)s; };
    auto converted = [&](int s) { return bars + 8u * (uint32_t)(kTcStages + s); };
    auto empty = [&](int s) { return bars + 8u * (uint32_t)(2 * kTcStages + s); };
    const uint32_t done_bar = bars + 8u * (uint32_t)(3 * kTcStages);

    if (warp == 8) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(tmem_slot)),
                     "r"(kTcTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < kTcStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(loaded(s)), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(converted(s)), "r"(kTcConverters));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(empty(s)), "r"(1));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(done_bar), "r"(1));
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 9) {
        if (lane == 0) {
            for (int c = 0; c < nk; ++c) {
                const int s = c % kTcStages, round = c / kTcStages;
                if (round > 0 && !mbar_wait(empty(s), (uint32_t)((round - 1) & 1), abort_flag)) {
                    *abort_flag = 1;
                    break;
                }
                const uint32_t st = sbuf + s * kTcStage;
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(loaded(s)),
                             "r"((mode == kTcSolve ? 2 : 4) * kTcPart)
                             : "memory");
                if (mode == kTcSolve) {
                    tma_load_2d(st, &tmap_a, a_col + c * kTcKC, a_row, loaded(s));
                    tma_load_2d(st + kTcPart, &tmap_b, b_col + c * kTcKC, b_row, loaded(s));
                } else {   // hi of A and B from tmap_a, lo of A and B from tmap_b
                    tma_load_2d(st, &tmap_a, a_col + c * kTcKC, a_row, loaded(s));
                    tma_load_2d(st + kTcPart, &tmap_a, b_col + c * kTcKC, b_row, loaded(s));
                    tma_load_2d(st + 2 * kTcPart, &tmap_b, a_col + c * kTcKC, a_row, loaded(s));
                    tma_load_2d(st + 3 * kTcPart, &tmap_b, b_col + c * kTcKC, b_row, loaded(s));
                }
            }
        }
    } else if (warp == 8) {
        if (lane == 0) {
            for (int c = 0; c < nk; ++c) {
                const int s = c % kTcStages, round = c / kTcStages;
                if (!mbar_wait(mode == kTcSolve ? converted(s) : loaded(s), (uint32_t)(round & 1), abort_flag)) {
                    *abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a_hi = sbuf + s * kTcStage, b_hi = a_hi + kTcPart, a_lo = a_hi + 2 * kTcPart,
                               b_lo = a_hi + 3 * kTcPart;
                const uint32_t d_hh = tmem + 128u * (uint32_t)(c % 3), d_x = tmem + 384u;
                for (int ks = 0; ks < kTcKC / 8; ++ks) {
                    const uint32_t kb = 32u * (uint32_t)ks;   // 8 TF32 = 32 bytes of each row
                    const uint64_t da[3] = {umma_desc_sw128(a_hi + kb), umma_desc_sw128(a_hi + kb),
                                            umma_desc_sw128(a_lo + kb)};
                    const uint64_t db[3] = {umma_desc_sw128(b_hi + kb), umma_desc_sw128(b_lo + kb),
                                            umma_desc_sw128(b_hi + kb)};
#pragma unroll
                    for (int t = 0; t < 3; ++t) {
                        const uint32_t dacc = t == 0 ? d_hh : d_x;
                        const uint32_t acc = t == 0 ? (c >= 3 || ks > 0 ? 1u : 0u) : (c > 0 || ks > 0 || t > 1 ? 1u : 0u);
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dacc),
                            "l"(da[t]), "l"(db[t]), "r"(kTcIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(empty(s))
                             : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(done_bar)
                         : "memory");
        }
    } else {
        // converters (a solve's operands only): item u of thread tid covers
        // row 8 g + r, 16-byte chunk q (swizzled position q ^ r); lanes r =
        // 0..7 of one chunk hit eight banks
        for (int c = 0; c < (mode == kTcSolve ? nk : 0); ++c) {
            const int s = c % kTcStages, round = c / kTcStages;
            if (!mbar_wait(loaded(s), (uint32_t)(round & 1), abort_flag)) {
                *abort_flag = 1;
                break;
            }
            unsigned char* st = buf + s * kTcStage;
#pragma unroll
            for (int u = 0; u < kCT * kTcKC / 4 / kTcConverters; ++u) {
                const int idx = tid + kTcConverters * u;
                const int r = idx & 7, q = (idx >> 3) & 7, g = idx >> 6;
                const int off = (8 * g + r) * 128 + ((q ^ r) << 4);
#pragma unroll
                for (int op = 0; op < 2; ++op) {
                    unsigned char* hi = st + op * kTcPart + off;
                    const float4 v = *reinterpret_cast<const float4*>(hi);
                    const uint32_t h0 = tf32_rn(v.x), h1 = tf32_rn(v.y), h2 = tf32_rn(v.z), h3 = tf32_rn(v.w);
                    const uint32_t l0 = tf32_rn(v.x - __uint_as_float(h0)), l1 = tf32_rn(v.y - __uint_as_float(h1)),
                                   l2 = tf32_rn(v.z - __uint_as_float(h2)), l3 = tf32_rn(v.w - __uint_as_float(h3));
                    *reinterpret_cast<uint4*>(hi) = make_uint4(h0, h1, h2, h3);
                    *reinterpret_cast<uint4*>(hi + 2 * kTcPart) = make_uint4(l0, l1, l2, l3);
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(converted(s)) : "memory");
        }
    }
    // an update's C entries of this thread, loaded while the last MMAs run
    // (C is neither operand: the K columns lie left of the tile)
    float4 cpre[16];
    if (warp < 8 && mode == kTcUpdate) {
        const int gr = r0 + 32 * (warp & 3) + lane;
        const float* src = aux.tensor + (size_t)min(gr, m - 1) * ld + c0 + 64 * (warp >> 2);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int gc = c0 + 64 * (warp >> 2) + 4 * q;
            cpre[q] = (gr < m && gc + 3 <= gr && gc + 3 < m) ? *reinterpret_cast<const float4*>(src + 4 * q)
                                                          : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    // epilogue: wait for the MMAs (every thread, bounded), then update C
    const bool done = mbar_wait(done_bar, 0u, nullptr);
    const bool ok = __syncthreads_and(done && !*abort_flag) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok && warp < 8) {
        const int hh = nk < 3 ? nk : 3;
        const int lrow = 32 * (warp & 3) + lane, gr = r0 + lrow;
        const int cmax = mode == kTcSolve ? min(m, c0 + kCT) : m;
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) {
            const int col = 64 * (warp >> 2) + 32 * ch;
            float sum[32];
            for (int bq = 0; bq <= hh; ++bq) {
                const int bk = bq < hh ? bq : 3;   // the cross-term bank last
                uint32_t v[32];
                const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(128 * bk + col);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                      "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                      "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int e = 0; e < 32; ++e) sum[e] = bq == 0 ? __uint_as_float(v[e]) : sum[e] + __uint_as_float(v[e]);
            }
            if (gr < m) {
                const int gc = c0 + col;
                float* dst = aux.tensor + (size_t)gr * ld + gc;
                if (mode == kTcSolve) {
                    // the tile's outer panel: its planes' rows and first column
                    const int span = J / pw;
                    const size_t po = (size_t)((span & 1) * aux.plane_rows + gr) * aux.plane_ld + (gc - span * pw * kCT);
                    float* ph = aux.plane_hi + po;
                    float* pl = aux.plane_lo + po;
#pragma unroll
                    for (int e = 0; e < 32; e += 4) {
                        float hv[4], lv[4];
#pragma unroll
                        for (int w = 0; w < 4; ++w) {
                            const uint32_t h = tf32_rn(sum[e + w]);
                            hv[w] = __uint_as_float(h);
                            lv[w] = __uint_as_float(tf32_rn(sum[e + w] - hv[w]));
                        }
                        if (gc + e + 3 < cmax) {
                            *reinterpret_cast<float4*>(dst + e) = make_float4(sum[e], sum[e + 1], sum[e + 2], sum[e + 3]);
                            *reinterpret_cast<float4*>(ph + e) = make_float4(hv[0], hv[1], hv[2], hv[3]);
                            *reinterpret_cast<float4*>(pl + e) = make_float4(lv[0], lv[1], lv[2], lv[3]);
                        } else {
#pragma unroll
                            for (int w = 0; w < 4; ++w)
                                if (gc + e + w < cmax) {
                                    dst[e + w] = sum[e + w];
                                    ph[e + w] = hv[w];
                                    pl[e + w] = lv[w];
                                }
                        }
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 32; e += 4) {
                        if (gc + e + 3 <= gr && gc + e + 3 < m) {
                            float4 x = cpre[8 * ch + e / 4];
                            x.x -= sum[e];
                            x.y -= sum[e + 1];
                            x.z -= sum[e + 2];
                            x.w -= sum[e + 3];
                            *reinterpret_cast<float4*>(dst + e) = x;
                        } else {
#pragma unroll
                            for (int w = 0; w < 4; ++w)
                                if (gc + e + w <= gr && gc + e + w < m) dst[e + w] -= sum[e + w];
                        }
                    }
                }
            }
        }
    }
    if (!ok && tid == 0) atomicMax(&Jp->status, SOPB_ERR_TIMEOUT);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 8) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols));
}

}  // namespace sopb
