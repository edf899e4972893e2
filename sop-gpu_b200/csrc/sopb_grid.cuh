// sopb_grid.cuh — the grid path: per-step kernels for jobs too large for one
// CTA (n > ~4096 beads, e.g. a 198k-bead capsid shell) and for jobs with
// hydrodynamic interactions, whose O(N^2) sums need the whole GPU.
//
// One step is a forces kernel followed by the integrator kernel(s).  Every
// `stride` steps the updater kernels run first; each reads the job's step
// counter on the device and returns at once when its frequency does not
// divide it, so a whole stride chunk is one fixed launch sequence that the
// host captures once in a CUDA graph and replays.  The step counter moves by
// `stride` in the chunk's last launch.
//
// Lists are index rows in global memory.  Possible pairs of large jobs come
// from a cell list (cells no smaller than pairs_threshold, 27-cell search,
// exact distance test) and each row is then sorted, so the rows equal the
// reference's brute-force rows (src/Updaters/possiblepairlist_kernel.cu:18-71)
// entry for entry.
#pragma once

#include "sopb_resident.cuh"

namespace sopb {

constexpr int kGridBlock = 256;
constexpr int kGridLpb = 4;
constexpr int kCellMax = 1 << 22;
constexpr int kSortCap = 2048;   // rows up to this length are sorted in shared memory

struct GridAux {
    // per-bead buffers of the grid path
    float4* F;           // potential forces of the current step
    // hydrodynamics (TEA / Cholesky)
    float4* rf;          // rho * g (random force)
    float4* mf;          // molecular force (+ pulling), then D F for Cholesky
    float4* xc;          // coordinate copy read during the O(N^2) sums
    float4* ci4;         // sum of squared normalised tensor rows (x,y,z), sum of entries (w)
    float* eps;          // per-bead epsilon share
    double* beta;        // beta' of the job (TEA), FP64
    float* tensor;       // Cholesky: (3n)^2 matrix, row-major
    int32_t ld;          // leading dimension of `tensor`
    float* linv;         // blocked Cholesky: inverses of the last two diagonal tiles' factors, 2 x 128 x 128
    float* plane_hi;     // blocked Cholesky: the solved tiles of the last two outer panels split into
    float* plane_lo;     //   TF32 hi and lo (bit patterns), [2 * plane_rows][plane_ld], by panel parity
    int32_t plane_rows;  // tile rows x 128
    int32_t plane_ld;    // outer-panel width in columns
    // reductions
    float4* part;        // per-CTA partial sums
    int32_t npart;
    // cell list
    int32_t* cell_count; // [kCellMax + 1]
    int32_t* cell_start; // [kCellMax + 1]
    int32_t* cell_beads; // [n]
    int32_t* bead_cell;  // [n]
    float* cell_geo;     // origin[3], size, dims[3] (as float), ncell
    int32_t use_cells;
    // near list of the Verlet rebuilds (null: none, every rebuild filters
    // the possible rows)
    int32_t* nr_j;       // [n * cap_nr] possible pairs within pairlist_cutoff + skin
    int32_t* nr_cnt;     // [n]
    float4* x_ref;       // coordinates it was built at
    int32_t* near;       // [3] drift bits, overflow, usable
    int32_t cap_nr;
};

__device__ __forceinline__ int64_t job_step(const JobDev* Jp) { return *(volatile const int64_t*)&Jp->step; }

// ---- potentials ------------------------------------------------------------
// Verlet-pair terms of bead i from its row (16-byte aligned), a 4-lane group:
// lane l takes entries 4l..4l+3 of every 16 with one 16-byte load, and the
// next block's indices are fetched before this block's four gathers, so the
// row load overlaps the coordinate gathers.
static_assert(kGridLpb == 4, "one int4 of row entries per lane");
__device__ __forceinline__ void pair_row_v4(const JobDev& J, const float4* __restrict__ xs,
                                            const int32_t* __restrict__ row, int cnt, float4 xi, int l, float3& f) {
    const float c8 = J.c8, cut2 = J.cut2;
    const int4* __restrict__ r4 = reinterpret_cast<const int4*>(row);
    int k = 4 * l;
    int4 nx = make_int4(0, 0, 0, 0);
    if (k < cnt) nx = __ldg(r4 + l);
    for (; k < cnt; k += 16) {
        const int4 cur = nx;
        if (k + 16 < cnt) nx = __ldg(r4 + (k >> 2) + 4);
        if (k + 3 < cnt) {
            const float4 x0 = xs[cur.x], x1 = xs[cur.y], x2 = xs[cur.z], x3 = xs[cur.w];
            pair_term(xi, x0, c8, cut2, f);
            pair_term(xi, x1, c8, cut2, f);
            pair_term(xi, x2, c8, cut2, f);
            pair_term(xi, x3, c8, cut2, f);
        } else {
            pair_term(xi, xs[cur.x], c8, cut2, f);
            if (k + 1 < cnt) pair_term(xi, xs[cur.y], c8, cut2, f);
            if (k + 2 < cnt) pair_term(xi, xs[cur.z], c8, cut2, f);
        }
    }
}

// All potentials of every bead at the current coordinates into aux.F; the
// tip's share accumulates per bead (indentation_kernel.cu:71-128).
// EXT: the job has a discrete surface or a pulling plane (a separate
// instantiation, so the common one keeps its register budget).
template <bool EXT>
__global__ void __launch_bounds__(kGridBlock)
k_g_forces(JobDev* __restrict__ Jp, GridAux aux) {
    __shared__ JobDev Js;
    load_job<kGridBlock>(Js, Jp);
    __syncthreads();
    const JobDev& J = Js;
    if (J.status) return;
    const int lpb = kGridLpb, l = threadIdx.x % lpb;
    const int groups = gridDim.x * (kGridBlock / lpb);
    const int g0 = blockIdx.x * (kGridBlock / lpb) + threadIdx.x / lpb;
    for (int base = 0; base < J.n; base += groups) {
        const int i = base + g0;
        const bool act = i < J.n;
        const float4 xi = J.x[act ? i : 0];
        float3 f = make_float3(0.f, 0.f, 0.f);
        if (act) {
            bonded_partial(J, global_bonded(J), J.x, i, xi, l, lpb, f);
            if ((J.cap_pl & 3) == 0) pair_row_v4(J, J.x, J.pl_j + (size_t)i * J.cap_pl, J.pl_cnt[i], xi, l, f);
            else pairs_partial(J, J.x, nullptr, nullptr, 0, i, xi, l, lpb, f);
            if (EXT && J.discrete) mica_partial(J, i, xi, l, lpb, f);
        }
        f = group_reduce(f, lpb);
        if (act && l == 0) {
            if (J.indent) {
                // read from the shared copy here, not held in registers over the pair loop
                IndentGeom ig;
                for (int c = 0; c < 3; ++c) { ig.tip[c] = J.tip[c]; ig.micaR[c] = J.micaR[c]; ig.micaN[c] = J.micaN[c]; }
                ig.tipR = J.tipR; ig.tipAp = J.tipAp; ig.tipBp = J.tipBp; ig.surfAp = J.surfAp; ig.surfBp = J.surfBp;
                float3 tf;
                if (EXT && J.discrete) tip_term(xi, ig, f, tf);
                else indentation_term(xi, ig, f, tf);
                float4 t = J.tipF[i];
                t.x += tf.x; t.y += tf.y; t.z += tf.z;
                J.tipF[i] = t;
            }
            if (EXT && J.plane) {
                const int mask = J.plane_mask[i];
                if (mask) J.plane_f[i] = plane_term(J, J.plane_displ, mask, xi, J.plane_r0[i], f);
            }
            aux.F[i] = make_float4(f.x, f.y, f.z, 0.f);
        }
    }
}

// ---- Langevin integrator (langevin_kernel.cu:17-58) -------------------------
__global__ void __launch_bounds__(kGridBlock)
k_g_langevin(JobDev* __restrict__ Jp, GridAux aux) {
    __shared__ JobDev Js;
    load_job<kGridBlock>(Js, Jp);
    __syncthreads();
    const JobDev& J = Js;
    if (J.status) return;
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < J.n; i += gridDim.x * kGridBlock) {
        float4 f4 = aux.F[i];
        float3 f = make_float3(f4.x, f4.y, f4.z);
        if (!J.minimization) {
            uint4 st = J.seeds[i];
            const float4 gg = gaussian4(st);
            J.seeds[i] = st;
            f.x += gg.x * J.var;
            f.y += gg.y * J.var;
            f.z += gg.z * J.var;
        }
        if (J.pulling) {
            const uint8_t fl = J.flags[i];
            if (fl == FLAG_FIXED) f = make_float3(0.f, 0.f, 0.f);
            if (fl == FLAG_PULLED) { f.x += J.pullF[0]; f.y += J.pullF[1]; f.z += J.pullF[2]; }
        }
        const float4 xi = J.x[i];
        const float dx = J.hOverZeta * f.x, dy = J.hOverZeta * f.y, dz = J.hOverZeta * f.z;
        J.x[i] = make_float4(xi.x + dx, xi.y + dy, xi.z + dz, xi.w);
        J.T[i] += J.tempNorm * (dx * dx + dy * dy + dz * dz);
    }
}

// ---- updaters ----------------------------------------------------------------
// Tip force: per-CTA partial sums of the per-bead accumulators (zeroed).
__global__ void __launch_bounds__(kGridBlock)
k_g_tip_partial(JobDev* __restrict__ Jp, GridAux aux) {
    __shared__ float red[kGridBlock / 32][4];
    const int64_t step = job_step(Jp);
    const JobDev& J = *Jp;
    if (!J.indent || J.status || step % J.stride != 0 || step % J.nav != 0) return;
    float3 p = make_float3(0.f, 0.f, 0.f);
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < J.n; i += gridDim.x * kGridBlock) {
        float4 t = J.tipF[i];
        p.x += t.x; p.y += t.y; p.z += t.z;
        J.tipF[i] = make_float4(0.f, 0.f, 0.f, t.w);
    }
    const float3 s = block_sum3<kGridBlock>(p, red);
    if (threadIdx.x == 0) aux.part[blockIdx.x] = make_float4(s.x, s.y, s.z, 0.f);
}

// One thread: the remaining host-side updaters of the reference in order
// (indentation tip, force-ramp cantilever, heating), reading their state
// from and writing it back to the descriptor.
__global__ void k_g_scalar_updaters(JobDev* __restrict__ Jp, GridAux aux) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    JobDev& J = *Jp;
    const int64_t step = job_step(Jp);
    if (J.status || step % J.stride != 0) return;
    StepScalars sc;
    sc.var = J.var;
    for (int c = 0; c < 3; ++c) {
        sc.pullF[c] = J.pullF[c]; sc.cant[c] = J.cant[c]; sc.chip[c] = J.chip[c];
        sc.ig.tip[c] = J.tip[c]; sc.ig.micaR[c] = J.micaR[c]; sc.ig.micaN[c] = J.micaN[c];
    }
    sc.V = J.V;
    sc.dx = J.dx;
    for (int c = 0; c < 4; ++c) sc.fav[c] = J.fav[c];
    sc.log_head = J.log_head;
    sc.plane_displ = J.plane_displ;
    sc.plane_cant = J.plane_cant;
    if (J.indent) {
        if (step == J.retraction_step) sc.V = -sc.V;
        if (step % J.nav == 0) {
            float3 s = make_float3(0.f, 0.f, 0.f);
            for (int b = 0; b < aux.npart; ++b) { float4 q = aux.part[b]; s.x += q.x; s.y += q.y; s.z += q.z; }
            tip_update(J, sc, s, step);
        }
    }
    if (J.pulling && J.ramp) {
        const float xt = __fmul_rn(J.deltax, (float)(step / J.pull_freq));
        const float4 xe = J.x[J.pulledEnd];
        const float xe3[3] = {xe.x, xe.y, xe.z};
        for (int c = 0; c < 3; ++c) sc.pullF[c] = __fmul_rn(J.k_trans, __fsub_rn(sc.cant[c], xe3[c]));
        for (int c = 0; c < 3; ++c) sc.cant[c] = __fadd_rn(J.cant0[c], __fmul_rn(xt, J.pullvec[c]));
        if (step % J.pull_freq == 0) log_pull(J, sc, xe, J.x[J.fixedEnd], step);
    }
    if (J.plane) plane_update(J, sc, J.x, step);
    if (J.heating && step % J.temp_freq == 0) {
        const float temp = __fadd_rn(J.initialT, __fmul_rn((float)(step / J.temp_freq), J.deltaT));
        sc.var = __fsqrt_rn(__fdiv_rn(__fmul_rn(__fmul_rn(2.0f, temp), J.zeta), J.h));
    }
    J.var = sc.var;
    for (int c = 0; c < 3; ++c) {
        J.pullF[c] = sc.pullF[c]; J.cant[c] = sc.cant[c]; J.chip[c] = sc.chip[c];
        J.tip[c] = sc.ig.tip[c]; J.micaR[c] = sc.ig.micaR[c];
    }
    J.V = sc.V;
    J.dx = sc.dx;
    for (int c = 0; c < 4; ++c) J.fav[c] = sc.fav[c];
    J.log_head = sc.log_head;
    J.plane_displ = sc.plane_displ;
    J.plane_cant = sc.plane_cant;
}

// Discrete surface at a tip update (after k_g_scalar_updaters moved dx):
// the surface beads follow dx when the surface moves (indentation.cu:446-455).
__global__ void __launch_bounds__(kGridBlock)
k_g_surf_move(JobDev* __restrict__ Jp) {
    const int64_t step = job_step(Jp);
    const JobDev& J = *Jp;
    if (!J.indent || !J.discrete || !J.moveSurface || J.status || step % J.stride != 0 || step % J.nav != 0) return;
    const float dx = J.dx;
    for (int q = blockIdx.x * kGridBlock + threadIdx.x; q < J.nsurf; q += gridDim.x * kGridBlock) {
        const float4 s0 = J.surf0[q];
        J.surf[q] = make_float4(__fadd_rn(s0.x, __fmul_rn(J.dir[0], dx)), __fadd_rn(s0.y, __fmul_rn(J.dir[1], dx)),
                                __fadd_rn(s0.z, __fmul_rn(J.dir[2], dx)), 0.f);
    }
}

// Every bead's surface-bead list (generateMicaList_kernel,
// indentation_kernel.cu:182-201) as a bitmask row, a warp per bead.
__global__ void __launch_bounds__(kGridBlock)
k_g_mica(JobDev* __restrict__ Jp) {
    const int64_t step = job_step(Jp);
    const JobDev& J = *Jp;
    if (!J.indent || !J.discrete || J.status || step % J.stride != 0 || step % J.nav != 0) return;
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (kGridBlock / 32);
    for (int i = blockIdx.x * (kGridBlock / 32) + (threadIdx.x >> 5); i < J.n; i += warps) {
        const float4 xi = J.x[i];
        uint32_t* row = J.mica + (size_t)i * J.Wm;
        for (int wd = 0; wd < J.Wm; ++wd) {
            const int q = 32 * wd + lane;
            const bool in = q < J.nsurf && dist2_rn(xi, J.surf[q]) < J.mica_cut2;
            const uint32_t m = __ballot_sync(0xffffffffu, in);
            if (lane == 0) row[wd] = m;
        }
    }
}

// Temperature-accumulator reset at nav (output_manager.cu:125-127).
__global__ void k_g_treset(JobDev* __restrict__ Jp) {
    const int64_t step = job_step(Jp);
    const JobDev& J = *Jp;
    if (J.status || step % J.stride != 0 || step % J.nav != 0) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < J.n; i += gridDim.x * blockDim.x) J.T[i] = 0.f;
}

// Possible pairs by brute force, one group of lanes per bead, order kept by
// ballot compaction (possiblepairlist_kernel.cu:18-71).
__global__ void __launch_bounds__(kGridBlock)
k_g_possible_brute(JobDev* __restrict__ Jp, int force) {
    __shared__ JobDev Js;
    load_job<kGridBlock>(Js, Jp);
    __syncthreads();
    const JobDev& J = Js;
    const int64_t step = J.step;
    if (J.status || (!force && (step % J.stride != 0 || step % J.pp_freq != 0))) return;
    const int lpb = 32, l = threadIdx.x % 32, n = J.n;
    int err = 0;
    for (int i = blockIdx.x * (kGridBlock / 32) + threadIdx.x / 32; i < n; i += gridDim.x * (kGridBlock / 32)) {
        const float4 xi = J.x[i];
        int32_t* row = J.pp_j + (size_t)i * J.cap_pp;
        int cnt = 0;
        const int c0 = J.cov_off[i], c1 = J.cov_off[i + 1], n0 = J.nat_off[i], n1 = J.nat_off[i + 1];
        for (int qb = 0; qb < n; qb += lpb) {
            const int q = qb + l;
            bool ok = q < n && q != i && within_cutoff(xi, J.x[q < n ? q : 0], J.pp_t);
            if (ok) {
                for (int k = c0; k < c1 && ok; ++k) ok = J.cov_j[k] != q;
                for (int k = n0; k < n1 && ok; ++k) ok = J.nat_j[k] != q;
            }
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (ok) {
                const int pos = cnt + __popc(m & ((1u << l) - 1u));
                if (pos < J.cap_pp) row[pos] = q;
                else err = SOPB_STATUS_CAPACITY;
            }
            cnt += __popc(m);
        }
        if (l == 0) J.pp_cnt[i] = cnt < J.cap_pp ? cnt : J.cap_pp;
    }
    if (err) atomicMax(&Jp->status, err);
}

// ---- cell list (large systems) ------------------------------------------------
__global__ void __launch_bounds__(kGridBlock)
k_cl_bounds(JobDev* __restrict__ Jp, GridAux aux, int force) {
    __shared__ float red[6][kGridBlock / 32];
    const JobDev& J = *Jp;
    const int64_t step = job_step(Jp);
    if (J.status || (!force && (step % J.stride != 0 || step % J.pp_freq != 0))) return;
    float mn[3] = {3.4e38f, 3.4e38f, 3.4e38f}, mx[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < J.n; i += gridDim.x * kGridBlock) {
        const float4 x = J.x[i];
        const float v[3] = {x.x, x.y, x.z};
        for (int c = 0; c < 3; ++c) { mn[c] = fminf(mn[c], v[c]); mx[c] = fmaxf(mx[c], v[c]); }
    }
    for (int o = 16; o > 0; o >>= 1)
        for (int c = 0; c < 3; ++c) {
            mn[c] = fminf(mn[c], __shfl_xor_sync(0xffffffffu, mn[c], o));
            mx[c] = fmaxf(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], o));
        }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int c = 0; c < 3; ++c) { red[c][w] = mn[c]; red[3 + c][w] = mx[c]; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < kGridBlock / 32; ++q)
            for (int c = 0; c < 3; ++c) { red[c][0] = fminf(red[c][0], red[c][q]); red[3 + c][0] = fmaxf(red[3 + c][0], red[3 + c][q]); }
        aux.part[blockIdx.x] = make_float4(red[0][0], red[1][0], red[2][0], 0.f);
        aux.part[gridDim.x + blockIdx.x] = make_float4(red[3][0], red[4][0], red[5][0], 0.f);
    }
}

// Cell geometry: cells no smaller than the threshold (slightly enlarged so a
// pair closer than the threshold is never two cells apart), at most kCellMax.
__global__ void k_cl_geometry(JobDev* __restrict__ Jp, GridAux aux, int nparts, int force) {
    const JobDev& J = *Jp;
    const int64_t step = job_step(Jp);
    if (threadIdx.x != 0 || J.status || (!force && (step % J.stride != 0 || step % J.pp_freq != 0))) return;
    float mn[3] = {3.4e38f, 3.4e38f, 3.4e38f}, mx[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    for (int b = 0; b < nparts; ++b) {
        const float4 a = aux.part[b], z = aux.part[nparts + b];
        mn[0] = fminf(mn[0], a.x); mn[1] = fminf(mn[1], a.y); mn[2] = fminf(mn[2], a.z);
        mx[0] = fmaxf(mx[0], z.x); mx[1] = fmaxf(mx[1], z.y); mx[2] = fmaxf(mx[2], z.z);
    }
    float size = J.pp_thr * 1.0001f + 1e-3f;
    int dims[3] = {1, 1, 1};
    bool ok = true;
    for (int c = 0; c < 3; ++c) ok = ok && isfinite(mn[c]) && isfinite(mx[c]) && mx[c] >= mn[c];
    if (!ok) {   // non-finite coordinates: one cell; the job is flagged after the step
        atomicMax(&Jp->status, SOPB_STATUS_NONFINITE);
        for (int c = 0; c < 3; ++c) mn[c] = 0.f;
    } else {
        for (int it = 0; it < 200; ++it) {   // bounded: each round grows the cells by 25%
            double tot = 1.0;
            for (int c = 0; c < 3; ++c) {
                dims[c] = (int)fminf(floorf((mx[c] - mn[c]) / size) + 1.0f, (float)kCellMax);
                tot *= dims[c];
            }
            if (tot <= (double)kCellMax) break;
            size *= 1.25f;
        }
        double tot = (double)dims[0] * dims[1] * dims[2];
        if (tot > (double)kCellMax) { dims[0] = dims[1] = dims[2] = 1; size = 3.0e38f; }
    }
    for (int c = 0; c < 3; ++c) aux.cell_geo[c] = mn[c];
    aux.cell_geo[3] = size;
    for (int c = 0; c < 3; ++c) aux.cell_geo[4 + c] = (float)dims[c];
    aux.cell_geo[7] = (float)(dims[0] * dims[1] * dims[2]);
}

__device__ __forceinline__ int cell_coord(float v, float o, float size, int dim) {
    int c = (int)floorf((v - o) / size);
    return c < 0 ? 0 : (c >= dim ? dim - 1 : c);
}

__global__ void __launch_bounds__(kGridBlock)
k_cl_count(JobDev* __restrict__ Jp, GridAux aux, int force) {
    const JobDev& J = *Jp;
    const int64_t step = job_step(Jp);
    if (J.status || (!force && (step % J.stride != 0 || step % J.pp_freq != 0))) return;
    const float o0 = aux.cell_geo[0], o1 = aux.cell_geo[1], o2 = aux.cell_geo[2], sz = aux.cell_geo[3];
    const int d0 = (int)aux.cell_geo[4], d1 = (int)aux.cell_geo[5], d2 = (int)aux.cell_geo[6];
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < J.n; i += gridDim.x * kGridBlock) {
        const float4 x = J.x[i];
        const int c = (cell_coord(x.z, o2, sz, d2) * d1 + cell_coord(x.y, o1, sz, d1)) * d0 + cell_coord(x.x, o0, sz, d0);
        aux.bead_cell[i] = c;
        atomicAdd(&aux.cell_count[c], 1);
    }
}

// Exclusive scan of the cell counts (one CTA); cell_count becomes the fill
// cursor.
__global__ void __launch_bounds__(1024)
k_cl_scan(JobDev* __restrict__ Jp, GridAux aux, int force) {
    __shared__ int32_t tot[1024];
    const JobDev& J = *Jp;
    const int64_t step = job_step(Jp);
    if (J.status || (!force && (step % J.stride != 0 || step % J.pp_freq != 0))) return;
    const int nc = (int)aux.cell_geo[7];
    const int per = (nc + 1023) / 1024;
    const int b0 = threadIdx.x * per, b1 = min(nc, b0 + per);
    int32_t s = 0;
    for (int c = b0; c < b1; ++c) s += aux.cell_count[c];
    tot[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int32_t run = 0;
        for (int t = 0; t < 1024; ++t) { const int32_t v = tot[t]; tot[t] = run; run += v; }
        aux.cell_start[nc] = run;
    }
    __syncthreads();
    int32_t run = tot[threadIdx.x];
    for (int c = b0; c < b1; ++c) {
        const int32_t v = aux.cell_count[c];
        aux.cell_start[c] = run;
        aux.cell_count[c] = run;
        run += v;
    }
}

__global__ void __launch_bounds__(kGridBlock)
k_cl_fill(JobDev* __restrict__ Jp, GridAux aux, int force) {
    const JobDev& J = *Jp;
    const int64_t step = job_step(Jp);
    if (J.status || (!force && (step % J.stride != 0 || step % J.pp_freq != 0))) return;
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < J.n; i += gridDim.x * kGridBlock) {
        const int pos = atomicAdd(&aux.cell_count[aux.bead_cell[i]], 1);
        aux.cell_beads[pos] = i;
    }
}

// Candidates from the 27 neighbouring cells with the exact test, appended
// unordered; one warp per bead.
__global__ void __launch_bounds__(kGridBlock)
k_cl_possible(JobDev* __restrict__ Jp, GridAux aux, int force) {
    __shared__ JobDev Js;
    load_job<kGridBlock>(Js, Jp);
    __syncthreads();
    const JobDev& J = Js;
    const int64_t step = J.step;
    if (J.status || (!force && (step % J.stride != 0 || step % J.pp_freq != 0))) return;
    const int l = threadIdx.x & 31;
    const float o0 = aux.cell_geo[0], o1 = aux.cell_geo[1], o2 = aux.cell_geo[2], sz = aux.cell_geo[3];
    const int d0 = (int)aux.cell_geo[4], d1 = (int)aux.cell_geo[5], d2 = (int)aux.cell_geo[6];
    int err = 0;
    for (int i = blockIdx.x * (kGridBlock / 32) + threadIdx.x / 32; i < J.n; i += gridDim.x * (kGridBlock / 32)) {
        const float4 xi = J.x[i];
        const int cx = cell_coord(xi.x, o0, sz, d0), cy = cell_coord(xi.y, o1, sz, d1), cz = cell_coord(xi.z, o2, sz, d2);
        const int c0 = J.cov_off[i], c1 = J.cov_off[i + 1], n0 = J.nat_off[i], n1 = J.nat_off[i + 1];
        int32_t* row = J.pp_j + (size_t)i * J.cap_pp;
        int cnt = 0;
        for (int dz = -1; dz <= 1; ++dz) {
            const int z = cz + dz;
            if (z < 0 || z >= d2) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int y = cy + dy;
                if (y < 0 || y >= d1) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = cx + dx;
                    if (x < 0 || x >= d0) continue;
                    const int c = (z * d1 + y) * d0 + x;
                    const int s0 = aux.cell_start[c], s1 = aux.cell_start[c + 1];
                    for (int kb = s0; kb < s1; kb += 32) {
                        const int k = kb + l;
                        int q = -1;
                        bool ok = false;
                        if (k < s1) {
                            q = aux.cell_beads[k];
                            ok = q != i && within_cutoff(xi, J.x[q], J.pp_t);
                            for (int t = c0; t < c1 && ok; ++t) ok = J.cov_j[t] != q;
                            for (int t = n0; t < n1 && ok; ++t) ok = J.nat_j[t] != q;
                        }
                        const unsigned m = __ballot_sync(0xffffffffu, ok);
                        if (ok) {
                            const int pos = cnt + __popc(m & ((1u << l) - 1u));
                            if (pos < J.cap_pp) row[pos] = q;
                            else err = SOPB_STATUS_CAPACITY;
                        }
                        cnt += __popc(m);
                    }
                }
            }
        }
        if (l == 0) J.pp_cnt[i] = cnt < J.cap_pp ? cnt : J.cap_pp;
    }
    if (err) atomicMax(&Jp->status, err);
}

// Sorts every possible-pairs row ascending (the brute-force order); one warp
// per row, bitonic sort in shared memory for rows up to kSortCap entries,
// odd-even transposition in place for longer rows.
__global__ void __launch_bounds__(128)
k_cl_sort_rows(JobDev* __restrict__ Jp, int force) {
    extern __shared__ int32_t buf[];   // 4 warps x kSortCap
    const JobDev& J = *Jp;
    const int64_t step = job_step(Jp);
    if (J.status || (!force && (step % J.stride != 0 || step % J.pp_freq != 0))) return;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    int32_t* sb = buf + w * kSortCap;
    for (int i = blockIdx.x * 4 + w; i < J.n; i += gridDim.x * 4) {
        const int cnt = J.pp_cnt[i];
        int32_t* row = J.pp_j + (size_t)i * J.cap_pp;
        if (cnt <= kSortCap) {
            int len = 1;
            while (len < cnt) len <<= 1;
            for (int k = l; k < len; k += 32) sb[k] = k < cnt ? row[k] : 0x7fffffff;
            __syncwarp();
            for (int size = 2; size <= len; size <<= 1) {
                for (int stride = size >> 1; stride > 0; stride >>= 1) {
                    for (int k = l; k < len; k += 32) {
                        const int p = k ^ stride;
                        if (p > k) {
                            const bool up = (k & size) == 0;
                            const int32_t a = sb[k], b = sb[p];
                            if ((a > b) == up) { sb[k] = b; sb[p] = a; }
                        }
                    }
                    __syncwarp();
                }
            }
            for (int k = l; k < cnt; k += 32) row[k] = sb[k];
            __syncwarp();
        } else {
            for (int pass = 0; pass < cnt; ++pass) {
                for (int k = 2 * l + (pass & 1); k + 1 < cnt; k += 64) {
                    const int32_t a = row[k], b = row[k + 1];
                    if (a > b) { row[k] = b; row[k + 1] = a; }
                }
                __syncwarp();
            }
        }
    }
}

// Near list of the Verlet rebuilds (a grid job with a skin): the possible
// pairs within pairlist_cutoff + skin, in the order of the possible rows,
// with the coordinates it was built at.  While no bead has moved more than
// half the skin since, every possible pair now closer than pairlist_cutoff
// was closer than pairlist_cutoff + skin then, so filtering the near rows with
// the same exact test gives the rows a filter of the possible rows gives.
// aux.near: [0] largest squared drift (float bits), [1] a near row overflowed
// its capacity, [2] the near list is usable.  [0] and [1] are cleared by
// k_g_near_commit, the last kernel of every rebuild.
__device__ __forceinline__ bool verlet_from_near(const JobDev& J, const GridAux& a, int64_t step, int force) {
    return !force && a.nr_j && a.near[2] && step % J.pp_freq != 0 && __int_as_float(a.near[0]) < J.drift2;
}

// Largest squared displacement since the near list was built, at a Verlet
// step that may reuse it.
__global__ void __launch_bounds__(kGridBlock)
k_g_drift(JobDev* __restrict__ Jp, GridAux a) {
    const JobDev& J = *Jp;
    const int64_t step = job_step(Jp);
    if (J.status || step % J.stride != 0 || step % J.pairs_freq != 0 || step % J.pp_freq == 0 || !a.near[2]) return;
    float d2 = 0.f;
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < J.n; i += gridDim.x * kGridBlock) {
        const float e = dist2_rn(a.x_ref[i], J.x[i]);
        d2 = fmaxf(d2, isfinite(e) ? e : INFINITY);   // fmaxf drops a NaN: count it as an infinite drift
    }
    for (int o = 16; o > 0; o >>= 1) d2 = fmaxf(d2, __shfl_xor_sync(0xffffffffu, d2, o));
    if ((threadIdx.x & 31) == 0 && d2 > 0.f) atomicMax(&a.near[0], __float_as_int(d2));   // non-negative floats order as ints
}

// Exclusive prefix sum over the warp's lanes, and the warp total.
__device__ __forceinline__ int warp_excl_scan(int v, int l, int& total) {
    int s = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, s, o);
        if (l >= o) s += t;
    }
    total = __shfl_sync(0xffffffffu, s, 31);
    return s - v;
}

// Appends the candidates of `hits` (bit u: q[u]) to a row in entry order:
// lane l holds entries 4l..4l+3 of the warp's 128, so its first hit goes
// after the hits of the lanes below.  Returns 1 when the row overflowed.
__device__ __forceinline__ int append_hits(int32_t* row, int cap, int& cnt, unsigned hits, const int (&q)[4], int l) {
    int total;
    int pos = cnt + warp_excl_scan(__popc(hits), l, total);
    int over = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u)
        if ((hits >> u) & 1u) {
            if (pos < cap) row[pos] = q[u];
            else over = 1;
            ++pos;
        }
    cnt += total;
    return over;
}

// Verlet rows (pairlist_kernel.cu:33-76), order kept: a warp per bead, each
// lane testing four consecutive candidates of the warp's 128 (four gathers in
// flight), an order-preserving warp scan placing the hits.  From the near
// rows when they are usable and no bead drifted too far; else from the
// possible rows, renewing the near rows at the current coordinates.
__global__ void __launch_bounds__(kGridBlock)
k_g_verlet(JobDev* __restrict__ Jp, GridAux a, int force) {
    __shared__ JobDev Js;
    load_job<kGridBlock>(Js, Jp);
    __syncthreads();
    const JobDev& J = Js;
    const int64_t step = J.step;
    if (J.status || (!force && (step % J.stride != 0 || step % J.pairs_freq != 0))) return;
    const bool near = verlet_from_near(J, a, step, force);
    const bool renew = !near && a.nr_j;
    const int srcw = near ? a.cap_nr : J.cap_pp;
    const bool vec = (srcw & 3) == 0;      // 16-byte aligned source rows
    const int l = threadIdx.x & 31;
    int err = 0, over = 0;
    for (int i = blockIdx.x * (kGridBlock / 32) + threadIdx.x / 32; i < J.n; i += gridDim.x * (kGridBlock / 32)) {
        const float4 xi = J.x[i];
        const int src = near ? a.nr_cnt[i] : J.pp_cnt[i];
        const int32_t* srow = near ? a.nr_j + (size_t)i * a.cap_nr : J.pp_j + (size_t)i * J.cap_pp;
        int32_t* row = J.pl_j + (size_t)i * J.cap_pl;
        int32_t* nrow = renew ? a.nr_j + (size_t)i * a.cap_nr : nullptr;
        int cnt = 0, ncnt = 0;
        for (int kb = 0; kb < src; kb += 128) {
            const int k = kb + 4 * l;
            int q[4] = {0, 0, 0, 0};
            if (vec && k + 3 < src) {
                const int4 v = __ldg(reinterpret_cast<const int4*>(srow + k));
                q[0] = v.x; q[1] = v.y; q[2] = v.z; q[3] = v.w;
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (k + u < src) q[u] = __ldg(srow + k + u);
            }
            float r2[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) r2[u] = k + u < src ? dist2_rn(xi, J.x[q[u]]) : 0.f;
            unsigned hits = 0u, nhits = 0u;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const bool cand = k + u < src;
                if (cand && r2[u] < J.pl_t) hits |= 1u << u;
                if (cand && r2[u] < J.nr_t) nhits |= 1u << u;
            }
            if (append_hits(row, J.cap_pl, cnt, hits, q, l)) err = SOPB_STATUS_CAPACITY;
            if (renew) over |= append_hits(nrow, a.cap_nr, ncnt, nhits, q, l);
        }
        if (l == 0) {
            J.pl_cnt[i] = cnt < J.cap_pl ? cnt : J.cap_pl;
            if (renew) {
                a.nr_cnt[i] = ncnt < a.cap_nr ? ncnt : a.cap_nr;
                a.x_ref[i] = xi;
            }
        }
    }
    if (err) atomicMax(&Jp->status, err);
    if (over) atomicOr(&a.near[1], 1);
}

// Closes a rebuild: the near list is usable after a rebuild that renewed it
// without overflow, unusable after new possible pairs without a Verlet
// rebuild, unchanged otherwise.  possible/verlet: an explicit rebuild (-1 in
// a run, where the step decides).
__global__ void k_g_near_commit(JobDev* __restrict__ Jp, GridAux a, int possible, int verlet) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || !a.nr_j) return;
    const JobDev& J = *Jp;
    const int64_t step = job_step(Jp);
    const bool force = verlet >= 0;
    if (!force) {
        const bool at = step % J.stride == 0;
        possible = at && step % J.pp_freq == 0;
        verlet = at && step % J.pairs_freq == 0;
    }
    if (J.status) a.near[2] = 0;
    else if (verlet && !verlet_from_near(J, a, step, force ? 1 : 0)) a.near[2] = a.near[1] ? 0 : 1;
    else if (possible && !verlet) a.near[2] = 0;
    a.near[0] = 0;
    a.near[1] = 0;
}

// Advances the job's step counter by `by` (last launch of a chunk) and flags
// non-finite coordinates.
__global__ void k_g_advance(JobDev* __restrict__ Jp, int by) {
    if (threadIdx.x == 0 && blockIdx.x == 0) Jp->step += by;
}

__global__ void __launch_bounds__(kGridBlock)
k_g_check_finite(JobDev* __restrict__ Jp) {
    const JobDev& J = *Jp;
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < J.n; i += gridDim.x * kGridBlock) {
        const float4 v = J.x[i];
        if (!(isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) atomicMax(&Jp->status, SOPB_STATUS_NONFINITE);
    }
}

}  // namespace sopb
