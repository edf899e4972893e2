// sopb_resident.cuh — the replica-resident Langevin step kernel.
//
// One CTA owns one job for a whole launch of `nsteps` steps.  Coordinates
// (ping-pong), Hybrid Taus states and the temperature accumulator sit in
// shared memory; every updater of the reference loop (indentation tip,
// force-ramp cantilever, possible pairs, temperature reset, Verlet pairlist,
// heating) runs inside the kernel at its step, so there is no host round
// trip and no launch per step (the reference launches 4-6 kernels per step
// and copies all coordinates to the host every `stride` steps for pulling,
// src/Potentials/pulling.cu:152-165).
//
// Neighbour lists.  The possible-pairs list of a job is a bitmask over its
// beads (n <= 2048, so at most 64 words a row), with bonded/native
// exclusions as a precomputed bitmask.  The Verlet list is a set of
// bead-major, order-preserving index rows in global memory (the reference's
// slot-major d_pairs transposed), cached in shared memory as a compact CSR
// copy (u16 byte offsets of the partners, in the lanes' order) as far as it
// fits the job's cache.  Both
// are rebuilt a warp per bead with ballots, so partners are always visited
// in increasing j, the reference's list order.
//
// One step is two phases.  Forces: a group of `lpb` lanes (a power of two
// <= 32, four by default) takes beads from a shared counter, strides
// over the bead's covalent, native and Verlet entries, combines the partial
// forces with xor-shuffles and stores the bead's force in shared memory.
// Integration: one thread per bead draws the noise and moves the bead.  A
// bead's arithmetic depends only on the job and on lpb, never on which group
// computed it or on the list's location (cache or global rows).
#pragma once

#include "sopb_device.cuh"

namespace sopb {

constexpr int kMaxResidentBeads = 2048;
// shared memory per bead that every resident job holds: coordinates, RNG
// state and force (16 B each), temperature and the cache's row offset
// (4 B each), pulling flag (1 B)
constexpr int kResidentSmemPerBead = 57;

// Shared-memory layout of a resident launch (byte offsets, 16-B aligned
// arrays).  The coordinates are followed by one far-away dummy bead that the
// padding of the Verlet cache points at.  The bonded maps (covalent and
// native CSR with parameters) are copied in when `bonded` is set; the Verlet
// cache takes `cache` u16 entries.
struct ResidentLayout {
    size_t x, F, sd, nat_par, Ts, off, cov_off, nat_off, cov_r0, cov_j, nat_j, flags, nbr, total;
};
__host__ __device__ inline size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }
__host__ __device__ inline ResidentLayout resident_layout(int n, int ncov, int nnat, int bonded, int cache) {
    ResidentLayout L;
    const size_t b = bonded ? 1 : 0;
    size_t o = 0;
    L.x = o;        o = align16(o + (size_t)(n + 1) * 16);
    L.F = o;        o = align16(o + (size_t)n * 16);
    L.sd = o;       o = align16(o + (size_t)n * 16);
    L.nat_par = o;  o = align16(o + b * (size_t)nnat * 8);
    L.Ts = o;       o = align16(o + (size_t)n * 4);
    L.off = o;      o = align16(o + (size_t)(n + 4) * 4);
    L.cov_off = o;  o = align16(o + b * (size_t)(n + 1) * 4);
    L.nat_off = o;  o = align16(o + b * (size_t)(n + 1) * 4);
    L.cov_r0 = o;   o = align16(o + b * (size_t)ncov * 4);
    L.cov_j = o;    o = align16(o + b * (size_t)ncov * 4);
    L.nat_j = o;    o = align16(o + b * (size_t)nnat * 4);
    L.flags = o;    o = align16(o + (size_t)n);
    L.nbr = o;      o = align16(o + (size_t)cache * 2);
    L.total = o;
    return L;
}

// Where a job's covalent and native maps are read from during a launch.
struct BondedView {
    const int32_t* cov_off;
    const int32_t* cov_j;
    const float* cov_r0;
    const int32_t* nat_off;
    const int32_t* nat_j;
    const float2* nat_par;
};

struct StepScalars {
    float var;
    float pullF[3];
    float cant[3];
    IndentGeom ig;
    float chip[3];
    float V, dx;
    float fav[4];
    int32_t err;
    int32_t nr_valid;   // the job's near list is usable (written back at the end)
    uint32_t log_head;  // event-log rows appended (written back at the end)
    float plane_displ, plane_cant;   // pulling plane (written back at the end)
};

// Cooperative copy of a job descriptor into shared memory (read by every
// thread as a broadcast instead of per-thread register copies).
template <int BLOCK>
__device__ __forceinline__ void load_job(JobDev& dst, const JobDev* src) {
    static_assert(sizeof(JobDev) % 4 == 0, "JobDev must be word sized");
    const int* s = reinterpret_cast<const int*>(src);
    int* d = reinterpret_cast<int*>(&dst);
    for (int w = threadIdx.x; w < (int)(sizeof(JobDev) / 4); w += BLOCK) d[w] = s[w];
}

__device__ __forceinline__ unsigned group_mask(int lpb) {
    return lpb == 32 ? 0xffffffffu : ((1u << lpb) - 1u);
}

// Sum over a lane group; `mask` names the lanes taking part (the whole
// warp, or just the group when groups of a warp run independently).
__device__ __forceinline__ float3 group_reduce(float3 f, int lpb, unsigned mask = 0xffffffffu) {
    for (int o = lpb >> 1; o > 0; o >>= 1) {
        f.x += __shfl_xor_sync(mask, f.x, o);
        f.y += __shfl_xor_sync(mask, f.y, o);
        f.z += __shfl_xor_sync(mask, f.z, o);
    }
    return f;
}

__device__ __forceinline__ int group_sum(int v, int lpb) {
    for (int o = lpb >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Covalent then native terms of bead i, strided over the group's lanes
// (the reference sums its kernels' contributions in this order,
// src/gsop.cu:80-85).  The maps are read-only for a launch.
__device__ __forceinline__ void bonded_partial(const JobDev& J, const BondedView& B, const float4* __restrict__ xs,
                                               int i, float4 xi, int l, int lpb, float3& f) {
    const int c0 = B.cov_off[i], c1 = B.cov_off[i + 1];
    const int n0 = B.nat_off[i], n1 = B.nat_off[i + 1];
    for (int k = c0 + l; k < c1; k += lpb) fene_term(xi, xs[B.cov_j[k]], B.cov_r0[k], J.ks, J.R2, f);
    for (int k = n0 + l; k < n1; k += lpb) native_term(xi, xs[B.nat_j[k]], B.nat_par[k], f);
}

__device__ __forceinline__ BondedView global_bonded(const JobDev& J) {
    return BondedView{J.cov_off, J.cov_j, J.cov_r0, J.nat_off, J.nat_j, J.nat_par};
}

// Verlet-pair terms of bead i from its global row (a bead beyond the
// shared-memory cache, or forces outside a step), lane l of lpb taking
// entries l, l+lpb, ... in that order.  Four entries are fetched per
// iteration so four gathers are in flight; the per-lane summation order is
// unchanged.
template <typename Idx>
__device__ __forceinline__ void pair_run(const JobDev& J, const float4* __restrict__ xs, const Idx* __restrict__ r,
                                         int cnt, float4 xi, int l, int lpb, float3& f) {
    const float c8 = J.c8, cut2 = J.cut2;
    int k = l;
    for (; k + 3 * lpb < cnt; k += 4 * lpb) {
        const int j0 = r[k], j1 = r[k + lpb], j2 = r[k + 2 * lpb], j3 = r[k + 3 * lpb];
        const float4 x0 = xs[j0], x1 = xs[j1], x2 = xs[j2], x3 = xs[j3];
        pair_term(xi, x0, c8, cut2, f);
        pair_term(xi, x1, c8, cut2, f);
        pair_term(xi, x2, c8, cut2, f);
        pair_term(xi, x3, c8, cut2, f);
    }
    for (; k < cnt; k += lpb) pair_term(xi, xs[r[k]], c8, cut2, f);
}

// The shared-memory cache of a bead's Verlet row: byte offsets of the
// partners' coordinates (16 j), the row padded to a multiple of four entries
// with the offset of the dummy bead, whose term is exactly zero (+0 or -0
// added).  Each full block of 4 lpb entries is stored lane by lane -- the
// four entries l, l + lpb, l + 2 lpb, l + 3 lpb of lane l side by side -- so
// that one 8-byte load fetches them; the rest of the row is in row order.
// A lane therefore visits the same entries in the same order as pair_run.
__device__ __forceinline__ int cache_pos(int k, int full, int lg) {
    if (k >= full) return k;
    const int blk = 4 << lg, b = k & ~(blk - 1), w = k & (blk - 1);
    return b + 4 * (w & ((1 << lg) - 1)) + (w >> lg);
}
__device__ __forceinline__ void pair_run_cached(const JobDev& J, const float4* __restrict__ xs,
                                                const uint16_t* __restrict__ rb, int cnt, float4 xi, int l, int lpb,
                                                float3& f) {
    const float c8 = J.c8, cut2 = J.cut2;
    const char* xb = reinterpret_cast<const char*>(xs);
    const int blk = 4 * lpb, full = cnt - cnt % blk;
    const uint16_t* q = rb + 4 * l;
    for (int b = 0; b < full; b += blk, q += blk) {
        const uint2 o = *reinterpret_cast<const uint2*>(q);
        const float4 x0 = *reinterpret_cast<const float4*>(xb + (o.x & 0xffffu));
        const float4 x1 = *reinterpret_cast<const float4*>(xb + (o.x >> 16));
        const float4 x2 = *reinterpret_cast<const float4*>(xb + (o.y & 0xffffu));
        const float4 x3 = *reinterpret_cast<const float4*>(xb + (o.y >> 16));
        pair_term(xi, x0, c8, cut2, f);
        pair_term(xi, x1, c8, cut2, f);
        pair_term(xi, x2, c8, cut2, f);
        pair_term(xi, x3, c8, cut2, f);
    }
    for (int k = full + l; k < cnt; k += lpb) pair_term(xi, *reinterpret_cast<const float4*>(xb + rb[k]), c8, cut2, f);
}

__device__ __forceinline__ void pairs_partial(const JobDev& J, const float4* __restrict__ xs, const int32_t* off,
                                              const uint16_t* nbr, int cap, int i, float4 xi, int l, int lpb,
                                              float3& f) {
    const int k1 = off ? off[i + 1] : 0x7fffffff;
    if (k1 <= cap) {
        const int k0 = off[i];
        pair_run_cached(J, xs, nbr + k0, k1 - k0, xi, l, lpb, f);
    } else {
        pair_run(J, xs, J.pl_j + (size_t)i * J.cap_pl, J.pl_cnt[i], xi, l, lpb, f);
    }
}

// generate_possiblepairs (src/Updaters/possiblepairlist_kernel.cu:18-71):
// every q of the job with |r| < pairs_threshold that is neither i nor a
// covalent or native partner, as a bitmask row.  A warp takes one bead;
// lane b tests bead 32w+b of word w and a ballot forms the word.  More than
// max_possiblePairs sets err (the reference writes past its rows there).
template <int BLOCK>
__device__ void build_possible(const JobDev& J, const float4* __restrict__ xs, int& err) {
    const int n = J.n, W = J.W, lane = threadIdx.x & 31;
    for (int i = threadIdx.x >> 5; i < n; i += BLOCK / 32) {
        const float4 xi = xs[i];
        const uint32_t* ex = J.ex_mask + (size_t)i * W;
        uint32_t* row = J.pp_mask + (size_t)i * W;
        int cnt = 0;
        for (int w = 0; w < W; ++w) {
            const int q = 32 * w + lane;
            const bool ok = q < n && within_cutoff(xi, xs[q < n ? q : 0], J.pp_t);
            const uint32_t bits = __ballot_sync(0xffffffffu, ok) & ~__ldg(&ex[w]);
            if (lane == 0) row[w] = bits;
            cnt += __popc(bits);
        }
        if (lane == 0 && cnt > J.max_pp) err = SOPB_STATUS_CAPACITY;
    }
}

// generate_pairs (src/Updaters/pairlist_kernel.cu:33-76): the possible pairs
// with |r| < pairlist_cutoff, in increasing j (the reference's order), as
// index rows.  A warp takes one bead: the possible-pairs words are held two
// per lane (W <= 64), lane b tests candidate 32w+b and a ballot places the
// hits.  The same scan writes the near list -- the possible pairs within
// pairlist_cutoff + skin, also in increasing j -- for the cheaper rebuilds
// that follow (build_verlet_near).  A Verlet row longer than its capacity
// sets err; a near row longer than its capacity sets *near_over.
template <int BLOCK>
__device__ void build_verlet(const JobDev& J, const float4* __restrict__ xs, int& err, int* near_over) {
    static_assert(kMaxResidentBeads <= 64 * 32, "two mask words per lane");
    const int n = J.n, W = J.W, lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    for (int i = threadIdx.x >> 5; i < n; i += BLOCK / 32) {
        const float4 xi = xs[i];
        const uint32_t* pm = J.pp_mask + (size_t)i * W;
        const uint32_t m0 = lane < W ? pm[lane] : 0u;
        const uint32_t m1 = lane + 32 < W ? pm[lane + 32] : 0u;
        int32_t* row = J.pl_j + (size_t)i * J.cap_pl;
        uint16_t* nrow = J.nr_j + (size_t)i * J.cap_nr;
        int cnt = 0, ncnt = 0;
        for (int w = 0; w < W; ++w) {
            const uint32_t m = __shfl_sync(0xffffffffu, w < 32 ? m0 : m1, w & 31);
            const int q = 32 * w + lane;
            const bool cand = ((m >> lane) & 1u) && q < n;
            const float r2 = cand ? dist2_rn(xi, xs[q]) : 0.f;
            const bool ok = cand && r2 < J.pl_t, nok = cand && r2 < J.nr_t;
            const uint32_t hit = __ballot_sync(0xffffffffu, ok), nhit = __ballot_sync(0xffffffffu, nok);
            if (ok) {
                const int pos = cnt + __popc(hit & below);
                if (pos < J.cap_pl) row[pos] = q;
            }
            if (nok) {
                const int pos = ncnt + __popc(nhit & below);
                if (pos < J.cap_nr) nrow[pos] = (uint16_t)q;
            }
            cnt += __popc(hit);
            ncnt += __popc(nhit);
        }
        if (lane == 0) {
            if (cnt > J.cap_pl) err = SOPB_STATUS_CAPACITY;
            J.pl_cnt[i] = cnt < J.cap_pl ? cnt : J.cap_pl;
            if (ncnt > J.cap_nr) atomicOr(near_over, 1);
            J.nr_cnt[i] = ncnt < J.cap_nr ? ncnt : J.cap_nr;
        }
    }
}

// The Verlet list from the near list: while no bead moved more than half the
// skin since the near list was built, every pair now closer than
// pairlist_cutoff was closer than pairlist_cutoff + skin then, so filtering
// the near rows (increasing j) with the same exact test gives the same rows
// as the full scan.  A warp per bead, lanes over 32 near entries at a time;
// the warp fetches its next bead's row length while it filters the current
// row, and a row's first kNearAhead x 32 entries are loaded before any of
// them is tested, so a row costs one global round trip, not one per 32.
constexpr int kNearAhead = 8;
template <int BLOCK>
__device__ void build_verlet_near(const JobDev& J, const float4* __restrict__ xs, int& err) {
    const int n = J.n, lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    int i = threadIdx.x >> 5;
    int ncnt = i < n ? J.nr_cnt[i] : 0;
    for (; i < n; i += BLOCK / 32) {
        const int ncnt_next = i + BLOCK / 32 < n ? J.nr_cnt[i + BLOCK / 32] : 0;
        const uint16_t* nrow = J.nr_j + (size_t)i * J.cap_nr;
        int q[kNearAhead];
#pragma unroll
        for (int u = 0; u < kNearAhead; ++u) {
            const int k = 32 * u + lane;
            q[u] = k < ncnt ? nrow[k] : 0;
        }
        const float4 xi = xs[i];
        int32_t* row = J.pl_j + (size_t)i * J.cap_pl;
        int cnt = 0;
        auto take = [&](int k, int qk) {
            const bool ok = k < ncnt && within_cutoff(xi, xs[qk], J.pl_t);
            const uint32_t hit = __ballot_sync(0xffffffffu, ok);
            if (ok) {
                const int pos = cnt + __popc(hit & below);
                if (pos < J.cap_pl) row[pos] = qk;
            }
            cnt += __popc(hit);
        };
#pragma unroll
        for (int u = 0; u < kNearAhead; ++u)
            if (32 * u < ncnt) take(32 * u + lane, q[u]);   // the same for the warp's lanes
        for (int kb = 32 * kNearAhead; kb < ncnt; kb += 32) {
            const int k = kb + lane;
            take(k, k < ncnt ? nrow[k] : 0);
        }
        if (lane == 0) {
            if (cnt > J.cap_pl) err = SOPB_STATUS_CAPACITY;
            J.pl_cnt[i] = cnt < J.cap_pl ? cnt : J.cap_pl;
        }
        ncnt = ncnt_next;
    }
}

// Verlet rebuild of a resident job: from the near list when it is valid and
// no bead drifted more than half the skin from where it was built, else a
// full scan that also rebuilds the near list at the current coordinates.
template <int BLOCK>
__device__ void rebuild_verlet(const JobDev& J, const float4* __restrict__ xs, int& valid, bool possible_changed,
                               int& err) {
    __shared__ int drift_bits, near_over;
    const int tid = threadIdx.x, n = J.n;
    if (tid == 0) {
        drift_bits = 0;
        near_over = 0;
    }
    __syncthreads();
    if (valid && !possible_changed) {
        float d2 = 0.f;
        for (int i = tid; i < n; i += BLOCK) {
            const float e = dist2_rn(J.x_ref[i], xs[i]);
            d2 = fmaxf(d2, isfinite(e) ? e : INFINITY);   // fmaxf drops a NaN: count it as an infinite drift
        }
        if (d2 > 0.f) atomicMax(&drift_bits, __float_as_int(d2));   // non-negative floats order as ints
    }
    __syncthreads();
    if (valid && !possible_changed && __int_as_float(drift_bits) < J.drift2) {
        build_verlet_near<BLOCK>(J, xs, err);
        return;
    }
    build_verlet<BLOCK>(J, xs, err, &near_over);
    for (int i = tid; i < n; i += BLOCK) J.x_ref[i] = xs[i];
    __syncthreads();
    valid = near_over || !(J.drift2 > 0.f) ? 0 : 1;   // drift2 0: the job keeps no near list
}

// Deterministic CTA sum of a float3 (fixed tree for a given BLOCK).
template <int BLOCK>
__device__ float3 block_sum3(float3 v, float (*red)[4]) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        v.z += __shfl_xor_sync(0xffffffffu, v.z, o);
    }
    __syncthreads();
    if (lane == 0) { red[w][0] = v.x; red[w][1] = v.y; red[w][2] = v.z; }
    __syncthreads();
    float3 s = make_float3(0.f, 0.f, 0.f);
    for (int q = 0; q < BLOCK / 32; ++q) { s.x += red[q][0]; s.y += red[q][1]; s.z += red[q][2]; }
    return s;
}

// Appends one row to the job's event-log ring (sopb_log_row layout: kind,
// pad, step, twelve floats); the host drains it with sopb_job_log.
__device__ __forceinline__ void log_row(const JobDev& J, uint32_t& head, int32_t kind, int64_t step, const float* v) {
    if (J.log_cap <= 0) return;
    float* r = J.log + (size_t)(head & (uint32_t)(J.log_cap - 1)) * 16;
    reinterpret_cast<int32_t*>(r)[0] = kind;
    reinterpret_cast<int32_t*>(r)[1] = 0;
    *reinterpret_cast<int64_t*>(r + 2) = step;
    for (int k = 0; k < 12; ++k) r[4 + k] = v[k];
    ++head;
}

// PullingPotential::savePullingData (src/Potentials/pulling.cu:167-190): the
// end-to-end distance, its projection and the applied force along the pull
// vector, from the coordinates of this step and the force just computed.
// The reference evaluates it on the host (IEEE, no contraction).
__device__ __noinline__ void log_pull(const JobDev& J, StepScalars& sc, float4 xp, float4 xf, int64_t step) {
    const float e[3] = {__fsub_rn(xp.x, xf.x), __fsub_rn(xp.y, xf.y), __fsub_rn(xp.z, xf.z)};
    auto dot3 = [](const float* a, const float* b) {
        return __fadd_rn(__fadd_rn(__fmul_rn(a[0], b[0]), __fmul_rn(a[1], b[1])), __fmul_rn(a[2], b[2]));
    };
    const float v[12] = {__fsqrt_rn(dot3(e, e)), dot3(e, J.pullvec), dot3(sc.pullF, J.pullvec),
                         sc.pullF[0], sc.pullF[1], sc.pullF[2], 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    log_row(J, sc.log_head, SOPB_LOG_PULL, step, v);
}

// PullingPlaneUpdater::update (src/Potentials/pulling_plane.cu:183-258), run
// every stride by one thread: the cantilever moves by deltax per update
// period; the plane takes one overdamped step of update-period length under
// the cantilever spring and the beads' springs, summed in bead order from
// the forces of the last step; every output period one log line with the
// distance between the centroids of the fixed and the pulled beads.  Host
// arithmetic in the reference: explicit _rn operations.
__device__ __noinline__ void plane_update(const JobDev& J, StepScalars& sc, const float4* __restrict__ xs, int64_t step) {
    const float xt = __fdiv_rn(__fmul_rn(J.plane_deltax, (float)step), (float)J.plane_freq);
    sc.plane_cant = xt;
    const int32_t* fixed = J.plane_idx;
    const int32_t* pulled = J.plane_idx + J.nplane_fixed;
    float ext = 0.0f;
    for (int k = 0; k < J.nplane_pulled; ++k) ext = __fadd_rn(ext, J.plane_f[pulled[k]]);
    const float cant = __fmul_rn(__fsub_rn(xt, sc.plane_displ), J.plane_kscant);
    const float mult = __fdiv_rn(__fmul_rn((float)J.plane_freq, J.h), J.plane_zeta);
    sc.plane_displ = __fadd_rn(sc.plane_displ, __fmul_rn(mult, __fsub_rn(cant, ext)));
    if (step % J.plane_ofreq == 0) {
        float cf[3] = {0.f, 0.f, 0.f}, cp[3] = {0.f, 0.f, 0.f};
        for (int k = 0; k < J.nplane_fixed; ++k) {
            const float4 q = xs[fixed[k]];
            cf[0] = __fadd_rn(cf[0], q.x); cf[1] = __fadd_rn(cf[1], q.y); cf[2] = __fadd_rn(cf[2], q.z);
        }
        for (int k = 0; k < J.nplane_pulled; ++k) {
            const float4 q = xs[pulled[k]];
            cp[0] = __fadd_rn(cp[0], q.x); cp[1] = __fadd_rn(cp[1], q.y); cp[2] = __fadd_rn(cp[2], q.z);
        }
        float d[3];
        for (int c = 0; c < 3; ++c)
            d[c] = __fsub_rn(__fdiv_rn(cp[c], (float)J.nplane_pulled), __fdiv_rn(cf[c], (float)J.nplane_fixed));
        const float e2e = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(d[0], d[0]), __fmul_rn(d[1], d[1])), __fmul_rn(d[2], d[2])));
        const float v[12] = {sc.plane_displ, xt, cant, ext, e2e, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        log_row(J, sc.log_head, SOPB_LOG_PLANE, step, v);
    }
}

// Discrete surface at a tip update: the surface beads follow dx when the
// surface moves (IndentationTipUpdater::update, indentation.cu:446-455), then
// every bead's list of surface beads within the cutoff is rebuilt
// (generateMicaList_kernel, indentation_kernel.cu:182-201) as a bitmask row,
// a warp per bead and a ballot per 32 surface beads.
template <int BLOCK>
__device__ void build_mica(const JobDev& J, const float4* __restrict__ xs, float dx) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (J.moveSurface) {
        for (int q = tid; q < J.nsurf; q += BLOCK) {
            const float4 s0 = J.surf0[q];
            J.surf[q] = make_float4(__fadd_rn(s0.x, __fmul_rn(J.dir[0], dx)), __fadd_rn(s0.y, __fmul_rn(J.dir[1], dx)),
                                    __fadd_rn(s0.z, __fmul_rn(J.dir[2], dx)), 0.f);
        }
        __syncthreads();
    }
    for (int i = w; i < J.n; i += BLOCK / 32) {
        const float4 xi = xs[i];
        uint32_t* row = J.mica + (size_t)i * J.Wm;
        for (int wd = 0; wd < J.Wm; ++wd) {
            const int q = 32 * wd + lane;
            bool in = false;
            if (q < J.nsurf) in = dist2_rn(xi, J.surf[q]) < J.mica_cut2;
            const uint32_t m = __ballot_sync(0xffffffffu, in);
            if (lane == 0) row[wd] = m;
        }
    }
    __syncthreads();
}

// IndentationTipUpdater::update (src/Potentials/indentation.cu:414-550) for
// the continuous surface, run by thread 0 after the CTA summed the tip force.
// Host-side arithmetic of the reference is IEEE without contraction, hence
// the explicit _rn intrinsics.
__device__ __noinline__ void tip_update(const JobDev& J, StepScalars& sc, float3 fsum, int64_t step) {
    const float inv = (float)J.nav;
    float f[3] = {__fdiv_rn(fsum.x, inv), __fdiv_rn(fsum.y, inv), __fdiv_rn(fsum.z, inv)};
    sc.dx = __fmul_rn((float)(step / J.nav), sc.V);
    if (J.moveSurface) {
        for (int c = 0; c < 3; ++c) sc.ig.micaR[c] = __fadd_rn(J.micaR0[c], __fmul_rn(J.dir[c], sc.dx));
    } else {
        for (int c = 0; c < 3; ++c) sc.chip[c] = __fadd_rn(J.chip0[c], __fmul_rn(J.dir[c], sc.dx));
    }
    float df[3], dr[3];
    for (int c = 0; c < 3; ++c) dr[c] = __fsub_rn(sc.chip[c], sc.ig.tip[c]);
    const float drw = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dr[0], dr[0]), __fmul_rn(dr[1], dr[1])), __fmul_rn(dr[2], dr[2])));
    for (int c = 0; c < 3; ++c) df[c] = __fadd_rn(-f[c], __fmul_rn(dr[c], J.cantKs));
    const float mult = __fdiv_rn(__fmul_rn(J.h, (float)J.nav), J.tipZeta);
    if (J.fixTrans) {
        float ct = __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(mult, df[0]), J.dir[0]), __fmul_rn(__fmul_rn(mult, df[1]), J.dir[1])),
                             __fmul_rn(__fmul_rn(mult, df[2]), J.dir[2]));
        for (int c = 0; c < 3; ++c) sc.ig.tip[c] = __fadd_rn(sc.ig.tip[c], __fmul_rn(ct, J.dir[c]));
    } else {
        for (int c = 0; c < 3; ++c) sc.ig.tip[c] = __fadd_rn(sc.ig.tip[c], __fmul_rn(mult, df[c]));
    }
    sc.fav[0] = f[0];
    sc.fav[1] = f[1];
    sc.fav[2] = f[2];
    sc.fav[3] = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(f[0], f[0]), __fmul_rn(f[1], f[1])), __fmul_rn(f[2], f[2])));
    const float v[12] = {sc.fav[0], sc.fav[1], sc.fav[2], sc.fav[3], drw, sc.dx,
                         sc.ig.tip[0], sc.ig.tip[1], sc.ig.tip[2], sc.chip[0], sc.chip[1], sc.chip[2]};
    log_row(J, sc.log_head, SOPB_LOG_TIP, step, v);
}

// Shared-memory cache of the Verlet rows as compact CSR: offsets by a CTA
// scan of the row counts padded to multiples of four, then for every bead
// whose padded row ends within `cap` entries its row in the layout that
// pair_run_cached reads (the beads after it read their global rows).  The
// dummy bead sits at index n, far from every bead.
template <int BLOCK>
__device__ void fill_cache(const JobDev& J, int32_t* off, uint16_t* nbr, int cap, int* tot_smem, float4* xs) {
    const int n = J.n, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int per = (n + BLOCK - 1) / BLOCK, b0 = tid * per, b1 = min(n, b0 + per);
    auto padded = [](int c) { return (c + 3) & ~3; };
    if (tid == 0) xs[n] = make_float4(1.0e18f, 1.0e18f, 1.0e18f, 0.f);
    int s = 0;
    for (int i = b0; i < b1; ++i) s += padded(J.pl_cnt[i]);
    int incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    __shared__ int wsum[BLOCK / 32];
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (tid == 0) {
        int run = 0;
        for (int q = 0; q < BLOCK / 32; ++q) { const int v = wsum[q]; wsum[q] = run; run += v; }
        *tot_smem = run;
    }
    __syncthreads();
    int run = wsum[w] + incl - s;
    for (int i = b0; i < b1; ++i) { off[i] = run; run += padded(J.pl_cnt[i]); }
    if (tid == 0) off[n] = *tot_smem;
    __syncthreads();
    {
        const int lg = __ffs(J.lpb) - 1, blk = 4 << lg;
        const uint16_t dummy = (uint16_t)(16 * n);
        // two beads per warp at a time, so that the loads of both rows are
        // in flight together
        for (int i = w; i < n; i += 2 * (BLOCK / 32)) {
            const int i2 = i + BLOCK / 32;
            const bool in1 = off[i + 1] <= cap, in2 = i2 < n && off[i2 + 1] <= cap;
            const int k0 = off[i], pc = in1 ? off[i + 1] - k0 : 0, cnt = in1 ? J.pl_cnt[i] : 0;
            const int k02 = in2 ? off[i2] : 0, pc2 = in2 ? off[i2 + 1] - k02 : 0, cnt2 = in2 ? J.pl_cnt[i2] : 0;
            const int full = pc - pc % blk, full2 = pc2 - pc2 % blk;
            const int32_t* r = J.pl_j + (size_t)i * J.cap_pl;
            const int32_t* r2 = J.pl_j + (size_t)(in2 ? i2 : i) * J.cap_pl;
            for (int kb = 0; kb < max(pc, pc2); kb += 128) {
                int v[4], v2[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = kb + 32 * u + lane;
                    v[u] = k < cnt ? r[k] : n;
                    v2[u] = k < cnt2 ? r2[k] : n;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = kb + 32 * u + lane;
                    if (k < pc) nbr[k0 + cache_pos(k, full, lg)] = k < cnt ? (uint16_t)(16 * v[u]) : dummy;
                    if (k < pc2) nbr[k02 + cache_pos(k, full2, lg)] = k < cnt2 ? (uint16_t)(16 * v2[u]) : dummy;
                }
            }
            if (!in2) break;   // every later bead ends beyond the cache as well
        }
    }
    __syncthreads();
}

// The updaters of one `stride` boundary in the reference order
// (creation order in src/gsop.cu:80-101; loop in src/gsop.cu:129-133).
// Returns 1 when the Verlet list was rebuilt.
template <int BLOCK>
__device__ __noinline__ int run_updaters(const JobDev& J, StepScalars& sc, const float4* __restrict__ xs, float* Ts,
                                         float (*red)[4], int64_t step, int& err) {
    const int tid = threadIdx.x, n = J.n;
    if (J.indent) {
        if (tid == 0 && step == J.retraction_step) sc.V = -sc.V;
        if (step % J.nav == 0) {
            float3 p = make_float3(0.f, 0.f, 0.f);
            for (int i = tid; i < n; i += BLOCK) {
                float4 t = J.tipF[i];
                p.x += t.x; p.y += t.y; p.z += t.z;
                J.tipF[i] = make_float4(0.f, 0.f, 0.f, t.w);
            }
            const float3 s = block_sum3<BLOCK>(p, red);
            if (tid == 0) tip_update(J, sc, s, step);
            if (J.discrete) {
                __syncthreads();
                build_mica<BLOCK>(J, xs, sc.dx);
            }
        }
    }
    if (J.pulling && J.ramp && tid == 0) {
        // PullingUpdater::update runs every stride (src/Potentials/pulling.cu:198-204)
        const float xt = __fmul_rn(J.deltax, (float)(step / J.pull_freq));
        const float4 xe = xs[J.pulledEnd];
        const float xe3[3] = {xe.x, xe.y, xe.z};
        for (int c = 0; c < 3; ++c) sc.pullF[c] = __fmul_rn(J.k_trans, __fsub_rn(sc.cant[c], xe3[c]));
        for (int c = 0; c < 3; ++c) sc.cant[c] = __fadd_rn(J.cant0[c], __fmul_rn(xt, J.pullvec[c]));
        if (step % J.pull_freq == 0) log_pull(J, sc, xe, xs[J.fixedEnd], step);
    }
    if (J.plane && tid == 0) plane_update(J, sc, xs, step);
    const bool pp = step % J.pp_freq == 0;
    if (pp) build_possible<BLOCK>(J, xs, err);
    if (step % J.nav == 0)
        for (int i = tid; i < n; i += BLOCK) Ts[i] = 0.0f;   // output_manager.cu:125-127
    const bool verlet = step % J.pairs_freq == 0;
    if (pp && !verlet && tid == 0) sc.nr_valid = 0;   // the near list no longer matches the possible pairs
    if (verlet) {
        if (pp) __syncthreads();
        int valid = sc.nr_valid;
        rebuild_verlet<BLOCK>(J, xs, valid, pp, err);
        if (tid == 0) sc.nr_valid = valid;
    }
    if (J.heating && tid == 0 && step % J.temp_freq == 0) {
        // TemperatureUpdater (src/Integrators/langevin.cu:129-135, 44-48)
        const float temp = __fadd_rn(J.initialT, __fmul_rn((float)(step / J.temp_freq), J.deltaT));
        sc.var = __fsqrt_rn(__fdiv_rn(__fmul_rn(__fmul_rn(2.0f, temp), J.zeta), J.h));
    }
    __syncthreads();
    return verlet ? 1 : 0;
}

// Shared-memory bytes of a job's resident launch.
__host__ __device__ inline size_t resident_smem_bytes(const JobDev& J) {
    return resident_layout(J.n, J.ncov, J.nnat, J.bsm, J.lcache).total;
}

// Register cap of 64 per thread: 1024 threads of resident CTAs per SM.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK)
k_resident_steps(JobDev* __restrict__ jobs, const int32_t* __restrict__ ids, const int64_t* __restrict__ steps) {
    const int64_t nsteps = steps[blockIdx.x];   // each job its own number of steps
    JobDev* Jp = &jobs[ids[blockIdx.x]];
    __shared__ JobDev Js;
    load_job<BLOCK>(Js, Jp);
    __syncthreads();
    const JobDev& J = Js;
    if (J.status != 0) return;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ StepScalars sc;
    __shared__ float red[BLOCK / 32][4];
    __shared__ int list_total;
    const int n = J.n, tid = threadIdx.x;
    const ResidentLayout lay = resident_layout(n, J.ncov, J.nnat, J.bsm, J.lcache);
    float4* xs = reinterpret_cast<float4*>(smem + lay.x);
    float4* F = reinterpret_cast<float4*>(smem + lay.F);
    uint4* sd = reinterpret_cast<uint4*>(smem + lay.sd);
    float* Ts = reinterpret_cast<float*>(smem + lay.Ts);
    int32_t* off = reinterpret_cast<int32_t*>(smem + lay.off);
    uint8_t* fl = smem + lay.flags;
    uint16_t* nbr = reinterpret_cast<uint16_t*>(smem + lay.nbr);
    for (int i = tid; i < n; i += BLOCK) {
        xs[i] = J.x[i];
        sd[i] = J.seeds[i];
        Ts[i] = J.T[i];
        fl[i] = J.pulling ? J.flags[i] : (uint8_t)FLAG_FREE;
    }
    __shared__ BondedView Bs;                 // read as a broadcast, not held in registers
    if (tid == 0) Bs = global_bonded(J);
    if (J.bsm) {
        // the maps are constant for the launch: one copy into shared memory
        int32_t* co = reinterpret_cast<int32_t*>(smem + lay.cov_off);
        int32_t* no = reinterpret_cast<int32_t*>(smem + lay.nat_off);
        int32_t* cj = reinterpret_cast<int32_t*>(smem + lay.cov_j);
        float* cr = reinterpret_cast<float*>(smem + lay.cov_r0);
        int32_t* nj = reinterpret_cast<int32_t*>(smem + lay.nat_j);
        float2* np = reinterpret_cast<float2*>(smem + lay.nat_par);
        for (int i = tid; i <= n; i += BLOCK) { co[i] = J.cov_off[i]; no[i] = J.nat_off[i]; }
        for (int k = tid; k < J.ncov; k += BLOCK) { cj[k] = J.cov_j[k]; cr[k] = J.cov_r0[k]; }
        for (int k = tid; k < J.nnat; k += BLOCK) { nj[k] = J.nat_j[k]; np[k] = J.nat_par[k]; }
        if (tid == 0) Bs = BondedView{co, cj, cr, no, nj, np};
    }
    const BondedView& B = Bs;
    if (tid == 0) {
        sc.var = J.var;
        for (int c = 0; c < 3; ++c) {
            sc.pullF[c] = J.pullF[c];
            sc.cant[c] = J.cant[c];
            sc.ig.tip[c] = J.tip[c];
            sc.ig.micaR[c] = J.micaR[c];
            sc.ig.micaN[c] = J.micaN[c];
            sc.chip[c] = J.chip[c];
        }
        sc.ig.tipR = J.tipR; sc.ig.tipAp = J.tipAp; sc.ig.tipBp = J.tipBp;
        sc.ig.surfAp = J.surfAp; sc.ig.surfBp = J.surfBp;
        sc.V = J.V; sc.dx = J.dx;
        for (int c = 0; c < 4; ++c) sc.fav[c] = J.fav[c];
        sc.err = 0;
        sc.nr_valid = J.nr_valid;
        sc.log_head = J.log_head;
        sc.plane_displ = J.plane_displ;
        sc.plane_cant = J.plane_cant;
    }
    __syncthreads();
    const int cap = J.lcache;
    fill_cache<BLOCK>(J, off, nbr, cap, &list_total, xs);

    const int lpb = J.lpb, l = tid % lpb;
    int err = 0;
    int64_t step = J.step;
    int phase = (int)(step % J.stride);       // steps since the last updater pass
    __shared__ int next_bead[2];              // per-step bead counters, double buffered
    if (tid < 2) next_bead[tid] = 0;
    __syncthreads();
    for (int64_t s = 0; s < nsteps; ++s, ++step) {
        if (phase == 0 && run_updaters<BLOCK>(J, sc, xs, Ts, red, step, err))
            fill_cache<BLOCK>(J, off, nbr, cap, &list_total, xs);
        if (++phase == J.stride) phase = 0;
        int* counter = &next_bead[s & 1];
        // forces: each warp claims one bead per lane group from a shared
        // counter, the groups sum their beads' terms and reduce by shuffles
        for (;;) {
            int base = 0;
            if ((tid & 31) == 0) base = atomicAdd(counter, 32 / lpb);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= n) break;
            const int i = base + (tid & 31) / lpb;
            float3 f = make_float3(0.f, 0.f, 0.f);
            const float4 xi = xs[i < n ? i : 0];
            if (i < n) {
                bonded_partial(J, B, xs, i, xi, l, lpb, f);
                pairs_partial(J, xs, off, nbr, cap, i, xi, l, lpb, f);
                if (J.discrete) mica_partial(J, i, xi, l, lpb, f);
            }
            f = group_reduce(f, lpb);
            if (l == 0 && i < n) {
                if (J.indent) {
                    float3 tf;
                    if (J.discrete) tip_term(xi, sc.ig, f, tf);
                    else indentation_term(xi, sc.ig, f, tf);
                    float4 t = J.tipF[i];
                    t.x += tf.x; t.y += tf.y; t.z += tf.z;
                    J.tipF[i] = t;
                }
                if (J.plane) {
                    const int mask = J.plane_mask[i];
                    if (mask) J.plane_f[i] = plane_term(J, sc.plane_displ, mask, xi, J.plane_r0[i], f);
                }
                F[i] = make_float4(f.x, f.y, f.z, 0.f);
            }
        }
        __syncthreads();
        if (tid == 0) *counter = 0;          // reused two steps from now, after a barrier
        // integrateLangevin_kernel (src/Integrators/langevin_kernel.cu:17-58),
        // one thread per bead, in place: every force of the step is final
        const float var = sc.var;
        for (int i = tid; i < n; i += BLOCK) {
            const float4 f4 = F[i];
            float3 f = make_float3(f4.x, f4.y, f4.z);
            if (!J.minimization) {
                uint4 st = sd[i];
                const float4 gg = gaussian4(st);
                sd[i] = st;
                f.x += gg.x * var;
                f.y += gg.y * var;
                f.z += gg.z * var;
            }
            const uint8_t fi = fl[i];
            if (fi == FLAG_FIXED) f = make_float3(0.f, 0.f, 0.f);
            if (fi == FLAG_PULLED) { f.x += sc.pullF[0]; f.y += sc.pullF[1]; f.z += sc.pullF[2]; }
            const float4 xi = xs[i];
            const float dx = J.hOverZeta * f.x, dy = J.hOverZeta * f.y, dz = J.hOverZeta * f.z;
            xs[i] = make_float4(xi.x + dx, xi.y + dy, xi.z + dz, xi.w);
            Ts[i] += J.tempNorm * (dx * dx + dy * dy + dz * dz);
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += BLOCK) {
        const float4 v = xs[i];
        if (!(isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) err = SOPB_STATUS_NONFINITE;
        J.x[i] = v;
        J.seeds[i] = sd[i];
        J.T[i] = Ts[i];
    }
    if (err) atomicMax(&sc.err, err);
    __syncthreads();
    if (tid == 0) {
        Jp->step = step;
        Jp->var = sc.var;
        for (int c = 0; c < 3; ++c) {
            Jp->pullF[c] = sc.pullF[c];
            Jp->cant[c] = sc.cant[c];
            Jp->tip[c] = sc.ig.tip[c];
            Jp->micaR[c] = sc.ig.micaR[c];
            Jp->chip[c] = sc.chip[c];
        }
        Jp->V = sc.V;
        Jp->dx = sc.dx;
        for (int c = 0; c < 4; ++c) Jp->fav[c] = sc.fav[c];
        Jp->nr_valid = sc.nr_valid;
        Jp->log_head = sc.log_head;
        Jp->plane_displ = sc.plane_displ;
        Jp->plane_cant = sc.plane_cant;
        if (sc.err) Jp->status = sc.err;
    }
}

// Potential forces only (SOPPotential::compute of every potential, no
// integrator) at the job's current coordinates and Verlet rows, with the
// step kernel's lane split; does not touch the tip accumulator.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1)
k_forces_only(const JobDev* __restrict__ jobs, const int32_t* __restrict__ ids, float4* __restrict__ out) {
    __shared__ JobDev Js;
    load_job<BLOCK>(Js, &jobs[ids[blockIdx.x]]);
    __syncthreads();
    const JobDev& J = Js;
    const int n = J.n, tid = threadIdx.x, lpb = J.lpb, g = tid / lpb, l = tid % lpb, ng = BLOCK / lpb;
    IndentGeom ig;
    for (int c = 0; c < 3; ++c) { ig.tip[c] = J.tip[c]; ig.micaR[c] = J.micaR[c]; ig.micaN[c] = J.micaN[c]; }
    ig.tipR = J.tipR; ig.tipAp = J.tipAp; ig.tipBp = J.tipBp; ig.surfAp = J.surfAp; ig.surfBp = J.surfBp;
    for (int base = 0; base < n; base += ng) {
        const int i = base + g;
        const bool act = i < n;
        const float4 xi = J.x[act ? i : 0];
        float3 f = make_float3(0.f, 0.f, 0.f);
        if (act) {
            bonded_partial(J, global_bonded(J), J.x, i, xi, l, lpb, f);
            pairs_partial(J, J.x, nullptr, nullptr, 0, i, xi, l, lpb, f);
            if (J.discrete) mica_partial(J, i, xi, l, lpb, f);
        }
        f = group_reduce(f, lpb);
        if (act && l == 0) {
            if (J.indent) {
                float3 tf;
                if (J.discrete) tip_term(xi, ig, f, tf);
                else indentation_term(xi, ig, f, tf);
            }
            if (J.plane) {
                const int mask = J.plane_mask[i];
                if (mask) plane_term(J, J.plane_displ, mask, xi, J.plane_r0[i], f);
            }
            out[i] = make_float4(f.x, f.y, f.z, 0.f);
        }
    }
}

// Rebuilds the possible-pairs and/or Verlet lists now, without the step gate.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1)
k_rebuild_lists(JobDev* __restrict__ jobs, const int32_t* __restrict__ ids, int possible, int verlet) {
    JobDev* Jp = &jobs[ids[blockIdx.x]];
    __shared__ JobDev Js;
    load_job<BLOCK>(Js, Jp);
    const JobDev& J = Js;
    __shared__ int errs;
    if (threadIdx.x == 0) errs = 0;
    __syncthreads();
    int err = 0;
    if (possible) build_possible<BLOCK>(J, J.x, err);
    __syncthreads();
    if (verlet) {
        int valid = 0;                      // a full scan, which also renews the near list
        rebuild_verlet<BLOCK>(J, J.x, valid, true, err);
        if (threadIdx.x == 0) Jp->nr_valid = valid;
    } else if (possible && threadIdx.x == 0) {
        Jp->nr_valid = 0;                   // the near list no longer matches the possible pairs
    }
    if (err) atomicMax(&errs, err);
    __syncthreads();
    if (threadIdx.x == 0 && errs) Jp->status = errs;
}

}  // namespace sopb
