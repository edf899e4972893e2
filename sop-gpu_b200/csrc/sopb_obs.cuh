// sopb_obs.cuh — on-device observables of a job, the quantities the
// reference's output manager writes to its .dat files every `outputtiming`
// steps (src/Updaters/output_manager.cu:73-222): the kinetic temperature
// averaged over beads and the nav window, the FENE, native and repulsive
// energies (covalentEnergy_kernel, nativeEnergy_kernel, pairsEnergy_kernel:
// per bead in FP32, summed in FP64 and halved, SOPPotential::sumEnergies,
// src/gsop.cu:255-271), the intact native contacts and the radius of
// gyration.  The reference copies coordinates and per-bead arrays to the
// host for these; here a grid of CTAs reduces them per job on the device in
// a fixed order (per-CTA FP64 partials, then one CTA over the partials).
#pragma once

#include "sopb_resident.cuh"

namespace sopb {

constexpr int kObsBlock = 256;
constexpr int kObsTerms = 9;   // FENE, native, repulsive, T, contacts, sum x, y, z, |r|^2

// Deterministic CTA sum of kObsTerms doubles (fixed shuffle tree, then warps
// in order); the result is valid in thread 0.
__device__ __forceinline__ void obs_block_sum(double (&v)[kObsTerms], double (*red)[kObsTerms]) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kObsTerms; ++q)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < kObsTerms; ++q) red[w][q] = v[q];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int ww = 1; ww < kObsBlock / 32; ++ww)
#pragma unroll
            for (int q = 0; q < kObsTerms; ++q) v[q] += red[ww][q];
}

__global__ void __launch_bounds__(kObsBlock)
k_obs_partial(const JobDev* __restrict__ Jp, double* __restrict__ part) {
    __shared__ JobDev Js;
    __shared__ double red[kObsBlock / 32][kObsTerms];
    load_job<kObsBlock>(Js, Jp);
    __syncthreads();
    const JobDev& J = Js;
    const float R_limit = sqrtf(J.R2), el_a6 = -J.c8 / 6.0f;
    double v[kObsTerms] = {};
    for (int i = blockIdx.x * kObsBlock + threadIdx.x; i < J.n; i += gridDim.x * kObsBlock) {
        const float4 xi = J.x[i];
        float fene = 0.f, nat = 0.f, pairs = 0.f;
        int contacts = 0;
        for (int k = J.cov_off[i]; k < J.cov_off[i + 1]; ++k) {
            const float4 xj = J.x[J.cov_j[k]];
            const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            const float d = sqrtf(dx * dx + dy * dy + dz * dz) - J.cov_r0[k];
            fene -= 0.5f * J.ks * J.R2 * logf(1.0f - d * d / J.R2);
        }
        for (int k = J.nat_off[i]; k < J.nat_off[i + 1]; ++k) {
            const int j = J.nat_j[k];
            const float4 xj = J.x[j];
            const float2 par = J.nat_par[k];   // (r0^2, -12 eh / r0^2)
            const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            const float r2 = dx * dx + dy * dy + dz * dz;
            const float s = par.x / r2, p6 = s * s * s;
            nat += (-par.y * par.x / 12.0f) * (p6 * p6 - 2.0f * p6);
            if (j > i) {   // each contact once (computeNativeCounts, output_manager.cu:166-186)
                const float dr = sqrtf(r2);
                if (dr < J.rlb || fabsf(sqrtf(par.x) - dr) <= R_limit) ++contacts;
            }
        }
        const int32_t* row = J.pl_j + (size_t)i * J.cap_pl;
        for (int k = 0; k < J.pl_cnt[i]; ++k) {
            const float4 xj = J.x[row[k]];
            const float dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < J.cut2) {
                const float s = 1.0f / r2;
                pairs += el_a6 * s * s * s;
            }
        }
        v[0] += fene;
        v[1] += nat;
        v[2] += pairs;
        v[3] += J.T[i];
        v[4] += contacts;
        v[5] += xi.x;
        v[6] += xi.y;
        v[7] += xi.z;
        v[8] += (double)xi.x * xi.x + (double)xi.y * xi.y + (double)xi.z * xi.z;
    }
    obs_block_sum(v, red);
    if (threadIdx.x == 0)
        for (int q = 0; q < kObsTerms; ++q) part[(size_t)blockIdx.x * kObsTerms + q] = v[q];
}

// out: T, E_fene, E_native, E_pairs, E_total, native contacts, Rg, TEA epsilon
__global__ void __launch_bounds__(32)
k_obs_final(const JobDev* __restrict__ Jp, const double* __restrict__ part, int nparts, double* __restrict__ out) {
    if (threadIdx.x != 0) return;
    const JobDev& J = *Jp;
    double v[kObsTerms] = {};
    for (int b = 0; b < nparts; ++b)
        for (int q = 0; q < kObsTerms; ++q) v[q] += part[(size_t)b * kObsTerms + q];
    const double n = (double)J.n;
    out[0] = v[3] / (n * (double)J.nav);
    out[1] = 0.5 * v[0];
    out[2] = 0.5 * v[1];
    out[3] = 0.5 * v[2];
    out[4] = out[1] + out[2] + out[3];
    out[5] = v[4];
    // Rg^2 = sum_{i<j} r_ij^2 / n^2 (computeRg_kernel) = <|r|^2> - |<r>|^2
    const double cx = v[5] / n, cy = v[6] / n, cz = v[7] / n;
    const double rg2 = v[8] / n - (cx * cx + cy * cy + cz * cz);
    out[6] = sqrt(rg2 > 0.0 ? rg2 : 0.0);
    out[7] = (J.hi && !J.hi_exact) ? (double)J.epsilon : 0.0;
}

}  // namespace sopb
