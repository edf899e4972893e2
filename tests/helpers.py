"""Shared inputs and tolerances of the parity tests."""
import functools

import numpy as np

import sopb
import sopb_synth as S

# Force parity bound, per component: |F_gpu - F_fp64| <= FORCE_RTOL * S where
# S is the FP32 rounding scale of the sum (for every term the magnitudes of
# the quantities it subtracts; oracle orc_job_forces), i.e. 1e-5 relative.
FORCE_RTOL = 1e-5


@functools.lru_cache(maxsize=64)
def system(n: int, seed: int) -> S.System:
    return S.make_system(n, seed)


def plain_params(**kw) -> sopb.Params:
    """The plain 200-bead pull configuration: T = 0.6 kcal/mol (300 K),
    dt = 0.08 tau_H (20 ps), pairlist every 10 steps at 20 A, FENE k = 20
    kcal/mol/A^2 (14 N/m) with R0 = 2 A, repulsive sigma 3.8 A el 1."""
    base = dict(timestep=0.08, zeta=50.0, temperature=0.6, pairs_freq=10, pairlist_cutoff=20.0,
                pairs_cutoff=20.0, pairs_threshold=200.0, nav=1000)
    base.update(kw)
    return sopb.default_params(**base)


def spec(n: int, seed: int, mode: str = "ramp", rng_seed: int = 1119727, **kw) -> sopb.JobSpec:
    s = system(n, seed)
    if mode == "ramp":
        p = plain_params(pulling=1, deltax=0.02, k_trans=0.05, fixedEnd=0, pulledEnd=n - 1, pullFreq=10, **kw)
        return sopb.JobSpec.from_system(s, p, fixed=[0], pulled=[n - 1], seed=rng_seed)
    if mode == "clamp":
        p = plain_params(pulling=1, fconst=2.5, fixedEnd=0, pulledEnd=n - 1, **kw)
        return sopb.JobSpec.from_system(s, p, fixed=[0], pulled=[n - 1], seed=rng_seed)
    if mode == "free":
        return sopb.JobSpec.from_system(s, plain_params(**kw), seed=rng_seed)
    if mode == "indent":
        x = s.xyz.astype(np.float64)
        top = x[:, 1].min()
        p = plain_params(indentation=1, indentationTipR=20.0, indentationKs=0.07, indentationDeltaX=0.05,
                         indentationTip=[float(x[:, 0].mean()), float(top - 22.0), float(x[:, 2].mean())],
                         indentationChip=[float(x[:, 0].mean()), float(top - 22.0), float(x[:, 2].mean())],
                         indentationDirection=[0.0, 1.0, 0.0],
                         indentationSurfaceR0=[0.0, float(x[:, 1].max() + 6.0), 0.0],
                         indentationSurfaceN=[0.0, -1.0, 0.0], indentationTipZeta=500.0,
                         indentationSurfA=1.0, indentationSurfB=-2.0, indentationSurfSigma=3.0, indentationSurfEl=0.2,
                         indentationFixTrans=1, nav=20, **kw)
        return sopb.JobSpec.from_system(s, p, seed=rng_seed)
    raise ValueError(mode)


def force_error(f, f64, abs64) -> float:
    """max over components of |f - f64| / (rounding scale + tiny)."""
    f = np.asarray(f, np.float64)[:, :3]
    return float(np.max(np.abs(f - f64[:, :3]) / (abs64[:, :3] + 1e-30)))
