"""Seeded request streams for the serving loop: pulling, force-clamp and
indentation jobs of mixed sizes, some with hydrodynamic interactions."""
import math

import numpy as np

import sopb
import sopb_serve
import sopb_synth as S
from helpers import plain_params


def job_spec(kind, n, seed, hi=False, rng_seed=1):
    s = S.make_system(int(n), seed)
    extra = {}
    if hi:
        extra = dict(hi_on=1, hi_a=1.9, hi_epsilon_freq=10, hi_capricious=0)
        if n <= 1500:
            # exact HI (Cholesky factor), refreshed every step up to the
            # reference's 128 beads and every 10 steps above
            extra["hi_exact"] = 1
            if n > 128:
                extra["hi_refresh"] = 10
    if kind == "ramp":
        p = plain_params(pulling=1, deltax=0.05, k_trans=0.05, pullFreq=100, fixedEnd=0, pulledEnd=n - 1, **extra)
        return sopb.JobSpec.from_system(s, p, fixed=[0], pulled=[n - 1], seed=rng_seed)
    if kind == "clamp":
        p = plain_params(pulling=1, fconst=2.5, fixedEnd=0, pulledEnd=n - 1, **extra)
        return sopb.JobSpec.from_system(s, p, fixed=[0], pulled=[n - 1], seed=rng_seed)
    x = s.xyz.astype(np.float64)
    top = x[:, 1].min()
    tip = [float(x[:, 0].mean()), float(top - 22.0), float(x[:, 2].mean())]
    p = plain_params(indentation=1, indentationTipR=20.0, indentationKs=0.07, indentationDeltaX=0.05,
                     indentationTip=tip, indentationChip=tip, indentationDirection=[0.0, 1.0, 0.0],
                     indentationSurfaceR0=[0.0, float(x[:, 1].max() + 6.0), 0.0],
                     indentationSurfaceN=[0.0, -1.0, 0.0], indentationTipZeta=500.0, indentationSurfA=1.0,
                     indentationSurfB=-2.0, indentationSurfSigma=3.0, indentationSurfEl=0.2,
                     indentationFixTrans=1, nav=100, **extra)
    return sopb.JobSpec.from_system(s, p, seed=rng_seed)


def poisson_stream(count, rate, seed, n_lo=50, n_hi=5000, steps_lo=10000, steps_hi=100000, hi_frac=0.3,
                   n_median=None):
    """`count` requests with exponential inter-arrival times (mean 1/rate s),
    sizes log-normal in [n_lo, n_hi], steps log-uniform in [steps_lo, steps_hi],
    kind uniform over ramp/clamp/indentation, `hi_frac` with HI."""
    rng = np.random.default_rng(seed)
    t = 0.0
    sizes = S.lognormal_sizes(count, n_lo, n_hi, seed, median=n_median)
    out = []
    for k in range(count):
        t += rng.exponential(1.0 / rate)
        kind = ("ramp", "clamp", "indent")[int(rng.integers(3))]
        hi = bool(rng.random() < hi_frac)
        steps = int(math.exp(rng.uniform(math.log(steps_lo), math.log(steps_hi))))
        spec = job_spec(kind, int(sizes[k]), seed * 7919 + k, hi=hi, rng_seed=seed + k)
        out.append(sopb_serve.Request(k, spec, steps, arrival=t, kind=kind + ("+hi" if hi else "")))
    return out
