"""The benchmark workloads as job specifications (seeded synthetic inputs).

The reference's benchmarks have no public dataset; these generators stand in
for them with the sizes of the benchmark configurations:
  * plain: one 200-bead chain, force-ramp pull of the last bead, first fixed;
  * batch512: 512 replicas, sizes log-normal in [60, 600], force clamp at
    U(100, 300) pN, each with its own chain, native map and RNG seed;
  * capsid: a shell of chain copies on an icosahedral lattice, nanoindented by
    a 10 nm tip against a substrate, cell-list pairlist;
  * hi: one n-bead globule with exact HI (Cholesky) or TEA.
Common parameters: T = 0.6 kcal/mol (300 K), dt = 0.08 tau_H (20 ps),
pairlist every 10 steps at 20 A, FENE k = 20 kcal/mol/A^2 with R0 = 2 A.
"""
from __future__ import annotations

import numpy as np

import sopb
import sopb_synth as S


def plain_params(defaults=None, **kw):
    """Parameters of the bench workloads over the reference defaults, from
    `defaults` (the library's sopb.default_params unless given: the CPU arm
    passes the oracle's own table so that it loads no product library)."""
    base = dict(timestep=0.08, zeta=50.0, temperature=0.6, pairs_freq=10, pairlist_cutoff=20.0, pairs_cutoff=20.0,
                pairs_threshold=200.0, nav=1000)
    base.update(kw)
    return (defaults or sopb.default_params)(**base)


def batch_specs(count=512, lo=60, hi=600, seed=2024, rank=0, defaults=None):
    """The ragged force-clamp batch (one independent copy per rank)."""
    base = seed + 7919 * rank
    sizes = S.lognormal_sizes(count, lo, hi, base)
    rng = np.random.default_rng(base + 1)
    f_pn = rng.uniform(100.0, 300.0, count)
    specs = []
    for k, n in enumerate(sizes):
        n = int(n)
        s = S.make_system(n, base * 1000 + k)
        p = plain_params(defaults, pulling=1, fconst=float(f_pn[k] / 70.0), fixedEnd=0, pulledEnd=n - 1)
        specs.append(sopb.JobSpec.from_system(s, p, fixed=[0], pulled=[n - 1], seed=1119727 + k))
    return specs


def plain_spec(seed=2024):
    """One 200-bead force-ramp pull: first bead fixed, last pulled."""
    s = S.make_system(200, seed)
    p = plain_params(pulling=1, deltax=0.5, k_trans=0.05, pullFreq=1000, fixedEnd=0, pulledEnd=199)
    return sopb.JobSpec.from_system(s, p, fixed=[0], pulled=[199], seed=1119727)


def batch_config(specs, chunk, world):
    """The `config` object of the batch512 line, shared by both arms."""
    return {"workload": "batch512_lognormal_60-600_clamp", "replicas": len(specs),
            "beads": int(sum(sp.n for sp in specs)), "langevin_steps_per_step": chunk, "pairs_freq": 10,
            "pairlist_cutoff_A": 20.0, "dt_tauH": 0.08, "parallelism": "replicas-dp%d" % world,
            "l2": "flushed between timed steps"}


def capsid_spec(copies_per_unit=3, chain_n=1100, cell_list=0):
    """A shell of 60 x copies_per_unit copies of a chain_n-bead chain on the
    icosahedral lattice (default: the 198k-bead shell, 180 copies of 1100
    beads), nanoindented by a 10 nm tip on a ramped cantilever against an
    attractive substrate; cell-list pairlist (automatic above 16384 beads,
    or cell_list 1)."""
    s, info = S.make_capsid(copies_per_unit=copies_per_unit, chain_n=chain_n)
    x = s.xyz.astype(np.float64)
    c = x.mean(axis=0)
    tipR = 100.0
    tip = [float(c[0]), float(x[:, 1].max() + tipR + 4.0), float(c[2])]
    p = plain_params(pairs_threshold=40.0, max_possiblePairs=2048, max_pairs=512, possiblepairs_freq=100000,
                     indentation=1, indentationTipR=tipR, indentationKs=0.07, indentationDeltaX=0.012,
                     indentationTip=tip, indentationChip=tip, indentationDirection=[0.0, -1.0, 0.0],
                     indentationSurfaceR0=[0.0, float(x[:, 1].min() - 10.0), 0.0],
                     indentationSurfaceN=[0.0, 1.0, 0.0], indentationTipZeta=5000.0,
                     indentationSurfA=1.0, indentationSurfB=-2.0, indentationSurfSigma=10.0, indentationSurfEl=0.2,
                     indentationFixTrans=1, nav=100, cell_list=cell_list)
    return sopb.JobSpec.from_system(s, p, seed=5032015), info


def hi_spec(n, exact, refresh=10, seed=4000):
    """The HI configuration: one n-bead globule (the plain configuration's
    generator and force-ramp pull), RPY radius 3.8 A; exact (Cholesky factor
    refreshed every `refresh` steps) or TEA (epsilon every 10 steps)."""
    s = S.make_system(n, seed)
    p = plain_params(pulling=1, deltax=0.5, k_trans=0.05, pullFreq=1000, fixedEnd=0, pulledEnd=n - 1,
                     hi_on=1, hi_a=3.8, hi_exact=1 if exact else 0, hi_refresh=refresh, hi_epsilon_freq=10,
                     hi_capricious=0, max_possiblePairs=4096)
    return sopb.JobSpec.from_system(s, p, fixed=[0], pulled=[n - 1], seed=1119727)
