"""Long-run statistics of a multi-run force-ramp pull, read from the files the
reference's output updaters write (and the `sopb-gpu` driver writes in the
same formats): the pulling lines <name>_<run>_pull.dat (step, end-to-end
distance, its projection, the force along the pull direction and the force
vector; src/Potentials/pulling.cu:167-190) and the energy lines
<name>_<run>.dat (step, T, FENE, native, repulsive and total energy, intact
native contacts, Rg; src/Updaters/output_manager.cu:339-360).

Used by make_ref_longrun_golden.py (the reference's CUDA build on a B200) and
by tests/test_gpu_longrun.py (this library), so both sides are reduced by the
same code.
"""
import os

import numpy as np


def read_runs(d, name, runs, first=1):
    """pull: (runs, lines, 3) step, end-to-end distance, force along the pull
    direction; dat: (runs, lines, 8) every .dat column."""
    pull, dat = [], []
    for r in range(first, first + runs):
        with open(os.path.join(d, "%s_%d_pull.dat" % (name, r))) as f:
            p = [[float(t) for t in l.split("\t")] for l in f if l.strip()]
        pull.append(np.array(p, np.float64)[:, [0, 1, 3]])
        with open(os.path.join(d, "%s_%d.dat" % (name, r))) as f:
            q = [[float(t) for t in l.split("\t")] for l in f if l.strip()]
        dat.append(np.array(q, np.float64))
    lp = min(len(p) for p in pull)
    ld = min(len(q) for q in dat)
    return np.stack([p[:lp] for p in pull]), np.stack([q[:ld] for q in dat])


def per_run(pull, dat):
    """Statistics with one independent value per run: the peak force and the
    extension it is reached at, the force averaged over the last fifth of the
    ramp (the stretched chain), the mean kinetic temperature over the .dat
    lines after the first, the mean total energy and the intact native
    contacts over the first half (the folded part of the run) and over the
    last fifth."""
    f, x = pull[:, :, 2], pull[:, :, 1]
    k = np.argmax(f, axis=1)
    nl, nd = pull.shape[1], dat.shape[1]
    return {
        "peak_force": f.max(axis=1),
        "extension_at_peak": x[np.arange(len(k)), k],
        "late_force": f[:, -nl // 5:].mean(axis=1),
        "temperature": dat[:, 1:, 1].mean(axis=1),
        # NaN for a run whose FENE energy is not finite (a bond beyond the
        # FENE limit: the reference prints nan and carries on)
        "energy_early": dat[:, 1:nd // 2, 5].mean(axis=1),
        "energy_late": dat[:, -nd // 5:, 5].mean(axis=1),
        "contacts_early": dat[:, 1:nd // 2, 6].mean(axis=1),
        "contacts_late": dat[:, -nd // 5:, 6].mean(axis=1),
    }


def nonfinite_energy_runs(dat):
    """Runs with a non-finite energy on any .dat line."""
    return set(np.nonzero(~np.isfinite(dat[:, :, 2:6]).all(axis=(1, 2)))[0].tolist())


def force_extension(pull, edges):
    """Per run, the mean force in each extension bin (NaN where a run has no
    line in the bin)."""
    x, f = pull[:, :, 1], pull[:, :, 2]
    out = np.full((pull.shape[0], len(edges) - 1), np.nan)
    for b in range(len(edges) - 1):
        m = (x >= edges[b]) & (x < edges[b + 1])
        cnt = m.sum(axis=1)
        s = np.where(m, f, 0.0).sum(axis=1)
        out[:, b] = np.where(cnt > 0, s / np.maximum(cnt, 1), np.nan)
    return out
