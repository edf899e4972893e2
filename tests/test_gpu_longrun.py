"""Long-run distributions against the reference's own CUDA build.

The reference validates itself by the statistics of long pulling runs
(force-extension curves, unfolding forces, the kinetic temperature;
docs/source/general_sop.rst:58-64).  Here 256 runs of the plain 200-bead
force-ramp pull, 1e5 steps each (the cantilever travels 700 A), were run by
the reference's CUDA path on a B200 (tests/golden/make_ref_longrun_golden.py;
its output files reduced to ref_gpu_longpull.npz).  The same config runs
through this library's `sopb-gpu` driver with its own random streams (the
seed shifted, so the two sets of runs are independent samples), and both
sets of files are reduced by the same code (tests/golden/longrun.py).

Bars, with one value per run (runs are independent; lines within a run are
not):
  * two-sample Kolmogorov-Smirnov test on each per-run statistic (peak force
    and the extension it is reached at, late force, mean temperature, early
    and late energy and intact contacts): p >= 1e-3 for each of the eight;
    the energies leave out the runs whose FENE energy is not finite (a start
    with a bond near the FENE limit: the reference prints nan and carries
    on), and those runs must be the same on both sides;
  * the mean force-extension curve in 5 A bins: difference within four
    standard errors of the difference in every bin that at least 64 runs of
    each side reach;
  * the mean kinetic temperature over all runs: within four standard errors,
    and both within 2% of the set 0.6 kcal/mol.
Set SOPB_LONGRUN_LOG to a file to collect the numbers (one JSON line).
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
GOLD = os.path.join(HERE, "golden")
CLI = os.path.join(REPO, "sop-gpu_b200", "sopb-gpu")
sys.path.insert(0, GOLD)
import longrun  # noqa: E402
import ref_cases  # noqa: E402

pytestmark = pytest.mark.gpu
NAME = "longpull"
SEED_SHIFT = 1000003


@pytest.fixture(scope="module")
def both(tmp_path_factory):
    g = np.load(os.path.join(GOLD, "ref_gpu_%s.npz" % NAME))
    c = ref_cases.CASES[NAME]
    d = str(tmp_path_factory.mktemp("longrun"))
    cfg = ref_cases.write_inputs(NAME, d)
    stride = 10                                       # min of nav and the updater frequencies (pairs_freq)
    seed = int(c["cfg"]["seed"]) + SEED_SHIFT
    r = subprocess.run([CLI, os.path.basename(cfg), "numsteps=%d" % (c["total"] - stride), "seed=%d" % seed],
                       cwd=d, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    ours = longrun.read_runs(d, NAME, c["runs"])
    ref = (g["pull"].astype(np.float64), g["dat"].astype(np.float64))
    return ref, ours


def test_same_line_layout(both):
    (rp, rd), (op, od) = both
    assert rp.shape == op.shape and rd.shape == od.shape
    assert np.array_equal(rp[:, :, 0], op[:, :, 0]) and np.array_equal(rd[:, :, 0], od[:, :, 0])
    assert rp.shape[0] == 256 and rp[0, -1, 0] >= 99000


def test_distributions_agree(both):
    from scipy import stats
    (rp, rd), (op, od) = both
    a, b = longrun.per_run(rp, rd), longrun.per_run(op, od)
    bad_ref, bad_ours = longrun.nonfinite_energy_runs(rd), longrun.nonfinite_energy_runs(od)
    out = {}
    for k in a:
        va, vb = a[k][np.isfinite(a[k])], b[k][np.isfinite(b[k])]
        res = stats.ks_2samp(va, vb)
        a[k], b[k] = va, vb
        out[k] = {"ref_mean": float(a[k].mean()), "ours_mean": float(b[k].mean()), "ks": float(res.statistic),
                  "p": float(res.pvalue)}
    # mean force-extension curve
    lo = min(rp[:, :, 1].min(), op[:, :, 1].min())
    hi = max(rp[:, :, 1].max(), op[:, :, 1].max())
    edges = np.arange(np.floor(lo / 5) * 5, hi + 5, 5.0)
    fa, fb = longrun.force_extension(rp, edges), longrun.force_extension(op, edges)
    worst = 0.0
    nbins = 0
    for k in range(len(edges) - 1):
        xa, xb = fa[:, k][~np.isnan(fa[:, k])], fb[:, k][~np.isnan(fb[:, k])]
        if len(xa) < 64 or len(xb) < 64:
            continue
        se = np.sqrt(xa.var(ddof=1) / len(xa) + xb.var(ddof=1) / len(xb))
        worst = max(worst, abs(xa.mean() - xb.mean()) / max(se, 1e-12))
        nbins += 1
    ta, tb = a["temperature"], b["temperature"]
    t_se = np.sqrt(ta.var(ddof=1) / len(ta) + tb.var(ddof=1) / len(tb))
    rec = {"runs": int(rp.shape[0]), "nonfinite_energy_runs_ref": sorted(bad_ref),
           "nonfinite_energy_runs_ours": sorted(bad_ours), "per_run": out, "force_extension_bins": nbins,
           "force_extension_worst_z": float(worst), "T_ref": float(ta.mean()), "T_ours": float(tb.mean()),
           "T_z": float(abs(ta.mean() - tb.mean()) / t_se)}
    path = os.environ.get("SOPB_LONGRUN_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(rec) + "\n")
    print(json.dumps(rec))
    assert bad_ref == bad_ours and len(bad_ref) <= 4, (bad_ref, bad_ours)
    for k, v in out.items():
        assert v["p"] >= 1e-3, (k, v)
    assert nbins >= 10 and worst <= 4.0, (nbins, worst)
    assert rec["T_z"] <= 4.0
    assert abs(ta.mean() / 0.6 - 1) < 0.02 and abs(tb.mean() / 0.6 - 1) < 0.02
