"""The oracle and the CUDA path against golden dumps of the reference's own
CUDA code run on a B200 (tests/golden/make_ref_gpu_golden.py).

Both sides read the same config file and inputs (ref_cases.py), parsed by
the library's config layer (sopb_config.py).  Bars:
  * Hybrid Taus states after k steps: bit-exact;
  * the Verlet list the reference built from its own coordinates: rebuilt
    from those coordinates, bit-exact;
  * potential forces of step 0: within FORCE_RTOL of FP64 for the oracle and
    the CUDA path; the reference itself (fast-math build) within
    REF_FORCE_RTOL of FP64;
  * coordinates after k steps: within 1e-5 A (measured: 1-4e-6 A after 100
    steps of pulling, clamp, indentation, heating and TEA runs); exact HI,
    compared in the reference-compatible noise mode, within 1e-3 A per step:
    integrateCholesky_D reads mforce[j] while other threads overwrite it
    (src/Integrators/bdhitea_kernel.cu:141-150), so the reference's own
    result depends on thread timing there.
"""
import os
import sys

import numpy as np
import pytest

import oracle_py as O
import sopb
import sopb_config as CFG
from helpers import FORCE_RTOL, force_error

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, GOLD)
import ref_cases  # noqa: E402

# The reference build uses the approximate sqrt and division of -use_fast_math
# (src/Makefile:14); its step-0 forces carry up to ~2e-4 of the FP32 rounding
# scale, mostly from FENE's r - r0 on near-relaxed bonds.
REF_FORCE_RTOL = 1e-3


def coord_tol(steps, name=""):
    if ref_cases.CASES.get(name, {}).get("cfg", {}).get("hi_exact") == "yes":
        return 1e-3 * steps
    return 1e-5


def cases():
    # the state-dump cases (the long-run statistics have their own test)
    return [c for c in ref_cases.CASES
            if os.path.exists(os.path.join(GOLD, "ref_gpu_%s.npz" % c)) and not ref_cases.CASES[c].get("longrun")]


def load(name):
    g = np.load(os.path.join(GOLD, "ref_gpu_%s.npz" % name))
    over = {"hi_b_mode": "reference"} if ref_cases.CASES[name]["cfg"].get("hi_exact") == "yes" else {}
    cfg = CFG.Config(text=ref_cases.config_text(name), overrides=over)
    jc = CFG.job_config(cfg)
    specs = CFG.job_specs(jc, ref_cases.systems(name))
    return g, jc, specs


def split(arr, nruns):
    return np.split(arr, nruns)


@pytest.mark.parametrize("name", cases())
def test_stride_and_layout(name):
    g, jc, specs = load(name)
    assert int(g["stride"]) == jc.params.stride
    assert g["forces_0"].shape[0] == sum(s.n for s in specs)


@pytest.mark.parametrize("name", cases())
def test_oracle_against_reference_cuda(name):
    g, jc, specs = load(name)
    c = ref_cases.CASES[name]
    for r, sp in enumerate(specs):
        o = O.OracleJob(sp)
        done = 0
        for s in c["dumps"]:
            assert o.advance(s - done) == 0
            done = s
            sl = slice(r * sp.n, (r + 1) * sp.n)
            assert np.array_equal(o.read(sopb.SEEDS), g["seeds_%d" % s][sl]), (name, r, s)
            dx = np.max(np.abs(o.read(sopb.COORDS)[:, :3] - g["coords_%d" % s][sl, :3]))
            assert dx < coord_tol(s, name), (name, r, s, dx)
        o.close()


@pytest.mark.parametrize("name", [c for c in cases() if not ref_cases.CASES[c]["cfg"].get("hi_on")])
def test_step0_forces_against_reference_cuda(name):
    g, jc, specs = load(name)
    for r, sp in enumerate(specs):
        o = O.OracleJob(sp)
        o.rebuild(True, True)
        f32, f64, a64 = o.forces()
        ref = g["forces_0"][r * sp.n:(r + 1) * sp.n]
        assert force_error(f32, f64, a64) <= FORCE_RTOL
        assert force_error(ref, f64, a64) <= REF_FORCE_RTOL
        o.close()


@pytest.mark.parametrize("name", cases())
def test_reference_verlet_list_rebuilt_bit_exact(name):
    g, jc, specs = load(name)
    c = ref_cases.CASES[name]
    p = jc.params
    for s in c["dumps"]:
        build = (s - 1) // p.pairs_freq * p.pairs_freq   # the list in force at step s-1
        if "coords_%d" % build not in g and build != 0:
            continue
        for r, sp in enumerate(specs):
            sl = slice(r * sp.n, (r + 1) * sp.n)
            o = O.OracleJob(sp)
            o.rebuild(True, False)                          # possible pairs at step 0
            if build:
                o.write(sopb.COORDS, g["coords_%d" % build][sl])
            o.rebuild(False, True)
            cnt, rows = o.pairlist(False, cap=g["pairs_%d" % s].shape[1])
            ref = g["pairs_%d" % s][sl]
            ref = np.where(ref >= 0, ref - r * sp.n, ref)     # reference rows hold global bead numbers
            assert np.array_equal(cnt, g["paircount_%d" % s][sl]), (name, s, r)
            assert np.array_equal(rows, ref), (name, s, r)
            o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", cases())
def test_cuda_path_against_reference_cuda(gpu_ctx, name):
    g, jc, specs = load(name)
    c = ref_cases.CASES[name]
    jobs = [gpu_ctx.job(sp) for sp in specs]
    done = 0
    for s in c["dumps"]:
        gpu_ctx.run(jobs, s - done)
        done = s
        for r, (j, sp) in enumerate(zip(jobs, specs)):
            sl = slice(r * sp.n, (r + 1) * sp.n)
            assert j.status() == 0
            assert np.array_equal(j.read(sopb.SEEDS), g["seeds_%d" % s][sl]), (name, r, s)
            dx = np.max(np.abs(j.read(sopb.COORDS)[:, :3] - g["coords_%d" % s][sl, :3]))
            assert dx < coord_tol(s, name), (name, r, s, dx)
            if "tip_%d" % s in g:
                tip = j.read(sopb.TIPSTATE)
                assert np.allclose(tip[:3], g["tip_%d" % s][:3], atol=1e-3)
    for j in jobs:
        j.destroy()
