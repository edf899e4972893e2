"""Continuous batching: requests arriving while others run are admitted as
memory frees up; each result equals the same job run alone."""
import numpy as np
import pytest

import sopb
import sopb_serve
from serve_mix import poisson_stream

pytestmark = pytest.mark.gpu


def test_served_results_equal_alone(gpu_ctx):
    reqs = poisson_stream(14, rate=400.0, seed=3, n_lo=40, n_hi=400, steps_lo=150, steps_hi=700, hi_frac=0.3)
    srv = sopb_serve.Server(gpu_ctx, quantum=100, keep_coords=True)
    res = {r.rid: r for r in srv.serve(reqs)}
    assert len(res) == len(reqs)
    assert srv.peak_inflight > 1                      # work of different requests overlapped
    for req in reqs:
        r = res[req.rid]
        assert r.status == 0, (req.kind, r.status)
        j = gpu_ctx.job(req.spec)
        gpu_ctx.run([j], req.steps)
        alone = j.read(sopb.COORDS)
        j.destroy()
        assert np.array_equal(r.coords, alone), req.kind


def test_admission_by_footprint(gpu_ctx):
    reqs = poisson_stream(10, rate=1000.0, seed=5, n_lo=60, n_hi=300, steps_lo=100, steps_hi=300, hi_frac=0.0)
    fps = [r.spec.footprint() for r in reqs]
    budget = int(sum(sorted(fps)[-3:]))               # about three jobs at a time
    srv = sopb_serve.Server(gpu_ctx, hbm_budget=budget, quantum=50)
    res = srv.serve(reqs)
    assert all(r.status == 0 for r in res) and len(res) == len(reqs)
    assert srv.peak_used <= budget
    s = sopb_serve.summarize(res, max(r.finished for r in res))
    assert s["ok"] == len(reqs) and s["p99_s"] >= s["p50_s"] > 0


def test_ragged_run_equals_separate_runs(gpu_ctx):
    # one call, a step count per job (resident and grid-path jobs): each job
    # ends where its own run of that length ends
    from helpers import spec
    specs = [spec(120, 3, "clamp"), spec(333, 4, "ramp"), spec(90, 5, "free"),
             spec(200, 6, "clamp", hi_on=1, hi_a=1.9, hi_epsilon_freq=10, hi_capricious=0)]
    steps = [37, 120, 0, 64]
    ref = []
    for sp, n in zip(specs, steps):
        j = gpu_ctx.job(sp)
        gpu_ctx.run([j], n)
        ref.append((j.read(sopb.COORDS), j.step()))
        j.destroy()
    jobs = [gpu_ctx.job(sp) for sp in specs]
    gpu_ctx.run(jobs, steps)
    for j, (x, st) in zip(jobs, ref):
        assert j.step() == st
        assert np.array_equal(j.read(sopb.COORDS), x)
        j.destroy()
