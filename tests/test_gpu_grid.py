"""The grid path (per-step kernels in CUDA graphs) against the oracle:
jobs forced onto it, cell-list possible pairs against brute force, and a
job too large for one CTA."""
import numpy as np
import pytest

import oracle_py as O
import sopb
from helpers import FORCE_RTOL, force_error, spec

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["ramp", "indent", "free", "clamp"])
def test_grid_path_tracks_oracle(gpu_ctx, mode):
    sp = spec(300, 41, mode, grid_path=1)
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    for chunk in (7, 23, 50):           # partial chunks, graph replays, partial again
        gpu_ctx.run([g], chunk)
        assert o.advance(chunk) == 0
    assert g.status() == 0 and g.step() == o.step() == 80
    assert np.array_equal(g.read(sopb.SEEDS), o.read(sopb.SEEDS))
    assert np.max(np.abs(g.read(sopb.COORDS) - o.read(sopb.COORDS))) < 1e-3
    assert np.allclose(g.read(sopb.TEMP), o.read(sopb.TEMP), rtol=1e-3, atol=1e-3)
    if mode == "ramp":
        assert np.array_equal(g.read(sopb.PULLSTATE)[3:], o.read(sopb.PULLSTATE)[3:])
    if mode == "indent":
        assert np.allclose(g.read(sopb.TIPSTATE)[:11], o.read(sopb.TIPSTATE)[:11], rtol=1e-4, atol=1e-4)
    g.destroy()


@pytest.mark.parametrize("n,thr", [(3000, 25.0), (8000, 30.0)])
def test_cell_list_rows_equal_brute_force(gpu_ctx, n, thr):
    sp = spec(n, 5, "free", pairs_threshold=thr, max_possiblePairs=2048, grid_path=1, cell_list=1)
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    g.rebuild(True, True)
    o.rebuild(True, True)
    for possible in (True, False):
        cg, rg = g.pairlist(possible, cap=2048)
        co, ro = o.pairlist(possible, cap=2048)
        assert np.array_equal(cg, co)
        assert np.array_equal(rg, ro)
    f32, f64, a64 = o.forces()
    assert force_error(g.read(sopb.FORCES), f64, a64) <= FORCE_RTOL
    g.destroy()


def test_large_job_on_grid_path(gpu_ctx):
    sp = spec(20000, 3, "clamp", pairs_threshold=30.0, max_possiblePairs=2048, max_pairs=512)
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    gpu_ctx.run([g], 30)
    assert o.advance(30) == 0
    assert g.status() == 0
    assert np.array_equal(g.read(sopb.SEEDS), o.read(sopb.SEEDS))
    assert np.max(np.abs(g.read(sopb.COORDS) - o.read(sopb.COORDS))) < 1e-3
    g.destroy()


def test_concurrent_grid_jobs_equal_alone(gpu_ctx):
    # grid-path jobs of one sopb_run execute side by side on their own
    # streams; each must equal itself run alone (no shared scratch)
    specs = [spec(100, 11, "clamp", hi_on=1, hi_exact=1, hi_a=1.9, hi_capricious=0),
             spec(300, 12, "ramp", hi_on=1, hi_exact=1, hi_refresh=10, hi_a=1.9, hi_capricious=0),
             spec(3000, 13, "clamp", pairs_threshold=30.0, max_possiblePairs=2048),
             spec(2000, 14, "free", hi_on=1, hi_a=1.9, hi_epsilon_freq=10, hi_capricious=0),
             spec(250, 15, "clamp")]                       # a resident job beside them
    alone = []
    for sp in specs:
        j = gpu_ctx.job(sp)
        gpu_ctx.run([j], 60)
        alone.append(j.read(sopb.COORDS))
        j.destroy()
    jobs = [gpu_ctx.job(sp) for sp in specs]
    for q in (20, 20, 20):
        gpu_ctx.run(jobs, q)
    for j, ref in zip(jobs, alone):
        assert j.status() == 0
        assert np.array_equal(j.read(sopb.COORDS), ref)
        j.destroy()


def test_grid_only_run_after_resident_run_on_the_same_stream(gpu_ctx):
    # a run of several grid jobs and no resident job, after a run of resident
    # jobs on the same stream, launches nothing of that earlier run: each
    # grid job equals itself run alone
    specs = [spec(200, 81, "clamp", grid_path=1), spec(260, 82, "ramp", grid_path=1)]
    alone = []
    for sp in specs:
        j = gpu_ctx.job(sp)
        gpu_ctx.run([j], 40)
        alone.append(j.read(sopb.COORDS))
        j.destroy()
    res = [gpu_ctx.job(spec(120 + 30 * k, 90 + k, "clamp")) for k in range(3)]
    gpu_ctx.run(res, [30, 20, 10])
    for j in res:
        assert j.status() == 0
        j.destroy()
    jobs = [gpu_ctx.job(sp) for sp in specs]
    gpu_ctx.run(jobs, 40)
    for j, ref in zip(jobs, alone):
        assert j.status() == 0
        assert np.array_equal(j.read(sopb.COORDS), ref)
        j.destroy()
