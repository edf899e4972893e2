"""Pulling plane and discrete-surface indentation through the C ABI against
the oracle: forces within the force bar, short trajectories, the plane and
tip lines of the event log; resident kernel and grid path."""
import numpy as np
import pytest

import oracle_py as O
import sopb
from helpers import FORCE_RTOL, force_error, plain_params, system

pytestmark = pytest.mark.gpu


def plane_spec(n=150, seed=17, **kw):
    s = system(n, seed)
    c = s.xyz.astype(np.float64).mean(axis=0)
    p = plain_params(pullingPlane=1, pullingPlaneDeltax=0.5, pullingPlaneKs=0.5, pullingPlaneKsCant=0.2,
                     pullingPlaneZeta=50.0, pullingPlaneDir=[0.0, 0.6, 0.8], pullingPlanePos=[float(v) for v in c],
                     pullingPlaneUpdateFreq=10, pullingPlaneOutputFreq=20, **kw)
    return sopb.JobSpec.from_system(s, p, seed=1357, plane_fixed=range(0, 5), plane_pulled=range(n - 5, n))


def surface_spec(n=200, seed=13, move=0, **kw):
    s = system(n, seed)
    x = s.xyz.astype(np.float64)
    top = x[:, 1].min()
    tip = [float(x[:, 0].mean()), float(top - 22.0), float(x[:, 2].mean())]
    p = plain_params(indentation=1, indentationTipR=20.0, indentationKs=0.07,
                     indentationDeltaX=-0.5 if move else 0.05, indentationTip=tip, indentationChip=tip,
                     indentationDirection=[0.0, 1.0, 0.0],
                     indentationSurfaceR0=[float(x[:, 0].mean()), float(x[:, 1].max() + 6.0), float(x[:, 2].mean())],
                     indentationSurfaceN=[0.0, -1.0, 0.0], indentationTipZeta=500.0, indentationSurfA=1.0,
                     indentationSurfB=-2.0, indentationSurfSigma=3.0, indentationSurfEl=0.2, indentationFixTrans=1,
                     indentationMoveSurface=move, indentationDiscreteSurf=1, indentationSurfaceSize=15,
                     indentationSurfaceStep=3.0, indentationPairsCutoff=12.0, nav=20, **kw)
    return sopb.JobSpec.from_system(s, p, seed=2468)


CASES = [("plane", {}), ("surface", {}), ("surface", {"move": 1})]


def make(kind, grid, extra):
    if kind == "plane":
        return plane_spec(grid_path=grid)
    return surface_spec(grid_path=grid, **extra)


@pytest.mark.parametrize("grid", [0, 1])
@pytest.mark.parametrize("kind,extra", CASES)
def test_forces_match_oracle(gpu_ctx, kind, extra, grid):
    sp = make(kind, grid, extra)
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    gpu_ctx.run([g], 1)                 # the step-0 updaters build the lists
    o.advance(1)
    o.write(sopb.COORDS, g.read(sopb.COORDS))
    f32, f64, a64 = o.forces()
    assert force_error(g.read(sopb.FORCES), f64, a64) <= FORCE_RTOL
    assert force_error(f32, f64, a64) <= FORCE_RTOL
    g.destroy()


@pytest.mark.parametrize("grid", [0, 1])
@pytest.mark.parametrize("kind,extra", CASES)
def test_trajectory_and_log_track_oracle(gpu_ctx, kind, extra, grid):
    sp = make(kind, grid, extra)
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    gpu_ctx.run([g], 120)
    gpu_ctx.run([g], 80)
    assert o.advance(200) == 0
    assert g.status() == 0
    assert np.max(np.abs(g.read(sopb.COORDS) - o.read(sopb.COORDS))) < 2e-3
    assert np.array_equal(g.read(sopb.SEEDS), o.read(sopb.SEEDS))
    lg, lo = g.log(), o.log()
    assert len(lg) == len(lo) > 0
    assert np.array_equal(lg["kind"], lo["kind"]) and np.array_equal(lg["step"], lo["step"])
    assert np.allclose(lg["v"], lo["v"], rtol=1e-3, atol=2e-3)
    g.destroy()


def test_plane_alone_equals_batch(gpu_ctx):
    sps = [plane_spec(), plane_spec(n=120, seed=5)]
    alone = []
    for sp in sps:
        j = gpu_ctx.job(sp)
        gpu_ctx.run([j], 100)
        alone.append((j.read(sopb.COORDS), j.log()))
        j.destroy()
    jobs = [gpu_ctx.job(sp) for sp in sps]
    gpu_ctx.run(jobs, 100)
    for j, (x, L) in zip(jobs, alone):
        assert np.array_equal(j.read(sopb.COORDS), x)
        assert np.array_equal(j.log(), L)
        j.destroy()
