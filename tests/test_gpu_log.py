"""The event log (sopb_job_log): the pulling and indentation updaters' lines
from the step kernel against the oracle's, for the resident kernel and the
grid path, and the ring's drain / wrap behaviour."""
import numpy as np
import pytest

import oracle_py as O
import sopb
from helpers import spec

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["ramp", "indent"])
@pytest.mark.parametrize("grid", [0, 1])
def test_log_rows_match_oracle(gpu_ctx, mode, grid):
    sp = spec(160, 41, mode, grid_path=grid)
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    gpu_ctx.run([g], 95)
    gpu_ctx.run([g], 105)
    o.advance(200)
    lg, lo = g.log(), o.log()
    assert len(lg) == len(lo) > 0
    assert np.array_equal(lg["kind"], lo["kind"]) and np.array_equal(lg["step"], lo["step"])
    # values follow the coordinates, which track the oracle within 2e-3 A
    # after 200 steps; the tip force is a sum over beads in another order
    assert np.allclose(lg["v"], lo["v"], rtol=1e-3, atol=2e-3)
    assert len(g.log()) == 0            # drained
    g.destroy()


def test_log_ring_wrap_is_reported(gpu_ctx):
    sp = spec(120, 5, "ramp", log_rows=8)
    g = gpu_ctx.job(sp)
    gpu_ctx.run([g], 200)                # 20 pulling lines into 8 slots
    with pytest.raises(sopb.SopbError) as e:
        g.log()
    assert e.value.code == sopb.ERR_CAPACITY
    gpu_ctx.run([g], 30)
    rows = g.log()
    assert list(rows["step"]) == [200, 210, 220]
    g.destroy()


def test_log_rows_of_a_served_batch_equal_alone(gpu_ctx):
    specs = [spec(n, 60 + k, "ramp", rng_seed=900 + k) for k, n in enumerate((90, 150, 260))]
    alone = []
    for sp in specs:
        j = gpu_ctx.job(sp)
        gpu_ctx.run([j], 100)
        alone.append(j.log())
        j.destroy()
    jobs = [gpu_ctx.job(sp) for sp in specs]
    gpu_ctx.run(jobs, [100, 40, 70])
    gpu_ctx.run(jobs, [0, 60, 30])
    for j, a in zip(jobs, alone):
        b = j.log()
        assert np.array_equal(a, b)
        j.destroy()
