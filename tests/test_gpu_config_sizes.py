"""Parity at the sizes the benchmark runs, against the CPU oracle.

* the 512-replica ragged force-clamp batch (113 612 beads, sizes 60-600):
  the whole batch advances 200 steps in one run, and 16 of its jobs, spread
  over the size range, are compared with the oracle;
* exact HI at 4000 beads (a 12 000 x 12 000 RPY tensor, factor refreshed
  every 10 steps): the blocked factor against an FP64 Cholesky of D, and a
  12-step trajectory (two factorisations) against the oracle's column
  Cholesky;
* a capsid-like shell on the grid path with the cell list and a 10 nm
  indentation tip: 180 copies of a 100-bead chain on the icosahedral 60 x 3
  lattice (18 000 beads, radius about 149 A), 50 steps.

Bars are those of the smaller parity tests: Hybrid Taus states bit-exact,
coordinates within 2e-3 A after 200 steps and 1e-3 A after 12 or 50.
"""
import numpy as np
import pytest

import oracle_py as O
import sopb
import sopb_workloads as W

pytestmark = pytest.mark.gpu


def test_batch512_sample_tracks_oracle():
    specs = W.batch_specs()
    assert len(specs) == 512 and sum(sp.n for sp in specs) == 113612
    sizes = np.array([sp.n for sp in specs])
    order = np.argsort(sizes, kind="stable")
    pick = [int(order[q]) for q in np.linspace(0, len(order) - 1, 16).round().astype(int)]
    assert sizes[pick[0]] == sizes.min() and sizes[pick[-1]] == sizes.max()
    with sopb.Context(0) as ctx:
        ctx.set_shape_policy(4, 1.0, 1024)      # the bench's policy
        jobs = [ctx.job(sp) for sp in specs]
        ctx.run(jobs, 200)
        ctx.sync()
        assert all(j.status() == 0 for j in jobs)
        got = {k: (jobs[k].read(sopb.COORDS), jobs[k].read(sopb.SEEDS)) for k in pick}
    oj = [O.OracleJob(specs[k]) for k in pick]
    assert O.jobs_advance(oj, 200) == 0
    for k, o in zip(pick, oj):
        x, s = got[k]
        assert np.array_equal(s, o.read(sopb.SEEDS)), k
        dx = float(np.max(np.abs(x - o.read(sopb.COORDS))))
        assert dx < 2e-3, (k, specs[k].n, dx)
        o.close()


def test_exact_hi_4000_beads_factor_and_trajectory(gpu_ctx):
    import torch
    n = 4000
    sp = W.hi_spec(n, exact=True, refresh=10)
    g = gpu_ctx.job(sp)
    x0 = g.read(sopb.COORDS)[:, :3].copy()
    gpu_ctx.run([g], 1)                          # step 0 factorises D at x0
    assert g.status() == 0
    L = torch.from_numpy(g.read(sopb.HIFACTOR)).cuda().double().tril_()
    D = torch.from_numpy(O.rpy_tensor(x0, sp.params.hi_a)).cuda()
    L64 = torch.linalg.cholesky(D)
    max_entry = float((L - L64).abs().max())
    rel = float(torch.linalg.matrix_norm(L @ L.T - D) / torch.linalg.matrix_norm(D))
    del L, L64, D
    torch.cuda.empty_cache()
    assert max_entry < 2e-4, max_entry
    assert rel < 2e-6, rel
    g.destroy()
    # 12 steps: factorisations at steps 0 and 10
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    gpu_ctx.run([g], 12)
    assert o.advance(12) == 0
    assert g.status() == 0
    assert np.array_equal(g.read(sopb.SEEDS), o.read(sopb.SEEDS))
    dx = float(np.max(np.abs(g.read(sopb.COORDS) - o.read(sopb.COORDS))))
    assert dx < 1e-3, dx
    g.destroy()
    o.close()


def test_capsid_shell_with_indentation_tracks_oracle(gpu_ctx):
    sp, info = W.capsid_spec(copies_per_unit=3, chain_n=100, cell_list=1)
    assert sp.n == 18000 and info["copies"] == 180 and info["inter_natives"] > 0
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    # the lists of the step-0 coordinates (cell list against the oracle's
    # brute force), as step 0 builds them
    g.rebuild(True, True)
    o.rebuild(True, True)
    for possible in (True, False):
        cg, rg = g.pairlist(possible, cap=2048)
        co, ro = o.pairlist(possible, cap=2048)
        assert np.array_equal(cg, co) and np.array_equal(rg, ro)
    for chunk in (10, 40):
        gpu_ctx.run([g], chunk)
        assert o.advance(chunk) == 0
    assert g.status() == 0 and g.step() == o.step() == 50
    assert np.array_equal(g.read(sopb.SEEDS), o.read(sopb.SEEDS))
    dx = float(np.max(np.abs(g.read(sopb.COORDS) - o.read(sopb.COORDS))))
    assert dx < 1e-3, dx
    assert np.allclose(g.read(sopb.TIPSTATE)[:11], o.read(sopb.TIPSTATE)[:11], rtol=1e-4, atol=1e-4)
    g.destroy()
    o.close()
