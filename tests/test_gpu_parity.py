"""Parity of the CUDA path (through the C ABI) against the CPU oracle.

Bars: Hybrid Taus states and neighbour lists bit-exact; potential forces
within 1e-5 of the summation scale (helpers.FORCE_RTOL); coordinates after
one step within 1e-5 A (the noise goes through the fast-math intrinsics the
reference build uses, the oracle through libm); a job's result is
bit-identical alone and inside a mixed batch.
"""
import numpy as np
import pytest

import oracle_py as O
import sopb
from helpers import FORCE_RTOL, force_error, spec, system

pytestmark = pytest.mark.gpu


def pair(ctx, sp):
    return ctx.job(sp), O.OracleJob(sp)


@pytest.mark.parametrize("n,steps", [(64, 1), (200, 37), (600, 5)])
def test_hybrid_taus_states_bit_exact(gpu_ctx, n, steps):
    g, o = pair(gpu_ctx, spec(n, 3, "free"))
    gpu_ctx.run([g], steps)
    assert o.advance(steps) == 0
    assert np.array_equal(g.read(sopb.SEEDS), o.read(sopb.SEEDS))
    g.destroy()


@pytest.mark.parametrize("n,seed", [(60, 1), (200, 11), (451, 5), (1100, 9), (1500, 4)])
def test_lists_bit_exact_on_identical_coordinates(gpu_ctx, n, seed):
    sp = spec(n, seed, "free", pairs_threshold=25.0)
    g, o = pair(gpu_ctx, sp)
    # perturb so the lists are not the generator's
    rng = np.random.default_rng(seed)
    x = g.read(sopb.COORDS)
    x[:, :3] += rng.normal(scale=0.7, size=(n, 3)).astype(np.float32)
    g.write(sopb.COORDS, x)
    o.write(sopb.COORDS, x)
    g.rebuild(True, True)
    o.rebuild(True, True)
    for possible in (True, False):
        cg, rg = g.pairlist(possible)
        co, ro = o.pairlist(possible)
        assert np.array_equal(cg, co)
        assert np.array_equal(rg, ro)
    g.destroy()


def test_lists_bit_exact_at_exact_cutoff_ties(gpu_ctx):
    # a cubic lattice with spacing 5 A: many pairs at exactly 20 A (excluded)
    # and at sqrt(k)*5 A around it
    pts = np.array([(i, j, k) for i in range(6) for j in range(6) for k in range(6)], np.float32) * 5.0
    n = len(pts)
    p = sopb.default_params(timestep=0.08, pairs_threshold=20.0, pairlist_cutoff=15.000001, pairs_freq=10)
    sp = sopb.JobSpec(pts, np.zeros((0, 2)), [], np.zeros((0, 2)), [], [], p, seed=3)
    g, o = pair(gpu_ctx, sp)
    g.rebuild(True, True)
    o.rebuild(True, True)
    for possible in (True, False):
        cg, rg = g.pairlist(possible)
        co, ro = o.pairlist(possible)
        assert np.array_equal(cg, co) and np.array_equal(rg, ro)
    assert (cg > 0).all()
    g.destroy()


@pytest.mark.parametrize("cut", [20.0, 13.7, 7.3])
def test_lists_bit_exact_within_ulps_of_the_cutoff(gpu_ctx, cut):
    # isolated pairs whose separation is the cutoff give or take a few ulps,
    # in random directions: the squared-distance threshold must classify
    # every one as sqrt(r^2) < cut does
    rng = np.random.default_rng(int(cut * 10))
    npair = 256
    u = rng.normal(size=(npair, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    d = np.float32(cut) * (1.0 + rng.integers(-6, 7, npair) * 6e-8)
    base = np.zeros((npair, 3))
    base[:, 0] = np.arange(npair) * 4.0 * cut
    xi = base.astype(np.float32)
    xj = (base + d[:, None] * u).astype(np.float32)
    pts = np.empty((2 * npair, 3), np.float32)
    pts[0::2], pts[1::2] = xi, xj
    p = sopb.default_params(timestep=0.08, pairs_threshold=cut, pairlist_cutoff=cut, pairs_freq=10)
    sp = sopb.JobSpec(pts, np.zeros((0, 2)), [], np.zeros((0, 2)), [], [], p, seed=3)
    g, o = pair(gpu_ctx, sp)
    g.rebuild(True, True)
    o.rebuild(True, True)
    for possible in (True, False):
        cg, rg = g.pairlist(possible)
        co, ro = o.pairlist(possible)
        assert np.array_equal(cg, co) and np.array_equal(rg, ro)
    assert 0 < cg.sum() < 2 * npair           # both sides of the cutoff occur
    g.destroy()


@pytest.mark.parametrize("n,shift", [(200, 0.0), (450, 0.0), (200, 2.5)])
def test_verlet_rebuild_from_near_list_is_exact(gpu_ctx, n, shift):
    # rebuilds after the first filter the near list (pairs within the
    # cutoff plus a skin); the rows must equal a full scan of the same
    # coordinates, and a displacement beyond half the skin must force the
    # full scan again
    sp = spec(n, 31, "clamp")
    g = gpu_ctx.job(sp)
    gpu_ctx.run([g], 30)                      # rebuilds at 0 (full), 10, 20
    x = g.read(sopb.COORDS)
    if shift:
        x[n // 2:, 0] += shift                   # half of the beads jump
        g.write(sopb.COORDS, x)
    gpu_ctx.run([g], 1)                       # rebuild at step 30 from x
    o = O.OracleJob(sp)
    o.write(sopb.COORDS, x)
    o.rebuild(True, True)
    cg, rg = g.pairlist(False)
    co, ro = o.pairlist(False)
    assert np.array_equal(cg, co) and np.array_equal(rg, ro)
    g.destroy()


@pytest.mark.parametrize("lpb", [1, 2, 4, 8, 32])
@pytest.mark.parametrize("mode", ["free", "indent"])
def test_forces_match_oracle(gpu_ctx, lpb, mode):
    sp = spec(300, 21, mode, lanes_per_bead=lpb)
    g, o = pair(gpu_ctx, sp)
    g.rebuild(True, True)
    o.rebuild(True, True)
    fg = g.read(sopb.FORCES)
    f32, f64, a64 = o.forces()
    assert force_error(fg, f64, a64) <= FORCE_RTOL
    assert force_error(f32, f64, a64) <= FORCE_RTOL
    g.destroy()


@pytest.mark.parametrize("mode,lpb", [("free", 0), ("ramp", 0), ("clamp", 0), ("indent", 0),
                                      ("free", 4), ("free", 8), ("free", 16)])
def test_one_step_matches_oracle(gpu_ctx, mode, lpb):
    # one step through the resident kernel and its shared-memory list cache
    # for several lane-group widths: a lost or doubled close pair would move
    # beads by ~1e-3 A
    g, o = pair(gpu_ctx, spec(200, 13, mode, lanes_per_bead=lpb))
    gpu_ctx.run([g], 1)
    o.advance(1)
    xg, xo = g.read(sopb.COORDS), o.read(sopb.COORDS)
    assert np.max(np.abs(xg - xo)) < 1e-5
    assert np.array_equal(g.read(sopb.SEEDS), o.read(sopb.SEEDS))
    g.destroy()


def test_list_representation_by_size(gpu_ctx):
    # bitmask lists while they fit in shared memory, index rows above
    for n, want_mask in ((600, True), (1500, False)):
        j = gpu_ctx.job(spec(n, 1, "free"))
        lpb, block = j.shape()
        assert block in (64, 128, 256, 512, 1024) and lpb in (1, 2, 4, 8, 16, 32)
        j.destroy()


@pytest.mark.parametrize("n", [300, 2500])
def test_forces_match_oracle_both_list_modes(gpu_ctx, n):
    sp = spec(n, 21, "free")
    g, o = pair(gpu_ctx, sp)
    g.rebuild(True, True)
    o.rebuild(True, True)
    f32, f64, a64 = o.forces()
    assert force_error(g.read(sopb.FORCES), f64, a64) <= FORCE_RTOL
    gpu_ctx.run([g], 30)
    o.advance(30)
    assert np.array_equal(g.read(sopb.SEEDS), o.read(sopb.SEEDS))
    assert np.max(np.abs(g.read(sopb.COORDS) - o.read(sopb.COORDS))) < 1e-3
    g.destroy()


@pytest.mark.parametrize("mode", ["ramp", "clamp", "indent", "free"])
def test_short_trajectory_tracks_oracle(gpu_ctx, mode):
    steps = 200
    g, o = pair(gpu_ctx, spec(150, 17, mode))
    gpu_ctx.run([g], steps)
    assert o.advance(steps) == 0
    assert g.status() == 0
    xg, xo = g.read(sopb.COORDS), o.read(sopb.COORDS)
    assert np.max(np.abs(xg - xo)) < 2e-3
    assert g.step() == o.step() == steps
    assert np.array_equal(g.read(sopb.SEEDS), o.read(sopb.SEEDS))
    Tg, To = g.read(sopb.TEMP), o.read(sopb.TEMP)
    assert np.allclose(Tg, To, rtol=1e-3, atol=1e-3)
    if mode == "ramp":
        sg, so = g.read(sopb.PULLSTATE), o.read(sopb.PULLSTATE)
        assert np.array_equal(sg[3:12], so[3:12])          # cantilever path: exact
        assert np.allclose(sg[:3], so[:3], atol=1e-4)       # spring force from coordinates
    if mode == "indent":
        tg, to = g.read(sopb.TIPSTATE), o.read(sopb.TIPSTATE)
        assert np.allclose(tg[:11], to[:11], rtol=1e-4, atol=1e-4)
    g.destroy()


def test_fixed_bead_is_exactly_fixed(gpu_ctx):
    g = gpu_ctx.job(spec(120, 8, "clamp"))
    x0 = g.read(sopb.COORDS)
    gpu_ctx.run([g], 500)
    x = g.read(sopb.COORDS)
    assert np.array_equal(x[0], x0[0])
    g.destroy()


def test_batch_invariance_alone_vs_mix(gpu_ctx):
    sizes = [60, 97, 200, 333, 600, 128, 450]
    specs = [spec(n, 100 + k, ["ramp", "clamp", "free", "indent"][k % 4], rng_seed=5000 + k) for k, n in enumerate(sizes)]
    alone = []
    for sp in specs:
        j = gpu_ctx.job(sp)
        gpu_ctx.run([j], 120)
        alone.append(j.read(sopb.COORDS))
        j.destroy()
    mix = [gpu_ctx.job(sp) for sp in specs]
    gpu_ctx.run(mix, 50)
    gpu_ctx.run(mix[::-1], 70)
    for j, a in zip(mix, alone):
        assert np.array_equal(j.read(sopb.COORDS), a)
        j.destroy()


def test_capacity_overflow_is_reported_and_isolated(gpu_ctx):
    bad = gpu_ctx.job(spec(100, 2, "free", max_pairs=3))
    good = gpu_ctx.job(spec(100, 2, "free"))
    gpu_ctx.run([bad, good], 20)
    gpu_ctx.sync()
    assert bad.status() == sopb.ERR_CAPACITY
    assert good.status() == 0
    step = bad.step()
    gpu_ctx.run([bad], 10)          # a failed job is not advanced further
    assert bad.step() == step
    bad.destroy()
    good.destroy()


def test_long_run_kinetic_temperature(gpu_ctx):
    g = gpu_ctx.job(spec(200, 31, "free", nav=1000))
    gpu_ctx.run([g], 2999)          # T accumulates from the reset at step 2000
    T = g.read(sopb.TEMP)
    assert abs(T.mean() / 999.0 - 0.6) < 0.05
    g.destroy()


def test_heating_updater_changes_noise(gpu_ctx):
    sp = spec(100, 6, "free", heating=1, initialT=0.1, deltaT=0.2, tempFreq=10)
    g, o = pair(gpu_ctx, sp)
    gpu_ctx.run([g], 45)
    o.advance(45)
    assert np.max(np.abs(g.read(sopb.COORDS) - o.read(sopb.COORDS))) < 1e-3
    g.destroy()
