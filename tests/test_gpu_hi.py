"""Hydrodynamic interactions on the CUDA path against the oracle: TEA with
all-pairs and listed couplings, and exact HI with the true Cholesky factor
(the reference's single-CTA factorisation up to 128 beads, the blocked one
above, refreshed every step or every hi_refresh steps) and with the
reference-compatible noise matrix."""
import numpy as np
import pytest

import oracle_py as O
import sopb
from helpers import spec

pytestmark = pytest.mark.gpu


def hi_spec(n, seed, mode="free", **kw):
    base = dict(hi_on=1, hi_a=1.9, hi_epsilon_freq=10, hi_capricious=0)
    base.update(kw)
    return spec(n, seed, mode, **base)


@pytest.mark.parametrize("n,unlisted,mode", [(100, 1, "free"), (100, 0, "free"), (257, 1, "clamp"), (257, 0, "ramp"),
                                             (1500, 1, "free")])
def test_tea_tracks_oracle(gpu_ctx, n, unlisted, mode):
    sp = hi_spec(n, 23, mode, hi_unlisted=unlisted)
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    steps = 25 if n < 1000 else 12
    gpu_ctx.run([g], steps)
    assert o.advance(steps) == 0
    assert g.status() == 0
    assert np.array_equal(g.read(sopb.SEEDS), o.read(sopb.SEEDS))
    dx = np.max(np.abs(g.read(sopb.COORDS) - o.read(sopb.COORDS)))
    assert dx < 1e-4, dx
    g.destroy()


@pytest.mark.parametrize("n,unlisted", [(100, 1), (300, 1), (300, 0), (2000, 1)])
def test_tea_beta_and_epsilon_match_oracle(gpu_ctx, n, unlisted):
    sp = hi_spec(n, 31, "free", hi_unlisted=unlisted)
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    gpu_ctx.run([g], 1)            # the TEA updater runs at step 0
    assert o.advance(1) == 0
    hg, ho = g.read(sopb.HISTATE), o.read(sopb.HISTATE)
    assert 0.0 < ho[1] < 1.0 and 0.0 < ho[0] < 1.0
    assert abs(hg[1] - ho[1]) <= 1e-5 * ho[1] and abs(hg[0] - ho[0]) <= 1e-5 * ho[0]
    g.destroy()


@pytest.mark.parametrize("bmode", [sopb.HI_B_CHOLESKY, sopb.HI_B_REFCOMPAT])
@pytest.mark.parametrize("n", [20, 40, 128])
def test_exact_hi_tracks_oracle(gpu_ctx, n, bmode):
    sp = hi_spec(n, 29, "clamp", hi_exact=1, hi_b_mode=bmode)
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    gpu_ctx.run([g], 5)
    assert o.advance(5) == 0
    assert g.status() == 0
    assert np.array_equal(g.read(sopb.SEEDS), o.read(sopb.SEEDS))
    dx = np.max(np.abs(g.read(sopb.COORDS) - o.read(sopb.COORDS)))
    assert dx < 1e-3, dx
    g.destroy()


def test_reference_noise_matrix_above_128_beads_is_unsupported(gpu_ctx):
    # the symmetrised-upper-block B exists for the reference's sizes only
    with pytest.raises(sopb.SopbError) as e:
        gpu_ctx.job(hi_spec(200, 1, hi_exact=1, hi_b_mode=sopb.HI_B_REFCOMPAT))
    assert e.value.code == sopb.ERR_UNSUPPORTED


@pytest.mark.parametrize("n", [20, 90, 128, 129, 200, 451])
def test_factor_matches_fp64_cholesky(gpu_ctx, n):
    # up to 128 beads the panel factor in one CTA, above it the tiled one
    sp = hi_spec(n, 37, "free", hi_exact=1)
    g = gpu_ctx.job(sp)
    x0 = g.read(sopb.COORDS)[:, :3].copy()
    gpu_ctx.run([g], 1)                       # step 0 factorises D at x0
    assert g.status() == 0
    L = np.tril(g.read(sopb.HIFACTOR).astype(np.float64))
    D = O.rpy_tensor(x0, sp.params.hi_a)
    L64 = np.linalg.cholesky(D)
    assert np.max(np.abs(L - L64)) < 2e-4
    assert np.linalg.norm(L @ L.T - D) / np.linalg.norm(D) < 2e-6
    g.destroy()


@pytest.mark.parametrize("w", [1, 2, 3, 4, 8])
def test_blocked_factor_panel_widths(w):
    # the factorisation's three streams (single-tile chain, tile-column rest,
    # trailing updates) for several outer-panel widths at 17 tile columns:
    # the factor against FP64, and bit-identical when the same job runs
    # again beside another exact-HI job, so that the streams interleave
    # differently
    n = 700
    sp = hi_spec(n, 47, "free", hi_exact=1)
    with sopb.Context(0) as ctx:
        ctx.set_hi_policy(w, 8)
        g = ctx.job(sp)
        x0 = g.read(sopb.COORDS)[:, :3].copy()
        ctx.run([g], 1)                       # step 0 factorises D at x0
        assert g.status() == 0
        L1 = np.tril(g.read(sopb.HIFACTOR))
        g2 = ctx.job(sp)
        other = ctx.job(hi_spec(900, 5, "free", hi_exact=1))
        ctx.run([g2, other], 1)
        assert g2.status() == 0 and other.status() == 0
        L2 = np.tril(g2.read(sopb.HIFACTOR))
    assert np.array_equal(L1, L2)
    L = L1.astype(np.float64)
    D = O.rpy_tensor(x0, sp.params.hi_a)
    assert np.max(np.abs(L - np.linalg.cholesky(D))) < 2e-4
    assert np.linalg.norm(L @ L.T - D) / np.linalg.norm(D) < 2e-6


@pytest.mark.parametrize("n,refresh", [(150, 1), (300, 1), (300, 10), (100, 10)])
def test_exact_hi_with_refresh_tracks_oracle(gpu_ctx, n, refresh):
    # the blocked factorisation above 128 beads and the refresh updater on
    # both paths against the oracle's column Cholesky
    sp = hi_spec(n, 41, "clamp", hi_exact=1, hi_refresh=refresh)
    g, o = gpu_ctx.job(sp), O.OracleJob(sp)
    steps = 23
    gpu_ctx.run([g], steps)
    assert o.advance(steps) == 0
    assert g.status() == 0
    assert np.array_equal(g.read(sopb.SEEDS), o.read(sopb.SEEDS))
    dx = np.max(np.abs(g.read(sopb.COORDS) - o.read(sopb.COORDS)))
    assert dx < 1e-3, dx
    g.destroy()


def test_stale_factor_differs_from_fresh_one(gpu_ctx):
    # with refresh 10 the factor read after 5 steps is still the step-0 one
    sp = hi_spec(200, 43, "free", hi_exact=1, hi_refresh=10)
    g = gpu_ctx.job(sp)
    gpu_ctx.run([g], 1)
    L0 = g.read(sopb.HIFACTOR).copy()
    gpu_ctx.run([g], 4)
    assert np.array_equal(np.tril(g.read(sopb.HIFACTOR)), np.tril(L0))
    gpu_ctx.run([g], 6)                       # step 10 refreshes
    assert not np.array_equal(np.tril(g.read(sopb.HIFACTOR)), np.tril(L0))
    g.destroy()


def test_hi_with_minimization_is_rejected(gpu_ctx):
    with pytest.raises(sopb.SopbError) as e:
        gpu_ctx.job(hi_spec(50, 1, minimization=1))
    assert e.value.code == sopb.ERR_INVALID
