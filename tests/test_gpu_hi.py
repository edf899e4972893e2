"""Hydrodynamic interactions on the CUDA path against the oracle: TEA with
all-pairs and listed couplings, and exact HI (n <= 128) with the true
Cholesky factor and with the reference-compatible noise matrix."""
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


def test_exact_hi_above_128_beads_is_reported_unsupported(gpu_ctx):
    with pytest.raises(sopb.SopbError) as e:
        gpu_ctx.job(hi_spec(200, 1, hi_exact=1))
    assert e.value.code == sopb.ERR_UNSUPPORTED


def test_hi_with_minimization_is_rejected(gpu_ctx):
    with pytest.raises(sopb.SopbError) as e:
        gpu_ctx.job(hi_spec(50, 1, minimization=1))
    assert e.value.code == sopb.ERR_INVALID
