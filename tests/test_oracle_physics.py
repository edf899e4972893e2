"""Known-answer checks of the oracle's restated kernels on hand-built
geometries, and of the loop semantics (updater order, stride, pulling)."""
import math

import numpy as np
import pytest

import oracle_py as O
import sopb
from helpers import spec, system


def two_bead(r, **kw):
    xyz = np.array([[0.0, 0.0, 0.0], [r, 0.0, 0.0]], np.float32)
    return xyz


def job(xyz, bonds=(), r0=(), natives=(), nr0=(), neh=(), **kw):
    p = sopb.default_params(timestep=0.08, **kw)
    s = sopb.JobSpec(xyz, np.array(bonds, np.int32).reshape(-1, 2), np.array(r0, np.float32),
                     np.array(natives, np.int32).reshape(-1, 2), np.array(nr0, np.float32),
                     np.array(neh, np.float32), p, seed=7)
    return O.OracleJob(s)


def test_fene_two_beads():
    # U = -(k/2) R0^2 log(1 - (r-r0)^2/R0^2);  F_1 = k (r-r0)/(1-(r-r0)^2/R0^2) * x_hat
    r, r0, k, R = 4.3, 3.8, 20.0, 2.0
    j = job(two_bead(r), bonds=[(0, 1)], r0=[r0])
    f32, f64, _ = j.forces()
    d = r - r0
    expect = k * d / (1 - d * d / (R * R))
    assert f64[0, 0] == pytest.approx(expect, rel=1e-6)
    assert f32[0, 0] == pytest.approx(expect, rel=1e-5)
    assert f32[1, 0] == pytest.approx(-expect, rel=1e-5)


def test_native_lj_zero_at_r0_and_known_value():
    r0, eh = 5.5, 1.5
    j = job(two_bead(r0), natives=[(0, 1)], nr0=[r0], neh=[eh])
    f32, f64, _ = j.forces()
    assert abs(f64[0, 0]) < 1e-12 and abs(f32[0, 0]) < 1e-5
    r = 6.2
    j = job(two_bead(r), natives=[(0, 1)], nr0=[r0], neh=[eh])
    f32, f64, _ = j.forces()
    # U = eh((r0/r)^12 - 2 (r0/r)^6); F_1,x = dU/dr = -12 eh/r ((r0/r)^12 - (r0/r)^6)
    s = r0 / r
    expect = -12.0 * eh / r * (s ** 12 - s ** 6)
    assert f64[0, 0] == pytest.approx(expect, rel=1e-6)  # coordinates are float32
    assert f32[0, 0] == pytest.approx(expect, rel=1e-5)


def test_repulsion_and_cutoffs():
    # pairlist cutoff 20: a pair at exactly 20.0 is not listed (sqrtf(400) < 20 is false)
    xyz = np.array([[0, 0, 0], [20.0, 0, 0], [0, 19.999998, 0], [0, 0, 4.0]], np.float32)
    j = job(xyz)
    j.rebuild(True, True)
    cnt, rows = j.pairlist(False, cap=3)
    assert 1 not in rows[0, :cnt[0]]
    assert 2 in rows[0, :cnt[0]] and 3 in rows[0, :cnt[0]]
    f32, f64, _ = j.forces()
    # bead 3 at 4 A: F_0,z = -6 el a^6 / r^7 (pointing away from bead 3)
    a, el = 3.8, 1.0
    fz = -6 * el * a ** 6 / 4.0 ** 7
    assert f64[0, 2] == pytest.approx(fz, rel=1e-6)
    assert f32[0, 2] == pytest.approx(fz, rel=1e-5)


def test_possible_pairs_exclude_bonded_and_native():
    xyz = np.array([[0, 0, 0], [3.8, 0, 0], [7.6, 0, 0], [0, 5.0, 0], [100, 0, 0]], np.float32)
    j = job(xyz, bonds=[(0, 1), (1, 2)], r0=[3.8, 3.8], natives=[(0, 3)], nr0=[5.0], neh=[1.5], pairs_threshold=50.0)
    j.rebuild(True, False)
    cnt, rows = j.pairlist(True, cap=4)
    assert list(rows[0, :cnt[0]]) == [2]           # 1 bonded, 3 native, 4 beyond threshold
    assert list(rows[3, :cnt[3]]) == [1, 2]        # increasing index order
    assert cnt[4] == 0


def test_rpy_block_both_branches():
    a = 1.9
    for r in (3.0, 5.0, 12.0):
        xyz = np.array([[0, 0, 0], [r * 0.6, r * 0.8, 0.0]], np.float32)
        D = O.rpy_tensor(xyz, a)
        e = np.array([0.6, 0.8, 0.0])
        ra = r / a
        if ra > 2:
            crr, cii = 0.75 / ra * (1 - 2 / ra ** 2), 0.75 / ra * (1 + 2 / (3 * ra ** 2))
        else:
            crr, cii = 3 * ra / 32, 1 - 9 * ra / 32
        want = crr * np.outer(e, e) + cii * np.eye(3)
        assert np.allclose(D[0:3, 3:6], want, atol=1e-12)
        assert np.allclose(D, D.T)


def test_gaussians_are_standard_normal():
    s = O.generate_seeds(99, 50000)
    g, s2 = O.rforce(s)
    assert not np.array_equal(s, s2)
    v = g.reshape(-1).astype(np.float64)
    assert abs(v.mean()) < 0.01 and abs(v.var() - 1.0) < 0.01
    assert abs(np.mean(v ** 4) - 3.0) < 0.05


def test_reference_exact_hi_noise_factor_is_biased():
    # integrateCholesky_L reads symmetrised upper 3x3 blocks of the factor
    # (bdhitea_kernel.cu:322-334): B'B'^T differs from D by ~10%.
    xyz = system(40, 5).xyz
    D = O.rpy_tensor(xyz, 1.9)
    M = O.cholesky_ref(D.astype(np.float32))
    L = np.tril(M).astype(np.float64)
    assert np.linalg.norm(L @ L.T - D) / np.linalg.norm(D) < 1e-5
    B = O.ref_b_matrix(40, M)
    err = np.linalg.norm(B @ B.T - D) / np.linalg.norm(D)
    assert 0.03 < err < 0.3


def test_ramp_cantilever_moves_per_pullfreq():
    sp = spec(60, 3, "ramp")
    j = O.OracleJob(sp)
    j.advance(35)     # updaters at 0,10,20,30 (stride = pullFreq = pairs_freq = 10)
    st = j.read(sopb.PULLSTATE)
    cant, cant0, vec = st[3:6], st[6:9], st[9:12]
    xt = np.float32(sp.params.deltax) * np.float32(30 // 10)
    assert np.allclose(cant, cant0 + xt * vec, atol=1e-6)
    assert abs(np.linalg.norm(vec) - 1.0) < 1e-6


def test_fixed_bead_never_moves_and_temperature_is_sane():
    sp = spec(80, 4, "clamp")
    j = O.OracleJob(sp)
    x0 = j.read(sopb.COORDS)
    assert j.advance(1000) == 0
    x = j.read(sopb.COORDS)
    assert np.array_equal(x[0], x0[0])
    assert not np.array_equal(x[79], x0[79])
    # kinetic temperature accumulator averaged over nav steps ~ T = 0.6
    T = j.read(sopb.TEMP).mean() / 1000.0
    assert 0.5 < T < 0.7


def test_capacity_overflow_is_an_error():
    sp = spec(60, 3, "free", max_pairs=4)
    j = O.OracleJob(sp)
    assert j.advance(1) == sopb.ERR_CAPACITY
