"""Covariance of the hydrodynamic noise against FP64.

The Ermak-McCammon step moves bead coordinates by (h/zeta) D F plus the
noise (h/zeta) rho B g (src/Integrators/bdhitea_kernel.cu:303-361 for the
exact factor, :364-456 for TEA), g standard normal from the Hybrid Taus
stream.  With no forces (no bonds, no natives, el = 0) every step's
displacement is one noise sample s = dx / ((h/zeta) rho) of covariance
B B^T.  Replicas of one system with their own RNG seeds are reset to the same
coordinates x0 before every step, so all samples share one covariance, and
the library's B is the one built at x0 (the exact factor at step 0, TEA's
coefficients from x0).

Against the FP64 target K (the normalised RPY tensor D of x0 for the exact
factor; for TEA, B_TEA B_TEA^T of the reference's TEA formula in FP64):
  * trace statistic t = mean(s^T K^-1 s) / (3n) - 1, zero for Cov = K, with
    standard deviation sqrt(2 / (3n N)) from sampling alone; bar
    |t| <= 1e-4 + 5 sigma;
  * ||C_hat - K||_F / ||K||_F against its sampling floor
    sqrt((||K||_F^2 + tr(K)^2) / N) / ||K||_F; bar 1.1 x the floor.
For contrast, the reference's own exact-HI noise matrix (symmetrised upper
3x3 blocks of its in-place factor, hi_b_mode reference) misses D, and the
trace statistic sees it at many sigma; TEA's own departure from D (the
method's approximation, not an implementation error) is stated beside it.
Set SOPB_NOISE_LOG to a file to collect the numbers (one JSON line each).
"""
import json
import math
import os

import numpy as np
import pytest

import oracle_py as O
import sopb
import sopb_synth as S
from helpers import plain_params

pytestmark = pytest.mark.gpu


def record(**kw):
    path = os.environ.get("SOPB_NOISE_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(kw) + "\n")
    print(json.dumps(kw))


def free_spec(xyz, seed, seeds, **kw):
    """No bonds, no natives, no repulsion: forces are identically zero."""
    p = plain_params(el=0.0, hi_on=1, hi_a=3.8, hi_capricious=0, hi_epsilon_freq=10, hi_refresh=1 << 30, **kw)
    e2 = np.zeros((0, 2), np.int32)
    return sopb.JobSpec(xyz, e2, [], e2, [], [], p, seeds=seeds, seed=seed)


def tea_model(D, n):
    """B_TEA B_TEA^T in FP64: beta' and epsilon from the off-diagonal entries
    (src/Integrators/bdhitea.cu:143-169), C_i = 1 / sqrt(1 + beta'^2 sum of
    the squared off-diagonal row entries) per component, and
    B[(i,a),(i,a)] = C_i[a], B[(i,a),(q,b)] = beta' D_iq[a][b] C_i[b] for
    q != i (src/Integrators/bdhitea_kernel.cu:364-456)."""
    import torch
    m = 3 * n
    off = D.clone()
    blk = torch.arange(m, device=D.device) // 3
    off[blk[:, None] == blk[None, :]] = 0.0
    eps = float(off.sum()) / (3.0 * n * (3.0 * n - 3.0))
    a = (3.0 * n - 1.0) * eps * eps - (3.0 * n - 2.0) * eps
    beta = 0.5 if abs(a) < 1e-7 else (1.0 - math.sqrt(1.0 - a)) / a
    c = 1.0 / torch.sqrt(1.0 + beta * beta * (off * off).sum(dim=1))        # C_i[a], row (i, a)
    cb = c.view(n, 3)[blk].reshape(m, 1, 3)                                  # C_i[b] for row (i, a)
    B = beta * off * cb.expand(m, n, 3).reshape(m, m)
    B += torch.diag(c)
    return B @ B.T, beta, eps


def sample(exact, n, replicas, steps, seed=4000, b_mode=sopb.HI_B_CHOLESKY):
    import torch
    xyz = S.make_system(n, seed).xyz
    # one ran2 stream for all replicas, as the reference seeds its runs
    # (src/Integrators/ht.cu:40-56): fresh streams from nearby positive
    # seeds start from the same empty shuffle table and repeat their first
    # draws, which would correlate the first beads of every replica
    states = sopb.generate_seeds(20011, replicas * n)
    specs = [free_spec(xyz, 0, states[r * n:(r + 1) * n], hi_exact=int(exact), hi_b_mode=b_mode)
             for r in range(replicas)]
    m = 3 * n
    stream = torch.cuda.Stream()
    with sopb.Context(0, stream=stream.cuda_stream) as ctx:
        jobs = [ctx.job(sp) for sp in specs]
        x0 = np.zeros((replicas * n, 4), np.float32)
        ctx.download_coords(jobs, x0)
        p = specs[0].params
        var = math.sqrt(2.0 * p.temperature * p.zeta / p.timestep)
        scale = (p.timestep / p.zeta) * var
        x0_dev = torch.from_numpy(x0[:, :3].copy()).double().cuda()
        host = np.zeros_like(x0)
        C = torch.zeros((m, m), dtype=torch.float64, device="cuda")
        S_list = []
        for _ in range(steps):
            ctx.upload_coords(jobs, x0)
            ctx.run(jobs, 1)
            ctx.download_coords(jobs, host)
            s = (torch.from_numpy(host[:, :3]).cuda().double() - x0_dev) / scale   # (replicas*n, 3)
            s = s.view(replicas, m)
            C.addmm_(s.T, s)
            S_list.append(s)
        assert all(j.status() == 0 for j in jobs)
    N = replicas * steps
    C /= N
    D = torch.from_numpy(O.rpy_tensor(xyz, 3.8)).cuda()
    return C, torch.cat(S_list), D, N


def stats(C, Sm, K, N, m):
    import torch
    L = torch.linalg.cholesky(K)
    z = torch.linalg.solve_triangular(L, Sm.T, upper=False)
    t = float((z * z).sum()) / (N * m) - 1.0
    sigma = math.sqrt(2.0 / (m * N))
    nk = float(torch.linalg.matrix_norm(K))
    rel = float(torch.linalg.matrix_norm(C - K)) / nk
    floor = math.sqrt((nk * nk + float(torch.trace(K)) ** 2) / N) / nk
    return t, sigma, rel, floor


@pytest.mark.parametrize("n,replicas,steps", [(1000, 50, 2000), (4000, 20, 5000)])
def test_exact_hi_noise_covariance_is_D(n, replicas, steps):
    C, Sm, D, N = sample(True, n, replicas, steps)
    t, sigma, rel, floor = stats(C, Sm, D, N, 3 * n)
    record(case="exact", n=n, samples=N, trace_stat=t, sigma=sigma, rel_frobenius=rel, floor=floor)
    assert abs(t) <= 1e-4 + 5 * sigma, (t, sigma)
    assert rel <= 1.1 * floor, (rel, floor)


def test_tea_noise_covariance_is_its_fp64_model():
    n, replicas, steps = 4000, 20, 5000
    C, Sm, D, N = sample(False, n, replicas, steps)
    K, beta, eps = tea_model(D, n)
    t, sigma, rel, floor = stats(C, Sm, K, N, 3 * n)
    import torch
    method = float(torch.linalg.matrix_norm(K - D) / torch.linalg.matrix_norm(D))
    record(case="tea", n=n, samples=N, trace_stat=t, sigma=sigma, rel_frobenius=rel, floor=floor,
           beta=beta, epsilon=eps, tea_vs_D=method)
    assert abs(t) <= 1e-4 + 5 * sigma, (t, sigma)
    assert rel <= 1.1 * floor, (rel, floor)


def test_reference_noise_matrix_misses_D():
    # the same statistic on the reference's symmetrised noise matrix (the
    # reference's own sizes, n <= 128) detects its departure from D
    n, replicas, steps = 100, 200, 2000
    C, Sm, D, N = sample(True, n, replicas, steps, b_mode=sopb.HI_B_REFCOMPAT)
    t, sigma, rel, floor = stats(C, Sm, D, N, 3 * n)
    Cl, Sl, _, _ = sample(True, n, replicas, steps)
    tl, _, rell, _ = stats(Cl, Sl, D, N, 3 * n)
    record(case="exact_vs_reference_B", n=n, samples=N, sigma=sigma, floor=floor, trace_stat_reference_B=t,
           rel_frobenius_reference_B=rel, trace_stat_true_L=tl, rel_frobenius_true_L=rell)
    assert abs(t) > 20 * sigma or rel > 2 * floor, (t, sigma, rel, floor)
    assert abs(tl) <= 1e-4 + 5 * sigma and rell <= 1.1 * floor, (tl, rell, floor)
