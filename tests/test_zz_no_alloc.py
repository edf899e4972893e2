"""The no-allocation entry point sopb_tea_coefficients_noalloc.

It is for callers that cannot call cudaMalloc (a host program that owns all
device memory through its own pool, or code ordering work on a stream where
an allocation would stall or break it).  It computes TEA's per-bead coupling
sums and the job's beta' and epsilon from caller-owned device buffers, with
its scratch in a static array of the library.  Here it is called through the
C ABI on device buffers the test owns, twice in a row, and compared with the
beta' and epsilon the TEA updater of sopb_run computes for the same
coordinates (read with SOPB_HISTATE).
"""
import ctypes

import numpy as np
import pytest

import sopb
from helpers import spec

pytestmark = pytest.mark.gpu

RTOL = 1e-5   # the bar of the TEA beta'/epsilon parity tests


@pytest.mark.parametrize("n", [300, 2000])
def test_noalloc_tea_coefficients_match_tea_updater(n):
    import torch
    sp = spec(n, 31, "free", hi_on=1, hi_a=1.9, hi_epsilon_freq=10, hi_capricious=0)
    with sopb.Context(0) as ctx:
        job = ctx.job(sp)
        ctx.run([job], 1)                     # the TEA updater runs at step 0
        ref = job.read(sopb.HISTATE)[:2]
        job.destroy()
    assert 0.0 < ref[0] < 1.0 and 0.0 < ref[1] < 1.0
    x = np.zeros((n, 4), np.float32)
    x[:, :3] = sp.xyz
    d_x = torch.from_numpy(x).cuda()
    d_ci = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    d_be = torch.empty(2, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for _ in range(2):                        # two calls in a row share the static scratch
        d_ci.fill_(float("nan"))
        d_be.fill_(float("nan"))
        rc = sopb.lib().sopb_tea_coefficients_noalloc(d_x.data_ptr(), n, ctypes.c_float(1.9), d_ci.data_ptr(),
                                                      d_be.data_ptr(), stream)
        assert rc == sopb.OK
        torch.cuda.synchronize()
        be = d_be.cpu().numpy()
        assert abs(be[0] - ref[0]) <= RTOL * ref[0], (be, ref)
        assert abs(be[1] - ref[1]) <= RTOL * ref[1], (be, ref)
        ci = d_ci.cpu().numpy()
        assert np.isfinite(ci).all()
        # epsilon is the mean of the per-bead sums over the off-diagonal entries
        assert abs(ci[:, 3].astype(np.float64).sum() / (3.0 * n * (3.0 * n - 3.0)) - be[1]) <= RTOL * be[1]
        outs.append((be, ci))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    d = torch.empty(8, dtype=torch.float32, device="cuda")
    rc = sopb.lib().sopb_tea_coefficients_noalloc(d.data_ptr(), (1 << 18) + 1, ctypes.c_float(1.9), d.data_ptr(),
                                                  d.data_ptr(), None)
    assert rc == sopb.ERR_CAPACITY
    assert sopb.lib().sopb_tea_coefficients_noalloc(None, 10, ctypes.c_float(1.9), None, None, None) == sopb.ERR_INVALID
