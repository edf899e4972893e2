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
    # a caller's pool may hand out buffers at any offset: float4 buffers off
    # a 16-byte boundary are refused instead of faulting
    buf = torch.zeros(64, dtype=torch.float32, device="cuda")
    base = buf.data_ptr()
    assert base % 256 == 0
    for xo, co, bo in ((4, 0, 0), (8, 0, 0), (0, 4, 0), (0, 0, 2)):
        rc = sopb.lib().sopb_tea_coefficients_noalloc(base + xo, 2, ctypes.c_float(1.9), base + 64 + co,
                                                      base + 128 + bo, None)
        assert rc == sopb.ERR_INVALID, (xo, co, bo)
    torch.cuda.synchronize()


def _noalloc_on_primary_context(x, n, a):
    import torch
    d_x = torch.from_numpy(x).cuda()
    d_ci = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    d_be = torch.empty(2, dtype=torch.float32, device="cuda")
    rc = sopb.lib().sopb_tea_coefficients_noalloc(d_x.data_ptr(), n, ctypes.c_float(a), d_ci.data_ptr(),
                                                  d_be.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == sopb.OK
    torch.cuda.synchronize()
    return d_ci.cpu().numpy(), d_be.cpu().numpy()


def test_noalloc_in_a_context_of_its_own():
    """A host that creates its own CUDA context (cuCtxCreate) gets the
    scratch address of that context, not the one cached for the primary
    context: the results are bit-identical to the primary context's, and the
    primary context still works after the other one is destroyed."""
    from cuda.bindings import driver as cu
    n, a = 500, 1.9
    sp = spec(n, 5, "free")
    x = np.zeros((n, 4), np.float32)
    x[:, :3] = sp.xyz
    ci0, be0 = _noalloc_on_primary_context(x, n, a)

    def ok(res):
        err = res[0] if isinstance(res, tuple) else res
        assert err == cu.CUresult.CUDA_SUCCESS, err
        return res[1] if isinstance(res, tuple) and len(res) > 1 else None

    ok(cu.cuInit(0))
    dev = ok(cu.cuDeviceGet(0))
    ctx = ok(cu.cuCtxCreate(0, dev))
    try:
        d_x = ok(cu.cuMemAlloc(x.nbytes))
        d_ci = ok(cu.cuMemAlloc(x.nbytes))
        d_be = ok(cu.cuMemAlloc(8))
        ok(cu.cuMemcpyHtoD(d_x, x.ctypes.data, x.nbytes))
        for _ in range(2):
            rc = sopb.lib().sopb_tea_coefficients_noalloc(int(d_x), n, ctypes.c_float(a), int(d_ci), int(d_be), None)
            assert rc == sopb.OK
            ok(cu.cuCtxSynchronize())
            ci = np.empty_like(x)
            be = np.empty(2, np.float32)
            ok(cu.cuMemcpyDtoH(ci.ctypes.data, d_ci, ci.nbytes))
            ok(cu.cuMemcpyDtoH(be.ctypes.data, d_be, be.nbytes))
            assert np.array_equal(be, be0) and np.array_equal(ci, ci0)
        for d in (d_x, d_ci, d_be):
            ok(cu.cuMemFree(d))
    finally:
        ok(cu.cuCtxDestroy(ctx))
    ci1, be1 = _noalloc_on_primary_context(x, n, a)
    assert np.array_equal(be1, be0) and np.array_equal(ci1, ci0)
