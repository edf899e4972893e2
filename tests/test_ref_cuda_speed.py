"""Speed against the reference's own CUDA path on the same GPU.

The reference's CUDA build (oracle/_ref/ref_gpu, compiled from the SOP-GPU
tree for sm_100a by oracle/build_ref.sh) times its runGPU loop on the speed
cases of tests/golden/ref_cases.py: the plain 200-bead ramp pull, 512
force-clamp replicas of one 200-bead system (the reference runs replicas of
one topology only), TEA at 4000 beads, exact HI at 128 beads (the largest
the reference runs) and the 198 000-bead capsid shell.  The same configs go through this
library's C ABI on the same inputs.  Both sides are timed on the host around
the whole loop with the device synchronised, set-up excluded.  Bar: this
library is faster on every case.  With SOPB_SPEED_LOG set, the numbers are
written there as JSON lines.
"""
import json
import os
import subprocess
import sys
import time

import pytest

import sopb
import sopb_config as CFG
from test_ref_gpu_golden import GOLD

sys.path.insert(0, GOLD)
import ref_cases  # noqa: E402

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_GPU = os.path.join(REPO, "oracle", "_ref", "ref_gpu")

pytestmark = pytest.mark.gpu

SPEED = [c for c in ref_cases.CASES if ref_cases.CASES[c].get("speed")]


def reference_rate(name, d):
    c = ref_cases.CASES[name]
    cfg = ref_cases.write_inputs(name, d)
    r = subprocess.run([REF_GPU, os.path.basename(cfg), d, str(c["total"])], cwd=d, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("ref_gpu_time")][0]
    return float(line.split()[2])


def our_rate(name):
    c = ref_cases.CASES[name]
    jc = CFG.job_config(CFG.Config(text=ref_cases.config_text(name)))
    specs = CFG.job_specs(jc, ref_cases.systems(name))
    ctx = sopb.Context(0)
    try:
        jobs = [ctx.job(sp) for sp in specs]
        ctx.run(jobs, min(c["total"], 200))       # warm-up: lists, caches, graphs
        ctx.sync()
        t0 = time.perf_counter()
        ctx.run(jobs, c["total"])
        ctx.sync()
        secs = time.perf_counter() - t0
        for j in jobs:
            assert j.status() == 0
        return sum(sp.n for sp in specs) * c["total"] / secs
    finally:
        ctx.close()


@pytest.mark.parametrize("name", SPEED)
def test_faster_than_reference_cuda(tmp_path, name):
    if not os.path.exists(REF_GPU):
        pytest.skip("the reference's CUDA build is not present")
    ref = reference_rate(name, str(tmp_path))
    ours = our_rate(name)
    log = os.environ.get("SOPB_SPEED_LOG")
    if log:
        with open(log, "a") as f:
            f.write(json.dumps({"case": name, "reference_cuda": ref, "sopb": ours, "ratio": ours / ref}) + "\n")
    assert ours > ref, (name, ours, ref)
