"""The C++ host mirror (plugin surface, config reader, .top/PDB IO) and its
command-line driver `sopb-gpu`, which has the reference's usage."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CLI = os.path.join(REPO, "sop-gpu_b200", "sopb-gpu")
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, GOLD)


def build():
    """Builds the driver when it is missing (a prebuilt one is used as is)."""
    if not os.path.exists(CLI):
        subprocess.check_call(["make", "-s", "-C", os.path.join(REPO, "sop-gpu_b200")])


def test_cli_config_parse_matches_reference():
    build()
    with open(os.path.join(GOLD, "config.json")) as f:
        g = json.load(f)
    args = [CLI, "--dump-config", os.path.join(GOLD, "config_sample.sop")]
    for k, t in g["keys"]:
        args += [k, t]
    out = subprocess.check_output(args).decode()
    got = dict(line.split("\t", 1) for line in out.splitlines())
    assert got == g["parsed"]


def test_cli_reports_errors_as_status(tmp_path):
    build()
    cfg = tmp_path / "bad.sop"
    cfg.write_text("topology\tnone.top\n")
    r = subprocess.run([CLI, str(cfg)], capture_output=True, text=True)
    assert r.returncode != 0 and "sopb-gpu:" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["pull2", "indent", "tea"])
def test_cli_run_matches_reference_cuda(tmp_path, name):
    import ref_cases
    build()
    d = str(tmp_path)
    cfg = ref_cases.write_inputs(name, d)
    c = ref_cases.CASES[name]
    g = np.load(os.path.join(GOLD, "ref_gpu_%s.npz" % name))
    stride = int(g["stride"])
    total = c["dumps"][-1]
    numsteps = total - stride        # the loop runs (numsteps/stride + 1) * stride steps
    r = subprocess.run([CLI, os.path.basename(cfg), "numsteps=%d" % numsteps], cwd=d, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    first = int(c["cfg"].get("firstrun", c["cfg"].get("run", "1")))
    n = c["n"]
    for k in range(c["runs"]):
        pdb = os.path.join(d, "%s_%d_final.pdb" % (name, first + k))
        x = np.array([[float(l[30:38]), float(l[38:46]), float(l[46:54])] for l in open(pdb) if l.startswith("ATOM")])
        ref = g["coords_%d" % total][k * n:(k + 1) * n, :3]
        assert np.max(np.abs(x - ref)) <= 5e-4 + 1e-4
