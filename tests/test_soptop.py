"""The topology builders against the reference's own topology creators
(run by tests/golden/make_soptop_golden.py).  `sopb-top` (src/sop-top.cpp):
the .top file and the Calpha coordinates PDB byte for byte, for plain,
side-chain-contact, covalent-linker and tandem models.  `sopb-top2`
(src/sop-top2.cpp): the coarse-grained PDB, .top and the two PSF files byte
for byte, for one- and two-bead-per-residue descriptions, segments or
chains, and an extra-bond file.  The one tolerated
difference: the reference leaves the alternate-location column of its linker
beads uninitialised (a NUL byte in the golden files); sopb-top writes a
space there."""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
GOLD = os.path.join(HERE, "golden")
TOOL = os.path.join(REPO, "sop-gpu_b200", "sopb-top")
TOOL2 = os.path.join(REPO, "sop-gpu_b200", "sopb-top2")
sys.path.insert(0, GOLD)
import soptop_cases  # noqa: E402


@pytest.fixture(scope="module")
def tool():
    if not (os.path.exists(TOOL) and os.path.exists(TOOL2)):
        subprocess.check_call(["make", "-s", "-C", os.path.join(REPO, "sop-gpu_b200")])
    return TOOL


@pytest.mark.parametrize("name", list(soptop_cases.CG_CASES))
def test_coarse_grained_model_matches_reference_tool(tmp_path, tool, name):
    g = np.load(os.path.join(GOLD, "soptop.npz"))
    cfg = soptop_cases.write_cg_case(name, str(tmp_path))
    r = subprocess.run([TOOL2, os.path.basename(cfg)], cwd=str(tmp_path), capture_output=True, text=True,
                       stdin=subprocess.DEVNULL)
    assert r.returncode == 0, r.stderr
    for f in (name + "_cg.pdb", name + ".top", name + ".psf", name + "_nat.psf"):
        with open(tmp_path / f, "rb") as fh:
            assert fh.read() == bytes(g[f]), f


@pytest.mark.parametrize("name", list(soptop_cases.CASES))
def test_model_matches_reference_tool(tmp_path, tool, name):
    g = np.load(os.path.join(GOLD, "soptop.npz"))
    cfg = soptop_cases.write_case(name, str(tmp_path))
    r = subprocess.run([tool, os.path.basename(cfg)], cwd=str(tmp_path), capture_output=True, text=True,
                       stdin=subprocess.DEVNULL)
    assert r.returncode == 0, r.stderr
    for f in (name + ".top", name + "_ca.pdb"):
        with open(tmp_path / f, "rb") as fh:
            mine = fh.read()
        assert mine == bytes(g[f]).replace(b"\x00", b" "), f


def test_existing_coordinates_kept_without_yes(tmp_path, tool):
    cfg = soptop_cases.write_case("basic", str(tmp_path))
    (tmp_path / "basic_ca.pdb").write_text("keep\n")
    r = subprocess.run([tool, os.path.basename(cfg)], cwd=str(tmp_path), input="n\n", capture_output=True, text=True)
    assert r.returncode == 0 and "Overwrite" in r.stdout
    assert (tmp_path / "basic_ca.pdb").read_text() == "keep\n"
    r = subprocess.run([tool, os.path.basename(cfg)], cwd=str(tmp_path), input="y\n", capture_output=True, text=True)
    assert (tmp_path / "basic_ca.pdb").read_text().startswith("ATOM")


def test_top_loads_into_the_simulation_format(tmp_path, tool):
    # the builder's output is read back by the simulation's topology reader
    import sopb_synth as S
    cfg = soptop_cases.write_case("basic", str(tmp_path))
    subprocess.run([tool, os.path.basename(cfg)], cwd=str(tmp_path), check=True, capture_output=True,
                   stdin=subprocess.DEVNULL)
    sysm = S.load_system(str(tmp_path / "basic.top"), str(tmp_path / "basic_ca.pdb"))
    assert sysm.n == 70 and len(sysm.bonds) >= 68 and len(sysm.natives) > 0
