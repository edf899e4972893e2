"""The oracle and the product's host code against golden vectors produced
by the reference's own host code (tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

import oracle_py as O
import sopb
import sopb_synth as S

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _seeds():
    with open(os.path.join(GOLD, "seeds.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("case", sorted(_seeds().keys()))
def test_oracle_seeds_match_reference(case):
    seed, count = (int(v) for v in case.split(":"))
    gold = np.array(_seeds()[case], np.uint64).astype(np.uint32).reshape(-1, 4)
    assert np.array_equal(O.generate_seeds(seed, count), gold)


@pytest.mark.parametrize("case", sorted(_seeds().keys()))
def test_library_seeds_match_reference(case):
    # host function of the C ABI: runs without a GPU
    seed, count = (int(v) for v in case.split(":"))
    gold = np.array(_seeds()[case], np.uint64).astype(np.uint32).reshape(-1, 4)
    assert np.array_equal(sopb.generate_seeds(seed, count), gold)


def test_multirun_seed_stream_is_one_sequence():
    # runnum replicas draw from one ran2 stream: replica k's states are the
    # k-th block of a single generateSeeds call (ht.cu:40-56)
    s = sopb.generate_seeds(1119727, 64)
    gold = np.array(_seeds()["1119727:256"], np.uint64).astype(np.uint32).reshape(-1, 4)
    assert np.array_equal(s, gold[:64])


def test_synthetic_inputs_read_identically_by_reference_parser():
    with open(os.path.join(GOLD, "topology.json")) as f:
        g = json.load(f)
    sys_ = S.make_system(g["n"], g["seed"])
    assert g["atoms"] == sys_.n
    gb = np.array([[b[0], b[1]] for b in g["bonds"]], np.int32)
    assert np.array_equal(gb, sys_.bonds)
    assert np.array_equal(np.array([float(b[2]) for b in g["bonds"]], np.float32), sys_.bonds_r0)
    gn = np.array([[b[0], b[1]] for b in g["natives"]], np.int32)
    assert np.array_equal(gn, sys_.natives)
    assert np.array_equal(np.array([float(b[2]) for b in g["natives"]], np.float32), sys_.natives_r0)
    assert np.array_equal(np.array([float(b[3]) for b in g["natives"]], np.float32), sys_.natives_eh)
    gx = np.array([[float(v) for v in r] for r in g["xyz"]], np.float32)
    assert np.array_equal(gx, sys_.xyz)


def test_python_file_readers_match_reference(tmp_path):
    with open(os.path.join(GOLD, "topology.json")) as f:
        g = json.load(f)
    sys_ = S.make_system(g["n"], g["seed"])
    S.save_system(str(tmp_path / "s"), sys_)
    back = S.load_system(str(tmp_path / "s.top"), str(tmp_path / "s.pdb"))
    assert np.array_equal(back.xyz, sys_.xyz)
    assert np.array_equal(back.bonds, sys_.bonds)
    assert np.array_equal(back.natives_r0, sys_.natives_r0)
