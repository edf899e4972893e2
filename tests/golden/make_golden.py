"""Generates the golden fixtures in this directory from the reference's own
host code (compiled from the SOP-GPU source tree by oracle/build_ref.sh).

    python tests/golden/make_golden.py [path-to-SOP-GPU]

Fixtures written:
  seeds.json     generateSeeds() over ran2 for several seeds (ht.cu:40-56)
  config.json    configreader parse of config_sample.sop (configreader.cpp)
  topology.json  SOP::load + readCoord of a synthetic system written by
                 sopb_synth (topio.cpp:36-80, pdbio.cpp:292-337)
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, os.path.join(REPO, "sop-gpu_b200"))
import sopb_synth  # noqa: E402

REF_HOST = os.path.join(REPO, "oracle", "_ref", "ref_host")

SEED_CASES = [(1119727, 256), (5032015, 64), (1, 16), (0, 8), (-12345, 8), (2147483000, 8)]

CONFIG_KEYS = [
    ("name", "str"), ("topology", "str"), ("coordinates", "str"), ("timestep", "float"), ("zeta", "float"),
    ("temperature", "float"), ("seed", "int"), ("runnum", "int"), ("firstrun", "int"), ("pulling", "bool"),
    ("indentation", "bool"), ("hi_on", "bool"), ("fixed", "ints"), ("pulled", "ints"), ("pullVector", "float3"),
    ("indentationChip", "float3"), ("pairs_freq", "int"), ("deltax", "float"), ("outputname", "str"),
    ("empty_list", "ints"), ("missing_key", "str"),
]


def run(*args):
    return subprocess.check_output([REF_HOST] + [str(a) for a in args]).decode()


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SOPB_REFERENCE_DIR", "/root/reference")
    subprocess.check_call([os.path.join(REPO, "oracle", "build_ref.sh"), ref])
    if not os.path.exists(REF_HOST):
        sys.exit("reference harness not built")
    # seeds
    seeds = {}
    for s, n in SEED_CASES:
        vals = [int(v) for v in run("seeds", s, n).split()]
        seeds["%d:%d" % (s, n)] = vals
    with open(os.path.join(HERE, "seeds.json"), "w") as f:
        json.dump(seeds, f)
    # config
    cfg = os.path.join(HERE, "config_sample.sop")
    args = []
    for k, t in CONFIG_KEYS:
        args += [k, t]
    out = run("config", cfg, *args)
    parsed = {}
    for line in out.splitlines():
        k, _, v = line.partition("\t")
        parsed[k] = v
    with open(os.path.join(HERE, "config.json"), "w") as f:
        json.dump({"keys": CONFIG_KEYS, "parsed": parsed}, f, indent=1)
    # topology + coordinates round trip
    sys_ = sopb_synth.make_system(48, 2024)
    tmp = os.path.join(HERE, "_tmp_sys")
    sopb_synth.save_system(tmp, sys_)
    top = run("top", tmp + ".top")
    coords = run("coords", tmp + ".top", tmp + ".pdb")
    os.remove(tmp + ".top")
    os.remove(tmp + ".pdb")
    bonds, natives = [], []
    for line in top.splitlines():
        t = line.split()
        if t[0] == "bond":
            bonds.append([int(t[1]), int(t[2]), t[3]])
        elif t[0] == "native":
            natives.append([int(t[1]), int(t[2]), t[3], t[4]])
        elif t[0] == "atoms":
            natoms = int(t[1])
    def is_row(toks):
        try:
            return len(toks) == 3 and all(float(t) == float(t) for t in toks)
        except ValueError:
            return False
    # SOP::load also prints progress lines; keep the coordinate rows only
    xyz = [l.split() for l in coords.splitlines() if is_row(l.split())]
    with open(os.path.join(HERE, "topology.json"), "w") as f:
        json.dump({"n": 48, "seed": 2024, "atoms": natoms, "bonds": bonds, "natives": natives, "xyz": xyz}, f)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
