"""Runs the reference's own topology creators (oracle/_ref/ref_sop_top and
ref_sop_top2, built from src/sop-top.cpp and src/sop-top2.cpp by
oracle/build_ref.sh) on every case of soptop_cases.py and packs the files
they write into soptop.npz (byte arrays named by file: "<case>.top",
"<case>_ca.pdb"; for the coarse-graining cases "<case>_cg.pdb",
"<case>.top", "<case>.psf", "<case>_nat.psf").

    python tests/golden/make_soptop_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, HERE)
import soptop_cases  # noqa: E402

REF = os.path.join(REPO, "oracle", "_ref", "ref_sop_top")
REF2 = os.path.join(REPO, "oracle", "_ref", "ref_sop_top2")


def main():
    arrays = {}
    for name in soptop_cases.CASES:
        with tempfile.TemporaryDirectory() as d:
            cfg = soptop_cases.write_case(name, d)
            subprocess.run([REF, os.path.basename(cfg)], cwd=d, check=True, stdout=subprocess.DEVNULL,
                           stdin=subprocess.DEVNULL)
            for f in (name + ".top", name + "_ca.pdb"):
                with open(os.path.join(d, f), "rb") as fh:
                    arrays[f] = np.frombuffer(fh.read(), np.uint8)
    for name in soptop_cases.CG_CASES:
        with tempfile.TemporaryDirectory() as d:
            cfg = soptop_cases.write_cg_case(name, d)
            subprocess.run([REF2, os.path.basename(cfg)], cwd=d, check=True, stdout=subprocess.DEVNULL,
                           stdin=subprocess.DEVNULL)
            for f in (name + "_cg.pdb", name + ".top", name + ".psf", name + "_nat.psf"):
                with open(os.path.join(d, f), "rb") as fh:
                    arrays[f] = np.frombuffer(fh.read(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "soptop.npz"), **arrays)
    print("cases:", ", ".join(list(soptop_cases.CASES) + list(soptop_cases.CG_CASES)))


if __name__ == "__main__":
    main()
