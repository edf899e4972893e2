"""Runs the reference's own CUDA path (oracle/_ref/ref_gpu, built from the
SOP-GPU source tree by oracle/build_ref.sh) on the long-run case of
ref_cases.py on a B200 and keeps what its output updaters wrote, reduced to
arrays by longrun.read_runs, in ref_gpu_<case>.npz beside this script.

    python tests/golden/make_ref_longrun_golden.py <workdir> [case [outdir]]

(outdir defaults to this directory.)
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, HERE)
import longrun  # noqa: E402
import ref_cases  # noqa: E402

REF_GPU = os.path.join(REPO, "oracle", "_ref", "ref_gpu")


def main():
    work = os.path.abspath(sys.argv[1] if len(sys.argv) > 1 else "longrun")
    name = sys.argv[2] if len(sys.argv) > 2 else "longpull"
    c = ref_cases.CASES[name]
    d = os.path.join(work, name)
    cfg = ref_cases.write_inputs(name, d)
    dumpdir = os.path.join(d, "dump")
    os.makedirs(dumpdir, exist_ok=True)
    with open(os.path.join(d, "ref_gpu.log"), "w") as log:
        subprocess.check_call([REF_GPU, os.path.basename(cfg), dumpdir, str(c["total"])], cwd=d, stdout=log,
                              stderr=subprocess.STDOUT)
    pull, dat = longrun.read_runs(d, name, c["runs"])
    out = sys.argv[3] if len(sys.argv) > 3 else HERE
    np.savez_compressed(os.path.join(out, "ref_gpu_%s.npz" % name), pull=pull.astype(np.float32),
                        dat=dat.astype(np.float32))
    print("case %s: %d runs, %d pulling lines, %d .dat lines each" % (name, pull.shape[0], pull.shape[1], dat.shape[1]))


if __name__ == "__main__":
    main()
