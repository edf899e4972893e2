"""Runs the reference's own CUDA path (oracle/_ref/ref_gpu, built from the
SOP-GPU source tree by oracle/build_ref.sh) on every case of ref_cases.py on
a B200 and packs the dumps into ref_gpu_<case>.npz.

    python tests/golden/make_ref_gpu_golden.py <outdir> [case ...]
    python tests/golden/make_ref_gpu_golden.py --pack <outdir> [case ...]

The .npz files are then committed next to this script.  Pair rows are
trimmed to the largest count (the reference pads them with -1).  The files
the reference's output updaters wrote during the run (.dat, DCD, restart
PDB, pulling and indentation lines) go into the same archive as byte arrays
under "file:<basename>".  --pack repacks an earlier run's directory without
running the reference again.
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, HERE)
import ref_cases  # noqa: E402

REF_GPU = os.path.join(REPO, "oracle", "_ref", "ref_gpu")


def main():
    args = sys.argv[1:]
    pack_only = bool(args) and args[0] == "--pack"
    if pack_only:
        args = args[1:]
    out = os.path.abspath(args[0] if args else "refgold")
    names = args[1:] or [c for c in ref_cases.CASES
                         if not ref_cases.CASES[c].get("speed") and not ref_cases.CASES[c].get("longrun")]
    for name in names:
        c = ref_cases.CASES[name]
        d = os.path.join(out, name)
        dumpdir = os.path.join(d, "dump")
        if not pack_only:
            cfg = ref_cases.write_inputs(name, d)
            os.makedirs(dumpdir, exist_ok=True)
            cmd = [REF_GPU, os.path.basename(cfg), dumpdir, str(c["total"])] + [str(s) for s in c["dumps"]]
            with open(os.path.join(d, "ref_gpu.log"), "w") as log:
                subprocess.check_call(cmd, cwd=d, stdout=log, stderr=subprocess.STDOUT)
        meta = dict(l.split() for l in open(os.path.join(dumpdir, "meta.txt")))
        N = int(meta["aminoCount"])
        mp = int(meta["max_pairs"])
        arrays = {"stride": np.int32(meta["stride"]),
                  "forces_0": np.fromfile(os.path.join(dumpdir, "forces_0.bin"), np.float32).reshape(N, 4)}
        for s in c["dumps"]:
            f = lambda w: os.path.join(dumpdir, "%s_%d.bin" % (w, s))
            arrays["coords_%d" % s] = np.fromfile(f("coords"), np.float32).reshape(N, 4)
            arrays["seeds_%d" % s] = np.fromfile(f("seeds"), np.uint32).reshape(N, 4)
            arrays["T_%d" % s] = np.fromfile(f("T"), np.float32)
            cnt = np.fromfile(f("paircount"), np.int32)
            rows = np.fromfile(f("pairs"), np.int32).reshape(mp, N).T
            arrays["paircount_%d" % s] = cnt
            arrays["pairs_%d" % s] = rows[:, : max(1, int(cnt.max()))].copy()
            if os.path.exists(f("tip")):
                arrays["tip_%d" % s] = np.fromfile(f("tip"), np.float32)
        for fname in ref_cases.output_files(d, name):
            with open(os.path.join(d, fname), "rb") as fh:
                arrays["file:" + fname] = np.frombuffer(fh.read(), np.uint8)
        np.savez_compressed(os.path.join(out, "ref_gpu_%s.npz" % name), **arrays)
        print("case %s: %d beads, stride %s" % (name, N, meta["stride"]))


if __name__ == "__main__":
    main()
