"""Output files in the reference's formats: energy .dat lines, DCD
trajectories, restart/final PDBs, pulling and indentation lines.

The golden files were written by the reference's own output updaters
during its CUDA runs on a B200 (tests/golden/make_ref_gpu_golden.py packs
them into ref_gpu_<case>.npz under "file:<name>").  On the CPU the oracle's
observables and event log are checked against those lines; on the GPU the
`sopb-gpu` driver runs each case and its files are compared with the
reference's file by file.

Bars: step columns, counts, file layouts and integer fields exact; printed
reals within the printed precision plus the trajectory tolerance of the
parity tests (the two runs agree to ~1e-5 A after 100 steps, energies to
~1e-5 relative: the trajectories and the reference's fast-math logf).
"""
import os
import struct
import subprocess
import sys

import numpy as np
import pytest

import oracle_py as O
from test_ref_gpu_golden import GOLD, load

sys.path.insert(0, GOLD)
import ref_cases  # noqa: E402

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(REPO, "sop-gpu_b200", "sopb-gpu")


def golden_cases(files_only=False):
    out = []
    for c in ref_cases.CASES:
        p = os.path.join(GOLD, "ref_gpu_%s.npz" % c)
        if not os.path.exists(p):
            continue
        if files_only and not ref_cases.CASES[c].get("files"):
            continue
        if any(k.startswith("file:") for k in np.load(p).files):
            out.append(c)
    return out


def gfile(g, name):
    return bytes(g["file:" + name])


# ---- readers -----------------------------------------------------------------
def read_dcd(buf):
    """Header fields and frames (k, 3, N) of a DCD without unit cell."""
    i32 = lambda o: struct.unpack_from("<i", buf, o)[0]
    assert i32(0) == 84 and buf[4:8] == b"CORD"
    hdr = dict(nfile=i32(8), npriv=i32(12), nsavc=i32(16), nstep=i32(20), delta=struct.unpack_from("<f", buf, 44)[0])
    assert i32(84) == 24 and i32(88) == 84 and i32(92) == 164 and i32(96) == 2 and i32(260) == 164
    assert i32(264) == 4 and i32(272) == 4
    hdr["zeros"] = [i32(o) for o in list(range(24, 44, 4)) + list(range(48, 84, 4))]
    n = i32(268)
    hdr["n"] = n
    hdr["titles"] = buf[100:260]
    frames = []
    o = 276
    while o < len(buf):
        fr = []
        for _ in range(3):
            assert i32(o) == 4 * n and i32(o + 4 + 4 * n) == 4 * n
            fr.append(np.frombuffer(buf, np.float32, n, o + 4))
            o += 8 + 4 * n
        frames.append(fr)
    assert o == len(buf)
    return hdr, np.array(frames, np.float32).reshape(-1, 3, n)


def dat_rows(text):
    return [l.split("\t") for l in text.decode().splitlines() if l.strip()]


def floats(rows):
    return np.array([[float(v) for v in r] for r in rows], np.float64)


def pdb_parts(text):
    atoms, rest = [], []
    for l in text.decode().split("\n"):
        if l.startswith("ATOM"):
            atoms.append((l[:30] + l[54:], (float(l[30:38]), float(l[38:46]), float(l[46:54]))))
        else:
            rest.append(l)
    return atoms, rest


# ---- the output updaters' arithmetic, restated for the oracle ------------------
def dat_line_values(obs, nav, n, rg, carry=0.0):
    """OutputManager columns from the observables of one run (T carries the
    previous run's FP64 average, output_manager.cu:144-155)."""
    t = (carry + obs[0] * n * nav) / (n * nav)
    e = np.float32(obs[1:4])
    vals = [np.float32(t)] + list(e) + [float(np.float64(e[0]) + e[1] + e[2]), int(obs[5]), np.float32(obs[6] if rg else 0.0)]
    return vals, t


def indentation_lines(rows, out_freq, nav, ks):
    """IndentationTipUpdater's output averages (indentation.cu:496-534) from
    the tip rows of the event log."""
    fav = np.zeros(4, np.float32)
    kdx = np.float32(0)
    lines = []
    for r in rows:
        v = r["v"].astype(np.float32)
        fav += v[:4]
        kdx = np.float32(kdx + np.float32(v[4] * np.float32(ks)))
        if r["step"] % out_freq == 0:
            factor = np.float32(out_freq // nav)
            a = fav / factor
            k = kdx / factor
            fmod = np.sqrt(np.float32(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]))
            lines.append([r["step"], v[5], a[3], fmod, abs(np.float32(v[4] * np.float32(ks))), k, a[0], a[1], a[2],
                          *v[6:9], *v[9:12]])
            fav[:] = 0
            kdx = np.float32(0)
    return np.array(lines, np.float64)


# ---- CPU: the golden files decode, and the oracle reproduces their lines ------
@pytest.mark.parametrize("name", golden_cases())
def test_reference_files_decode(name):
    g, jc, specs = load(name)
    c = ref_cases.CASES[name]
    cfg = dict(ref_cases.COMMON, **c["cfg"])
    first = int(c["cfg"].get("firstrun", c["cfg"].get("run", "1")))
    dcdfreq = int(cfg["dcdfreq"])
    last = (c["total"] - 1) // jc.params.stride * jc.params.stride
    nframes = last // dcdfreq + 1
    extra = 0
    if cfg.get("indentationShowTipSurf") == "yes" or cfg.get("indentationDiscreteSurf") == "yes":
        extra = 2 + int(cfg["indentationSurfaceSize"]) ** 2
    for r, sp in enumerate(specs):
        hdr, fr = read_dcd(gfile(g, "%s_%d.dcd" % (name, first + r)))
        assert (hdr["nfile"], hdr["npriv"], hdr["nsavc"], hdr["nstep"], hdr["delta"]) == (dcdfreq, dcdfreq, dcdfreq, 0, 0.0)
        assert hdr["zeros"] == [0] * 14 and hdr["n"] == sp.n + extra
        assert fr.shape == (nframes, 3, sp.n + extra)
        assert np.array_equal(fr[0][:, : sp.n].T, sp.xyz.astype(np.float32))     # step 0: the input coordinates


@pytest.mark.parametrize("name", golden_cases())
def test_oracle_reproduces_dat_lines(name):
    g, jc, specs = load(name)
    c = ref_cases.CASES[name]
    cfg = dict(ref_cases.COMMON, **c["cfg"])
    first = int(c["cfg"].get("firstrun", c["cfg"].get("run", "1")))
    rg = cfg.get("computeRg") == "yes"
    tea = cfg.get("hi_on") == "yes"
    nav = jc.params.nav
    rows = [floats(dat_rows(gfile(g, "%s_%d.dat" % (name, first + r)))) for r in range(len(specs))]
    steps = rows[0][:, 0].astype(np.int64)
    orcs = [O.OracleJob(sp) for sp in specs]
    done = 0
    for k, s in enumerate(steps):
        carry = 0.0
        for r, o in enumerate(orcs):
            assert o.advance(int(s) - done) == 0
            vals, carry = dat_line_values(o.observables(), nav, specs[r].n, rg, carry)
            got = rows[r][k]
            # step, T, FENE, native, repulsive, total, contacts, Rg [, TEA eps]
            assert got[0] == s and len(got) == 8 + int(tea)
            assert got[6] == vals[5]                                   # intact native contacts
            want = np.array(vals[:5] + [vals[6]], np.float64)
            have = np.concatenate([got[1:6], got[7:8]])
            # FENE energies follow the trajectories (1e-5 A apart after 20 steps)
            # and the reference's fast-math logf: 1e-5 relative
            assert np.allclose(have, want, rtol=1e-5, atol=1.5e-5), (s, have, want)
            if tea:
                assert abs(got[8] - o.observables()[7]) <= 1e-6 + 1e-5 * abs(got[8])
        done = int(s)


@pytest.mark.parametrize("name", [c for c in golden_cases() if ref_cases.CASES[c]["cfg"].get("deltax")])
def test_oracle_reproduces_pulling_lines(name):
    g, jc, specs = load(name)
    c = ref_cases.CASES[name]
    first = int(c["cfg"].get("firstrun", c["cfg"].get("run", "1")))
    for r, sp in enumerate(specs):
        ref = floats(dat_rows(gfile(g, "%s_%d_pull.dat" % (name, first + r))))
        o = O.OracleJob(sp)
        assert o.advance(c["total"]) == 0
        L = o.log()
        assert np.array_equal(L["kind"], np.ones(len(L)))
        assert np.array_equal(L["step"], ref[:, 0].astype(np.int64))
        assert np.allclose(L["v"][:, :6], ref[:, 1:], atol=5.01e-4 + 1e-4)


@pytest.mark.parametrize("name", [c for c in golden_cases() if ref_cases.CASES[c]["cfg"].get("pullingPlane")])
def test_oracle_reproduces_plane_lines(name):
    g, jc, specs = load(name)
    c = ref_cases.CASES[name]
    first = int(c["cfg"].get("firstrun", c["cfg"].get("run", "1")))
    for r, sp in enumerate(specs):
        ref = floats(dat_rows(gfile(g, "%s_%d_plane.dat" % (name, first + r))))
        o = O.OracleJob(sp)
        assert o.advance(c["total"]) == 0
        L = o.log()
        assert np.all(L["kind"] == 3)
        assert np.array_equal(L["step"], ref[:, 0].astype(np.int64))
        # printed with %f: 6 decimals
        assert np.allclose(L["v"][:, :5], ref[:, 1:], rtol=1e-5, atol=1.5e-6)


@pytest.mark.parametrize("name", [c for c in golden_cases() if ref_cases.CASES[c]["cfg"].get("indentation")])
def test_oracle_reproduces_indentation_lines(name):
    g, jc, specs = load(name)
    c = ref_cases.CASES[name]
    cfg = dict(ref_cases.COMMON, **c["cfg"])
    ref = floats(dat_rows(gfile(g, "%s_indent.dat" % name)))
    o = O.OracleJob(specs[0])
    assert o.advance(c["total"]) == 0
    L = o.log()
    assert np.all(L["kind"] == 2) and np.array_equal(L["step"], np.arange(len(L)) * jc.params.nav)
    got = indentation_lines(L, int(cfg.get("indentationOutputFreq", 1000)), jc.params.nav, float(cfg["indentationKs"]))
    assert got.shape == ref.shape
    assert np.array_equal(got[:, 0], ref[:, 0])
    assert np.allclose(got[:, 1:], ref[:, 1:], rtol=1e-5, atol=2e-5)


# ---- GPU: the driver's files against the reference's ------------------------------
def run_cli(name, d):
    c = ref_cases.CASES[name]
    cfg = ref_cases.write_inputs(name, d)
    g = np.load(os.path.join(GOLD, "ref_gpu_%s.npz" % name))
    stride = int(g["stride"])
    numsteps = c["total"] - stride      # the loop runs (numsteps/stride + 1) * stride steps
    r = subprocess.run([CLI, os.path.basename(cfg), "numsteps=%d" % numsteps], cwd=d, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("name", golden_cases())
def test_cli_files_match_reference(tmp_path, name):
    if not os.path.exists(CLI):
        subprocess.check_call(["make", "-s", "-C", os.path.join(REPO, "sop-gpu_b200")])
    d = str(tmp_path)
    g = run_cli(name, d)
    ref_names = sorted(k[5:] for k in g.files if k.startswith("file:"))
    mine = ref_cases.output_files(d, name)
    assert set(ref_names) <= set(mine), set(ref_names) - set(mine)
    for f in ref_names:
        want = gfile(g, f)
        with open(os.path.join(d, f), "rb") as fh:
            have = fh.read()
        if f.endswith(".dcd"):
            h1, f1 = read_dcd(have)
            h0, f0 = read_dcd(want)
            h1.pop("titles"), h0.pop("titles")
            assert h1 == h0
            assert f1.shape == f0.shape
            assert np.max(np.abs(f1 - f0)) <= 1e-4, f
        elif f.endswith("_restart") or f.endswith(".pdb"):
            a1, r1 = pdb_parts(have)
            a0, r0 = pdb_parts(want)
            assert r1 == r0 and [a for a, _ in a1] == [a for a, _ in a0], f
            assert np.max(np.abs(np.array([x for _, x in a1]) - np.array([x for _, x in a0]))) <= 1.01e-3, f
        elif f.endswith(".vmd"):
            assert have == want
        else:
            l1, l0 = dat_rows(have), dat_rows(want)
            assert [len(r) for r in l1] == [len(r) for r in l0], f
            assert [r[0] for r in l1] == [r[0] for r in l0], f
            v1, v0 = floats(l1), floats(l0)
            # printed precision (%5.3f pulling, %8.5f others) plus the runs' spread
            atol = 1.01e-3 if f.endswith("_pull.dat") else 2e-4
            assert np.allclose(v1, v0, rtol=2e-6, atol=atol), (f, np.max(np.abs(v1 - v0)))
