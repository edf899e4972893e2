"""Cases for golden fixtures made by the reference's own CUDA path on B200
(tests/golden/make_ref_gpu_golden.py) and checked by
tests/test_ref_gpu_golden.py.  Each case is a config file in the reference's
format plus seeded synthetic inputs; both sides read the same files."""
import functools
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "sop-gpu_b200"))
import sopb_synth as S  # noqa: E402

COMMON = {
    "timestep": "0.08", "zeta": "50.0", "temperature": "0.6", "kspring_cov": "20.0", "R_limit": "2.0",
    "a": "3.8", "el": "1.0", "pairs_cutoff": "20.0", "pairlist_cutoff": "20.0", "pairs_threshold": "200.0",
    "pairs_freq": "10", "possiblepairs_freq": "100000", "max_covalent": "8", "max_native": "128",
    "block_size": "128", "outputtiming": "1000000", "dcdfreq": "1000000", "restartfreq": "1000000",
    "name": "case", "topology": "<name>.top", "coordinates": "<name>_<run>.pdb",
    "outputname": "<name>_<run>.dat", "DCDfile": "<name>_<run>.dcd", "restartname": "<name>_<run>_restart",
    "finalcoord": "<name>_<run>_final.pdb", "reffilename": "<name>.ref.pdb", "numsteps": "0",
}

CASES = {
    "pull2": dict(n=200, sys_seed=11, runs=2, total=100, dumps=[1, 10, 90, 91, 100], cfg={
        "runnum": "2", "firstrun": "1", "seed": "1119726", "nav": "100", "max_pairs": "256",
        "max_possiblePairs": "256", "pulling": "on", "deltax": "0.02", "k_trans": "0.05", "pullFreq": "10",
        "fixed": "0", "pulled": "199", "fixedEnd": "0", "pulledEnd": "199", "pullDirection": "endToEnd",
        "pullOutput": "<name>_<run>_pull.dat"}),
    "clampvec": dict(n=150, sys_seed=17, runs=1, total=50, dumps=[1, 50], cfg={
        "run": "3", "seed": "4242", "nav": "1000", "max_pairs": "200", "max_possiblePairs": "200",
        "pulling": "on", "fconst": "2.5", "fixed": "0 to 2", "pulled": "149", "fixedEnd": "0", "pulledEnd": "149",
        "pullDirection": "vector", "pullVector": "0.6 0.8 0.0"}),
    "tea": dict(n=100, sys_seed=23, runs=1, total=30, dumps=[1, 10, 30], cfg={
        "run": "1", "seed": "777", "nav": "1000", "max_pairs": "128", "max_possiblePairs": "128",
        "hi_on": "yes", "hi_a": "1.9", "hi_unlisted": "yes", "hi_capricious": "no", "hi_epsilon_freq": "10"}),
    "tealist": dict(n=100, sys_seed=23, runs=1, total=30, dumps=[1, 30], cfg={
        "run": "1", "seed": "778", "nav": "1000", "max_pairs": "128", "max_possiblePairs": "128",
        "hi_on": "yes", "hi_a": "1.9", "hi_unlisted": "no", "hi_capricious": "no", "hi_epsilon_freq": "10"}),
    "chol": dict(n=40, sys_seed=29, runs=1, total=10, dumps=[1, 10], cfg={
        "run": "1", "seed": "99", "nav": "1000", "max_pairs": "64", "max_possiblePairs": "64",
        "hi_on": "yes", "hi_exact": "yes", "hi_a": "1.9"}),
    "indent": dict(n=200, sys_seed=13, runs=1, total=100, dumps=[1, 40, 100], cfg={
        "run": "1", "seed": "31337", "nav": "20", "max_pairs": "256", "max_possiblePairs": "256",
        "indentation": "on", "indentationTipR": "20.0", "indentationKs": "0.07", "indentationDeltaX": "0.05",
        "indentationDirection": "0.0 1.0 0.0", "indentationSurfaceN": "0.0 -1.0 0.0", "indentationTipZeta": "500",
        "indentationSurfA": "1.0", "indentationSurfB": "-2.0", "indentationSurfSigma": "3.0",
        "indentationSurfEl": "0.2", "indentationFixTrans": "yes", "indentationOutput": "<name>_indent.dat"}),
    # output files every few strides: .dat (with Rg), DCD, restart PDB and
    # pulling lines for two runs
    "pullout": dict(n=200, sys_seed=11, runs=2, total=100, dumps=[100], files=True, cfg={
        "runnum": "2", "firstrun": "1", "seed": "1119726", "nav": "100", "max_pairs": "256",
        "max_possiblePairs": "256", "pulling": "on", "deltax": "0.02", "k_trans": "0.05", "pullFreq": "10",
        "fixed": "0", "pulled": "199", "fixedEnd": "0", "pulledEnd": "199", "pullDirection": "endToEnd",
        "pullOutput": "<name>_<run>_pull.dat", "outputtiming": "20", "dcdfreq": "20", "restartfreq": "50",
        "computeRg": "yes"}),
    # indentation lines averaged over two tip updates, the tip and surface
    # beads in the DCD and PDB files
    "indentout": dict(n=200, sys_seed=13, runs=1, total=120, dumps=[120], files=True, cfg={
        "run": "1", "seed": "31337", "nav": "20", "max_pairs": "256", "max_possiblePairs": "256",
        "indentation": "on", "indentationTipR": "20.0", "indentationKs": "0.07", "indentationDeltaX": "0.05",
        "indentationDirection": "0.0 1.0 0.0", "indentationSurfaceN": "0.0 -1.0 0.0", "indentationTipZeta": "500",
        "indentationSurfA": "1.0", "indentationSurfB": "-2.0", "indentationSurfSigma": "3.0",
        "indentationSurfEl": "0.2", "indentationFixTrans": "yes", "indentationOutput": "<name>_indent.dat",
        "indentationOutputFreq": "40", "outputtiming": "20", "dcdfreq": "40", "restartfreq": "60",
        "indentationShowTipSurf": "yes", "indentationSurfaceSize": "5", "indentationSurfaceStep": "10.0",
        "indentationCantLength": "50.0", "indentationSurfConnectFile": "<name>_mica.vmd"}),
    # the TEA epsilon column
    "teaout": dict(n=100, sys_seed=23, runs=1, total=30, dumps=[30], files=True, cfg={
        "run": "1", "seed": "777", "nav": "1000", "max_pairs": "128", "max_possiblePairs": "128",
        "hi_on": "yes", "hi_a": "1.9", "hi_unlisted": "yes", "hi_capricious": "no", "hi_epsilon_freq": "10",
        "outputtiming": "10", "dcdfreq": "10"}),
    # pulling plane, two runs (one plane displacement each)
    "plane": dict(n=150, sys_seed=17, runs=2, total=100, dumps=[1, 50, 100], files=True, cfg={
        "runnum": "2", "firstrun": "1", "seed": "2468", "nav": "1000", "max_pairs": "200",
        "max_possiblePairs": "200", "pullingPlane": "on", "pullingPlaneDeltax": "0.5", "pullingPlaneKs": "0.5",
        "pullingPlaneKsCant": "0.2", "pullingPlaneZeta": "50", "pullingPlaneDir": "0.0 0.6 0.8",
        "plane_fixed": "0 to 4", "plane_pulled": "145 to 149", "pullingPlaneUpdateFreq": "10",
        "pullingPlaneOutputFreq": "20", "pullingPlaneOutput": "<name>_<run>_plane.dat", "outputtiming": "50",
        "dcdfreq": "50"}),
    # indentation on a discrete surface (surface-bead lists), chip moving
    "mica": dict(n=200, sys_seed=13, runs=1, total=100, dumps=[1, 40, 100], files=True, cfg={
        "run": "1", "seed": "4711", "nav": "20", "max_pairs": "256", "max_possiblePairs": "256",
        "indentation": "on", "indentationTipR": "20.0", "indentationKs": "0.07", "indentationDeltaX": "0.05",
        "indentationDirection": "0.0 1.0 0.0", "indentationSurfaceN": "0.0 -1.0 0.0", "indentationTipZeta": "500",
        "indentationSurfA": "1.0", "indentationSurfB": "-2.0", "indentationSurfSigma": "3.0",
        "indentationSurfEl": "0.2", "indentationFixTrans": "yes", "indentationOutput": "<name>_indent.dat",
        "indentationOutputFreq": "20", "indentationDiscreteSurf": "yes", "indentationSurfaceSize": "15",
        "indentationSurfaceStep": "3.0", "indentationPairsCutoff": "12.0", "indentationCantLength": "50.0",
        "indentationSurfConnectFile": "<name>_mica.vmd", "outputtiming": "20", "dcdfreq": "40"}),
    # the same with the surface moving towards the tip
    "micamove": dict(n=200, sys_seed=13, runs=1, total=100, dumps=[1, 40, 100], files=True, cfg={
        "run": "1", "seed": "4712", "nav": "20", "max_pairs": "256", "max_possiblePairs": "256",
        "indentation": "on", "indentationTipR": "20.0", "indentationKs": "0.07", "indentationDeltaX": "-0.5",
        "indentationDirection": "0.0 1.0 0.0", "indentationSurfaceN": "0.0 -1.0 0.0", "indentationTipZeta": "500",
        "indentationSurfA": "1.0", "indentationSurfB": "-2.0", "indentationSurfSigma": "3.0",
        "indentationSurfEl": "0.2", "indentationFixTrans": "yes", "indentationOutput": "<name>_indent.dat",
        "indentationOutputFreq": "20", "indentationDiscreteSurf": "yes", "indentationSurfaceSize": "15",
        "indentationSurfaceStep": "3.0", "indentationPairsCutoff": "12.0", "indentationMoveSurface": "yes",
        "indentationCantLength": "50.0", "indentationSurfConnectFile": "<name>_mica.vmd", "outputtiming": "20",
        "dcdfreq": "40"}),
    # speed comparisons with the reference's CUDA path (timed, no dumps):
    # the plain 200-bead ramp pull, 512 force-clamp replicas of one 200-bead
    # system, TEA at 4000 beads
    "speed_plain": dict(n=200, sys_seed=2024, runs=1, total=20000, dumps=[], speed=True, cfg={
        "run": "1", "seed": "1119726", "nav": "1000", "max_pairs": "256", "max_possiblePairs": "256",
        "pulling": "on", "deltax": "0.5", "k_trans": "0.05", "pullFreq": "1000", "fixed": "0", "pulled": "199",
        "fixedEnd": "0", "pulledEnd": "199", "pullDirection": "endToEnd"}),
    "speed_batch": dict(n=200, sys_seed=2024, runs=512, total=2000, dumps=[], speed=True, cfg={
        "runnum": "512", "firstrun": "1", "seed": "1119726", "nav": "1000", "max_pairs": "256",
        "max_possiblePairs": "256", "pulling": "on", "fconst": "2.0", "fixed": "0", "pulled": "199",
        "fixedEnd": "0", "pulledEnd": "199", "pullDirection": "endToEnd"}),
    "speed_tea": dict(n=4000, sys_seed=4000, runs=1, total=20, dumps=[], speed=True, cfg={
        "run": "1", "seed": "777", "nav": "1000", "max_pairs": "1024", "max_possiblePairs": "4096",
        "hi_on": "yes", "hi_a": "3.8", "hi_unlisted": "yes", "hi_capricious": "no", "hi_epsilon_freq": "10"}),
    # exact HI at the reference's largest size (CHOLSIZE = 3 x 128), the
    # factor refreshed every step
    "speed_exact": dict(n=128, sys_seed=29, runs=1, total=2000, dumps=[], speed=True, cfg={
        "run": "1", "seed": "99", "nav": "1000", "max_pairs": "128", "max_possiblePairs": "128",
        "hi_on": "yes", "hi_exact": "yes", "hi_a": "1.9"}),
    # the 198 000-bead shell indented by a 10 nm tip, 200 steps
    "speed_capsid": dict(n=198000, sys_seed=7, runs=1, total=200, dumps=[], speed=True, system="capsid", cfg={
        "run": "1", "seed": "5032015", "nav": "100", "pairs_threshold": "40.0", "max_possiblePairs": "2048",
        "max_pairs": "512", "possiblepairs_freq": "100000", "indentation": "on", "indentationTipR": "100.0",
        "indentationKs": "0.07", "indentationDeltaX": "0.012", "indentationDirection": "0.0 -1.0 0.0",
        "indentationSurfaceN": "0.0 1.0 0.0", "indentationTipZeta": "5000", "indentationSurfA": "1.0",
        "indentationSurfB": "-2.0", "indentationSurfSigma": "10.0", "indentationSurfEl": "0.2",
        "indentationFixTrans": "yes"}),
    # long-run statistics: 256 runs of the plain 200-bead force-ramp pull for
    # 1e5 steps (cantilever 1.4 A per 200 steps, 700 A in all), pulling lines
    # every 200 steps and .dat lines every 1000; made by
    # make_ref_longrun_golden.py, compared by tests/test_gpu_longrun.py
    "longpull": dict(n=200, sys_seed=2024, runs=256, total=100000, dumps=[], longrun=True, cfg={
        "runnum": "256", "firstrun": "1", "seed": "1119726", "nav": "1000", "max_pairs": "256",
        "max_possiblePairs": "256", "pulling": "on", "deltax": "1.4", "k_trans": "0.05", "pullFreq": "200",
        "fixed": "0", "pulled": "199", "fixedEnd": "0", "pulledEnd": "199", "pullDirection": "endToEnd",
        "pullOutput": "<name>_<run>_pull.dat", "outputtiming": "1000", "dcdfreq": "100000000",
        "restartfreq": "100000000"}),
    "heat": dict(n=100, sys_seed=6, runs=1, total=45, dumps=[45], cfg={
        "run": "1", "seed": "5", "nav": "1000", "max_pairs": "128", "max_possiblePairs": "128",
        "heating": "on", "initialT": "0.1", "deltaT": "0.2", "tempFreq": "10"}),
    "minim": dict(n=100, sys_seed=6, runs=1, total=20, dumps=[20], cfg={
        "run": "1", "seed": "5", "nav": "1000", "max_pairs": "128", "max_possiblePairs": "128",
        "minimization": "yes"}),
}


@functools.lru_cache(maxsize=4)
def _capsid():
    return S.make_capsid()[0]


def systems(name):
    """The case's systems, one per run (run k > 0 is a perturbed copy)."""
    c = CASES[name]
    if c.get("system") == "capsid":
        return [_capsid()]
    base = S.make_system(c["n"], c["sys_seed"])
    out = [base]
    rng = np.random.default_rng(c["sys_seed"])
    for _ in range(1, c["runs"]):
        x = base.xyz.astype(np.float64) + rng.normal(scale=0.3, size=base.xyz.shape)
        out.append(S.System(S._round_pdb(x), base.bonds, base.bonds_r0, base.natives, base.natives_r0, base.natives_eh))
    return out


def config_text(name):
    c = CASES[name]
    cfg = dict(COMMON)
    cfg.update(c["cfg"])
    cfg["name"] = name
    if c.get("system") == "capsid":
        # a 10 nm tip over the shell, the substrate under it (the capsid
        # workload's geometry)
        x = systems(name)[0].xyz.astype(np.float64)
        m = x.mean(axis=0)
        tip = "%.4f %.4f %.4f" % (m[0], x[:, 1].max() + 104.0, m[2])
        cfg["indentationChip"] = tip
        cfg["indentationTip"] = tip
        cfg["indentationSurfaceR0"] = "0.0 %.4f 0.0" % (x[:, 1].min() - 10.0)
    elif c["cfg"].get("indentation") == "on":
        x = systems(name)[0].xyz.astype(np.float64)
        top = x[:, 1].min()
        tip = "%.4f %.4f %.4f" % (x[:, 0].mean(), top - 22.0, x[:, 2].mean())
        cfg["indentationChip"] = tip
        cfg["indentationTip"] = tip
        if c["cfg"].get("indentationDiscreteSurf") == "yes":    # the bead square under the chain
            cfg["indentationSurfaceR0"] = "%.4f %.4f %.4f" % (x[:, 0].mean(), x[:, 1].max() + 6.0, x[:, 2].mean())
        else:
            cfg["indentationSurfaceR0"] = "0.0 %.4f 0.0" % (x[:, 1].max() + 6.0)
    if c["cfg"].get("pullingPlane") == "on":
        x = systems(name)[0].xyz.astype(np.float64)
        cfg["pullingPlanePos"] = "%.4f %.4f %.4f" % tuple(x.mean(axis=0))
    return "".join("%s\t%s\n" % (k, v) for k, v in cfg.items())


# the files the reference's output updaters write for a case, by basename
OUTPUT_SUFFIXES = (".dat", ".dcd", "_restart", "_final.pdb", ".vmd")


def output_files(d, name):
    """Output files of a case found in directory d (not the input PDBs)."""
    out = []
    for f in sorted(os.listdir(d)):
        if f.startswith(name) and f.endswith(OUTPUT_SUFFIXES):
            out.append(f)
    return out


def write_inputs(name, d):
    """Writes <name>.top, <name>_<run>.pdb and <name>.sop into directory d."""
    os.makedirs(d, exist_ok=True)
    c = CASES[name]
    syss = systems(name)
    S.write_top(os.path.join(d, name + ".top"), syss[0])
    first = int(c["cfg"].get("firstrun", c["cfg"].get("run", "1")))
    for k, s in enumerate(syss):
        S.write_pdb(os.path.join(d, "%s_%d.pdb" % (name, first + k)), s.xyz)
    path = os.path.join(d, name + ".sop")
    with open(path, "w") as f:
        f.write(config_text(name))
    return path
