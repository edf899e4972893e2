"""The reference's config-file layer for the Langevin-step parameters.

File syntax and value parsing follow src/IO/configreader.cpp:
  * a line is `name value  # comment`; lines starting with '#', ' ', '\\t'
    or '\\n' are skipped (:26-39); later lines override earlier ones;
  * `<key>` masks are replaced by other keys' values, in the map's sorted
    key order (getMaskedParameter, :77-86);
  * booleans: yes/true/on/y and no/false/off/n, case-insensitive (:122-129);
  * integer arrays: whitespace separated with `a to b` ranges, `empty` or
    `none` for an empty list (:88-118); float3: three numbers (:131-141).

`job_config()` maps the keys the hot path reads onto sopb params with the
reference defaults and mandatory-key checks, and computes the updater period
`stride` exactly as runGPU does (src/gsop.cu:117-122), output updaters
included.
"""
from __future__ import annotations

import dataclasses
import re
from typing import Dict, List, Optional

import numpy as np

import sopb


class ConfigError(ValueError):
    pass


class Config:
    def __init__(self, path: Optional[str] = None, text: Optional[str] = None, overrides: Optional[Dict[str, str]] = None):
        self.values: Dict[str, str] = {}
        if path is not None:
            with open(path) as f:
                text = f.read()
        for line in (text or "").splitlines(keepends=True):
            if not line or line[0] in "# \n\t":
                continue
            m = re.match(r"([^ \t\n]+)[ \t]?(.*)", line, re.S)
            name, rest = m.group(1), m.group(2)
            self.values[name] = rest.split("#")[0].split("\n")[0].strip()
        for k, v in (overrides or {}).items():
            self.values[k] = str(v)

    def has(self, key: str) -> bool:
        return key in self.values

    def raw(self, key: str) -> str:
        if key not in self.values:
            raise ConfigError("Parameter '%s' not specified" % key)
        return self.values[key]

    def masked(self, key: str) -> str:
        v = self.raw(key)
        for k in sorted(self.values):
            v = v.replace("<%s>" % k, self.values[k])
        return v

    def get_str(self, key: str, default: Optional[str] = None) -> str:
        if not self.has(key):
            if default is None:
                raise ConfigError("Parameter '%s' not specified" % key)
            return default
        return self.masked(key)

    def get_bool(self, key: str, default: Optional[bool] = None) -> bool:
        if not self.has(key):
            if default is None:
                raise ConfigError("Parameter '%s' not specified" % key)
            return default
        v = self.raw(key).lower()
        if v in ("yes", "true", "on", "y"):
            return True
        if v in ("no", "false", "off", "n"):
            return False
        raise ConfigError("Wrong value '%s' for boolean parameter '%s'" % (v, key))

    def get_int(self, key: str, default: Optional[int] = None) -> int:
        if not self.has(key):
            if default is None:
                raise ConfigError("Parameter '%s' not specified" % key)
            return default
        return int(float(self.masked(key).split()[0])) if "." in self.masked(key).split()[0] else int(self.masked(key).split()[0])

    def get_float(self, key: str, default: Optional[float] = None) -> float:
        if not self.has(key):
            if default is None:
                raise ConfigError("Parameter '%s' not specified" % key)
            return default
        return float(np.float32(float(self.masked(key).split()[0])))

    def get_ints(self, key: str, default: Optional[List[int]] = None) -> List[int]:
        if not self.has(key):
            if default is None:
                raise ConfigError("Parameter '%s' not specified" % key)
            return list(default)
        v = self.raw(key).lower()
        if v in ("empty", "none"):
            return []
        out: List[int] = []
        toks = v.split()
        i = 0
        while i < len(toks):
            if toks[i] == "to":
                if not out:
                    raise ConfigError("In parameters of array type, 'to' keyword must be preceeded by number")
                out.extend(range(out[-1] + 1, int(toks[i + 1]) + 1))
                i += 2
            else:
                out.append(int(toks[i]))
                i += 1
        return out

    def get_float3(self, key: str, default=None) -> List[float]:
        if not self.has(key):
            if default is None:
                raise ConfigError("Parameter '%s' not specified" % key)
            return list(default)
        v = [float(np.float32(float(t))) for t in self.raw(key).split()]
        if len(v) != 3:
            raise ConfigError("Float3 parameter '%s' has %d components; must have 3." % (key, len(v)))
        return v


@dataclasses.dataclass
class JobConfig:
    params: sopb.Params
    fixed: List[int]
    pulled: List[int]
    seed: int             # seed + firstrun (src/Integrators/langevin.cu:23)
    ntr: int              # runs of this process (runnum, or 1 with `run`)
    firstrun: int
    numsteps: int
    topology: str
    coordinates: List[str]   # per run, <run> substituted
    plane_fixed: List[int] = dataclasses.field(default_factory=list)
    plane_pulled: List[int] = dataclasses.field(default_factory=list)


def job_config(cfg: Config) -> JobConfig:
    p = sopb.default_params()
    g = cfg
    run = g.get_int("run", -1)
    if run == -1:
        ntr, firstrun = g.get_int("runnum"), g.get_int("firstrun")
    else:
        ntr, firstrun = 1, run
    p.timestep = g.get_float("timestep")
    for k in ("zeta", "temperature", "kspring_cov", "R_limit", "R_limit_bond", "a", "el", "pairs_cutoff", "pairlist_cutoff",
              "pairs_threshold", "k_trans", "hi_a", "hi_epsmax"):
        setattr(p, k, g.get_float(k, getattr(p, k)))
    for k in ("pairs_freq", "possiblepairs_freq", "max_pairs", "max_possiblePairs", "nav"):
        setattr(p, k, g.get_int(k, getattr(p, k)))
    p.minimization = int(g.get_bool("minimization", False))
    p.heating = int(g.get_bool("heating", False))
    if p.heating:
        p.tempFreq, p.initialT, p.deltaT = g.get_int("tempFreq"), g.get_float("initialT"), g.get_float("deltaT")
    fixed: List[int] = []
    pulled: List[int] = []
    p.pulling = int(g.get_bool("pulling", False))
    if p.pulling:
        p.deltax = g.get_float("deltax", 0.0)
        p.fconst = g.get_float("fconst", 0.0)
        if p.deltax == 0 and p.fconst == 0:
            raise ConfigError("Either 'deltax' or 'fconst' parameter should be specified to initiate pulling")
        if g.has("fixed_beads") or g.has("pulled_beads"):
            raise ConfigError("'fixed_beads' and 'pulled_beads' parameters are deprecated. Use 'fixed' and 'pulled' instead")
        fixed, pulled = g.get_ints("fixed"), g.get_ints("pulled")
        d = g.get_str("pullDirection", "endToEnd")
        if d == "vector":
            p.pull_direction = sopb.PULL_VECTOR
            sopb.set_param(p, "pullVector", g.get_float3("pullVector"))
        elif d == "endToEnd":
            p.pull_direction = sopb.PULL_END_TO_END
        else:
            raise ConfigError("'pullDirection' parameter should be set to 'endToEnd' or 'vector'.")
        p.fixedEnd, p.pulledEnd = g.get_int("fixedEnd"), g.get_int("pulledEnd")
        p.pullFreq = g.get_int("pullFreq", p.nav)
    p.indentation = int(g.get_bool("indentation", False))
    if p.indentation:
        if ntr > 1:
            raise ConfigError("Many-runs-per-GPU mode is not supported by indentation potential.")
        if g.get_bool("indentationDiscreteSurf", False):
            # the surface as a square of beads (indentation.cu:137-201)
            p.indentationDiscreteSurf = 1
            p.indentationSurfaceSize = g.get_int("indentationSurfaceSize", 51)
            p.indentationSurfaceStep = g.get_float("indentationSurfaceStep", 1.4)
            p.indentationPairsCutoff = g.get_float("indentationPairsCutoff", 40.0)
        chip = g.get_float3("indentationChip")
        sopb.set_param(p, "indentationChip", chip)
        sopb.set_param(p, "indentationTip", g.get_float3("indentationTip", chip))
        for k in ("indentationDirection", "indentationSurfaceR0", "indentationSurfaceN"):
            sopb.set_param(p, k, g.get_float3(k))
        for k in ("indentationTipR", "indentationKs", "indentationDeltaX"):
            setattr(p, k, g.get_float(k))
        p.indentationMoveSurface = int(g.get_bool("indentationMoveSurface", False))
        p.indentationFixTrans = int(g.get_bool("indentationFixTrans", False))
        sig, el = g.get_float("indentationSigma", 1.0), g.get_float("indentationEl", 1.0)
        p.indentationTipSigma = g.get_float("indentationTipSigma", sig)
        p.indentationSurfSigma = g.get_float("indentationSurfSigma", sig)
        p.indentationTipEl = g.get_float("indentationTipEl", el)
        p.indentationSurfEl = g.get_float("indentationSurfEl", el)
        for k, d in (("indentationTipA", 0.0), ("indentationTipB", 1.0), ("indentationSurfA", 0.0), ("indentationSurfB", 1.0),
                     ("indentationTipZeta", 5000.0)):
            setattr(p, k, g.get_float(k, d))
        p.indentationRetractionStep = g.get_int("indentationRetractionStep", -1)
    plane_fixed: List[int] = []
    plane_pulled: List[int] = []
    p.pullingPlane = int(g.get_bool("pullingPlane", False))
    if p.pullingPlane:
        # PullingPlanePotential ctor (src/Potentials/pulling_plane.cu:35-135)
        p.pullingPlaneDeltax = g.get_float("pullingPlaneDeltax", 0.0)
        if p.pullingPlaneDeltax == 0:
            raise ConfigError("'pullingPlaneDeltax' parameter should be specified to initiate this->")
        if g.has("plane_fixed_beads") or g.has("plane_pulled_beads"):
            raise ConfigError("'plane_fixed_beads' and 'plane_pulled_beads' parameters are deprecated. "
                              "Use 'plane_fixed' and 'plane_pulled' instead")
        for k, d in (("pullingPlaneKs", 0.05), ("pullingPlaneKsCant", 0.05), ("pullingPlaneZeta", 200.0)):
            setattr(p, k, g.get_float(k, d))
        plane_fixed, plane_pulled = g.get_ints("plane_fixed"), g.get_ints("plane_pulled")
        sopb.set_param(p, "pullingPlaneDir", g.get_float3("pullingPlaneDir"))
        sopb.set_param(p, "pullingPlanePos", g.get_float3("pullingPlanePos"))
        p.pullingPlaneUpdateFreq = g.get_int("pullingPlaneUpdateFreq", p.nav)
        p.pullingPlaneOutputFreq = g.get_int("pullingPlaneOutputFreq", p.nav)
    p.hi_on = int(g.get_bool("hi_on", False))
    if p.hi_on:
        if p.minimization:
            raise ConfigError("Using minimization with BDHI integrator is not supported and will never be.")
        p.hi_exact = int(g.get_bool("hi_exact", False))
        if not p.hi_exact:
            p.hi_capricious = int(g.get_bool("hi_capricious", True))
            p.hi_epsilon_freq = g.get_int("hi_epsilon_freq")
            p.hi_unlisted = int(g.get_bool("hi_unlisted", True))
        p.hi_b_mode = {"cholesky": sopb.HI_B_CHOLESKY, "reference": sopb.HI_B_REFCOMPAT}[g.get_str("hi_b_mode", "cholesky")]
        p.hi_refresh = g.get_int("hi_refresh", 1)
    p.verlet_skin = g.get_float("verlet_skin", 0.0)   # near list of the Verlet rebuilds (this library)
    # runGPU's stride: nav and every updater's frequency (src/gsop.cu:117-122)
    freqs = [p.nav, p.possiblepairs_freq, g.get_int("outputtiming", 10000), p.pairs_freq, g.get_int("dcdfreq", 10000)]
    if p.indentation and g.get_bool("indentationShowTipSurf", False):
        freqs.append(g.get_int("outputtiming", 10000))
    if p.pulling and p.deltax != 0:
        freqs.append(p.pullFreq)
    if p.pullingPlane:
        freqs.append(p.pullingPlaneUpdateFreq)
    if p.heating:
        freqs.append(p.tempFreq)
    if p.hi_on and not p.hi_exact:
        freqs.append(p.hi_epsilon_freq)
    if p.hi_on and p.hi_exact and p.hi_refresh > 1:
        freqs.append(p.hi_refresh)      # the factor refresh is an updater of this library
    p.stride = min(freqs)
    seed = g.get_int("seed") + firstrun
    coords = [g.get_str("coordinates").replace("<run>", str(r + firstrun)) for r in range(ntr)]
    return JobConfig(p, fixed, pulled, seed, ntr, firstrun, g.get_int("numsteps"), g.get_str("topology"), coords,
                     plane_fixed, plane_pulled)


def job_specs(jc: JobConfig, systems) -> List["sopb.JobSpec"]:
    """One JobSpec per run; Hybrid Taus states drawn for all runs from one
    ran2 stream and split per run, as the reference's multi-run layout does."""
    n = systems[0].n
    seeds = sopb.generate_seeds(jc.seed, n * jc.ntr)
    out = []
    for r, s in enumerate(systems):
        out.append(sopb.JobSpec.from_system(s, jc.params, fixed=jc.fixed, pulled=jc.pulled,
                                            seeds=seeds[r * n:(r + 1) * n], plane_fixed=jc.plane_fixed,
                                            plane_pulled=jc.plane_pulled))
    return out
