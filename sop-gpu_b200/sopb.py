"""ctypes binding of the sopb C ABI (include/sopb.h).

This is the Python face of the library used by the test-suite, the benchmark
and the serving loop.  It loads the in-tree ``libsopb.so`` and fails loudly
when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Iterable, List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsopb.so")

# status codes (include/sopb.h)
OK, ERR_INVALID, ERR_CAPACITY, ERR_NONFINITE, ERR_CUDA, ERR_TIMEOUT, ERR_NOMEM, ERR_UNSUPPORTED, ERR_HI, ERR_NODEVICE = range(10)
PULL_END_TO_END, PULL_VECTOR = 0, 1
HI_B_CHOLESKY, HI_B_REFCOMPAT = 0, 1
COORDS, SEEDS, TEMP, FORCES, TIPFORCES, PULLSTATE, TIPSTATE, HISTATE, HIFACTOR, OBSERVABLES = range(10)
OBSERVABLE_NAMES = ("T", "E_fene", "E_native", "E_pairs", "E_total", "native_contacts", "Rg", "tea_eps")
# event-log rows (sopb_log_row): pulling lines every pullFreq, tip lines every nav
LOG_PULL, LOG_TIP, LOG_PLANE = 1, 2, 3
LOG_ROW = np.dtype([("kind", "<i4"), ("pad", "<i4"), ("step", "<i8"), ("v", "<f4", (12,))])

F3 = C.c_float * 3


class Params(C.Structure):
    """sopb_params: the reference's config keys for one job."""

    _fields_ = [
        ("timestep", C.c_float), ("zeta", C.c_float), ("temperature", C.c_float),
        ("minimization", C.c_int32), ("heating", C.c_int32), ("initialT", C.c_float), ("deltaT", C.c_float),
        ("tempFreq", C.c_int32),
        ("kspring_cov", C.c_float), ("R_limit", C.c_float),
        ("a", C.c_float), ("el", C.c_float), ("pairs_cutoff", C.c_float),
        ("pairlist_cutoff", C.c_float), ("pairs_freq", C.c_int32), ("pairs_threshold", C.c_float),
        ("possiblepairs_freq", C.c_int32), ("max_pairs", C.c_int32), ("max_possiblePairs", C.c_int32),
        ("nav", C.c_int32), ("stride", C.c_int32),
        ("pulling", C.c_int32), ("deltax", C.c_float), ("k_trans", C.c_float), ("fconst", C.c_float),
        ("pullFreq", C.c_int32), ("pull_direction", C.c_int32), ("pullVector", F3),
        ("fixedEnd", C.c_int32), ("pulledEnd", C.c_int32),
        ("indentation", C.c_int32), ("indentationChip", F3), ("indentationTip", F3),
        ("indentationDirection", F3), ("indentationSurfaceR0", F3), ("indentationSurfaceN", F3),
        ("indentationTipR", C.c_float), ("indentationKs", C.c_float), ("indentationDeltaX", C.c_float),
        ("indentationMoveSurface", C.c_int32), ("indentationFixTrans", C.c_int32),
        ("indentationTipSigma", C.c_float), ("indentationTipEl", C.c_float), ("indentationTipA", C.c_float),
        ("indentationTipB", C.c_float),
        ("indentationSurfSigma", C.c_float), ("indentationSurfEl", C.c_float), ("indentationSurfA", C.c_float),
        ("indentationSurfB", C.c_float),
        ("indentationTipZeta", C.c_float), ("indentationRetractionStep", C.c_int64),
        ("hi_on", C.c_int32), ("hi_exact", C.c_int32), ("hi_a", C.c_float), ("hi_epsilon_freq", C.c_int32),
        ("hi_capricious", C.c_int32), ("hi_unlisted", C.c_int32), ("hi_epsmax", C.c_float),
        ("hi_b_mode", C.c_int32), ("hi_refresh", C.c_int32), ("lanes_per_bead", C.c_int32),
        ("cell_list", C.c_int32), ("grid_path", C.c_int32), ("R_limit_bond", C.c_float),
        ("log_rows", C.c_int32),
        ("indentationDiscreteSurf", C.c_int32), ("indentationSurfaceSize", C.c_int32),
        ("indentationSurfaceStep", C.c_float), ("indentationPairsCutoff", C.c_float),
        ("pullingPlane", C.c_int32), ("pullingPlaneDeltax", C.c_float), ("pullingPlaneKs", C.c_float),
        ("pullingPlaneKsCant", C.c_float), ("pullingPlaneZeta", C.c_float), ("pullingPlaneDir", F3),
        ("pullingPlanePos", F3), ("pullingPlaneUpdateFreq", C.c_int32), ("pullingPlaneOutputFreq", C.c_int32),
        ("verlet_skin", C.c_float), ("reserved2", C.c_int32 * 3),
    ]


class JobDesc(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("xyz", C.c_void_p),
        ("nbonds", C.c_int32), ("bonds", C.c_void_p), ("bonds_r0", C.c_void_p),
        ("nnatives", C.c_int32), ("natives", C.c_void_p), ("natives_r0", C.c_void_p), ("natives_eh", C.c_void_p),
        ("nfixed", C.c_int32), ("fixed", C.c_void_p), ("npulled", C.c_int32), ("pulled", C.c_void_p),
        ("seeds", C.c_void_p), ("seed", C.c_int32), ("reserved", C.c_int32),
        ("params", Params),
        ("nplane_fixed", C.c_int32), ("plane_fixed", C.c_void_p),
        ("nplane_pulled", C.c_int32), ("plane_pulled", C.c_void_p),
    ]


_lib = None


def lib() -> C.CDLL:
    """The loaded libsopb.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libsopb.so not built at %s (run `make -C sop-gpu_b200`)" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
        sig = {
            "sopb_version": ([], C.c_int),
            "sopb_status_string": ([C.c_int], C.c_char_p),
            "sopb_default_params": ([vp], None),
            "sopb_generate_seeds": ([i32, i64, vp], C.c_int),
            "sopb_context_create": ([i32, vp, vp], C.c_int),
            "sopb_context_destroy": ([vp], C.c_int),
            "sopb_context_sync": ([vp], C.c_int),
            "sopb_context_set_shape_policy": ([vp, i32, C.c_float, i32], C.c_int),
            "sopb_context_set_hi_policy": ([vp, i32, i32], C.c_int),
            "sopb_job_footprint": ([vp, vp], C.c_int),
            "sopb_job_create": ([vp, vp, vp], C.c_int),
            "sopb_job_destroy": ([vp], C.c_int),
            "sopb_run": ([vp, vp, i32, i64], C.c_int),
            "sopb_run_on": ([vp, vp, i32, i64, vp], C.c_int),
            "sopb_run_ragged": ([vp, vp, i32, vp, vp], C.c_int),
            "sopb_job_status": ([vp], C.c_int),
            "sopb_job_step": ([vp, vp], C.c_int),
            "sopb_job_size": ([vp, vp], C.c_int),
            "sopb_job_shape": ([vp, vp, vp], C.c_int),
            "sopb_job_read": ([vp, i32, vp], C.c_int),
            "sopb_job_write": ([vp, i32, vp], C.c_int),
            "sopb_job_pairlist": ([vp, i32, vp, vp, i32], C.c_int),
            "sopb_job_rebuild_lists": ([vp, i32, i32], C.c_int),
            "sopb_job_log": ([vp, vp, i32, vp], C.c_int),
            "sopb_jobs_upload_coords": ([vp, vp, i32, vp], C.c_int),
            "sopb_jobs_download_coords": ([vp, vp, i32, vp], C.c_int),
            "sopb_tea_coefficients_noalloc": ([vp, i32, C.c_float, vp, vp, vp], C.c_int),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


class SopbError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        msg = lib().sopb_status_string(code).decode()
        super().__init__("%s: %s (status %d)" % (what, msg, code) if what else "%s (status %d)" % (msg, code))


def check(code: int, what: str = "") -> None:
    if code != OK:
        raise SopbError(code, what)


def default_params(**kw) -> Params:
    """Reference defaults, with keyword overrides (config-key names)."""
    p = Params()
    lib().sopb_default_params(C.byref(p))
    for k, v in kw.items():
        set_param(p, k, v)
    return p


def set_param(p: Params, key: str, value) -> None:
    cur = getattr(p, key)
    if isinstance(cur, C.Array):
        for i, v in enumerate(value):
            cur[i] = v
    else:
        setattr(p, key, value)


def params_dict(p: Params) -> Dict[str, object]:
    out = {}
    for name, _ in Params._fields_:
        v = getattr(p, name)
        out[name] = list(v) if isinstance(v, C.Array) else v
    return out


def generate_seeds(seed: int, count: int) -> np.ndarray:
    out = np.zeros((count, 4), np.uint32)
    check(lib().sopb_generate_seeds(int(seed), int(count), out.ctypes.data), "generate_seeds")
    return out


class JobSpec:
    """Host-side description of one job (a SOP system plus its parameters).

    Keeps the numpy arrays alive while a ``JobDesc`` points at them.
    """

    def __init__(self, xyz, bonds, bonds_r0, natives, natives_r0, natives_eh, params: Params,
                 fixed: Sequence[int] = (), pulled: Sequence[int] = (), seeds: Optional[np.ndarray] = None, seed: int = 0,
                 plane_fixed: Sequence[int] = (), plane_pulled: Sequence[int] = ()):
        self.xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        self.bonds = np.ascontiguousarray(bonds, np.int32).reshape(-1, 2)
        self.bonds_r0 = np.ascontiguousarray(bonds_r0, np.float32).reshape(-1)
        self.natives = np.ascontiguousarray(natives, np.int32).reshape(-1, 2)
        self.natives_r0 = np.ascontiguousarray(natives_r0, np.float32).reshape(-1)
        self.natives_eh = np.ascontiguousarray(natives_eh, np.float32).reshape(-1)
        self.fixed = np.ascontiguousarray(fixed, np.int32).reshape(-1)
        self.pulled = np.ascontiguousarray(pulled, np.int32).reshape(-1)
        self.seeds = None if seeds is None else np.ascontiguousarray(seeds, np.uint32).reshape(-1, 4)
        self.seed = int(seed)
        self.params = params
        self.plane_fixed = np.ascontiguousarray(plane_fixed, np.int32).reshape(-1)
        self.plane_pulled = np.ascontiguousarray(plane_pulled, np.int32).reshape(-1)

    @classmethod
    def from_system(cls, sys_, params: Params, **kw) -> "JobSpec":
        return cls(sys_.xyz, sys_.bonds, sys_.bonds_r0, sys_.natives, sys_.natives_r0, sys_.natives_eh, params, **kw)

    @property
    def n(self) -> int:
        return int(self.xyz.shape[0])

    def desc(self) -> JobDesc:
        d = JobDesc()
        d.n = self.n
        d.xyz = self.xyz.ctypes.data
        d.nbonds = self.bonds.shape[0]
        d.bonds = self.bonds.ctypes.data
        d.bonds_r0 = self.bonds_r0.ctypes.data
        d.nnatives = self.natives.shape[0]
        d.natives = self.natives.ctypes.data
        d.natives_r0 = self.natives_r0.ctypes.data
        d.natives_eh = self.natives_eh.ctypes.data
        d.nfixed = self.fixed.shape[0]
        d.fixed = self.fixed.ctypes.data
        d.npulled = self.pulled.shape[0]
        d.pulled = self.pulled.ctypes.data
        d.seeds = self.seeds.ctypes.data if self.seeds is not None else None
        d.seed = self.seed
        d.params = self.params
        d.nplane_fixed = self.plane_fixed.shape[0]
        d.plane_fixed = self.plane_fixed.ctypes.data
        d.nplane_pulled = self.plane_pulled.shape[0]
        d.plane_pulled = self.plane_pulled.ctypes.data
        return d

    def footprint(self) -> int:
        out = C.c_size_t(0)
        d = self.desc()
        check(lib().sopb_job_footprint(C.byref(d), C.byref(out)), "footprint")
        return int(out.value)


class Job:
    def __init__(self, ctx: "Context", handle: C.c_void_p, n: int):
        self.ctx = ctx
        self.handle = handle
        self.n = n

    def read(self, what: int) -> np.ndarray:
        shapes = {COORDS: ((self.n, 4), np.float32), SEEDS: ((self.n, 4), np.uint32), TEMP: ((self.n,), np.float32),
                  FORCES: ((self.n, 4), np.float32), TIPFORCES: ((self.n, 4), np.float32),
                  PULLSTATE: ((12,), np.float32), TIPSTATE: ((16,), np.float32), HISTATE: ((4,), np.float32),
                  HIFACTOR: ((3 * self.n, 3 * self.n), np.float32), OBSERVABLES: ((8,), np.float64)}
        shape, dt = shapes[what]
        out = np.zeros(shape, dt)
        check(lib().sopb_job_read(self.handle, what, out.ctypes.data), "job_read")
        return out

    def write(self, what: int, arr: np.ndarray) -> None:
        dt = np.uint32 if what == SEEDS else np.float32
        a = np.ascontiguousarray(arr, dt)
        check(lib().sopb_job_write(self.handle, what, a.ctypes.data), "job_write")

    def coords(self) -> np.ndarray:
        return self.read(COORDS)

    def status(self) -> int:
        return lib().sopb_job_status(self.handle)

    def shape(self):
        """(lanes per bead, CTA size) of this job's resident kernel."""
        l, b = C.c_int32(0), C.c_int32(0)
        check(lib().sopb_job_shape(self.handle, C.byref(l), C.byref(b)), "job_shape")
        return int(l.value), int(b.value)

    def step(self) -> int:
        s = C.c_int64(0)
        check(lib().sopb_job_step(self.handle, C.byref(s)), "job_step")
        return int(s.value)

    def pairlist(self, possible: bool = False, cap: Optional[int] = None):
        cap = cap or max(1, self.n - 1)
        counts = np.zeros(self.n, np.int32)
        rows = np.zeros((self.n, cap), np.int32)
        check(lib().sopb_job_pairlist(self.handle, int(possible), counts.ctypes.data, rows.ctypes.data, cap), "pairlist")
        return counts, rows

    def rebuild(self, possible: bool = True, verlet: bool = True) -> None:
        check(lib().sopb_job_rebuild_lists(self.handle, int(possible), int(verlet)), "rebuild")

    def log(self, max_rows: int = 1 << 16) -> np.ndarray:
        """Drains the event log: rows of LOG_ROW, oldest first.  Raises when
        the ring wrapped since the last drain (rows were lost)."""
        out = np.zeros(max_rows, LOG_ROW)
        got = C.c_int32(0)
        check(lib().sopb_job_log(self.handle, out.ctypes.data, max_rows, C.byref(got)), "job_log")
        return out[: got.value]

    def destroy(self) -> None:
        if self.handle:
            check(lib().sopb_job_destroy(self.handle), "job_destroy")
            self.handle = None


class Context:
    """A device context: bead pools, job table and a stream."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        h = C.c_void_p()
        check(lib().sopb_context_create(device, stream, C.byref(h)), "context_create")
        self.handle = h
        self.jobs: List[Job] = []

    def job(self, spec: JobSpec) -> Job:
        h = C.c_void_p()
        d = spec.desc()
        check(lib().sopb_job_create(self.handle, C.byref(d), C.byref(h)), "job_create")
        j = Job(self, h, spec.n)
        self.jobs.append(j)
        return j

    @staticmethod
    def _handles(jobs: Sequence[Job]):
        arr = (C.c_void_p * len(jobs))(*[j.handle for j in jobs])
        return arr

    def run(self, jobs: Sequence[Job], nsteps, stream: Optional[int] = None) -> None:
        """Advances `jobs` by `nsteps` steps (one count for all, or one per
        job), asynchronously, on the context stream or on `stream` (a
        cudaStream_t handle, e.g. a torch stream's cuda_stream)."""
        arr = self._handles(jobs)
        if not np.isscalar(nsteps):
            n = np.ascontiguousarray(nsteps, np.int64)
            if n.shape != (len(jobs),):
                raise ValueError("one step count per job")
            check(lib().sopb_run_ragged(self.handle, arr, len(jobs), n.ctypes.data, stream), "run_ragged")
            return
        if stream is None:
            check(lib().sopb_run(self.handle, arr, len(jobs), int(nsteps)), "run")
        else:
            check(lib().sopb_run_on(self.handle, arr, len(jobs), int(nsteps), stream), "run_on")

    def sync(self) -> None:
        check(lib().sopb_context_sync(self.handle), "sync")

    def set_shape_policy(self, lanes_per_bead: int = 4, beads_per_group: float = 1.0, max_block: int = 1024) -> None:
        """Resident-kernel shape for jobs created from now on (autotuner knob)."""
        check(lib().sopb_context_set_shape_policy(self.handle, int(lanes_per_bead), float(beads_per_group),
                                                  int(max_block)), "set_shape_policy")

    def set_hi_policy(self, chol_panel_tiles: int = 4, hi_ctas_per_sm: int = 8) -> None:
        """HI launch policy for jobs created from now on (autotuner knob):
        exact-HI outer-panel width in 128-column tiles, and the CTAs per SM
        the O(N^2) HI sums are sliced for."""
        check(lib().sopb_context_set_hi_policy(self.handle, int(chol_panel_tiles), int(hi_ctas_per_sm)),
              "set_hi_policy")

    def upload_coords(self, jobs: Sequence[Job], xyzw: np.ndarray) -> None:
        arr = self._handles(jobs)
        check(lib().sopb_jobs_upload_coords(self.handle, arr, len(jobs), xyzw.ctypes.data), "upload")

    def download_coords(self, jobs: Sequence[Job], xyzw: np.ndarray) -> None:
        arr = self._handles(jobs)
        check(lib().sopb_jobs_download_coords(self.handle, arr, len(jobs), xyzw.ctypes.data), "download")

    def close(self) -> None:
        if self.handle:
            check(lib().sopb_context_destroy(self.handle), "context_destroy")
            self.handle = None
            for j in self.jobs:
                j.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
