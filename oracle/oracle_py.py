"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU
baseline leg of bench.py.  It shares the job description layout of
include/sopb.h (the Params / JobDesc ctypes structures) so both sides read
identical inputs.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "sop-gpu_b200"))
import sopb  # noqa: E402  (structure layouts only: sopb.py loads libsopb.so only when lib() is called)

LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def build() -> None:
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
        sig = {
            "orc_default_params": ([vp], None),
            "orc_generate_seeds": ([i32, i64, vp], None),
            "orc_rforce_n": ([i32, vp, vp], None),
            "orc_hybrid_taus": ([vp, i32, vp], None),
            "orc_job_create": ([vp], vp),
            "orc_job_destroy": ([vp], None),
            "orc_job_status": ([vp], C.c_int),
            "orc_job_step": ([vp], i64),
            "orc_job_advance": ([vp, i64], C.c_int),
            "orc_jobs_advance": ([vp, i32, i64, i32], C.c_int),
            "orc_job_forces": ([vp, vp, vp, vp], None),
            "orc_job_read": ([vp, i32, vp], None),
            "orc_job_write": ([vp, i32, vp], None),
            "orc_job_rebuild": ([vp, i32, i32], None),
            "orc_job_pairlist": ([vp, i32, vp, vp, i32], None),
            "orc_job_observables": ([vp, vp], None),
            "orc_job_log": ([vp, vp, i32], i32),
            "orc_rpy_tensor": ([i32, vp, C.c_float, vp], None),
            "orc_cholesky_ref": ([i32, vp], None),
            "orc_ref_b_matrix": ([i32, vp, vp], None),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def default_params(**kw) -> "sopb.Params":
    """The reference defaults from the oracle's own table, with keyword
    overrides (config-key names); loads no product library."""
    p = sopb.Params()
    lib().orc_default_params(C.byref(p))
    for k, v in kw.items():
        sopb.set_param(p, k, v)
    return p


def generate_seeds(seed: int, count: int) -> np.ndarray:
    out = np.zeros((count, 4), np.uint32)
    lib().orc_generate_seeds(int(seed), int(count), out.ctypes.data)
    return out


def rforce(seeds: np.ndarray):
    """One rforce() per state: returns (gaussians (n,4) f32, advanced states)."""
    s = np.ascontiguousarray(seeds, np.uint32).copy()
    out = np.zeros((s.shape[0], 4), np.float32)
    lib().orc_rforce_n(s.shape[0], s.ctypes.data, out.ctypes.data)
    return out, s


def hybrid_taus(seed4: Sequence[int], draws: int) -> np.ndarray:
    s = np.ascontiguousarray(seed4, np.uint32).copy()
    out = np.zeros(draws, np.uint32)
    lib().orc_hybrid_taus(s.ctypes.data, draws, out.ctypes.data)
    return out


class OracleJob:
    """CPU restatement of one job (same description as sopb.JobSpec)."""

    def __init__(self, spec: "sopb.JobSpec"):
        d = spec.desc()
        self.n = spec.n
        self.h = lib().orc_job_create(C.byref(d))
        if not self.h:
            raise ValueError("oracle rejected the job description")

    def advance(self, nsteps: int) -> int:
        return lib().orc_job_advance(self.h, int(nsteps))

    def step(self) -> int:
        return int(lib().orc_job_step(self.h))

    def status(self) -> int:
        return lib().orc_job_status(self.h)

    def read(self, what: int) -> np.ndarray:
        shapes = {sopb.COORDS: ((self.n, 4), np.float32), sopb.SEEDS: ((self.n, 4), np.uint32),
                  sopb.TEMP: ((self.n,), np.float32), sopb.FORCES: ((self.n, 4), np.float32),
                  sopb.TIPFORCES: ((self.n, 4), np.float32), sopb.PULLSTATE: ((12,), np.float32),
                  sopb.TIPSTATE: ((16,), np.float32), sopb.HISTATE: ((4,), np.float32)}
        shape, dt = shapes[what]
        out = np.zeros(shape, dt)
        lib().orc_job_read(self.h, what, out.ctypes.data)
        return out

    def write(self, what: int, arr: np.ndarray) -> None:
        dt = np.uint32 if what == sopb.SEEDS else np.float32
        a = np.ascontiguousarray(arr, dt)
        lib().orc_job_write(self.h, what, a.ctypes.data)

    def forces(self):
        """(FP32 restatement, FP64 mirror, sum of |terms|) at current coords."""
        f32 = np.zeros((self.n, 4), np.float32)
        f64 = np.zeros((self.n, 4), np.float64)
        a64 = np.zeros((self.n, 4), np.float64)
        lib().orc_job_forces(self.h, f32.ctypes.data, f64.ctypes.data, a64.ctypes.data)
        return f32, f64, a64

    def rebuild(self, possible: bool = True, verlet: bool = True) -> None:
        lib().orc_job_rebuild(self.h, int(possible), int(verlet))

    def pairlist(self, possible: bool = False, cap: Optional[int] = None):
        cap = cap or max(1, self.n - 1)
        counts = np.zeros(self.n, np.int32)
        rows = np.zeros((self.n, cap), np.int32)
        lib().orc_job_pairlist(self.h, int(possible), counts.ctypes.data, rows.ctypes.data, cap)
        return counts, rows

    def observables(self) -> np.ndarray:
        """T, E_fene, E_native, E_pairs, E_total, native contacts, Rg, TEA eps."""
        out = np.zeros(8, np.float64)
        lib().orc_job_observables(self.h, out.ctypes.data)
        return out

    def log(self, max_rows: int = 1 << 16) -> np.ndarray:
        """Drains the pulling / indentation event log (sopb.LOG_ROW rows)."""
        out = np.zeros(max_rows, sopb.LOG_ROW)
        got = lib().orc_job_log(self.h, out.ctypes.data, max_rows)
        return out[:got]

    def close(self) -> None:
        if self.h:
            lib().orc_job_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def jobs_advance(jobs: Sequence[OracleJob], nsteps: int, nthreads: int = 0) -> int:
    arr = (C.c_void_p * len(jobs))(*[j.h for j in jobs])
    return lib().orc_jobs_advance(arr, len(jobs), int(nsteps), int(nthreads))


def rpy_tensor(xyz: np.ndarray, a: float) -> np.ndarray:
    x = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    n = x.shape[0]
    D = np.zeros((3 * n, 3 * n), np.float64)
    lib().orc_rpy_tensor(n, x.ctypes.data, float(a), D.ctypes.data)
    return D


def cholesky_ref(M: np.ndarray) -> np.ndarray:
    A = np.ascontiguousarray(M, np.float32).copy()
    lib().orc_cholesky_ref(A.shape[0], A.ctypes.data)
    return A


def ref_b_matrix(n: int, M: np.ndarray) -> np.ndarray:
    A = np.ascontiguousarray(M, np.float32)
    B = np.zeros((3 * n, 3 * n), np.float64)
    lib().orc_ref_b_matrix(n, A.ctypes.data, B.ctypes.data)
    return B
