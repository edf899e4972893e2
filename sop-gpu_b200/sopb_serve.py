"""Continuous-batching serving loop over the sopb C ABI.

Requests (a job spec plus a number of steps) arrive at any time.  The loop:
  1. admits waiting requests while their device footprint fits the HBM
     budget and a slot is free (admission by footprint, sopb_job_footprint);
  2. advances every in-flight job by one quantum of steps with one sopb_run
     call: all resident jobs share one ragged launch, so work of jobs that
     arrived at different times overlaps on the device;
  3. retires finished jobs (reads their final coordinates, frees their
     state) and records completion latency.
State (coordinates, lists, RNG states, HI buffers) stays on the device for
a job's whole life.  A job's result does not depend on what it shares the
GPU with: its launch shape is a function of the job alone.
"""
from __future__ import annotations

import collections
import dataclasses
import heapq
import time
from typing import Callable, Deque, Dict, List, Optional

import numpy as np

import sopb


@dataclasses.dataclass
class Request:
    rid: int
    spec: "sopb.JobSpec"
    steps: int
    arrival: float = 0.0          # seconds on the serving clock
    kind: str = ""


@dataclasses.dataclass
class Result:
    rid: int
    n: int
    steps: int
    kind: str
    arrival: float
    admitted: float
    finished: float
    status: int
    coords: Optional[np.ndarray]

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class Server:
    def __init__(self, ctx: "sopb.Context", hbm_budget: int = 64 << 30, max_inflight: int = 2048,
                 quantum: int = 1000, keep_coords: bool = False):
        self.ctx = ctx
        self.budget = hbm_budget
        self.max_inflight = max_inflight
        self.quantum = quantum
        self.keep_coords = keep_coords
        self.waiting: Deque[Request] = collections.deque()
        self.inflight: Dict[int, dict] = {}
        self.used = 0
        self.peak_used = 0
        self.peak_inflight = 0
        self.results: List[Result] = []
        self.t0 = time.perf_counter()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def submit(self, req: Request) -> None:
        self.waiting.append(req)

    def _admit(self) -> None:
        while self.waiting and len(self.inflight) < self.max_inflight:
            req = self.waiting[0]
            fp = req.spec.footprint()
            if self.used + fp > self.budget and self.inflight:
                break                     # wait for memory to free up
            self.waiting.popleft()
            try:
                job = self.ctx.job(req.spec)
            except sopb.SopbError as e:
                self.results.append(Result(req.rid, req.spec.n, req.steps, req.kind, req.arrival, self.now(),
                                           self.now(), e.code, None))
                continue
            self.used += fp
            self.peak_used = max(self.peak_used, self.used)
            self.inflight[req.rid] = dict(req=req, job=job, done=0, fp=fp, admitted=self.now())
            self.peak_inflight = max(self.peak_inflight, len(self.inflight))

    def _retire(self, rid: int) -> None:
        st = self.inflight.pop(rid)
        job = st["job"]
        status = job.status()
        coords = job.read(sopb.COORDS) if self.keep_coords else None
        job.destroy()
        self.used -= st["fp"]
        r = st["req"]
        self.results.append(Result(rid, r.spec.n, r.steps, r.kind, r.arrival, st["admitted"], self.now(), status, coords))

    def step(self) -> int:
        """One serving iteration: admit, advance one quantum, retire."""
        self._admit()
        if not self.inflight:
            return 0
        # jobs needing a full quantum share one launch; the rest finish now
        groups: Dict[int, List[int]] = collections.defaultdict(list)
        for rid, st in self.inflight.items():
            left = st["req"].steps - st["done"]
            groups[min(self.quantum, left)].append(rid)
        for nsteps, rids in sorted(groups.items(), reverse=True):
            self.ctx.run([self.inflight[r]["job"] for r in rids], nsteps)
            for r in rids:
                self.inflight[r]["done"] += nsteps
        self.ctx.sync()
        finished = [rid for rid, st in self.inflight.items() if st["done"] >= st["req"].steps]
        for rid in finished:
            self._retire(rid)       # a failed job stops advancing; its status is reported here
        return len(finished)

    def serve(self, arrivals: List[Request], until_idle: bool = True) -> List[Result]:
        """Replays `arrivals` (sorted by arrival time, seconds) on the real
        clock, serving until every request finished."""
        pending = collections.deque(sorted(arrivals, key=lambda r: r.arrival))
        self.t0 = time.perf_counter()
        while pending or self.waiting or self.inflight:
            t = self.now()
            while pending and pending[0].arrival <= t:
                self.submit(pending.popleft())
            if not self.inflight and not self.waiting and pending:
                time.sleep(max(0.0, min(0.01, pending[0].arrival - t)))
                continue
            self.step()
        return self.results


def summarize(results: List[Result], wall: float) -> dict:
    ok = [r for r in results if r.status == 0]
    lat = np.array([r.latency for r in ok]) if ok else np.zeros(1)
    bead_steps = float(sum(r.n * r.steps for r in ok))
    return {
        "jobs": len(results), "ok": len(ok), "failed": len(results) - len(ok),
        "bead_steps": bead_steps, "wall_s": wall, "throughput": bead_steps / wall if wall > 0 else 0.0,
        "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
        "mean_s": float(lat.mean()),
    }
