"""Continuous-batching serving loop over the sopb C ABI.

Requests (a job spec plus a number of steps) arrive at any time.  The loop
admits waiting requests while their device footprint fits the HBM budget
(admission by footprint, sopb_job_footprint), advances the in-flight jobs
and retires finished ones (status, optional coordinates, asynchronous
destroy), recording completion latency.

Two kinds of job share the GPU:
  - replica-resident jobs (no HI, up to 2048 beads): one CTA holds a whole
    job, so they run best together, many jobs per launch;
  - grid-path jobs (HI or above 2048 beads): chains of small launches.
A resident CTA needs an empty SM, which a GPU kept busy by small CTAs
rarely offers, so the two kinds alternate in phases:
  - batch phase: every resident job with steps left runs up to
    `batch_quantum` steps in one ragged launch on the batch stream (each
    job's CTA stops at its own count), started when no grid quantum is in
    flight so that its CTAs find empty SMs; grid quanta then fill the SMs it
    leaves free;
  - grid phase: grid jobs run quanta of about `slice_us` of device time on
    `grid_lanes` streams (sopb_run_on), one quantum per lane at a time, the
    jobs with the least remaining work first; a lane takes the next quantum
    as soon as its previous one finished.  When resident jobs are waiting
    and no batch launch runs, no new quanta start, and the next batch launch
    begins once the running ones drain.
State stays on the device for a job's whole life, and a job's result does
not depend on what it shares the GPU with (its launch shape is a function
of the job alone).
"""
from __future__ import annotations

import collections
import dataclasses
import time
from typing import Deque, Dict, List, Optional

import numpy as np

import sopb

# jobs the library runs with the replica-resident kernel (one CTA per job)
RESIDENT_MAX_BEADS = 2048


def on_grid_path(spec: "sopb.JobSpec") -> bool:
    p = spec.params
    return spec.n > RESIDENT_MAX_BEADS or bool(p.hi_on) or bool(p.grid_path)


def step_cost(spec: "sopb.JobSpec") -> float:
    """Device time of one step of a grid-path job alone, microseconds, on
    B200 (sizes quanta and orders jobs): a per-step launch chain, all-pairs
    O(n^2) sums for HI and the amortised O((3n)^3) factorisation for exact
    HI (fitted to 87 us per TEA step and 3.6 ms per exact step, refresh 10,
    at 4000 beads), O(n) otherwise."""
    p, n = spec.params, float(spec.n)
    if not p.hi_on:
        return 20.0 + 5e-4 * n
    cost = 40.0 + 3e-6 * n * n
    if p.hi_exact:
        cost += 20.0 + 5.6e-7 * n ** 3 / max(1, int(p.hi_refresh))
    return cost


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
                 quantum: int = 1000, keep_coords: bool = False, slice_us: float = 1.0e4, grid_lanes: int = 16,
                 batch_quantum: int = 2000):
        import torch
        self.torch = torch
        self.ctx = ctx
        self.budget = hbm_budget
        self.max_inflight = max_inflight
        self.quantum = quantum          # upper bound of a grid job's quantum, steps
        self.slice_us = slice_us
        self.keep_coords = keep_coords
        self.batch_stream = torch.cuda.Stream()
        self.lanes = [torch.cuda.Stream() for _ in range(grid_lanes)]
        self.waiting: Deque[Request] = collections.deque()
        self.inflight: Dict[int, dict] = {}
        self.chain: Deque[tuple] = collections.deque()   # batch phase: (event, finishing rids)
        self.batch_quantum = batch_quantum
        self.grid_turn = False          # a grid round is due after a batch phase
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
            st = dict(req=req, job=job, done=0, fp=fp, admitted=self.now(), grid=on_grid_path(req.spec),
                      event=None, lane=None, q=0, queued=False)
            if st["grid"]:
                st["cost"] = step_cost(req.spec)
                q = int(self.slice_us / st["cost"]) // 10 * 10
                st["q"] = max(10, min(self.quantum, q))
            self.inflight[req.rid] = st
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

    def _poll_chain(self) -> bool:
        moved = False
        while self.chain and self.chain[0][0].query():
            _, rids = self.chain.popleft()
            for rid in rids:
                st = self.inflight[rid]
                if st["done"] >= st["req"].steps:
                    self._retire(rid)
                else:
                    st["queued"] = False      # more steps in a later batch phase
            moved = True
        return moved

    def _start_batch(self) -> None:
        """Up to `batch_quantum` more steps of every waiting resident job in
        one ragged launch (sopb_run_ragged: each job its own step count)."""
        members = [rid for rid, st in self.inflight.items() if not st["grid"] and not st["queued"]]
        left = [min(self.batch_quantum, self.inflight[r]["req"].steps - self.inflight[r]["done"]) for r in members]
        for rid, n in zip(members, left):
            self.inflight[rid]["queued"] = True
            self.inflight[rid]["done"] += n
        self.ctx.run([self.inflight[r]["job"] for r in members], left, stream=self.batch_stream.cuda_stream)
        ev = self.torch.cuda.Event()
        ev.record(self.batch_stream)
        self.chain.append((ev, members))
        self.grid_turn = True            # grid quanta fill the SMs the batch leaves free

    def _poll_grid(self, launch: bool) -> bool:
        """Retires grid jobs whose last quantum finished; with `launch`, starts
        quanta on free lanes, least remaining work first (a lane runs one
        quantum at a time, so the GPU holds at most one per lane)."""
        moved = False
        idle = []
        busy = set()
        for rid in [r for r, st in self.inflight.items() if st["grid"]]:
            st = self.inflight[rid]
            if st["event"] is not None:
                if not st["event"].query():
                    busy.add(id(st["lane"]))
                    continue
                st["event"] = None
                moved = True
            if st["done"] >= st["req"].steps:
                self._retire(rid)
                continue
            idle.append(rid)
        if not launch:
            return moved
        free = [ln for ln in self.lanes if id(ln) not in busy]
        idle.sort(key=lambda r: (self.inflight[r]["req"].steps - self.inflight[r]["done"]) * self.inflight[r]["cost"])
        for rid, lane in zip(idle, free):
            st = self.inflight[rid]
            n = min(st["q"], st["req"].steps - st["done"])
            st["lane"] = lane
            self.ctx.run([st["job"]], n, stream=lane.cuda_stream)
            st["done"] += n
            ev = self.torch.cuda.Event()
            ev.record(lane)
            st["event"] = ev
            moved = True
        return moved

    def step(self) -> bool:
        """One pass of the loop: admit, poll, and start whatever may start."""
        self._admit()
        moved = self._poll_chain()
        if self.grid_turn:                   # grid quanta beside the placed batch launch
            self.grid_turn = False
            moved |= self._poll_grid(launch=True)
        if self.chain:                       # batch launch running: keep the lanes busy
            return self._poll_grid(launch=True) or moved
        waiting_resident = any(not st["grid"] and not st["queued"] for st in self.inflight.values())
        if waiting_resident:
            # drain the grid quanta in flight, then the batch phase
            moved |= self._poll_grid(launch=False)
            if all(st["event"] is None for st in self.inflight.values() if st["grid"]):
                self._start_batch()
                moved = True
            return moved
        return self._poll_grid(launch=True) or moved

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
            if not self.step():
                time.sleep(2e-4)
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
