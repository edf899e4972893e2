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
Resident jobs run in ragged launches of up to `batch_quantum` steps (each
job's CTA stops at its own count) on a pool of highest-priority streams:
as soon as resident jobs are waiting and a pool stream is free, they start,
beside any batch already running, and the block scheduler hands their CTAs
the next SMs that the short grid-path kernels free.  Grid jobs run quanta of
about `slice_us` of device time on `grid_lanes` lowest-priority streams
(sopb_run_on), one quantum per lane at a time; a lane takes the next quantum
as soon as its previous one finished.  The jobs with the most time left (by
the measured device time of their last quantum, the cost model before
that; they set when the stream is done) get the `long_lanes` lanes at the
greatest priority, one level above the resident batches; the rest go least
remaining work first.
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
    B200, which sizes a job's first quantum and orders jobs until its own
    quanta have been timed: a per-step launch chain, all-pairs O(n^2) sums
    for HI and, for exact HI, the factorisation amortised over its refresh
    period -- up to 128 beads one CTA (about 0.023 n^2 us), above it the
    chain of 3n/128 tile columns (about 3.8 n us) plus the O(n^2) apply --
    (fitted to 66 us per TEA step and 1.79 ms per exact step with refresh 10
    at 4000 beads, 71 and 224 us per exact step with refresh 1 at 40 and 90
    beads), O(n) otherwise."""
    p, n = spec.params, float(spec.n)
    if not p.hi_on:
        return 20.0 + 5e-4 * n
    cost = 40.0 + 2e-6 * n * n
    if p.hi_exact:
        refresh = max(1, int(p.hi_refresh))
        if n <= 128:
            cost += 25.0 + 0.023 * n * n / refresh
        else:
            cost += 8e-6 * n * n + 3.8 * n / refresh
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
                 batch_quantum: int = 2000, batch_streams: int = 4, long_lanes: int = 4):
        import torch
        self.torch = torch
        self.ctx = ctx
        self.budget = hbm_budget
        self.max_inflight = max_inflight
        self.quantum = quantum          # upper bound of a grid job's quantum, steps
        self.slice_us = slice_us
        self.keep_coords = keep_coords
        lo, hi = torch.cuda.Stream.priority_range() if hasattr(torch.cuda.Stream, "priority_range") else (0, -1)
        # the first `long_lanes` lanes take the grid jobs with the most time
        # left (they set when the stream is done) at the greatest priority;
        # resident batches one level below; the other lanes at the least
        # (the library runs an exact-HI factorisation's chain one level above
        # its lane where there is one)
        self.batch_streams = [torch.cuda.Stream(priority=min(lo, hi + 1)) for _ in range(batch_streams)]
        self.long_lanes = min(long_lanes, grid_lanes)
        self.lanes = [torch.cuda.Stream(priority=hi if k < self.long_lanes else lo) for k in range(grid_lanes)]
        self.waiting: Deque[Request] = collections.deque()
        self.inflight: Dict[int, dict] = {}
        self.chain: List[tuple] = []    # running batch launches: (event, stream, rids)
        self.batch_quantum = batch_quantum
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
                      event=None, start=None, qn=0, lane=None, q=0, queued=False, meas=None)
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
        for item in [c for c in self.chain if c[0].query()]:
            self.chain.remove(item)
            for rid in item[2]:
                st = self.inflight[rid]
                if st["done"] >= st["req"].steps:
                    self._retire(rid)
                else:
                    st["queued"] = False      # more steps in a later batch launch
            moved = True
        return moved

    def _start_batch(self) -> bool:
        """Up to `batch_quantum` more steps of every waiting resident job in
        one ragged launch (sopb_run_ragged: each job its own step count) on a
        free batch stream, beside the batch launches already running."""
        members = [rid for rid, st in self.inflight.items() if not st["grid"] and not st["queued"]]
        busy = {id(c[1]) for c in self.chain}
        free = [b for b in self.batch_streams if id(b) not in busy]
        if not members or not free:
            return False
        stream = free[0]
        left = [min(self.batch_quantum, self.inflight[r]["req"].steps - self.inflight[r]["done"]) for r in members]
        for rid, n in zip(members, left):
            self.inflight[rid]["queued"] = True
            self.inflight[rid]["done"] += n
        self.ctx.run([self.inflight[r]["job"] for r in members], left, stream=stream.cuda_stream)
        ev = self.torch.cuda.Event()
        ev.record(stream)
        self.chain.append((ev, stream, members))
        return True

    def _poll_grid(self, launch: bool) -> bool:
        """Retires grid jobs whose last quantum finished; with `launch`, starts
        quanta on free lanes: the jobs with the most time left on the long
        lanes, the others least work first (a lane runs one quantum at a
        time, so the GPU holds at most one per lane)."""
        moved = False
        idle = []
        busy = set()
        for rid in [r for r, st in self.inflight.items() if st["grid"]]:
            st = self.inflight[rid]
            if st["event"] is not None:
                if not st["event"].query():
                    busy.add(id(st["lane"]))
                    continue
                # measured time per step of this job (device time of its last
                # quantum on its lane), which ranks the jobs by time left
                us = st["start"].elapsed_time(st["event"]) * 1e3 / max(1, st["qn"])
                st["meas"] = us if st["meas"] is None else 0.5 * (st["meas"] + us)
                st["event"] = None
                moved = True
            if st["done"] >= st["req"].steps:
                self._retire(rid)
                continue
            idle.append(rid)
        if not launch:
            return moved
        def work(r):
            st = self.inflight[r]
            per = st["meas"] if st["meas"] is not None else st["cost"]
            return (st["req"].steps - st["done"]) * per
        # the jobs with the most work left go to free long lanes, the others
        # (least work first) to free ordinary lanes
        long_free = [ln for ln in self.lanes[:self.long_lanes] if id(ln) not in busy]
        rest_free = [ln for ln in self.lanes[self.long_lanes:] if id(ln) not in busy]
        idle.sort(key=work, reverse=True)
        pairs = list(zip(idle, long_free))
        rest = sorted(idle[len(pairs):], key=work)
        pairs += list(zip(rest, rest_free))
        for rid, lane in pairs:
            st = self.inflight[rid]
            n = min(st["q"], st["req"].steps - st["done"])
            st["lane"] = lane
            t0 = self.torch.cuda.Event(enable_timing=True)
            t0.record(lane)
            self.ctx.run([st["job"]], n, stream=lane.cuda_stream)
            st["done"] += n
            ev = self.torch.cuda.Event(enable_timing=True)
            ev.record(lane)
            st["start"], st["event"], st["qn"] = t0, ev, n
            moved = True
        return moved

    def step(self) -> bool:
        """One pass of the loop: admit, retire what finished, start the
        resident jobs that wait and the grid quanta that fit the lanes."""
        self._admit()
        moved = self._poll_chain()
        moved |= self._start_batch()
        moved |= self._poll_grid(launch=True)
        return moved

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
