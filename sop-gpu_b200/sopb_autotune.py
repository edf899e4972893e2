"""Autotuner of the launch policies over a job mix.

Two policies of a context decide how its jobs are launched, and both are
functions of the job and the policy only, so tuning them on the mix that
will run keeps every job's result independent of what it shares the GPU
with:
  * the resident kernel's shape (lanes per bead, beads per lane group, CTA
    size cap) for the jobs of up to 2048 beads without HI;
  * the HI policy of grid-path HI jobs: the exact-HI factorisation's
    outer-panel width in 128-column tiles and the CTAs per SM that the
    O(N^2) TEA and D F sums are sliced for.
The tuner creates the jobs under each candidate, runs a warm-up, then times
`repeats` runs of a fixed number of steps on the device and keeps the best
of them (the runs of one candidate differ by a few per cent; a trial is
long enough that candidates ten per cent apart separate).  The fastest
candidates are left set on the context.
"""
from __future__ import annotations

import itertools
from typing import Iterable, List, Optional, Sequence, Tuple

import sopb

Policy = Tuple[int, float, int]   # (lanes per bead, beads per lane group, max CTA size)
HiPolicy = Tuple[int, int]        # (outer-panel tile columns, CTAs per SM of the O(N^2) sums)

DEFAULT_CANDIDATES: List[Policy] = [
    (lpb, bpg, maxb)
    for lpb, bpg, maxb in itertools.product((2, 4, 8, 16), (1.0, 2.0), (512, 1024))
]
DEFAULT_HI_CANDIDATES: List[HiPolicy] = list(itertools.product((2, 4, 8), (2, 4, 8)))


def _timed(ctx: "sopb.Context", jobs, steps: int, repeats: int) -> float:
    """Best of `repeats` device-timed runs of `steps` steps (seconds)."""
    import torch
    stream = torch.cuda.Stream()
    best = float("inf")
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx.sync()
        e0.record(stream)
        ctx.run(jobs, steps, stream=stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    return best


def time_policy(ctx: "sopb.Context", specs: Sequence["sopb.JobSpec"], policy: Policy, steps: int,
                repeats: int = 2) -> float:
    ctx.set_shape_policy(*policy)
    jobs = [ctx.job(s) for s in specs]
    try:
        ctx.run(jobs, 10)                      # list builds at step 0 and warm-up
        ctx.sync()
        return _timed(ctx, jobs, steps, repeats)
    finally:
        for j in jobs:
            j.destroy()


def time_hi_policy(ctx: "sopb.Context", specs: Sequence["sopb.JobSpec"], policy: HiPolicy, steps: int,
                   repeats: int = 2) -> float:
    ctx.set_hi_policy(*policy)
    jobs = [ctx.job(s) for s in specs]
    try:
        ctx.run(jobs, 10)                      # the first factorisation and list builds
        ctx.sync()
        return _timed(ctx, jobs, steps, repeats)
    finally:
        for j in jobs:
            j.destroy()


def autotune(ctx: "sopb.Context", specs: Sequence["sopb.JobSpec"], steps: int = 1000,
             candidates: Optional[Iterable[Policy]] = None, log=None, repeats: int = 2,
             hi_steps: int = 20, hi_candidates: Optional[Iterable[HiPolicy]] = None) -> dict:
    """Tunes the resident shape on the mix's resident jobs and the HI policy
    on its HI jobs (each job kind, exact and TEA, represented by its largest
    job).  Returns {"policy": best shape, "table": [(policy, s, bead-steps/s)],
    "hi_policy": best HI policy or None, "hi_table": [...]} and sets both."""
    resident = [s for s in specs if not s.params.hi_on and s.n <= 2048 and not s.params.grid_path]
    hi = [s for s in specs if s.params.hi_on]
    out = {"policy": None, "table": [], "hi_policy": None, "hi_table": []}
    if resident:
        beads = sum(s.n for s in resident)
        for pol in (candidates or DEFAULT_CANDIDATES):
            dt = time_policy(ctx, resident, pol, steps, repeats)
            out["table"].append((pol, dt, beads * steps / dt))
            if log:
                log("autotune lpb=%d bpg=%g maxb=%d: %.3e bead-steps/s" % (pol[0], pol[1], pol[2], beads * steps / dt))
        out["policy"] = min(out["table"], key=lambda t: t[1])[0]
        ctx.set_shape_policy(*out["policy"])
    if hi:
        reps = []
        for exact in (1, 0):
            kind = [s for s in hi if bool(s.params.hi_exact) == bool(exact)]
            if kind:
                reps.append(max(kind, key=lambda s: s.n))
        beads = sum(s.n for s in reps)
        for pol in (hi_candidates or DEFAULT_HI_CANDIDATES):
            dt = time_hi_policy(ctx, reps, pol, hi_steps, repeats)
            out["hi_table"].append((pol, dt, beads * hi_steps / dt))
            if log:
                log("autotune hi panel=%d ctas/sm=%d: %.3e bead-steps/s" % (pol[0], pol[1], beads * hi_steps / dt))
        out["hi_policy"] = min(out["hi_table"], key=lambda t: t[1])[0]
        ctx.set_hi_policy(*out["hi_policy"])
    return out
