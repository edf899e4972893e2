"""Autotuner of the resident kernel's launch shape over a job mix.

The shape of a job (lanes per bead, CTA size) is a function of the job and
of the context's shape policy only, so tuning the policy on the mix that
will run keeps every job's result independent of what it shares the GPU
with.  The tuner creates the mix under each candidate policy, times a short
run on the device and leaves the fastest policy set on the context.
"""
from __future__ import annotations

import itertools
import time
from typing import Iterable, List, Optional, Sequence, Tuple

import sopb

Policy = Tuple[int, float, int]   # (lanes per bead, beads per lane group, max CTA size)

DEFAULT_CANDIDATES: List[Policy] = [
    (lpb, bpg, maxb)
    for lpb, bpg, maxb in itertools.product((4, 8, 16), (1.0, 2.0, 4.0), (1024,))
]


def time_policy(ctx: "sopb.Context", specs: Sequence["sopb.JobSpec"], policy: Policy, steps: int) -> float:
    ctx.set_shape_policy(*policy)
    jobs = [ctx.job(s) for s in specs]
    try:
        ctx.run(jobs, 10)                      # list builds at step 0 and warm-up
        ctx.sync()
        t0 = time.perf_counter()
        ctx.run(jobs, steps)
        ctx.sync()
        return time.perf_counter() - t0
    finally:
        for j in jobs:
            j.destroy()


def autotune(ctx: "sopb.Context", specs: Sequence["sopb.JobSpec"], steps: int = 100,
             candidates: Optional[Iterable[Policy]] = None, log=None) -> dict:
    """Returns {"policy": best, "table": [(policy, seconds, bead-steps/s)]} and
    sets the best policy on `ctx`."""
    beads = sum(s.n for s in specs)
    table = []
    for pol in (candidates or DEFAULT_CANDIDATES):
        dt = time_policy(ctx, specs, pol, steps)
        table.append((pol, dt, beads * steps / dt))
        if log:
            log("autotune lpb=%d bpg=%g maxb=%d: %.3e bead-steps/s" % (pol[0], pol[1], pol[2], beads * steps / dt))
    best = min(table, key=lambda t: t[1])[0]
    ctx.set_shape_policy(*best)
    return {"policy": best, "table": table}
