"""The near list of the Verlet rebuilds (verlet_skin) is exact: a job keeping
one (default skin 4 A, or a 0.3 A skin that is renewed every few rebuilds)
follows, bit for bit, the same job whose every Verlet rebuild filters all
possible pairs (skin < 0).  Both launch paths, and a schedule where the
possible pairs are rebuilt at steps without a Verlet rebuild."""
import numpy as np
import pytest

import sopb
from helpers import spec

pytestmark = pytest.mark.gpu

CASES = {
    "resident": dict(n=300, mode="ramp", kw=dict()),
    "resident_pp_between": dict(n=300, mode="clamp", kw=dict(nav=10, pairs_freq=20, possiblepairs_freq=30,
                                                             pairs_threshold=30.0)),
    "grid": dict(n=300, mode="ramp", kw=dict(grid_path=1)),
    "grid_cells": dict(n=6000, mode="free", kw=dict(grid_path=1, cell_list=1, pairs_threshold=30.0,
                                                    max_possiblePairs=2048, max_pairs=512, temperature=2.0)),
    "grid_pp_between": dict(n=3000, mode="clamp", kw=dict(grid_path=1, cell_list=1, nav=10, pairs_freq=20,
                                                          possiblepairs_freq=30, pairs_threshold=30.0,
                                                          max_possiblePairs=2048, max_pairs=512)),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_near_list_trajectory_equals_full_filter(gpu_ctx, case):
    c = CASES[case]
    jobs = [gpu_ctx.job(spec(c["n"], 23, c["mode"], verlet_skin=skin, **c["kw"])) for skin in (-1.0, 0.0, 0.3)]
    for chunk in (30, 170, 200):
        gpu_ctx.run(jobs, chunk)
    full = jobs[0]
    for j in jobs:
        assert j.status() == 0 and j.step() == 400
    for j in jobs[1:]:
        assert np.array_equal(j.read(sopb.COORDS), full.read(sopb.COORDS))
        for possible in (True, False):
            cg, rg = j.pairlist(possible, cap=2048)
            cf, rf = full.pairlist(possible, cap=2048)
            assert np.array_equal(cg, cf) and np.array_equal(rg, rf)
    for j in jobs:
        j.destroy()


def test_skin_outside_range_is_rejected(gpu_ctx):
    for bad in (float("nan"), float("inf"), 5000.0):
        with pytest.raises(sopb.SopbError):
            gpu_ctx.job(spec(100, 1, "free", verlet_skin=bad))
