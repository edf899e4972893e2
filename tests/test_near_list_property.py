"""The argument behind the near list of the Verlet rebuilds, checked in
FP32 on the CPU with the kernels' arithmetic (differences, squares and sums
rounded to nearest; r^2 < t with t the smallest float whose square root
reaches the cutoff): while every bead stays within half the skin, less
0.01 A, of where the near list was built, filtering the near rows gives the
same Verlet rows, entry for entry and in order, as filtering all possible
pairs; a pair that closes by more than the skin is what the drift bound
keeps out."""
import math

import numpy as np

PAIRLIST_CUTOFF = 20.0
POSSIBLE_CUTOFF = 40.0


def threshold(cut):
    t = np.float32(cut) * np.float32(cut)
    while t > 0 and math.sqrt(float(np.nextafter(t, np.float32(0)))) >= cut:
        t = np.nextafter(t, np.float32(0))
    while math.sqrt(float(t)) < cut:
        t = np.nextafter(t, np.float32(np.inf))
    return np.float32(t)


def dist2(x, i, q):
    d = (x[q] - x[i]).astype(np.float32)
    return np.float32(np.float32(d[..., 0] * d[..., 0]) + np.float32(d[..., 1] * d[..., 1])) + np.float32(
        d[..., 2] * d[..., 2])


def rows(x, candidates, t):
    out = []
    for i, cand in enumerate(candidates):
        cand = np.asarray(cand, np.int64)
        keep = dist2(x, i, cand) < t if len(cand) else np.zeros(0, bool)
        out.append(cand[keep])
    return out


def possible_rows(x):
    n = len(x)
    t = threshold(POSSIBLE_CUTOFF)
    return [np.array([q for q in range(n) if q != i and dist2(x, i, np.array([q]))[0] < t]) for i in range(n)]


def test_near_rows_give_the_full_filter_while_drift_is_below_half_the_skin():
    rng = np.random.default_rng(7)
    skin = 4.0
    limit = 0.5 * skin - 0.01
    x_ref = rng.uniform(0.0, 60.0, size=(300, 3)).astype(np.float32)
    poss = possible_rows(x_ref)
    near = rows(x_ref, poss, threshold(PAIRLIST_CUTOFF + skin))
    t = threshold(PAIRLIST_CUTOFF)
    for trial in range(6):
        # every bead moves by up to the limit, in a random direction
        step = rng.normal(size=x_ref.shape)
        step *= (rng.uniform(0.0, 1.0, size=(len(x_ref), 1)) * limit) / np.linalg.norm(step, axis=1, keepdims=True)
        x = (x_ref + step).astype(np.float32)
        full, from_near = rows(x, poss, t), rows(x, near, t)
        for a, b in zip(full, from_near):
            assert np.array_equal(a, b)


def test_a_pair_closing_by_more_than_the_skin_is_missed_without_the_bound():
    skin = 4.0
    x_ref = np.array([[0.0, 0.0, 0.0], [24.5, 0.0, 0.0]], np.float32)
    poss = [np.array([1]), np.array([0])]
    near = rows(x_ref, poss, threshold(PAIRLIST_CUTOFF + skin))
    assert all(len(r) == 0 for r in near)              # 24.5 A apart: not near
    x = np.array([[2.3, 0.0, 0.0], [22.2, 0.0, 0.0]], np.float32)   # each moved 2.3 A > skin / 2
    full = rows(x, poss, threshold(PAIRLIST_CUTOFF))
    assert len(full[0]) == 1                           # 19.9 A: a Verlet pair the near rows lack
