"""The exact-HI factorisation's stream schedule, checked on the CPU.

chol_refresh (sop-gpu_b200/csrc/sopb_api.cu) factorises the tiled tensor on
three streams -- the chain of single tiles (hp), the rest of each tile
column (ms) and the trailing updates (la) -- ordered by events.  This test
replays the same sequence of launches, event records and waits on a model
of CUDA's stream semantics (a launch follows the stream's earlier work and
every event the stream waited for; an event stands for the work on its
stream when it was recorded) and records what each launch reads and writes:
tensor tiles, the two inverse buffers (by tile-column parity) and the TF32
hi/lo plane slots (by outer-panel parity).  It then requires every pair of
launches that touch the same storage, one of them writing, to be ordered by
the dependency graph the way they are in the host's launch order.  The GPU
computes then what that serial order computes, whatever the interleaving.
The model follows the C++ function line by line; a change there needs the
same change here.
"""
import itertools

import pytest

R = 4   # ring of events per kind (sopb_job::kLkRing)


class Model:
    def __init__(self):
        self.ops = []            # (name, reads, writes)
        self.anc = []            # ancestor bitsets
        self.front = {}          # stream -> set of op indices the next op follows
        self.ev = {}             # event -> set of op indices

    def launch(self, s, name, reads=(), writes=()):
        deps = self.front.get(s, set())
        a = 0
        for d in deps:
            a |= self.anc[d] | (1 << d)
        self.ops.append((name, frozenset(reads), frozenset(writes)))
        self.anc.append(a)
        k = len(self.ops) - 1
        self.front[s] = {k}
        return k

    def rec(self, e, s):
        self.ev[e] = set(self.front.get(s, set()))

    def wait(self, s, e):
        self.front[s] = self.front.get(s, set()) | self.ev.get(e, set())

    def races(self):
        bad = []
        for b, (nb, rb, wb) in enumerate(self.ops):
            for a in range(b):
                na, ra, wa = self.ops[a]
                if (wa & (rb | wb)) or (ra & wb):
                    if not (self.anc[b] >> a) & 1:
                        bad.append((na, nb, sorted(wa & (rb | wb) | ra & wb)[:3]))
        return bad


def refresh(M, T, W, hp, ms, la, st):
    """One chol_refresh, launch for launch."""
    def ten_tiles(tiles, jc0, i0):
        # the tile of each CTA of an update, as k_chol_tc maps blockIdx.x
        out = []
        for b in range(tiles):
            J, top = jc0, i0
            while J < T - 1 and b >= T - top:
                b -= T - top
                J += 1
                top = J
            out.append((top + b, J))
        return out

    def plane(I, k):
        pan = k // W
        return ("plane", pan & 1, I, k - pan * W)

    def update(s, tiles, jc0, i0, k0, k1):
        if tiles > 0 and k1 > k0:
            rd, wr = set(), set()
            for (I, J) in ten_tiles(tiles, jc0, i0):
                rd.add(("ten", I, J))
                wr.add(("ten", I, J))
                for k in range(k0, k1):
                    rd.add(plane(I, k))
                    rd.add(plane(J, k))
            M.launch(s, "update c%d i%d k%d-%d" % (jc0, i0, k0, k1), rd, wr)

    def tiles_from(jc0, i0, jc1):
        return T - i0 + sum(T - J for J in range(jc0 + 1, jc1))

    def solve(s, J, i0, i1):
        if i1 > i0:
            rd = {("inv", J & 1)} | {("ten", I, J) for I in range(i0, i1)}
            wr = {("ten", I, J) for I in range(i0, i1)} | {plane(I, J) for I in range(i0, i1)}
            M.launch(s, "solve c%d i%d-%d" % (J, i0, i1), rd, wr)

    def potrf(J):
        M.launch(hp, "potrf %d" % J, {("ten", J, J)}, {("ten", J, J), ("inv", J & 1)})

    e_pot = [("pot", r) for r in range(R)]
    e_s1 = [("s1", r) for r in range(R)]
    e_cu = [("cu", r) for r in range(R)]
    e_sr = [("sr", r) for r in range(R)]
    M.rec("hp_fork", st)
    M.wait(hp, "hp_fork")
    M.wait(ms, "hp_fork")
    M.launch(hp, "assemble", (), {("ten", I, J) for I in range(T) for J in range(I + 1)})
    rest_pending = False
    for P0 in range(0, T, W):
        P1 = min(T, P0 + W)
        for J in range(P0, P1):
            if J >= 2:
                M.wait(hp, e_sr[(J - 2) % R])
            if J > P0:
                if J == P0 + 1 and P0 > 0:
                    M.wait(hp, "np2")
                update(hp, 1, J, J, P0, J)
                if J + 1 < T:
                    M.wait(ms, e_s1[(J - 1) % R])
                    update(ms, T - J - 1, J, J + 1, P0, J)
                    M.rec(e_cu[J % R], ms)
            potrf(J)
            M.rec(e_pot[J % R], hp)
            if J + 1 < T:
                if J > P0:
                    M.wait(hp, e_cu[J % R])
                elif P0 > 0:
                    M.wait(hp, "np1")
                solve(hp, J, J + 1, J + 2)
                M.rec(e_s1[J % R], hp)
            if J + 2 < T:
                M.wait(ms, e_pot[J % R])
                solve(ms, J, J + 2, T)
                M.rec(e_sr[J % R], ms)
        if P1 < T:
            Q1 = min(T, P1 + W)
            if P1 >= 2:
                M.wait(hp, e_sr[(P1 - 2) % R])
            if rest_pending:
                M.wait(hp, "la_join")
            update(hp, 1, P1, P1, P0, P1)
            M.wait(ms, e_s1[(P1 - 1) % R])
            if rest_pending:
                M.wait(ms, "la_join")
            update(ms, T - P1 - 1, P1, P1 + 1, P0, P1)
            M.rec("np1", ms)
            if Q1 > P1 + 1:
                update(ms, tiles_from(P1 + 1, P1 + 1, Q1), P1 + 1, P1 + 1, P0, P1)
            M.rec("np2", ms)
            if Q1 < T:
                M.wait(la, e_s1[(P1 - 1) % R])
                M.wait(la, e_sr[(P1 - 1) % R])
                update(la, tiles_from(Q1, Q1, T), Q1, Q1, P0, P1)
                M.rec("la_join", la)
                rest_pending = True
    M.rec("hp_join", hp)
    M.rec("ms_join", ms)
    M.wait(st, "hp_join")
    M.wait(st, "ms_join")
    if rest_pending:
        M.wait(st, "la_join")


@pytest.mark.parametrize("alias", [False, True])
@pytest.mark.parametrize("T,W", [(t, w) for t, w in itertools.product([1, 2, 3, 5, 8, 13, 17], [1, 2, 3, 4, 8])]
                         + [(94, 4)])   # 4000 beads with the default outer-panel width
def test_factorisation_schedule_has_no_race(T, W, alias):
    # alias: the caller's stream already at the greatest priority, so the
    # chain and the trailing updates share one stream
    M = Model()
    hp, ms, la, st = "hp", "ms", ("hp" if alias else "la"), "st"
    for _ in range(2):           # two refreshes with the step's apply between
        refresh(M, T, W, hp, ms, la, st)
        M.launch(st, "apply", {("ten", I, J) for I in range(T) for J in range(I + 1)}, ())
    assert M.races() == []


def test_a_missing_wait_is_caught():
    # the check itself: the same schedule without the chain's wait for the
    # rest of the column (e_cu) lets a solve read a tile still being updated
    M = Model()
    orig = Model.wait

    def wait(self, s, e):
        if isinstance(e, tuple) and e[0] == "cu":
            return
        orig(self, s, e)

    M.wait = wait.__get__(M)
    refresh(M, 9, 4, "hp", "ms", "la", "st")
    assert M.races()
