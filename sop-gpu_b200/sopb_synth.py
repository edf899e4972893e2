"""Seeded synthetic SOP systems in the reference's file formats.

A self-avoiding C-alpha random walk (3.8 A bonds, beads >= 4 A apart) grown
inside a sphere sized for a compact globule (Rg ~ 2.2 N^0.38 A), native
contacts |i-j| > 2 within 8 A with eps_h = 1.5 kcal/mol, r0 = the initial
distance.  Coordinates and parameters are rounded exactly as the reference's
writers round them (PDB ``%8.3f``, .top ``%10.5f``; src/IO/pdbio.cpp:265-280,
src/IO/topio.cpp:211-234) and re-read as its readers read them (atof, then
float), so every implementation starts from identical inputs.

There is no public dataset behind the reference's benchmarks; these seeded
inputs stand in for them with the sizes named by the benchmark configs.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional, Sequence

import numpy as np

BOND = 3.8
MIN_DIST = 4.0
NATIVE_CUTOFF = 8.0
EH = 1.5


@dataclasses.dataclass
class System:
    """One SOP chain system: coordinates and topology, in reference units."""

    xyz: np.ndarray            # (n, 3) float32, PDB-rounded
    bonds: np.ndarray          # (nb, 2) int32
    bonds_r0: np.ndarray       # (nb,) float32
    natives: np.ndarray        # (nn, 2) int32
    natives_r0: np.ndarray     # (nn,) float32
    natives_eh: np.ndarray     # (nn,) float32

    @property
    def n(self) -> int:
        return int(self.xyz.shape[0])


def _round_pdb(x: np.ndarray) -> np.ndarray:
    # "%8.3f" then atof -> double -> float (src/IO/pdbio.cpp:292-337, gsop.cu:185-199)
    return np.array([float("%8.3f" % v) for v in x.reshape(-1)], dtype=np.float64).astype(np.float32).reshape(x.shape)


def _round_top(x: np.ndarray) -> np.ndarray:
    # "%10.5f" then atof -> float (src/IO/topio.cpp:211-234, 268-304)
    return np.array([float("%10.5f" % v) for v in x.reshape(-1)], dtype=np.float64).astype(np.float32).reshape(x.shape)


def target_radius(n: int) -> float:
    """Radius of the confining sphere for an n-bead compact globule."""
    rg = 2.2 * n ** 0.38
    return math.sqrt(5.0 / 3.0) * rg


def random_walk(n: int, seed: int, radius: Optional[float] = None, shape: Optional[Sequence[float]] = None) -> np.ndarray:
    """Self-avoiding walk of n beads confined to a sphere (or an axis-aligned
    ellipsoid with semi-axes `shape`).  Returns float64 (n, 3)."""
    rng = np.random.default_rng(seed)
    if shape is None:
        r = radius if radius is not None else target_radius(n)
        axes = np.array([r, r, r])
    else:
        axes = np.asarray(shape, dtype=np.float64)
    pos = np.zeros((n, 3))
    reach = BOND + MIN_DIST
    pos[0] = rng.normal(size=3) * axes * 0.1
    i = 1
    fails = 0
    while i < n:
        cand = rng.normal(size=(96, 3))
        cand /= np.linalg.norm(cand, axis=1, keepdims=True)
        cand = pos[i - 1] + BOND * cand
        cand = cand[np.sum((cand / axes) ** 2, axis=1) <= 1.0]
        if i > 1 and len(cand):
            prev = pos[: i - 1]
            box = np.all(np.abs(prev - pos[i - 1]) < reach, axis=1)
            nb = prev[box]
            if len(nb):
                d2 = np.sum((cand[:, None, :] - nb[None, :, :]) ** 2, axis=2)
                cand = cand[np.min(d2, axis=1) >= MIN_DIST * MIN_DIST]
        if len(cand):
            # mild pull toward the centre keeps the walk compact
            w = np.exp(-np.sum((cand / axes) ** 2, axis=1) * 1.5)
            pos[i] = cand[rng.choice(len(cand), p=w / w.sum())]
            i += 1
            fails = 0
        else:
            fails += 1
            i -= min(i - 1, 3 + fails)
            if fails > 200:
                axes = axes * 1.05
                fails = 0
    return pos


def topology(xyz: np.ndarray, native_cutoff: float = NATIVE_CUTOFF, eh: float = EH):
    """Bonds (i, i+1) and native contacts |i-j| > 2 within `native_cutoff`."""
    n = xyz.shape[0]
    x = xyz.astype(np.float64)
    bonds = np.stack([np.arange(n - 1), np.arange(1, n)], axis=1).astype(np.int32)
    b_r0 = np.linalg.norm(x[1:] - x[:-1], axis=1)
    nat = []
    r0 = []
    for i in range(n):
        d = np.linalg.norm(x[i + 3:] - x[i], axis=1)
        js = np.nonzero(d < native_cutoff)[0]
        for j in js:
            nat.append((i, i + 3 + int(j)))
            r0.append(d[j])
    natives = np.array(nat, dtype=np.int32).reshape(-1, 2)
    return bonds, _round_top(b_r0), natives, _round_top(np.array(r0)), np.full(len(r0), eh, np.float32)


def make_system(n: int, seed: int) -> System:
    """A seeded n-bead globular chain with its native map."""
    xyz = _round_pdb(random_walk(n, seed))
    b, br0, nat, nr0, neh = topology(xyz)
    return System(xyz, b, br0, nat, nr0, neh)


def lognormal_sizes(count: int, lo: int, hi: int, seed: int, median: Optional[float] = None, sigma: float = 0.6) -> np.ndarray:
    """Seeded log-normal sizes clipped to [lo, hi]."""
    rng = np.random.default_rng(seed)
    med = median if median is not None else math.sqrt(lo * hi)
    s = np.exp(rng.normal(math.log(med), sigma, size=count))
    return np.clip(np.rint(s), lo, hi).astype(np.int64)


# ---------------------------------------------------------------------------
# Reference file formats
# ---------------------------------------------------------------------------
def write_top(path: str, sys_: System, pairs: Optional[np.ndarray] = None) -> None:
    """.top as written by SOP::save (src/IO/topio.cpp:146-208): space
    delimited (the strtok(" ") reader rejects tabs)."""
    with open(path, "w") as f:
        f.write("; Created by sopb_synth\n\n[ atoms ]\n")
        f.write(";   nr       type  resnr residue  atom   cgnr     charge       mass\n")
        for i in range(sys_.n):
            f.write("%6d%11s%7d%7s%7s%7s%11.2f%11.3f\n" % (i, "CA", i + 1, "ALA", "CA", "A", 1.0, 0.0))
        f.write("\n[ bonds ]\n;  ai    aj funct            c0            c1            c2            c3\n")
        for (i, j), r0 in zip(sys_.bonds, sys_.bonds_r0):
            f.write("%5d %5d %5d %10.5f\n" % (i, j, 1, r0))
        f.write("\n[ native ]\n;  ai    aj funct            c0            c1            c2            c3\n")
        for (i, j), r0, eh in zip(sys_.natives, sys_.natives_r0, sys_.natives_eh):
            f.write("%5d %5d %5d %10.5f %10.5f\n" % (i, j, 1, r0, eh))
        f.write("\n[ pairs ]\n;  ai    aj funct            c0            c1            c2            c3\n")
        if pairs is not None:
            for i, j in pairs:
                f.write("%5d %5d %5d\n" % (i, j, 1))


def write_pdb(path: str, xyz: np.ndarray) -> None:
    """ATOM records as PDBAtom::fprint writes them (src/IO/pdbio.cpp:265-280)."""
    with open(path, "w") as f:
        hexid = xyz.shape[0] >= 100000
        for i, (x, y, z) in enumerate(xyz):
            serial = ("%5x" % (i + 1)) if hexid else ("%5d" % (i + 1))
            f.write("ATOM  %s %-4s%c%3s %c%4d    %8.3f%8.3f%8.3f%6.2f%6.2f\n"
                    % (serial, "CA", " ", "ALA", "A", (i + 1) % 10000, x, y, z, 1.0, 0.0))
        f.write("END")


def read_top(path: str):
    """Reads [ atoms ], [ bonds ], [ native ], [ pairs ] like SOP::load."""
    atoms = 0
    bonds, b_r0, nat, n_r0, n_eh, pairs = [], [], [], [], [], []
    section = None
    with open(path) as f:
        for line in f:
            if not line or line[0] in ";\n\0":
                continue
            if line[0] == "[":
                for tag, name in (("[ atoms ]", "atoms"), ("[ bonds ]", "bonds"), ("[ native ]", "native"), ("[ pairs ]", "pairs")):
                    if line.startswith(tag):
                        section = name
                        break
                else:
                    raise ValueError("malformed section header: %r" % line)
                continue
            tok = line.split(" ")
            tok = [t for t in tok if t not in ("",)]
            if section == "atoms":
                atoms += 1
            elif section == "bonds":
                bonds.append((int(tok[0]), int(tok[1])))
                b_r0.append(float(tok[3]))
            elif section == "native":
                nat.append((int(tok[0]), int(tok[1])))
                n_r0.append(float(tok[3]))
                n_eh.append(float(tok[4]))
            elif section == "pairs":
                pairs.append((int(tok[0]), int(tok[1])))
            else:
                raise ValueError("line outside any section: %r" % line)
    return (atoms, np.array(bonds, np.int32).reshape(-1, 2), np.array(b_r0, np.float64).astype(np.float32),
            np.array(nat, np.int32).reshape(-1, 2), np.array(n_r0, np.float64).astype(np.float32),
            np.array(n_eh, np.float64).astype(np.float32), np.array(pairs, np.int32).reshape(-1, 2))


def read_pdb(path: str) -> np.ndarray:
    """Fixed-column ATOM coordinates (src/IO/pdbio.cpp:80-152)."""
    out = []
    with open(path) as f:
        for line in f:
            if line.startswith("ATOM"):
                out.append((float(line[30:38]), float(line[38:46]), float(line[46:54])))
    return np.array(out, np.float64).astype(np.float32)


def load_system(top_path: str, pdb_path: str) -> System:
    n, b, br0, nat, nr0, neh, _ = read_top(top_path)
    xyz = read_pdb(pdb_path)
    if xyz.shape[0] != n:
        raise ValueError("read coordinates for %d beads, topology has %d" % (xyz.shape[0], n))
    return System(xyz, b, br0, nat, nr0, neh)


def save_system(prefix: str, sys_: System) -> None:
    os.makedirs(os.path.dirname(prefix) or ".", exist_ok=True)
    write_top(prefix + ".top", sys_)
    write_pdb(prefix + ".pdb", sys_.xyz)


# ---------------------------------------------------------------------------
# Large assembly: a capsid-like shell of chain copies on an icosahedral lattice
# ---------------------------------------------------------------------------
def icosahedral_rotations() -> np.ndarray:
    """The 60 proper rotations of the icosahedron (closure of a 5-fold and a
    3-fold generator)."""
    phi = (1.0 + 5.0 ** 0.5) / 2.0

    def rot(axis, ang):
        a = np.asarray(axis, np.float64)
        a /= np.linalg.norm(a)
        K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
        return np.eye(3) + math.sin(ang) * K + (1 - math.cos(ang)) * K @ K

    gens = [rot((0.0, 1.0, phi), 2 * math.pi / 5), rot((1.0, 1.0, 1.0), 2 * math.pi / 3)]
    group = [np.eye(3)]
    frontier = [np.eye(3)]
    while frontier:
        nxt = []
        for g in frontier:
            for h in gens:
                m = h @ g
                if not any(np.allclose(m, q, atol=1e-8) for q in group):
                    group.append(m)
                    nxt.append(m)
        frontier = nxt
    assert len(group) == 60
    return np.array(group)


def make_capsid(copies_per_unit: int = 3, chain_n: int = 1100, seed: int = 7, radius: float = 140.0,
                slab: float = 22.0, native_cutoff: float = NATIVE_CUTOFF):
    """A shell of 60 x copies_per_unit copies of an n-bead chain.

    Each copy is a flattened globule (semi-axes a, a, `slab`) whose short axis
    points along the radius; copies are placed by the icosahedral group from
    `copies_per_unit` seed directions in one asymmetric unit.  The radius
    starts at `radius` and grows by 3% until no two beads of different copies
    are closer than 4 A (180 copies of 1100 beads need ~33 nm).  Natives:
    |i-j| > 2 within 8 A inside a copy, and every inter-copy pair within 8 A.
    Returns (System, info)."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    vol = chain_n * 210.0                              # A^3 per bead in a compact globule
    a = math.sqrt(vol / (4.0 / 3.0 * math.pi * slab))
    chains = []
    for k in range(copies_per_unit):
        x = random_walk(chain_n, seed * 101 + k, shape=(a, a, slab))
        chains.append(x - x.mean(axis=0))
    G = icosahedral_rotations()
    # seed directions: the best-spread of 3000 random draws (largest minimum
    # angle between any two of the 60 x k images)
    best, best_sep = None, -1.0
    for _ in range(3000):
        d = rng.normal(size=(copies_per_unit, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        P = np.einsum("gij,kj->gki", G, d).reshape(-1, 3)
        cosm = P @ P.T
        np.fill_diagonal(cosm, -1.0)
        sep = math.acos(min(1.0, float(cosm.max())))
        if sep > best_sep:
            best, best_sep = d, sep
    seeds = list(best)
    R = radius
    while True:
        blocks = []
        for g in G:
            for k, d in enumerate(seeds):
                u = g @ d
                # frame with z along u
                e1 = np.cross(u, [0.0, 0.0, 1.0])
                if np.linalg.norm(e1) < 1e-6:
                    e1 = np.cross(u, [0.0, 1.0, 0.0])
                e1 /= np.linalg.norm(e1)
                e2 = np.cross(u, e1)
                F = np.stack([e1, e2, u], axis=1)
                blocks.append(chains[k] @ F.T + R * u)
        X = np.concatenate(blocks)
        tree = cKDTree(X)
        copy_id = np.repeat(np.arange(len(blocks)), chain_n)
        close = tree.query_pairs(4.0, output_type="ndarray")
        clash = np.any(copy_id[close[:, 0]] != copy_id[close[:, 1]]) if len(close) else False
        if not clash:
            break
        R *= 1.03
    X = X - 0.0
    xyz = _round_pdb(X)
    n = xyz.shape[0]
    # bonds within copies
    ii = np.arange(n - 1)
    same = copy_id[ii] == copy_id[ii + 1]
    bonds = np.stack([ii[same], ii[same] + 1], axis=1).astype(np.int32)
    x64 = xyz.astype(np.float64)
    b_r0 = np.linalg.norm(x64[bonds[:, 1]] - x64[bonds[:, 0]], axis=1)
    tree = cKDTree(x64)
    pairs = tree.query_pairs(native_cutoff, output_type="ndarray")
    pi, pj = np.minimum(pairs[:, 0], pairs[:, 1]), np.maximum(pairs[:, 0], pairs[:, 1])
    inter = copy_id[pi] != copy_id[pj]
    intra = (~inter) & (pj - pi > 2)
    keep = inter | intra
    pi, pj = pi[keep], pj[keep]
    order = np.lexsort((pj, pi))
    natives = np.stack([pi[order], pj[order]], axis=1).astype(np.int32)
    n_r0 = np.linalg.norm(x64[natives[:, 1]] - x64[natives[:, 0]], axis=1)
    sys_ = System(xyz, bonds, _round_top(b_r0), natives, _round_top(n_r0), np.full(len(n_r0), EH, np.float32))
    info = {"radius_A": R, "copies": len(blocks), "chain_n": chain_n, "inter_natives": int(inter[keep].sum()),
            "slab_A": slab, "min_separation_rad": best_sep}
    return sys_, info
