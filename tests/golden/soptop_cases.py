"""Cases for the topology builder: a seeded synthetic all-atom structure
(backbone N, CA, C, O and side-chain atoms, two chains, an SSBOND record)
and configs in the reference topology creator's format.  Used by
make_soptop_golden.py (golden files from the reference's own sop-top) and by
tests/test_soptop.py."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "sop-gpu_b200"))
import sopb_synth as S  # noqa: E402

RESNAMES = ["ALA", "GLY", "SER", "LEU", "VAL", "THR", "ASP", "ASN", "ILE", "PHE"]


def structure(seed=5, chains=(("A", 45), ("B", 25)), segments=False):
    """PDB text of the structure (with segment names PRO<chain> in columns
    73-76 when `segments`); residues made CYS/LYS/GLU for the SS bond and the
    covalent linker."""
    rng = np.random.default_rng(seed)
    n = sum(c for _, c in chains)
    ca = S.random_walk(n, seed).astype(np.float64)
    lines = []
    atom = 0
    res = []
    k = 0
    for ch, cnt in chains:
        for r in range(1, cnt + 1):
            res.append((ch, r, k))
            k += 1
    names = {i: RESNAMES[rng.integers(len(RESNAMES))] for i in range(n)}
    # an SS bond between the closest pair of residues of different chains
    ia = [i for c, r, i in res if c == chains[0][0]]
    ib = [i for c, r, i in res if c != chains[0][0]]
    d = np.linalg.norm(ca[ia][:, None, :] - ca[ib][None, :, :], axis=2)
    p, q = np.unravel_index(np.argmin(d), d.shape)
    ss = (ia[p], ib[q])
    names[ss[0]] = names[ss[1]] = "CYS"
    names[7] = "LYS"          # chain A resid 8
    names[29] = "GLU"         # chain A resid 30
    for c, r, i in res:
        if c != chains[0][0] and names[i] in ("LYS", "GLU"):
            names[i] = "ALA"
    for c, r, i in res:
        x = ca[i]
        occ = 0.5 + rng.random() * 1.5
        beta = 0.2 + rng.random() * 2.0
        gly = names[i] == "GLY"
        atoms = [("N", x + rng.normal(scale=0.9, size=3)), ("CA", x), ("C", x + rng.normal(scale=0.9, size=3)),
                 ("O", x + rng.normal(scale=1.3, size=3))]
        if not gly:
            atoms.append(("CB", x + rng.normal(scale=1.2, size=3)))
            if rng.random() < 0.6:
                atoms.append(("CG", x + rng.normal(scale=2.2, size=3)))
        for nm, pos in atoms:
            atom += 1
            lines.append("ATOM  %5d %-4s%c%3s %c%4d    %8.3f%8.3f%8.3f%6.2f%6.2f%s\n"
                         % (atom, " " + nm if len(nm) < 4 else nm, " ", names[i], c, r, pos[0], pos[1], pos[2],
                            occ, beta, ("      PRO" + c) if segments else ""))
    sa, sb = res[ss[0]], res[ss[1]]
    head = "SSBOND %3d CYS %c %4d    CYS %c %4d\n" % (1, sa[0], sa[1], sb[0], sb[1])
    return head + "".join(lines) + "END\n"


BASE = {"structure": "aa.pdb"}

CASES = {
    "basic": {"eh": "1.5"},
    "sidechain": {"eh": "O", "SC_limit_bond": "4.0", "covalentRepulsion": "yes", "pairs_threshold": "25.0"},
    "linker": {"eh": "B", "covLinkersCount": "1", "covLinker1": "LYS8-GLU30", "covLinkersCutoff": "30.0",
               "R_limit_bond": "7.0", "SS_cutoff": "40.0"},
    "tandem": {"eh": "1.2", "createTandem": "yes", "linkerLength": "3", "monomerCount": "2", "fixedEnd": "0",
               "pulledEnd": "44", "pairs_threshold": "30.0"},
    "tandemvec": {"eh": "1.0", "createTandem": "yes", "linkerLength": "2", "monomerCount": "3", "fixedEnd": "0",
                  "pulledEnd": "69", "tandemDirection": "vector", "tandemVectorX": "1.0", "tandemVectorY": "0.5",
                  "tandemVectorZ": "0.0", "covalentRepulsion": "yes", "pairs_threshold": "20.0"},
}


def write_case(name, d):
    """Writes aa.pdb and <name>.conf into d; returns the config path."""
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "aa.pdb"), "w") as f:
        f.write(structure())
    cfg = dict(BASE, topology=name + ".top", coordinates=name + "_ca.pdb", **CASES[name])
    path = os.path.join(d, name + ".conf")
    with open(path, "w") as f:
        f.write("".join("%s %s\n" % kv for kv in cfg.items()))
    return path


# ---- the coarse-graining builder (sop-top2) ---------------------------------
MASSES = "MASS 1 N 14.007\nMASS 2 C 12.011\nMASS 3 O 15.999\nMASS 4 S 32.06\n"


def cgconfig(kind):
    """Bead descriptions: one Calpha bead per residue ("ca"), or a backbone
    and a side-chain bead ("bbsc", GLY backbone only, charged LYS/GLU)."""
    out = [MASSES]
    for rn in sorted(set(RESNAMES + ["CYS", "LYS", "GLU"])):
        out.append("RESI %s\n" % rn)
        if kind == "ca":
            out.append("BEAD CA CA\nREPR N CA C O CB CG\nCOOR CA\nCONN +CA\nCHAR 0.0\nENDBEAD\n")
        else:
            sc = rn != "GLY"
            q = {"LYS": 1.0, "GLU": -1.0}.get(rn, 0.0)
            out.append("BEAD BB B\nREPR N CA C O\nCOOR N CA C\nCONN +BB%s\nCHAR 0.0\nENDBEAD\n"
                       % (" SC" if sc else ""))
            if sc:
                out.append("BEAD SC S\nREPR CB CG\nCOOR CB CG\nCONN BB\nCHAR %.1f\nENDBEAD\n" % q)
        out.append("ENDRESI\n")
    return "".join(out)


CG_CASES = {
    "cg_ca": {"kind": "ca", "segments": True, "cfg": {"eh": "1.5", "R_limit_bond": "8.0", "SC_limit_bond": "5.0"}},
    "cg_bbsc": {"kind": "bbsc", "segments": True, "cfg": {"eh": "O", "R_limit_bond": "7.0", "SC_limit_bond": "4.5",
                                                          "Ks": "15.0", "additional_bonds": "ss.conn"}},
    "cg_chains": {"kind": "bbsc", "segments": False, "cfg": {"eh": "B", "use_chains": "yes", "R_limit_bond": "9.0",
                                                             "SC_limit_bond": "3.5"}},
}


def write_cg_case(name, d):
    """Writes aa.pdb, the bead descriptions, an extra-bond file and
    <name>.conf into d; returns the config path."""
    c = CG_CASES[name]
    os.makedirs(d, exist_ok=True)
    text = structure(segments=c["segments"])
    with open(os.path.join(d, "aa.pdb"), "w") as f:
        f.write(text)
    with open(os.path.join(d, "cg.inp"), "w") as f:
        f.write(cgconfig(c["kind"]))
    ss = text.splitlines()[0]
    seg1, seg2 = "PRO" + ss[15], "PRO" + ss[29]
    with open(os.path.join(d, "ss.conn"), "w") as f:
        f.write("CONN %s %d SC %s %d SC\n" % (seg1, int(ss[17:21]), seg2, int(ss[31:35])))
    cfg = {"cgconfig": "cg.inp", "structure": "aa.pdb", "coordinates": name + "_cg.pdb", "topology": name + ".top",
           "topology_psf": name + ".psf", "topology_natpsf": name + "_nat.psf"}
    cfg.update(c["cfg"])
    path = os.path.join(d, name + ".conf")
    with open(path, "w") as f:
        f.write("".join("%s %s\n" % kv for kv in cfg.items()))
    return path
