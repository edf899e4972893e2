// sopb-top — builds a SOP model (.top topology and Calpha coordinates) from
// an all-atom PDB, with the reference topology creator's usage and rules:
//   sopb-top <config>
// (src/sop-top.cpp:21-478 and the model rules of src/sop.hpp:77-247).
//
// One bead per residue at its Calpha.  Beads i < j are
//   * covalently bonded when consecutive in the same chain and closer than
//     covalent_cutoff, when an SSBOND record names their residues and they
//     are closer than SS_cutoff, or when a covLinker<k> key names them and
//     they are closer than covLinkersCutoff;
//   * a native contact when not bonded, not within two residues of each
//     other in one chain, and their Calphas are closer than R_limit_bond or
//     (SC_limit_bond > 0) two side-chain atoms of theirs are closer than it;
//   * a possible (repulsive) pair when neither, or bonded with
//     covalentRepulsion on, and closer than pairs_threshold.
// Bonds and contacts take the Calpha distance as r0; a contact's eh is the
// `eh` key, or the geometric mean of the beads' occupancy ('O') or beta ('B')
// columns.  createTandem repeats the monomer monomerCount times joined by
// linkers of linkerLength beads.  Output: the .top file (topio.cpp:82-170
// layout) and the coordinates PDB with CONECT records; an existing
// coordinates file is overwritten only after a 'y' on standard input.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "sopb_mirror.h"

using namespace sopb_host;

namespace {

struct PdbAtomRec {
    int id = 0;
    std::string name, resName;
    char altLoc = ' ', chain = ' ';
    int resid = 0;
    double x = 0, y = 0, z = 0, occupancy = 0, beta = 0;   // PDBAtom keeps doubles
};
struct SsBond { char chain1, chain2; int resid1, resid2; };
struct Linker { std::string res1, res2; int resid1, resid2; };
struct Bond { int i, j; float r0; };
struct Native { int i, j; float r0, eh; };

std::string field(const std::string& line, size_t at, size_t len) {
    return at < line.size() ? line.substr(at, len) : std::string();
}

// PDBAtom::parse and PDBSSBond::parse (src/IO/pdbio.cpp:93-191): fixed columns.
void read_pdb_all(const std::string& path, std::vector<PdbAtomRec>& atoms, std::vector<SsBond>& ss) {
    std::ifstream f(path);
    if (!f) throw Error(SOPB_ERR_INVALID, "cannot open structure " + path);
    std::string line;
    while (std::getline(f, line)) {
        if (line.compare(0, 6, "SSBOND") == 0) {
            SsBond b;
            b.chain1 = line.size() > 15 ? line[15] : ' ';
            b.resid1 = std::atoi(field(line, 17, 4).c_str());
            b.chain2 = line.size() > 29 ? line[29] : ' ';
            b.resid2 = std::atoi(field(line, 31, 4).c_str());
            ss.push_back(b);
        }
        if (line.compare(0, 4, "ATOM") == 0) {
            PdbAtomRec a;
            a.id = std::atoi(field(line, 6, 5).c_str());
            std::string nm = field(line, 12, 4);
            const size_t s0 = nm.find_first_not_of(' ');
            nm = s0 == std::string::npos ? "" : nm.substr(s0);
            const size_t s1 = nm.find(' ');
            a.name = s1 == std::string::npos ? nm : nm.substr(0, s1);
            a.altLoc = line.size() > 16 ? line[16] : ' ';
            a.resName = field(line, 17, 3);
            a.chain = line.size() > 21 ? line[21] : ' ';
            a.resid = std::atoi(field(line, 22, 4).c_str());
            a.x = std::atof(field(line, 30, 8).c_str());
            a.y = std::atof(field(line, 38, 8).c_str());
            a.z = std::atof(field(line, 46, 8).c_str());
            a.occupancy = std::atof(field(line, 54, 6).c_str());
            a.beta = std::atof(field(line, 60, 6).c_str());
            atoms.push_back(a);
        }
    }
}

// getDistanceAtoms (src/sop.hpp:226-233): differences of the double
// coordinates rounded to float, the rest in float.
float dist(const PdbAtomRec& a, const PdbAtomRec& b) {
    const float x = (float)(a.x - b.x), y = (float)(a.y - b.y), z = (float)(a.z - b.z);
    return std::sqrt(x * x + y * y + z * z);
}

class Builder {
public:
    explicit Builder(const Config& g) : cfg(g) {}
    void run();

private:
    bool covalent(int i, int j) const;
    bool native(int i, int j) const;
    bool possible(int i, int j) const;
    float r0(int i, int j) const;
    float eh_of(int i, int j) const;
    void tandem();
    void save_top(const std::string& path) const;

    const Config& cfg;
    std::vector<PdbAtomRec> atoms;
    std::vector<SsBond> ss;
    std::vector<Linker> linkers;
    std::vector<int> ca;                       // atom index of each bead's Calpha
    std::vector<int> first, last;              // atom range of each bead's residue
    std::vector<PdbAtomRec> beads;
    std::vector<Bond> bonds;
    std::vector<Native> natives;
    std::vector<std::pair<int, int>> pairs;
    float eh = 1.5f, R_limit_bond = 8.0f, SC_limit_bond = 0.0f, a = 3.8f, pairs_threshold = 1000.0f;
    float covalent_cutoff = 10.0f, SS_cutoff = 10.0f, linker_cutoff = 5.0f;
    bool covalentLJ = false;
};

bool Builder::covalent(int i, int j) const {
    const PdbAtomRec &A = atoms[ca[i]], &B = atoms[ca[j]];
    if ((A.resid == B.resid + 1 && A.chain == B.chain) || (B.resid == A.resid + 1 && B.chain == A.chain))
        if (dist(A, B) < covalent_cutoff && std::abs(i - j) == 1) return true;
    for (const SsBond& s : ss) {
        const bool fwd = A.resid == s.resid1 && A.chain == s.chain1 && B.resid == s.resid2 && B.chain == s.chain2;
        const bool bwd = A.resid == s.resid2 && A.chain == s.chain2 && B.resid == s.resid1 && B.chain == s.chain1;
        if ((fwd || bwd) && dist(A, B) < SS_cutoff) return true;
    }
    // the first linker that names the two residues decides
    for (const Linker& l : linkers) {
        const bool fwd = A.resid == l.resid1 && A.resName.compare(0, 3, l.res1, 0, 3) == 0 && B.resid == l.resid2 &&
                         B.resName.compare(0, 3, l.res2, 0, 3) == 0;
        const bool bwd = A.resid == l.resid2 && A.resName.compare(0, 3, l.res2, 0, 3) == 0 && B.resid == l.resid1 &&
                         B.resName.compare(0, 3, l.res1, 0, 3) == 0;
        if (fwd || bwd) return dist(A, B) < linker_cutoff;
    }
    return false;
}

bool Builder::native(int i, int j) const {
    if (covalent(i, j)) return false;
    const PdbAtomRec &A = atoms[ca[i]], &B = atoms[ca[j]];
    const bool near_in_chain = std::abs(A.resid - B.resid) <= 2 && A.chain == B.chain;
    if (near_in_chain) return false;
    if (dist(A, B) < R_limit_bond) return true;
    if (SC_limit_bond > 0.0f) {
        auto backbone = [](const std::string& n) { return n == "CA" || n == "N" || n == "C" || n == "O"; };
        for (int p = first[i]; p <= last[i]; ++p)
            for (int q = first[j]; q <= last[j]; ++q)
                if (!backbone(atoms[p].name) && !backbone(atoms[q].name) && dist(atoms[p], atoms[q]) < SC_limit_bond)
                    return true;
    }
    return false;
}

bool Builder::possible(int i, int j) const {
    if (!(pairs_threshold > 0.0f)) return false;
    const float dr = dist(atoms[ca[i]], atoms[ca[j]]);
    if (covalent(i, j)) return covalentLJ && dr < pairs_threshold;
    if (native(i, j)) return false;
    return i != j && dr < pairs_threshold;
}

float Builder::r0(int i, int j) const {
    const float dr = dist(atoms[ca[i]], atoms[ca[j]]);
    if (dr < 1.0f && i != j) std::printf("WARNING: Residues %d and %d are closer than 1.0A!\n", i, j);
    return (native(i, j) || covalent(i, j)) ? dr : a;
}

float Builder::eh_of(int i, int j) const {
    // getOccupancy / getBeta return floats (sop.hpp:240-247)
    if (eh == -1.0f) return std::sqrt((float)atoms[ca[i]].occupancy * (float)atoms[ca[j]].occupancy);
    if (eh == -2.0f) return std::sqrt((float)atoms[ca[i]].beta * (float)atoms[ca[j]].beta);
    return eh;
}

void Builder::run() {
    const Config& g = cfg;
    const std::string ehs = g.str("eh", "1.5");
    if (ehs == "O") {
        std::printf("Taking eh's values from occupancy column.\n");
        eh = -1.0f;
    } else if (ehs == "B") {
        std::printf("Taking eh's values from beta column.\n");
        eh = -2.0f;
    } else {
        eh = (float)std::atof(ehs.c_str());
        if (eh == 0.0f) std::printf("WARNING: Value of eh in a configuration file is not valid; eh is set to 0.\n");
    }
    R_limit_bond = g.real("R_limit_bond", 8.0f);
    SC_limit_bond = g.real("SC_limit_bond", 0.0f);
    covalentLJ = g.boolean("covalentRepulsion", false);
    a = g.real("a", 3.8f);
    pairs_threshold = g.real("pairs_threshold", 1000.0f);
    covalent_cutoff = g.real("covalent_cutoff", 10.0f);
    SS_cutoff = g.real("SS_cutoff", 10.0f);
    const int nlink = (int)g.integer("covLinkersCount", 0);
    if (nlink > 0) {
        linker_cutoff = g.real("covLinkersCutoff", 5.0f);
        for (int k = 1; k <= nlink; ++k) {
            // "<RES><resid>-<RES><resid>" (sop-top.cpp:97-113)
            const std::string v = g.str("covLinker" + std::to_string(k));
            const size_t dash = v.find_first_of("-\t");
            if (dash == std::string::npos) throw Error(SOPB_ERR_INVALID, "covLinker" + std::to_string(k) + ": expected RES1-RES2");
            const std::string l = v.substr(0, dash), r = v.substr(dash + 1);
            Linker L{l.substr(0, 3), r.substr(0, 3), std::atoi(l.c_str() + std::min<size_t>(3, l.size())),
                     std::atoi(r.c_str() + std::min<size_t>(3, r.size()))};
            linkers.push_back(L);
            std::printf("Covalent linker between residues %s%d and %s%d will be added.\n", L.res1.c_str(), L.resid1,
                        L.res2.c_str(), L.resid2);
        }
    }
    read_pdb_all(g.str("structure"), atoms, ss);
    std::printf("Found %zu atoms and %zu SS-bonds.\n", atoms.size(), ss.size());
    for (size_t k = 0; k < atoms.size(); ++k)
        if (atoms[k].name == "CA") ca.push_back((int)k);
    const int n = (int)ca.size();
    std::printf("Found %d residues.\n", n);
    if (n == 0) throw Error(SOPB_ERR_INVALID, "no CA atoms in " + g.str("structure"));
    // residue atom ranges as the reference forms them (sop-top.cpp:148-175):
    // a new residue at every change of (resid, chain); bead i's range runs
    // from its residue's second atom to the first atom of the next residue
    // (bead 0 from atom 0, the last bead to the last atom)
    std::vector<int> group(atoms.size());
    {
        int idx = -1, lr = -1;
        char lc = 0;
        for (size_t k = 0; k < atoms.size(); ++k) {
            if (lr != atoms[k].resid || lc != atoms[k].chain) {
                lr = atoms[k].resid;
                lc = atoms[k].chain;
                ++idx;
            }
            group[k] = idx;
        }
    }
    first.assign(n, 0);
    last.assign(n, 0);
    last[n - 1] = (int)atoms.size() - 1;
    {
        size_t idx = 0;
        for (int i = 0; i < n - 1; ++i) {
            while (idx + 1 < atoms.size() && group[idx] == group[idx + 1]) ++idx;
            ++idx;
            last[i] = (int)idx;
            first[i + 1] = (int)idx + 1;
        }
    }
    for (int i = 0; i < n; ++i) beads.push_back(atoms[ca[i]]);
    for (int i = 0; i < n; ++i) {
        for (int j = i + 1; j < n; ++j) {
            if (covalent(i, j)) bonds.push_back({i, j, r0(i, j)});
            if (native(i, j)) natives.push_back({i, j, r0(i, j), eh_of(i, j)});
            if (possible(i, j)) pairs.emplace_back(i, j);
        }
    }
    std::printf("Total per monomer:\n%d amino acids\n%zu covalent bonds\n%zu native contacts\n%zu pairs\n=======\n", n,
                bonds.size(), natives.size(), pairs.size());
    if (g.boolean("createTandem", false)) tandem();
    save_top(g.str("topology"));
    const std::string coord = g.str("coordinates");
    bool write = true;
    if (FILE* t = std::fopen(coord.c_str(), "r")) {
        std::fclose(t);
        std::printf("Coordinates file '%s' exists. Overwrite (y/n)? ", coord.c_str());
        std::fflush(stdout);
        const int ch = std::getchar();
        write = ch == 'y';
    }
    if (write) {
        std::vector<Atom> out;
        for (const PdbAtomRec& b : beads) {
            Atom q;
            q.name = b.name;
            q.resName = b.resName;
            q.altLoc = b.altLoc;
            q.chain = b.chain;
            q.resid = b.resid;
            q.occupancy = b.occupancy;
            q.beta = b.beta;
            q.x = b.x;
            q.y = b.y;
            q.z = b.z;
            out.push_back(q);
        }
        std::vector<int32_t> bl;
        for (const Bond& b : bonds) { bl.push_back(b.i); bl.push_back(b.j); }
        save_pdb(coord, out, {}, bl);
    }
}

// createTandem (sop-top.cpp:265-448): monomerCount copies along the monomer's
// end-to-end direction (or tandemVector), linkers of linkerLength GLY beads
// at both ends and between copies, bonds of length a along the linkers, no
// contacts between copies; every other pair repulsive.  Slot arithmetic as
// the reference lays the arrays out.
void Builder::tandem() {
    const Config& g = cfg;
    const int L = (int)g.integer("linkerLength");
    const int M = (int)g.integer("monomerCount");
    const std::string dir = g.str("tandemDirection", "endToEnd");
    const int f0 = (int)g.integer("fixedEnd"), l0 = (int)g.integer("pulledEnd");
    const int n = (int)beads.size(), nb = (int)bonds.size(), nn = (int)natives.size();
    if (f0 < 0 || f0 >= n || l0 < 0 || l0 >= n) throw Error(SOPB_ERR_INVALID, "tandem ends out of range");
    const int tn = M * n + (M + 1) * L;
    const int tb = M * nb + (M + 1) * (L + 1) - 2;
    const int tnat = M * nn;
    long long tp = ((long long)tn * tn - tn) / 2 - tnat;
    if (!covalentLJ) tp -= tb;
    std::printf("Building a tandem of %d\n", M);
    std::vector<PdbAtomRec> ta(tn);
    std::vector<Bond> tbo(std::max(tb, 0), Bond{0, 0, 0.0f});
    std::vector<Native> tna(tnat);
    PdbAtomRec link;
    link.resName = "GLY";
    link.name = "CA";
    link.chain = 'l';
    link.occupancy = beads[0].occupancy;
    link.beta = beads[0].beta;
    link.resid = 1;
    link.id = 1;
    const float rx = (float)(beads[l0].x - beads[f0].x), ry = (float)(beads[l0].y - beads[f0].y),
                rz = (float)(beads[l0].z - beads[f0].z);
    float r, rxn, ryn, rzn;
    if (dir == "vector") {
        const float vx = g.real("tandemVectorX"), vy = g.real("tandemVectorY"), vz = g.real("tandemVectorZ");
        r = std::sqrt(vx * vx + vy * vy + vz * vz);
        rxn = vx / r; ryn = vy / r; rzn = vz / r;
    } else {
        r = std::sqrt(rx * rx + ry * ry + rz * rz);
        rxn = rx / r; ryn = ry / r; rzn = rz / r;
    }
    auto put_bond = [&](long long slot, const Bond& b) {
        if (slot >= 0 && slot < (long long)tbo.size()) tbo[slot] = b;
    };
    for (int i = 0; i < M; ++i)
        for (int j = 0; j < n; ++j) {
            PdbAtomRec q = beads[j];
            q.x += i * (rx + rxn * a * (L + 1));
            q.y += i * (ry + ryn * a * (L + 1));
            q.z += i * (rz + rzn * a * (L + 1));
            ta[i * (n + L) + j + L] = q;
        }
    for (int k = 0; k < L; ++k) {
        PdbAtomRec q = link;
        q.x = beads[f0].x - (k + 1) * a * rxn;
        q.y = beads[f0].y - (k + 1) * a * ryn;
        q.z = beads[f0].z - (k + 1) * a * rzn;
        ta[L - (k + 1)] = q;
    }
    for (int i = 0; i < M; ++i)
        for (int k = 0; k < L; ++k) {
            PdbAtomRec q = link;
            q.x = beads[l0].x + (rx + (L + 1) * a * rxn) * i + (k + 1) * a * rxn;
            q.y = beads[l0].y + (ry + (L + 1) * a * ryn) * i + (k + 1) * a * ryn;
            q.z = beads[l0].z + (rz + (L + 1) * a * rzn) * i + (k + 1) * a * rzn;
            ta[(i + 1) * n + (i + 1) * L + k] = q;
        }
    for (int i = 0; i < M; ++i)
        for (int j = 0; j < nb; ++j)
            put_bond((long long)i * (nb + L + 1) + L + j,
                     Bond{bonds[j].i + i * (n + L) + L, bonds[j].j + i * (n + L) + L, bonds[j].r0});
    for (int k = 0; k < L; ++k) put_bond(k, Bond{k, k + 1, a});
    if (L > 0) tbo[L - 1].j = f0 + L;
    int kmax = L + 1;
    for (int i = 0; i < M; ++i) {
        if (i == M - 1) kmax = L;
        for (int k = 0; k < kmax; ++k)
            put_bond((long long)(i + 1) * (nb + L) + i + k,
                     Bond{(i + 1) * (n + L) + k - 1, (i + 1) * (n + L) + k, a});
        const long long s = (long long)(i + 1) * (nb + L) + i;
        if (s >= 0 && s < (long long)tbo.size()) tbo[s].i = i * (n + L) + L + l0;
        if (i != M - 1) {
            const long long s2 = (long long)(i + 1) * (nb + L) + i + L;
            if (s2 >= 0 && s2 < (long long)tbo.size()) tbo[s2].j = (i + 1) * (n + L) + L + f0;
        }
    }
    for (int i = 0; i < M; ++i)
        for (int j = 0; j < nn; ++j)
            tna[i * nn + j] = Native{natives[j].i + i * (n + L) + L, natives[j].j + i * (n + L) + L, natives[j].r0,
                                     natives[j].eh};
    std::set<std::pair<int, int>> excl;
    if (!covalentLJ)
        for (const Bond& b : tbo) { excl.insert({b.i, b.j}); excl.insert({b.j, b.i}); }
    for (const Native& q : tna) { excl.insert({q.i, q.j}); excl.insert({q.j, q.i}); }
    std::vector<std::pair<int, int>> tpairs(std::max<long long>(tp, 0), {0, 0});
    size_t idx = 0;
    for (int i = 0; i < tn && idx < tpairs.size(); ++i)
        for (int j = i + 1; j < tn && idx < tpairs.size(); ++j)
            if (!excl.count({i, j})) tpairs[idx++] = {i, j};
    std::printf("Total per %d-mer:\n%d amino acids\n%zu covalent bonds\n%zu native contacts\n%zu pairs\n=======\n", M,
                tn, tbo.size(), tna.size(), tpairs.size());
    beads = ta;
    bonds = tbo;
    natives = tna;
    pairs = tpairs;
}

// SOP::save (src/IO/topio.cpp:82-170): GROMACS-like sections, a term's
// trailing parameters only while they are non-zero.
void Builder::save_top(const std::string& path) const {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw Error(SOPB_ERR_INVALID, "cannot write " + path);
    std::fprintf(f, "; Created by topio.cpp utility\n\n");
    std::fprintf(f, "[ atoms ]\n");
    std::fprintf(f, ";   nr       type  resnr residue  atom   cgnr     charge       mass\n");
    for (size_t i = 0; i < beads.size(); ++i) {
        const PdbAtomRec& b = beads[i];
        std::fprintf(f, "%6d%11s%7d%7s%7s%7c%11.2f%11.3f\n", (int)i, b.name.c_str(), b.resid, b.resName.c_str(),
                     b.name.c_str(), b.chain, (double)b.occupancy, (double)b.beta);
    }
    auto term = [&](int i, int j, float c0, float c1) {
        std::fprintf(f, "%5d %5d %5d", i, j, 1);
        if (c0 != 0.0f) {
            std::fprintf(f, " %10.5f", (double)c0);
            if (c1 != 0.0f) std::fprintf(f, " %10.5f", (double)c1);
        }
        std::fprintf(f, "\n");
    };
    std::fprintf(f, "\n[ bonds ]\n");
    std::fprintf(f, ";  ai    aj funct            c0            c1            c2            c3\n");
    for (const Bond& b : bonds) term(b.i, b.j, b.r0, 0.0f);
    std::fprintf(f, "\n[ native ]\n");
    std::fprintf(f, ";  ai    aj funct            c0            c1            c2            c3\n");
    for (const Native& q : natives) term(q.i, q.j, q.r0, q.eh);
    std::fprintf(f, "\n[ pairs ]\n");
    std::fprintf(f, ";  ai    aj funct            c0            c1            c2            c3\n");
    for (const auto& q : pairs) term(q.first, q.second, 0.0f, 0.0f);
    std::fclose(f);
}

}  // namespace

int main(int argc, char** argv) {
    std::printf("==========================\nSOP model builder (sopb-top)\n==========================\n");
    if (argc < 2) {
        std::fprintf(stderr, "ERROR: Configuration file should be specified.\n");
        return 2;
    }
    try {
        Config cfg(argv[1]);
        Builder(cfg).run();
        return 0;
    } catch (const Error& e) {
        std::fprintf(stderr, "sopb-top: %s\n", e.what());
        return e.code ? e.code : 1;
    }
}
