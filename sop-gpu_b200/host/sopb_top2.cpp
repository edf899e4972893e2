// sopb-top2 — coarse-grains an all-atom PDB by a bead description file into
// a SOP model, with the reference's second topology creator's usage:
//   sopb-top2 <config>
// (src/sop-top2.cpp:136-765, bead descriptions src/TopologyCreator/aatocg.cpp,
// file formats src/TopologyCreator/pdbio.cpp, psfio.cpp, topio.cpp).
//
// The bead description (`cgconfig`) lists, per residue name, its beads: the
// atoms a bead stands for (REPR: its mass is the sum of MASS entries keyed by
// their first letters, its occupancy and beta the mean of theirs), the atoms
// whose mean position is its position (COOR), its charge (CHAR) and its
// covalent partners (CONN: a bead of the same residue, or '+NAME' in the
// next residue).  Residues are grouped per segment (columns 73-76, or the
// chain with use_chains) by residue number.  Native contacts join beads that
// are neither bonded nor 1-3 bonded and whose positions are closer than
// R_limit_bond, or two of whose represented atoms are closer than
// SC_limit_bond.  Output: the coarse-grained PDB (charge and mass in the
// occupancy and beta columns), the .top file (bonds and contacts, no pairs),
// and optionally PSF files of the bonds and of the contacts.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "sopb_mirror.h"

using namespace sopb_host;

namespace {

struct AaAtom {
    std::string name, resName, segment;
    char altLoc = ' ', chain = ' ';
    int resid = 0;
    double x = 0, y = 0, z = 0, occupancy = 0, beta = 0;
};

struct BeadDef {
    std::string name, type;
    double mass = 0.0, charge = 0.0;
    std::vector<std::string> repr, coor, conn;
};
struct ResDef {
    std::string resname;
    std::vector<BeadDef> beads;
};
struct CgConfig {
    std::vector<ResDef> residues;
    std::vector<std::pair<char, double>> masses;
};

struct Bead {
    std::string name, type, resname, segment;
    int resid = 0;
    double x = 0, y = 0, z = 0, m = 0, q = 0, occupancy = 0, beta = 0;
    std::vector<std::string> conn;
    std::vector<const AaAtom*> represents;
};
struct Bond { int i, j; float b0; };
struct Native { int i, j; float eh, r0; };

std::vector<std::string> tokens(const std::string& line) {
    std::vector<std::string> t;
    std::string cur;
    for (char c : line) {
        if (c == ' ' || c == '\t' || c == '\n' || c == '\r') {
            if (!cur.empty()) t.push_back(cur);
            cur.clear();
        } else {
            cur += c;
        }
    }
    if (!cur.empty()) t.push_back(cur);
    return t;
}

// readCGConfiguration (aatocg.cpp:13-96): records by their first four
// letters; a bead's charge carries over to the next bead unless given.
CgConfig read_cgconfig(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw Error(SOPB_ERR_INVALID, "cannot open cgconfig " + path);
    CgConfig c;
    ResDef res;
    BeadDef bead;
    std::string line;
    while (std::getline(f, line)) {
        const std::string k = line.substr(0, 4);
        const std::vector<std::string> t = tokens(line);
        if (k == "MASS" && t.size() >= 4) c.masses.emplace_back(t[2][0], std::atof(t[3].c_str()));
        if (k == "RESI" && t.size() >= 2) res.resname = t[1].substr(0, 4);
        if (k == "ENDR") {
            c.residues.push_back(res);
            res.beads.clear();
        }
        if (k == "BEAD" && t.size() >= 3) {
            bead.name = t[1].substr(0, 4);
            bead.type = t[2].substr(0, 4);
        }
        if (k == "ENDB") {
            res.beads.push_back(bead);
            bead.repr.clear();
            bead.coor.clear();
            bead.conn.clear();
        }
        if (k == "REPR") bead.repr.insert(bead.repr.end(), t.begin() + 1, t.end());
        if (k == "COOR") bead.coor.insert(bead.coor.end(), t.begin() + 1, t.end());
        if (k == "CONN") bead.conn.insert(bead.conn.end(), t.begin() + 1, t.end());
        if (k == "CHAR" && t.size() >= 2) bead.charge = std::atof(t[1].c_str());
    }
    for (ResDef& r : c.residues)
        for (BeadDef& b : r.beads) {
            b.mass = 0.0;
            for (const std::string& a : b.repr)
                for (const auto& m : c.masses)
                    if (!a.empty() && m.first == a[0]) b.mass += m.second;
        }
    return c;
}

// readPDB (TopologyCreator/pdbio.cpp:46-89, 178-232): ATOM and HETATM
// records, fixed columns, the segment in columns 73-76.
std::vector<AaAtom> read_aa_pdb(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw Error(SOPB_ERR_INVALID, "cannot open structure " + path);
    std::vector<AaAtom> atoms;
    std::string line;
    auto col = [&](size_t at, size_t len) { return at < line.size() ? line.substr(at, len) : std::string(); };
    while (std::getline(f, line)) {
        const bool atom = line.compare(0, 5, "ATOM ") == 0 || line.compare(0, 6, "HETATM") == 0;
        if (!atom) continue;
        AaAtom a;
        const std::vector<std::string> nm = tokens(col(12, 4));
        a.name = nm.empty() ? "" : nm[0];
        a.altLoc = line.size() > 16 ? line[16] : ' ';
        a.resName = col(17, 3);
        a.chain = line.size() > 21 ? line[21] : ' ';
        a.resid = std::atoi(col(22, 4).c_str());
        a.x = std::atof(col(30, 8).c_str());
        a.y = std::atof(col(38, 8).c_str());
        a.z = std::atof(col(46, 8).c_str());
        a.occupancy = std::atof(col(54, 6).c_str());
        a.beta = std::atof(col(60, 6).c_str());
        a.segment = col(72, 4);
        for (char& ch : a.segment)
            if (ch == '\r' || ch == '\n') ch = ' ';
        atoms.push_back(a);
    }
    return atoms;
}

double dist(double ax, double ay, double az, double bx, double by, double bz) {
    const double dx = ax - bx, dy = ay - by, dz = az - bz;
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}

class Builder2 {
public:
    explicit Builder2(const Config& g) : cfg(g) {}
    void run();

private:
    void add_bond(int i, int j, double b0);
    void connect(int j, const std::string& conn);
    int find_bead(const std::string& seg, int resid, const std::string& name) const;
    bool bonded(int i, int j) const;
    bool bonded13(int i, int j) const;
    void write_pdb(const std::string& path) const;
    void write_psf(const std::string& path, const std::vector<std::pair<int, int>>& links) const;
    void write_top(const std::string& path) const;

    const Config& cfg;
    std::vector<AaAtom> atoms;
    std::vector<Bead> beads;
    std::vector<Bond> bonds;
    std::vector<Native> natives;
    std::vector<std::vector<int>> nb, nb13;
};

void Builder2::add_bond(int i, int j, double b0) {
    // addBond (sop-top2.cpp:656-675): each unordered pair once
    for (const Bond& b : bonds)
        if ((b.i == i && b.j == j) || (b.i == j && b.j == i)) return;
    if (i != j) bonds.push_back({i, j, (float)b0});
}

// addConnection (sop-top2.cpp:586-654).  '+NAME' takes the first bead of the
// next residue number after this bead (the reference's name test never
// advances past it); a plain name a bead of the same residue, searched
// forward, then backward.  Both ends must share the segment.
void Builder2::connect(int j, const std::string& conn) {
    const Bead& b = beads[j];
    const int n = (int)beads.size();
    auto bond_to = [&](int l) { add_bond(j, l, dist(b.x, b.y, b.z, beads[l].x, beads[l].y, beads[l].z)); };
    if (!conn.empty() && conn[0] == '+') {
        int l = j + 1;
        while (l < n && beads[l].resid != b.resid + 1) ++l;
        if (l < n && beads[j].segment == beads[l].segment) bond_to(l);
    } else if (!conn.empty() && conn[0] == '-') {
        int l = j - 1;
        while (l > 0 && beads[l].resid != b.resid - 1) --l;
        while (l > 0 && beads[l].name != conn.substr(1)) --l;
        if (l > 0 && beads[j].segment == beads[l].segment) bond_to(l);
    } else {
        int l = j + 1;
        while (l < n && beads[l].resid == b.resid && beads[l].name != conn) ++l;
        if (l < n && beads[j].segment == beads[l].segment && beads[l].resid == b.resid) {
            bond_to(l);
            return;
        }
        l = j - 1;
        while (l >= 0 && beads[l].resid == b.resid && beads[l].name != conn) --l;
        if (l >= 0 && beads[j].segment == beads[l].segment && beads[l].resid == b.resid) bond_to(l);
    }
}

int Builder2::find_bead(const std::string& seg, int resid, const std::string& name) const {
    // findBead (sop-top2.cpp:574-584): first three characters of the segment,
    // first two of the bead name
    for (size_t i = 0; i < beads.size(); ++i)
        if (beads[i].segment.compare(0, 3, seg, 0, 3) == 0 && beads[i].resid == resid &&
            beads[i].name.compare(0, 2, name, 0, 2) == 0)
            return (int)i;
    return -1;
}

bool Builder2::bonded(int i, int j) const { return std::find(nb[i].begin(), nb[i].end(), j) != nb[i].end(); }
bool Builder2::bonded13(int i, int j) const { return std::find(nb13[i].begin(), nb13[i].end(), j) != nb13[i].end(); }

void Builder2::run() {
    const Config& g = cfg;
    const CgConfig conf = read_cgconfig(g.str("cgconfig"));
    atoms = read_aa_pdb(g.str("structure"));
    std::printf("Found %zu atoms.\n", atoms.size());
    if (g.boolean("use_chains", false))
        for (AaAtom& a : atoms) a.segment = std::string(1, a.chain);
    // the residue tree: segments in order of appearance, residues of a
    // segment by residue number in order of appearance
    struct TreeRes { std::string resname; int resid; std::vector<const AaAtom*> atoms; };
    struct TreeSeg { std::string name; std::vector<TreeRes> res; };
    std::vector<TreeSeg> tree;
    for (const AaAtom& a : atoms) {
        auto s = std::find_if(tree.begin(), tree.end(), [&](const TreeSeg& t) { return t.name == a.segment; });
        if (s == tree.end()) {
            tree.push_back({a.segment, {}});
            s = tree.end() - 1;
        }
        auto r = std::find_if(s->res.begin(), s->res.end(), [&](const TreeRes& t) { return t.resid == a.resid; });
        if (r == s->res.end()) {
            s->res.push_back({a.resName, a.resid, {}});
            r = s->res.end() - 1;
        }
        r->atoms.push_back(&a);
    }
    std::printf("Found %zu segments.\n", tree.size());
    for (const TreeSeg& s : tree)
        for (const TreeRes& r : s.res) {
            const ResDef* def = nullptr;   // the last description of this residue name
            for (const ResDef& d : conf.residues)
                if (d.resname == r.resname) def = &d;
            if (!def) continue;
            for (const BeadDef& bd : def->beads) {
                Bead b;
                b.m = bd.mass;
                b.q = bd.charge;
                b.name = bd.name;
                b.type = bd.type;
                b.resname = r.resname;
                b.segment = s.name;
                b.resid = r.resid;
                b.conn = bd.conn;
                int cnt = 0;
                for (const AaAtom* a : r.atoms)
                    for (const std::string& c : bd.coor)
                        if (a->name == c) {
                            b.x += a->x;
                            b.y += a->y;
                            b.z += a->z;
                            ++cnt;
                        }
                if (cnt) {
                    b.x /= (double)cnt;
                    b.y /= (double)cnt;
                    b.z /= (double)cnt;
                }
                cnt = 0;
                for (const AaAtom* a : r.atoms)
                    for (const std::string& c : bd.repr)
                        if (a->name == c) {
                            b.represents.push_back(a);
                            b.beta += a->beta;
                            b.occupancy += a->occupancy;
                            ++cnt;
                        }
                b.beta /= cnt;
                b.occupancy /= cnt;
                beads.push_back(b);
            }
        }
    const int n = (int)beads.size();
    std::printf("Coarse-grained beads: %d.\n", n);
    for (int j = 0; j < n; ++j)
        for (const std::string& c : beads[j].conn) connect(j, c);
    const std::string extra = g.str("additional_bonds", "NONE");
    if (extra.compare(0, 4, "NONE") != 0) {
        // CONN seg1 resid1 bead1 seg2 resid2 bead2 (sop-top2.cpp:340-372)
        std::ifstream f(extra);
        std::string line;
        while (std::getline(f, line)) {
            if (line.compare(0, 4, "CONN") != 0) continue;
            const std::vector<std::string> t = tokens(line);
            if (t.size() < 7) continue;
            const int i = find_bead(t[1], std::atoi(t[2].c_str()), t[3]);
            const int j = find_bead(t[4], std::atoi(t[5].c_str()), t[6]);
            if (i >= 0 && j >= 0)
                add_bond(i, j, dist(beads[i].x, beads[i].y, beads[i].z, beads[j].x, beads[j].y, beads[j].z));
        }
    }
    std::sort(bonds.begin(), bonds.end(), [](const Bond& a, const Bond& b) { return a.i != b.i ? a.i < b.i : a.j < b.j; });
    nb.assign(n, {});
    for (const Bond& b : bonds) {
        nb[b.i].push_back(b.j);
        nb[b.j].push_back(b.i);
    }
    // 1-3 pairs i < k through a common partner (sop-top2.cpp:380-398)
    std::vector<std::pair<int, int>> b13;
    for (int i = 0; i < n; ++i)
        for (int j : nb[i])
            for (int k : nb[j])
                if (i < k) b13.emplace_back(i, k);
    std::sort(b13.begin(), b13.end());
    nb13.assign(n, {});
    for (const auto& p : b13) {
        nb13[p.first].push_back(p.second);
        nb13[p.second].push_back(p.first);
    }
    const std::string ehs = g.str("eh");
    const double cutoff = g.real("R_limit_bond", 8.0f), cutoff_aa = g.real("SC_limit_bond", 5.0f);
    for (int j = 0; j < n; ++j)
        for (int k = j + 1; k < n; ++k) {
            const double r0 = dist(beads[j].x, beads[j].y, beads[j].z, beads[k].x, beads[k].y, beads[k].z);
            double eh;
            if (ehs == "O") eh = std::sqrt(beads[j].occupancy * beads[k].occupancy);
            else if (ehs == "B") eh = std::sqrt(beads[j].beta * beads[k].beta);
            else if (std::atof(ehs.c_str()) != 0) eh = std::atof(ehs.c_str());
            else throw Error(SOPB_ERR_INVALID, "eh must be a number, 'O' or 'B'");
            if (bonded(j, k) || bonded13(j, k)) continue;
            bool add = r0 < cutoff;
            for (size_t l = 0; !add && l < beads[j].represents.size(); ++l)
                for (size_t m = 0; !add && m < beads[k].represents.size(); ++m) {
                    const AaAtom *p = beads[j].represents[l], *q = beads[k].represents[m];
                    add = dist(p->x, p->y, p->z, q->x, q->y, q->z) < cutoff_aa;
                }
            if (add) natives.push_back({j, k, (float)eh, (float)r0});
        }
    double pot = 0.0;
    for (const Native& q : natives) pot += q.eh;
    std::printf("Bonds: %zu. Native contacts: %zu. Total energy: %f\n", bonds.size(), natives.size(), pot);
    write_pdb(g.str("coordinates"));
    const std::string psf = g.str("topology_psf", "NONE"), natpsf = g.str("topology_natpsf", "NONE");
    if (psf.compare(0, 4, "NONE") != 0) {
        std::vector<std::pair<int, int>> l;
        for (const Bond& b : bonds) l.emplace_back(b.i + 1, b.j + 1);
        write_psf(psf, l);
    }
    if (natpsf.compare(0, 4, "NONE") != 0) {
        std::vector<std::pair<int, int>> l;
        for (const Native& q : natives) l.emplace_back(q.i + 1, q.j + 1);
        write_psf(natpsf, l);
    }
    write_top(g.str("topology"));
}

// writePDB (TopologyCreator/pdbio.cpp:261-312): charge and mass in the
// occupancy and beta columns, the segment's first letter as the chain.
void Builder2::write_pdb(const std::string& path) const {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw Error(SOPB_ERR_INVALID, "cannot write " + path);
    const bool hex = beads.size() >= 100000;
    for (size_t i = 0; i < beads.size(); ++i) {
        const Bead& b = beads[i];
        std::fprintf(f, hex ? "ATOM  %5x %-4s%c%3s %c%4d    %8.3f%8.3f%8.3f%6.2f%6.2f\n"
                            : "ATOM  %5d %-4s%c%3s %c%4d    %8.3f%8.3f%8.3f%6.2f%6.2f\n",
                     (int)i + 1, b.name.c_str(), ' ', b.resname.c_str(), b.segment.empty() ? '\0' : b.segment[0],
                     b.resid, b.x, b.y, b.z, b.q, b.m);
    }
    std::fprintf(f, "END");
    std::fclose(f);
}

// writePSF (psfio.cpp:498-637): atoms, then the bond list four pairs a line,
// empty angle, dihedral, improper and cross-term sections.
void Builder2::write_psf(const std::string& path, const std::vector<std::pair<int, int>>& links) const {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw Error(SOPB_ERR_INVALID, "cannot write " + path);
    std::fprintf(f, "PSF\n\n       1 !NTITLE\n REMARKS generated by psfio.c utility\n\n");
    std::fprintf(f, "%8d !NATOM\n", (int)beads.size());
    for (size_t i = 0; i < beads.size(); ++i) {
        const Bead& b = beads[i];
        const float q = (float)b.q, m = (float)b.m;
        std::fprintf(f, "%8d %-5s%-4d %-4s %-5s%-5s ", (int)i + 1, b.segment.c_str(), b.resid, b.resname.c_str(),
                     b.name.c_str(), b.name.c_str());
        if (q >= 0) std::fprintf(f, " %7.6f", (double)q);
        else std::fprintf(f, "%8.6f", (double)q);
        std::fprintf(f, "      %8.4f\n", (double)m);
    }
    std::fprintf(f, "\n%8d !NBOND: bonds\n", (int)links.size());
    for (size_t i = 0; i < links.size(); ++i) {
        std::fprintf(f, "%8d%8d", links[i].first, links[i].second);
        if (i != 0 && i % 4 == 3) std::fprintf(f, "\n");
    }
    std::fprintf(f, "\n\n%8d !NTHETA: angles\n\n\n", 0);
    std::fprintf(f, "%8d !NPHI: dihedrals\n\n\n", 0);
    std::fprintf(f, "%8d !IMNPHI: impropers\n\n\n", 0);
    std::fprintf(f, "%8d !NCRTERM: cross-terms\n\n\n", 0);
    std::fclose(f);
}

// writeTOP (TopologyCreator/topio.cpp:113-186): no pairs section entries.
void Builder2::write_top(const std::string& path) const {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw Error(SOPB_ERR_INVALID, "cannot write " + path);
    std::fprintf(f, "; Created by topio.c utility\n\n[ atoms ]\n");
    std::fprintf(f, ";   nr       type  resnr residue  atom   cgnr     charge       mass\n");
    for (size_t i = 0; i < beads.size(); ++i) {
        const Bead& b = beads[i];
        std::fprintf(f, "%6d%11s%7d%7s%7s%7c%11.2f%11.3f\n", (int)i, b.name.c_str(), b.resid, b.resname.c_str(),
                     b.name.c_str(), b.segment.empty() ? '\0' : b.segment[0], (double)(float)b.q, (double)(float)b.m);
    }
    auto term = [&](int i, int j, float c0, float c1) {
        std::fprintf(f, "%5d %5d %5d", i, j, 1);
        if (c0 != 0.0f) {
            std::fprintf(f, " %10.5f", (double)c0);
            if (c1 != 0.0f) std::fprintf(f, " %10.5f", (double)c1);
        }
        std::fprintf(f, "\n");
    };
    std::fprintf(f, "\n[ bonds ]\n;  ai    aj funct            c0            c1            c2            c3\n");
    for (const Bond& b : bonds) term(b.i, b.j, b.b0, 0.0f);
    std::fprintf(f, "\n[ native ]\n;  ai    aj funct            c0            c1            c2            c3\n");
    for (const Native& q : natives) term(q.i, q.j, q.r0, q.eh);
    std::fprintf(f, "\n[ pairs ]\n;  ai    aj funct            c0            c1            c2            c3\n\n");
    std::fclose(f);
}

}  // namespace

int main(int argc, char** argv) {
    std::printf("==========================\nSOP coarse-grained model builder (sopb-top2)\n==========================\n");
    if (argc < 2) {
        std::fprintf(stderr, "ERROR: Configuration file should be specified.\n");
        return 2;
    }
    try {
        Config cfg(argv[1]);
        Builder2(cfg).run();
        return 0;
    } catch (const Error& e) {
        std::fprintf(stderr, "sopb-top2: %s\n", e.what());
        return e.code ? e.code : 1;
    }
}
