// sopb_mirror.cpp — config reader, topology/PDB IO, plugin surface and the
// stride loop of SOP-GPU's host code, over the sopb C ABI.
#include "sopb_mirror.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace sopb_host {

void check(int code, const char* what) {
    if (code != SOPB_OK) throw Error(code, std::string(what) + ": " + sopb_status_string(code));
}

// ---------------------------------------------------------------------------
// Config: `name value # comment` lines; lines starting with '#', ' ', '\t' or
// '\n' are skipped; later lines override (src/IO/configreader.cpp:21-58).
// ---------------------------------------------------------------------------
static std::string trim(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}
static std::string lower(std::string s) {
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}
static std::string replace_all(std::string s, const std::string& from, const std::string& to) {
    if (from.empty()) return s;
    size_t pos = 0;
    while ((pos = s.find(from, pos)) != std::string::npos) {
        s.replace(pos, from.size(), to);
        pos += to.size();
    }
    return s;
}

Config::Config(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw Error(SOPB_ERR_INVALID, "cannot open config file " + path);
    std::string line;
    while (std::getline(f, line)) {
        if (line.empty() || line[0] == '#' || line[0] == ' ' || line[0] == '\t') continue;
        const size_t e = line.find_first_of(" \t");
        const std::string name = line.substr(0, e);
        std::string value = e == std::string::npos ? "" : line.substr(e + 1);
        const size_t h = value.find('#');
        if (h != std::string::npos) value = value.substr(0, h);
        values_[name] = trim(value);
    }
}

std::string Config::raw(const std::string& key) const {
    auto it = values_.find(key);
    if (it == values_.end()) throw Error(SOPB_ERR_INVALID, "Parameter '" + key + "' not specified");
    return it->second;
}

// getMaskedParameter (configreader.cpp:77-86): every <other-key> replaced,
// in the map's key order.
std::string Config::str(const std::string& key) const {
    std::string v = raw(key);
    for (const auto& kv : values_) v = replace_all(v, "<" + kv.first + ">", kv.second);
    return v;
}
std::string Config::str(const std::string& key, const std::string& def) const { return has(key) ? str(key) : def; }

int64_t Config::integer(const std::string& key) const {
    std::istringstream is(str(key));
    int64_t v = 0;
    is >> v;
    return v;
}
int64_t Config::integer(const std::string& key, int64_t def) const { return has(key) ? integer(key) : def; }

float Config::real(const std::string& key) const {
    std::istringstream is(str(key));
    float v = 0.0f;
    is >> v;
    return v;
}
float Config::real(const std::string& key, float def) const { return has(key) ? real(key) : def; }

bool Config::boolean(const std::string& key) const {
    const std::string v = lower(raw(key));
    if (v == "yes" || v == "true" || v == "on" || v == "y") return true;
    if (v == "no" || v == "false" || v == "off" || v == "n") return false;
    throw Error(SOPB_ERR_INVALID, "Wrong value '" + v + "' for boolean parameter '" + key + "'");
}
bool Config::boolean(const std::string& key, bool def) const { return has(key) ? boolean(key) : def; }

// getArrayParameter (configreader.cpp:88-118): `a to b` ranges, empty/none.
std::vector<int> Config::ints(const std::string& key) const {
    const std::string v = lower(raw(key));
    std::vector<int> out;
    if (v == "empty" || v == "none") return out;
    std::istringstream is(v);
    std::string t;
    while (is >> t) {
        if (t == "to") {
            if (out.empty()) throw Error(SOPB_ERR_INVALID, "'to' must follow a number in '" + key + "'");
            int to = 0;
            is >> to;
            for (int i = out.back() + 1; i <= to; ++i) out.push_back(i);
        } else {
            out.push_back(std::atoi(t.c_str()));
        }
    }
    return out;
}
std::vector<int> Config::ints(const std::string& key, const std::vector<int>& def) const {
    return has(key) ? ints(key) : def;
}

void Config::float3(const std::string& key, float out[3]) const {
    std::istringstream is(raw(key));
    std::vector<float> v;
    float x;
    while (is >> x) v.push_back(x);
    if (v.size() != 3) throw Error(SOPB_ERR_INVALID, "Float3 parameter '" + key + "' must have 3 components");
    for (int c = 0; c < 3; ++c) out[c] = v[c];
}
void Config::float3(const std::string& key, float out[3], const float def[3]) const {
    if (has(key)) float3(key, out);
    else for (int c = 0; c < 3; ++c) out[c] = def[c];
}

// ---------------------------------------------------------------------------
// .top (src/IO/topio.cpp:36-80, 204-240) and PDB (src/IO/pdbio.cpp:80-152)
// ---------------------------------------------------------------------------
Topology Topology::load(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw Error(SOPB_ERR_INVALID, "cannot open topology " + path);
    Topology t;
    std::string line;
    enum { NONE, ATOMS, BONDS, NATIVES, PAIRS } sec = NONE;
    int lineno = 0;
    while (std::getline(f, line)) {
        ++lineno;
        if (line.empty() || line[0] == ';') continue;
        if (line[0] == '[') {
            if (line.compare(0, 9, "[ atoms ]") == 0) sec = ATOMS;
            else if (line.compare(0, 9, "[ bonds ]") == 0) sec = BONDS;
            else if (line.compare(0, 10, "[ native ]") == 0) sec = NATIVES;
            else if (line.compare(0, 9, "[ pairs ]") == 0) sec = PAIRS;
            else throw Error(SOPB_ERR_INVALID, "malformed section header at " + path + ":" + std::to_string(lineno));
            continue;
        }
        // the reference tokenises on single spaces only (strtok(" "))
        std::vector<std::string> tok;
        {
            std::string cur;
            for (char ch : line) {
                if (ch == ' ' || ch == '\r') { if (!cur.empty()) tok.push_back(cur); cur.clear(); }
                else cur += ch;
            }
            if (!cur.empty()) tok.push_back(cur);
        }
        if (tok.empty()) continue;
        switch (sec) {
        case ATOMS: {
            Atom a;
            a.resid = t.natoms + 1;
            a.occupancy = 1.0;
            if (tok.size() >= 8) {
                a.resid = std::atoi(tok[2].c_str());
                a.resName = tok[3];
                a.name = tok[4];
                a.chain = tok[5][0];
                a.occupancy = std::atof(tok[6].c_str());
                a.beta = std::atof(tok[7].c_str());
            }
            t.atoms.push_back(a);
            t.natoms++;
            break;
        }
        case BONDS:
            t.bonds.push_back(std::atoi(tok[0].c_str()));
            t.bonds.push_back(std::atoi(tok[1].c_str()));
            t.bonds_r0.push_back(tok.size() > 3 ? (float)std::atof(tok[3].c_str()) : 0.0f);
            break;
        case NATIVES:
            t.natives.push_back(std::atoi(tok[0].c_str()));
            t.natives.push_back(std::atoi(tok[1].c_str()));
            t.natives_r0.push_back(tok.size() > 3 ? (float)std::atof(tok[3].c_str()) : 0.0f);
            t.natives_eh.push_back(tok.size() > 4 ? (float)std::atof(tok[4].c_str()) : 0.0f);
            break;
        case PAIRS:
            t.pairs.push_back(std::atoi(tok[0].c_str()));
            t.pairs.push_back(std::atoi(tok[1].c_str()));
            break;
        default:
            throw Error(SOPB_ERR_INVALID, "line outside any section at " + path + ":" + std::to_string(lineno));
        }
    }
    return t;
}

std::vector<float> read_coords(const std::string& path, int expect) {
    std::ifstream f(path);
    if (!f) throw Error(SOPB_ERR_INVALID, "coordinates file " + path + " can not be found");
    std::vector<float> xyz;
    std::string line;
    while (std::getline(f, line)) {
        if (line.compare(0, 4, "ATOM") != 0 || line.size() < 54) continue;
        xyz.push_back((float)std::atof(line.substr(30, 8).c_str()));
        xyz.push_back((float)std::atof(line.substr(38, 8).c_str()));
        xyz.push_back((float)std::atof(line.substr(46, 8).c_str()));
    }
    if ((int)xyz.size() != 3 * expect)
        throw Error(SOPB_ERR_INVALID, "read " + std::to_string(xyz.size() / 3) + " beads from " + path +
                                          ", topology has " + std::to_string(expect));
    return xyz;
}

// savePDB (src/IO/pdbio.cpp:194-221) with PDBAtom::fprint's format
// (:265-280): atom ids in hexadecimal from 100000 atoms on; CONECT lines
// group consecutive bonds that share their first bead.
void save_pdb(const std::string& path, const std::vector<Atom>& atoms, const std::vector<Atom>& extra,
              const std::vector<int32_t>& bonds) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw Error(SOPB_ERR_INVALID, "cannot write " + path);
    const bool hex = atoms.size() + extra.size() >= 100000;
    int id = 0;
    for (const std::vector<Atom>* set : {&atoms, &extra})
        for (const Atom& a : *set)
            std::fprintf(f, hex ? "ATOM  %5x %-4s%c%3s %c%4d    %8.3f%8.3f%8.3f%6.2f%6.2f\n"
                                : "ATOM  %5d %-4s%c%3s %c%4d    %8.3f%8.3f%8.3f%6.2f%6.2f\n",
                         ++id, a.name.c_str(), a.altLoc, a.resName.c_str(), a.chain, a.resid, (double)a.x, (double)a.y,
                         (double)a.z, a.occupancy, a.beta);
    int last = -1;
    for (size_t b = 0; b + 1 < bonds.size(); b += 2) {
        if (bonds[b] != last) {
            if (last != -1) std::fputc('\n', f);
            std::fprintf(f, "CONECT%5d", bonds[b] + 1);
            last = bonds[b];
        }
        std::fprintf(f, "%5d", bonds[b + 1] + 1);
    }
    std::fprintf(f, "\nEND");
    std::fclose(f);
}

// ---------------------------------------------------------------------------
// plugins
// ---------------------------------------------------------------------------
void SOPPotential::compute() {
    std::vector<float> f;
    for (sopb_job* j : sim->jobs) {
        int32_t n = 0;
        sopb_job_size(j, &n);
        f.resize(4 * (size_t)n);
        check(sopb_job_read(j, SOPB_FORCES, f.data()), "compute");
    }
}

void SOPIntegrator::integrate() { sim->run(1); }

namespace {
struct NamedPotential : SOPPotential {
    explicit NamedPotential(const char* n) { name = n; }
};
struct NamedUpdater : SOPUpdater {
    NamedUpdater(const char* n, int f) { name = n; frequency = f; }
};
struct ListUpdater : SOPUpdater {
    int possible;
    ListUpdater(const char* n, int f, int p) : possible(p) { name = n; frequency = f; }
    void update() override {
        for (sopb_job* j : sim->jobs) check(sopb_job_rebuild_lists(j, possible, !possible), name.c_str());
    }
};
struct NamedIntegrator : SOPIntegrator {
    NamedIntegrator(const char* n, float hh) { name = n; h = hh; }
};
}  // namespace

Simulation::Simulation(const Config& c, int device) : cfg(c) {
    // initParameters (src/sop-gpu.cpp:67-88)
    const int run = (int)cfg.integer("run", -1);
    if (run == -1) {
        ntr = (int)cfg.integer("runnum");
        firstrun = (int)cfg.integer("firstrun");
    } else {
        ntr = 1;
        firstrun = run;
    }
    numsteps = cfg.integer("numsteps");
    top = Topology::load(cfg.str("topology"));
    for (int r = 0; r < ntr; ++r)
        coords.push_back(read_coords(replace_all(cfg.str("coordinates"), "<run>", std::to_string(r + firstrun)), top.natoms));
    initFF();
    check(sopb_context_create(device >= 0 ? device : (int)cfg.integer("device", 0), nullptr, &ctx), "context");
    const int n = top.natoms;
    seeds.resize(4 * (size_t)n * ntr);
    const int32_t seed = (int32_t)cfg.integer("seed", (int64_t)time(nullptr)) + firstrun;   // langevin.cu:23
    check(sopb_generate_seeds(seed, (int64_t)n * ntr, seeds.data()), "seeds");
    for (int r = 0; r < ntr; ++r) {
        sopb_job_desc d{};
        d.n = n;
        d.xyz = coords[r].data();
        d.nbonds = (int32_t)top.bonds_r0.size();
        d.bonds = top.bonds.data();
        d.bonds_r0 = top.bonds_r0.data();
        d.nnatives = (int32_t)top.natives_r0.size();
        d.natives = top.natives.data();
        d.natives_r0 = top.natives_r0.data();
        d.natives_eh = top.natives_eh.data();
        d.nfixed = (int32_t)fixed.size();
        d.fixed = fixed.data();
        d.npulled = (int32_t)pulled.size();
        d.pulled = pulled.data();
        d.nplane_fixed = (int32_t)plane_fixed.size();
        d.plane_fixed = plane_fixed.data();
        d.nplane_pulled = (int32_t)plane_pulled.size();
        d.plane_pulled = plane_pulled.data();
        d.seeds = seeds.data() + 4 * (size_t)r * n;
        d.params = params;
        sopb_job* j = nullptr;
        check(sopb_job_create(ctx, &d, &j), "job");
        jobs.push_back(j);
    }
}

Simulation::~Simulation() {
    if (ctx) sopb_context_destroy(ctx);
}

// initFF (src/gsop.cu:66-106): the same plugins in the same order, their
// config keys mapped onto the job parameters.
void Simulation::initFF() {
    sopb_params& p = params;
    sopb_default_params(&p);
    const Config& g = cfg;
    p.timestep = g.real("timestep");
    p.zeta = g.real("zeta", p.zeta);
    p.temperature = g.real("temperature", p.temperature);
    p.kspring_cov = g.real("kspring_cov", p.kspring_cov);
    p.R_limit = g.real("R_limit", p.R_limit);
    p.R_limit_bond = g.real("R_limit_bond", p.R_limit_bond);
    p.a = g.real("a", p.a);
    p.el = g.real("el", p.el);
    p.pairs_cutoff = g.real("pairs_cutoff", p.pairs_cutoff);
    p.pairlist_cutoff = g.real("pairlist_cutoff", p.pairlist_cutoff);
    p.pairs_freq = (int32_t)g.integer("pairs_freq", p.pairs_freq);
    p.pairs_threshold = g.real("pairs_threshold", p.pairs_threshold);
    p.possiblepairs_freq = (int32_t)g.integer("possiblepairs_freq", p.possiblepairs_freq);
    p.max_pairs = (int32_t)g.integer("max_pairs", p.max_pairs);
    p.max_possiblePairs = (int32_t)g.integer("max_possiblePairs", p.max_possiblePairs);
    p.nav = (int32_t)g.integer("nav", p.nav);
    p.minimization = g.boolean("minimization", false);
    p.heating = g.boolean("heating", false);
    if (p.heating) {
        p.tempFreq = (int32_t)g.integer("tempFreq");
        p.initialT = g.real("initialT");
        p.deltaT = g.real("deltaT");
    }
    if (g.has("stage")) throw Error(SOPB_ERR_INVALID, "Parameter `stage` is no longer supported");
    potentials.emplace_back(new NamedPotential("Covalent"));
    potentials.emplace_back(new NamedPotential("Native"));
    potentials.emplace_back(new NamedPotential("Long Range"));
    // createIndentationPotential (indentation.cu:19-66): tip updater first
    if (g.boolean("indentation", false)) {
        if (ntr > 1) throw Error(SOPB_ERR_INVALID, "Many-runs-per-GPU mode is not supported by indentation potential.");
        p.indentation = 1;
        if (g.boolean("indentationDiscreteSurf", false)) {
            // the surface as a square of beads (indentation.cu:137-201)
            p.indentationDiscreteSurf = 1;
            p.indentationSurfaceSize = (int32_t)g.integer("indentationSurfaceSize", 51);
            p.indentationSurfaceStep = g.real("indentationSurfaceStep", 1.4f);
            p.indentationPairsCutoff = g.real("indentationPairsCutoff", 40.0f);
        }
        g.float3("indentationChip", p.indentationChip);
        g.float3("indentationTip", p.indentationTip, p.indentationChip);
        g.float3("indentationDirection", p.indentationDirection);
        g.float3("indentationSurfaceR0", p.indentationSurfaceR0);
        g.float3("indentationSurfaceN", p.indentationSurfaceN);
        p.indentationTipR = g.real("indentationTipR");
        p.indentationKs = g.real("indentationKs");
        p.indentationDeltaX = g.real("indentationDeltaX");
        p.indentationMoveSurface = g.boolean("indentationMoveSurface", false);
        p.indentationFixTrans = g.boolean("indentationFixTrans", false);
        const float sig = g.real("indentationSigma", 1.0f), el = g.real("indentationEl", 1.0f);
        p.indentationTipSigma = g.real("indentationTipSigma", sig);
        p.indentationSurfSigma = g.real("indentationSurfSigma", sig);
        p.indentationTipEl = g.real("indentationTipEl", el);
        p.indentationSurfEl = g.real("indentationSurfEl", el);
        p.indentationTipA = g.real("indentationTipA", 0.0f);
        p.indentationTipB = g.real("indentationTipB", 1.0f);
        p.indentationSurfA = g.real("indentationSurfA", 0.0f);
        p.indentationSurfB = g.real("indentationSurfB", 1.0f);
        p.indentationTipZeta = g.real("indentationTipZeta", 5000.0f);
        p.indentationRetractionStep = g.integer("indentationRetractionStep", -1);
        updaters.emplace_back(new NamedUpdater("Indentation", p.nav));
        // the tip and surface beads of the output files; a discrete surface
        // forces them (indentation.cu:24-32)
        if (p.indentationDiscreteSurf || g.boolean("indentationShowTipSurf", false))
            updaters.emplace_back(new NamedUpdater("AdditionalAminos", (int)g.integer("outputtiming", 10000)));
        potentials.emplace_back(new NamedPotential("Indentation"));
    }
    // createPullingPotential (pulling.cu:22-35)
    if (g.boolean("pulling", false)) {
        p.pulling = 1;
        p.deltax = g.real("deltax", 0.0f);
        p.k_trans = g.real("k_trans", p.k_trans);
        p.fconst = g.real("fconst", 0.0f);
        if (p.deltax == 0.0f && p.fconst == 0.0f)
            throw Error(SOPB_ERR_INVALID, "Either 'deltax' or 'fconst' parameter should be specified to initiate pulling");
        if (g.has("fixed_beads") || g.has("pulled_beads"))
            throw Error(SOPB_ERR_INVALID, "'fixed_beads' and 'pulled_beads' are deprecated; use 'fixed' and 'pulled'");
        for (int i : g.ints("fixed")) fixed.push_back(i);
        for (int i : g.ints("pulled")) pulled.push_back(i);
        const std::string dir = g.str("pullDirection", "endToEnd");
        if (dir == "vector") {
            p.pull_direction = SOPB_PULL_VECTOR;
            g.float3("pullVector", p.pullVector);
        } else if (dir == "endToEnd") {
            p.pull_direction = SOPB_PULL_END_TO_END;
        } else {
            throw Error(SOPB_ERR_INVALID, "'pullDirection' parameter should be set to 'endToEnd' or 'vector'.");
        }
        p.fixedEnd = (int32_t)g.integer("fixedEnd");
        p.pulledEnd = (int32_t)g.integer("pulledEnd");
        p.pullFreq = (int32_t)g.integer("pullFreq", p.nav);
        potentials.emplace_back(new NamedPotential("Pulling"));
        if (p.deltax != 0.0f) updaters.emplace_back(new NamedUpdater("Pulling", p.pullFreq));
    }
    // createPullingPlanePotential (pulling_plane.cu:17-30)
    if (g.boolean("pullingPlane", false)) {
        p.pullingPlane = 1;
        p.pullingPlaneDeltax = g.real("pullingPlaneDeltax", 0.0f);
        if (p.pullingPlaneDeltax == 0.0f)
            throw Error(SOPB_ERR_INVALID, "'pullingPlaneDeltax' parameter should be specified to initiate this->");
        if (g.has("plane_fixed_beads") || g.has("plane_pulled_beads"))
            throw Error(SOPB_ERR_INVALID,
                        "'plane_fixed_beads' and 'plane_pulled_beads' parameters are deprecated. Use 'plane_fixed' and 'plane_pulled' instead");
        p.pullingPlaneKs = g.real("pullingPlaneKs", p.pullingPlaneKs);
        p.pullingPlaneKsCant = g.real("pullingPlaneKsCant", p.pullingPlaneKsCant);
        p.pullingPlaneZeta = g.real("pullingPlaneZeta", p.pullingPlaneZeta);
        for (int i : g.ints("plane_fixed")) plane_fixed.push_back(i);
        for (int i : g.ints("plane_pulled")) plane_pulled.push_back(i);
        g.float3("pullingPlaneDir", p.pullingPlaneDir);
        g.float3("pullingPlanePos", p.pullingPlanePos);
        p.pullingPlaneUpdateFreq = (int32_t)g.integer("pullingPlaneUpdateFreq", p.nav);
        p.pullingPlaneOutputFreq = (int32_t)g.integer("pullingPlaneOutputFreq", p.nav);
        potentials.emplace_back(new NamedPotential("Pulling Plane"));
        updaters.emplace_back(new NamedUpdater("Pulling Plane", p.pullingPlaneUpdateFreq));
    }
    updaters.emplace_back(new ListUpdater("Possiblepairlist", p.possiblepairs_freq, 1));
    updaters.emplace_back(new NamedUpdater("DAT output", (int)g.integer("outputtiming", 10000)));
    updaters.emplace_back(new ListUpdater("Pairlist", p.pairs_freq, 0));
    updaters.emplace_back(new NamedUpdater("DCD output", (int)g.integer("dcdfreq", 10000)));
    const bool hi = g.boolean("hi_on", false);
    if (p.heating) updaters.emplace_back(new NamedUpdater("TemperatureUpdater", p.tempFreq));
    if (hi) {
        if (p.minimization) throw Error(SOPB_ERR_INVALID, "Using minimization with BDHI integrator is not supported");
        p.hi_on = 1;
        p.hi_a = g.real("hi_a", p.hi_a);
        p.hi_exact = g.boolean("hi_exact", false);
        if (!p.hi_exact) {
            p.hi_capricious = g.boolean("hi_capricious", true);
            p.hi_epsilon_freq = (int32_t)g.integer("hi_epsilon_freq");
            p.hi_epsmax = g.real("hi_epsmax", p.hi_epsmax);
            p.hi_unlisted = g.boolean("hi_unlisted", true);
            updaters.emplace_back(new NamedUpdater("BDHI-TEA updater", p.hi_epsilon_freq));
        }
        p.hi_refresh = (int32_t)g.integer("hi_refresh", 1);
        if (p.hi_exact && p.hi_refresh > 1) updaters.emplace_back(new NamedUpdater("Cholesky refresh", p.hi_refresh));
        const std::string bm = g.str("hi_b_mode", "cholesky");
        p.hi_b_mode = bm == "reference" ? SOPB_HI_B_REFCOMPAT : SOPB_HI_B_CHOLESKY;
        integrator.reset(new NamedIntegrator("BDHI-TEA", p.timestep));
    } else {
        integrator.reset(new NamedIntegrator("Langevin", p.timestep));
    }
    p.log_rows = 4096;   // event-log ring of the pulling, indentation and plane lines
    p.verlet_skin = g.real("verlet_skin", 0.0f);   // near list of the Verlet rebuilds (this library)
    // runGPU's stride (src/gsop.cu:117-122)
    stride = p.nav;
    for (auto& u : updaters) stride = std::min(stride, u->frequency);
    p.stride = stride;
    for (auto& q : potentials) q->sim = this;
    for (auto& u : updaters) u->sim = this;
    integrator->sim = this;
}

void Simulation::run(int64_t nsteps) {
    check(sopb_run(ctx, jobs.data(), (int32_t)jobs.size(), nsteps), "run");
    check(sopb_context_sync(ctx), "sync");
    for (size_t r = 0; r < jobs.size(); ++r) {
        const int st = sopb_job_status(jobs[r]);
        if (st != SOPB_OK)
            throw Error(st, "run " + std::to_string(r + firstrun) + ": " + sopb_status_string(st));
    }
}

SOPPotential* Simulation::potentialByName(const std::string& n) const {
    for (auto& q : potentials) if (q->name == n) return q.get();
    throw Error(SOPB_ERR_INVALID, "Unable to find requested potential '" + n + "'");
}

SOPUpdater* Simulation::updaterByName(const std::string& n) const {
    for (auto& u : updaters) if (u->name == n) return u.get();
    throw Error(SOPB_ERR_INVALID, "Unable to find requested updater '" + n + "'");
}

}  // namespace sopb_host
