// sopb_mirror.h — the reference's host-side surface over the sopb C ABI.
//
// SOP-GPU's host code reads a key/value config file, a .top topology and PDB
// coordinates, creates its plugins (potentials, updaters, one integrator) in
// a fixed order and runs the stride loop (src/gsop.h:69-105,
// src/gsop.cu:66-163).  This mirror keeps that surface -- the same plugin
// class names, plugin names, frequencies and creation order, the same config
// keys and file formats -- and runs the step through the C ABI, where every
// plugin's work is fused on the device.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sopb.h"

namespace sopb_host {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& what) : std::runtime_error(what), code(c) {}
};

// ---- config (src/IO/configreader.cpp) --------------------------------------
class Config {
public:
    explicit Config(const std::string& path);
    Config() = default;
    void set(const std::string& key, const std::string& value) { values_[key] = value; }
    bool has(const std::string& key) const { return values_.count(key) != 0; }
    std::string raw(const std::string& key) const;
    std::string str(const std::string& key) const;                  // <key> masks applied
    std::string str(const std::string& key, const std::string& def) const;
    int64_t integer(const std::string& key) const;
    int64_t integer(const std::string& key, int64_t def) const;
    float real(const std::string& key) const;
    float real(const std::string& key, float def) const;
    bool boolean(const std::string& key) const;
    bool boolean(const std::string& key, bool def) const;
    std::vector<int> ints(const std::string& key) const;
    std::vector<int> ints(const std::string& key, const std::vector<int>& def) const;
    void float3(const std::string& key, float out[3]) const;
    void float3(const std::string& key, float out[3], const float def[3]) const;

private:
    std::map<std::string, std::string> values_;   // sorted, as the reference's std::map
};

// ---- topology and coordinates (src/IO/topio.cpp, src/IO/pdbio.cpp) --------
struct Atom {                      // one PDB ATOM record (PDBAtom)
    std::string name = "CA", resName = "ALA";
    char altLoc = ' ', chain = 'A';
    int resid = 0;
    double occupancy = 0.0, beta = 0.0;
    double x = 0.0, y = 0.0, z = 0.0;
};
struct Topology {
    int natoms = 0;
    std::vector<Atom> atoms;           // [ atoms ] section, in file order
    std::vector<int32_t> bonds;        // (i, j) pairs
    std::vector<float> bonds_r0;
    std::vector<int32_t> natives;
    std::vector<float> natives_r0, natives_eh;
    std::vector<int32_t> pairs;        // [ pairs ] section (initial possible pairs)
    static Topology load(const std::string& path);
};
std::vector<float> read_coords(const std::string& path, int expect);         // xyz[3n]
// savePDB (src/IO/pdbio.cpp:194-221): the atoms, then `extra` (the tip and
// surface beads of an indentation run), then CONECT records of the bonds.
void save_pdb(const std::string& path, const std::vector<Atom>& atoms, const std::vector<Atom>& extra,
              const std::vector<int32_t>& bonds);

// ---- DCD trajectories (src/IO/dcdio.cpp:56-194) ------------------------------
// CHARMM/NAMD binary layout: an 84-byte header record, two 80-character
// title lines, the atom count, then per frame the X, Y and Z blocks, each
// framed by its byte length.  No unit cell.
void dcd_write_header(const std::string& path, int natoms, int nsavc, float delta);
void dcd_append_frame(const std::string& path, const std::vector<float>& X, const std::vector<float>& Y,
                      const std::vector<float>& Z);

// ---- plugin surface (src/gsop.h:69-105) -------------------------------------
class Simulation;

class SOPPotential {
public:
    virtual ~SOPPotential() = default;
    std::string name;
    // The device sums every potential into one force per bead inside
    // sopb_run; compute() evaluates that sum once (SOPB_FORCES) for a run.
    virtual void compute();
    virtual int getEnergiesCount() const { return 0; }
    Simulation* sim = nullptr;
};

class SOPUpdater {
public:
    virtual ~SOPUpdater() = default;
    std::string name;
    int frequency = 1;
    // Runs on the device at its step inside sopb_run; update() applies it
    // now, outside the step gate, where that has a meaning (list rebuilds).
    virtual void update() {}
    Simulation* sim = nullptr;
};

class SOPIntegrator {
public:
    virtual ~SOPIntegrator() = default;
    std::string name;
    float h = 0.0f;
    // One step of every potential and the integrator for all runs.
    virtual void integrate();
    Simulation* sim = nullptr;
};

// ---- the simulation (initGPU / initFF / runGPU) ---------------------------------
class Simulation {
public:
    explicit Simulation(const Config& cfg, int device = -1);
    ~Simulation();
    void initFF();                         // plugins in the reference's creation order
    void run(int64_t nsteps);              // sopb_run over every run of the job
    // the reference's loop: (numsteps/stride + 1) * stride steps with the
    // output updaters (.dat, DCD, restart PDB, pulling and indentation lines)
    // at their steps, then the final PDB of every run
    void runGPU();
    SOPPotential* potentialByName(const std::string& n) const;
    SOPUpdater* updaterByName(const std::string& n) const;

    const Config& cfg;
    Topology top;
    int ntr = 1, firstrun = 0;
    int64_t numsteps = 0;
    int stride = 1;
    sopb_params params{};
    std::vector<int32_t> fixed, pulled;
    std::vector<int32_t> plane_fixed, plane_pulled;   // pulling plane masks
    std::vector<std::vector<float>> coords;     // per run, xyz[3n]
    std::vector<uint32_t> seeds;                // all runs, one ran2 stream
    sopb_context* ctx = nullptr;
    std::vector<sopb_job*> jobs;
    std::vector<std::unique_ptr<SOPPotential>> potentials;
    std::vector<std::unique_ptr<SOPUpdater>> updaters;
    std::unique_ptr<SOPIntegrator> integrator;
};

void check(int code, const char* what);

}  // namespace sopb_host
