// sopb_output.cpp — the reference's output updaters over the sopb C ABI:
// the energy .dat files (OutputManager, src/Updaters/output_manager.cu),
// DCD trajectories and restart PDBs (DcdOutputManager,
// src/Updaters/dcd_manager.cpp; src/IO/dcdio.cpp), the pulling lines
// (PullingPotential::savePullingData, src/Potentials/pulling.cu:167-190), the
// indentation lines (IndentationTipUpdater::update,
// src/Potentials/indentation.cu:414-550) and the tip/surface beads written
// into DCD and PDB files (IndentationAminoUpdater, indentation.cu:238-365,
// 553-582).
//
// The reference stops its loop at every stride to run these on the host.
// Here the run advances from one output step to the next in one call; the
// values the reference reads at an output step come from the device at that
// step (SOPB_OBSERVABLES, coordinates), and the per-update lines of the
// pulling and indentation updaters, which run inside the step kernel, come
// from the job's event log (sopb_job_log) after the run that made them.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <deque>
#include <numeric>

#include "sopb_mirror.h"

namespace sopb_host {

namespace {

std::string replace_run(std::string s, int run) {
    const std::string key = "<run>", val = std::to_string(run);
    for (size_t pos = 0; (pos = s.find(key, pos)) != std::string::npos; pos += val.size()) s.replace(pos, key.size(), val);
    return s;
}

FILE* open_or_throw(const std::string& path, const char* mode) {
    FILE* f = std::fopen(path.c_str(), mode);
    if (!f) throw Error(SOPB_ERR_INVALID, "cannot open " + path);
    return f;
}

void put_i32(std::vector<unsigned char>& b, int32_t v) {
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    b.insert(b.end(), p, p + 4);
}
void put_f32(std::vector<unsigned char>& b, float v) {
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    b.insert(b.end(), p, p + 4);
}
void put_title(std::vector<unsigned char>& b, const std::string& t) {
    std::string s = t.substr(0, 80);
    s.resize(80, ' ');
    b.insert(b.end(), s.begin(), s.end());
}

int64_t gcd64(int64_t a, int64_t b) { return b == 0 ? a : gcd64(b, a % b); }
int64_t lcm64(int64_t a, int64_t b) { return a / gcd64(a, b) * b; }

}  // namespace

// write_header (src/IO/dcdio.cpp:100-148): NFILE = NPRIV = NSAVC = the
// output frequency, as the reference's DcdOutputManager sets them.
void dcd_write_header(const std::string& path, int natoms, int nsavc, float delta) {
    std::vector<unsigned char> b;
    put_i32(b, 84);
    b.insert(b.end(), {'C', 'O', 'R', 'D'});
    put_i32(b, nsavc);           // NFILE
    put_i32(b, nsavc);           // NPRIV
    put_i32(b, nsavc);           // NSAVC
    put_i32(b, 0);               // NPRIV - NSAVC
    for (int k = 0; k < 5; ++k) put_i32(b, 0);
    put_f32(b, delta);
    for (int k = 0; k < 9; ++k) put_i32(b, 0);
    put_i32(b, 24);
    put_i32(b, 84);
    put_i32(b, 164);
    put_i32(b, 2);
    put_title(b, "REMARKS CREATED BY sopb-gpu");
    char date[64];
    const std::time_t now = std::time(nullptr);
    std::strftime(date, sizeof(date), "%a %b %d %H:%M:%S %Y", std::localtime(&now));
    put_title(b, std::string("REMARKS DATE: ") + date);
    put_i32(b, 164);
    put_i32(b, 4);
    put_i32(b, natoms);
    put_i32(b, 4);
    FILE* f = open_or_throw(path, "wb");
    std::fwrite(b.data(), 1, b.size(), f);
    std::fclose(f);
}

// write_frame (src/IO/dcdio.cpp:174-194): three Fortran records.
void dcd_append_frame(const std::string& path, const std::vector<float>& X, const std::vector<float>& Y,
                      const std::vector<float>& Z) {
    FILE* f = open_or_throw(path, "ab");
    const int32_t len = (int32_t)(X.size() * 4);
    for (const std::vector<float>* v : {&X, &Y, &Z}) {
        std::fwrite(&len, 4, 1, f);
        std::fwrite(v->data(), 4, v->size(), f);
        std::fwrite(&len, 4, 1, f);
    }
    std::fclose(f);
}

// ---------------------------------------------------------------------------
// The output updaters of one simulation.
// ---------------------------------------------------------------------------
class OutputManagers {
public:
    explicit OutputManagers(Simulation& s);
    // The updaters due at `step` (a multiple of the stride), in the
    // reference's creation order: AdditionalAminos, DAT output, DCD output.
    void at_step(int64_t step);
    // After a run that ended at `step`: the event-log lines it made, and the
    // frames that waited for the tip state of their step.
    void after_run(int64_t step);
    // The next step after `step` at which at_step has work, or INT64_MAX.
    int64_t next_event(int64_t step) const;
    // Steps one run may span without overrunning a job's event-log ring.
    int64_t max_run() const { return max_run_; }
    // The final coordinates of every run (src/gsop.cu:149-160).
    void final_pdbs();

private:
    struct Frame {
        int64_t step;
        bool dcd, restart;
        std::vector<float> x;   // xyzw of every run
    };
    void tip_row(const sopb_log_row& r);
    void write_frame(const Frame& fr);
    void amino_update();

    Simulation& sim;
    const Config& cfg;
    const int n;
    int64_t dat_freq, dcd_freq, restart_freq, amino_freq = 0;
    std::vector<std::string> dat_files, dcd_files, restart_files, pull_files, plane_files;
    std::string indent_file;
    bool rg, tea, pull_log, indent_log, show_tip, plane_log;
    int width, print_runs;
    std::vector<Atom> atoms, extra;
    std::deque<Frame> pending;
    std::deque<int64_t> amino_steps;           // AdditionalAminos updates waiting for the tip state
    int64_t max_run_ = INT64_MAX;
    // indentation: state after the last tip update, and the output averages
    int64_t indent_freq = 1000;
    float tip[3] = {0, 0, 0}, chip[3] = {0, 0, 0}, dx = 0.0f;
    float fav[4] = {0, 0, 0, 0}, kdx_av = 0.0f, ks = 0.0f;
    float dir[3] = {0, 0, 0}, cantvec[3] = {0, 0, 0};
    std::vector<float> surf0;                   // surface beads at dx = 0, xyz
    int64_t tip_step = -1;
};

OutputManagers::OutputManagers(Simulation& s)
    : sim(s), cfg(s.cfg), n(s.top.natoms) {
    const Config& g = cfg;
    const sopb_params& p = s.params;
    dat_freq = g.integer("outputtiming", 10000);
    dcd_freq = g.integer("dcdfreq", 10000);
    restart_freq = g.integer("restartfreq", 100000);
    rg = g.boolean("computeRg", false);
    tea = p.hi_on != 0;
    width = (int)g.integer("outputcolwidth", 16);
    print_runs = (int)g.integer("printruns", 10);
    pull_log = p.pulling && p.deltax != 0.0f;
    indent_log = p.indentation != 0;
    // a discrete surface forces the tip and surface beads into the files
    // (indentation.cu:24-32)
    show_tip = indent_log && (p.indentationDiscreteSurf || g.boolean("indentationShowTipSurf", false));
    plane_log = p.pullingPlane != 0;
    atoms = s.top.atoms;
    if (p.pulling) {
        // the beta column marks pulled (2) and fixed (1) beads
        // (src/Potentials/pulling.cu:96-125)
        for (Atom& a : atoms) a.beta = 0.0;
        for (int32_t i : s.pulled) atoms[i].beta = 2.0;
        for (int32_t i : s.fixed) atoms[i].beta = 1.0;
    }
    if (plane_log) {
        // the pulling plane's masks, created after pulling (pulling_plane.cu:98-117)
        for (Atom& a : atoms) a.beta = 0.0;
        for (int32_t i : s.plane_pulled) atoms[i].beta = 2.0;
        for (int32_t i : s.plane_fixed) atoms[i].beta = 1.0;
    }
    for (int r = 0; r < s.ntr; ++r) {
        const int run = r + s.firstrun;
        dat_files.push_back(replace_run(g.str("outputname", "energy." + g.str("name", "unnamed") + "_<run>.dat"), run));
        dcd_files.push_back(replace_run(g.str("DCDfile", g.str("name", "unnamed") + "_<run>.dcd"), run));
        restart_files.push_back(
            replace_run(g.str("restartname", "restart." + g.str("name", "unnamed") + "_<run>.pdb"), run));
        if (pull_log)
            pull_files.push_back(replace_run(g.str("pullOutput", "pull." + g.str("name", "unnamed") + "_<run>.dat"), run));
        if (plane_log)
            plane_files.push_back(
                replace_run(g.str("pullingPlaneOutput", "pullplane." + g.str("name", "unnamed") + "_<run>.dat"), run));
    }
    if (indent_log) {
        indent_freq = g.integer("indentationOutputFreq", 1000);
        indent_file = g.str("indentationOutput", "indentation." + g.str("name", "unnamed") + "_<run>.dat");
        ks = p.indentationKs;
        const float nrm = std::sqrt(p.indentationDirection[0] * p.indentationDirection[0] +
                                    p.indentationDirection[1] * p.indentationDirection[1] +
                                    p.indentationDirection[2] * p.indentationDirection[2]);
        for (int c = 0; c < 3; ++c) {
            dir[c] = p.indentationDirection[c] / nrm;
            tip[c] = p.indentationTip[c];
            chip[c] = p.indentationChip[c];
        }
    }
    if (show_tip) {
        // IndentationAminoUpdater ctor (indentation.cu:240-365): the
        // cantilever base shifted sideways by indentationCantLength, the tip,
        // and a square of surface beads around indentationSurfaceR0
        amino_freq = dat_freq;
        const float* r0 = p.indentationDirection;
        float r[3];
        if (r0[0] != 0.0f) {
            r[1] = 1.0f;
            r[2] = 0.0f;
            r[0] = -r[1] * r0[1] / r0[0];
            const float len = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            for (float& v : r) v /= len;
        } else {
            r[0] = 1.0f;
            r[1] = r[2] = 0.0f;
        }
        const float cl = g.real("indentationCantLength", 500.0f);
        for (int c = 0; c < 3; ++c) cantvec[c] = r[c] * cl;
        const int S = (int)g.integer("indentationSurfaceSize", 51);
        const float step = g.real("indentationSurfaceStep", 1.4f);
        const float* nn = p.indentationSurfaceN;
        const float* m0 = p.indentationSurfaceR0;
        float r1[3];
        if (nn[0] == 0.0f) { r1[0] = 1.0f; r1[1] = 0.0f; r1[2] = 0.0f; }
        else if (nn[1] == 0.0f) { r1[0] = 0.0f; r1[1] = 1.0f; r1[2] = 0.0f; }
        else if (nn[2] == 0.0f) { r1[0] = 0.0f; r1[1] = 0.0f; r1[2] = 1.0f; }
        else { r1[0] = 0.0f; r1[1] = 1.0f; r1[2] = -(nn[1] / nn[2]) * r1[1]; }
        const float nr1 = std::sqrt(r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2]);
        for (float& v : r1) v /= nr1;
        const float r2[3] = {nn[1] * r1[2] - nn[2] * r1[1], nn[2] * r1[0] - nn[0] * r1[2], nn[0] * r1[1] - nn[1] * r1[0]};
        Atom base, tipa;
        base.name = tipa.name = "CA";
        base.resName = tipa.resName = "TIP";
        base.chain = tipa.chain = 'T';
        base.resid = 1;
        tipa.resid = 2;
        base.occupancy = tipa.occupancy = 0.0;
        base.x = chip[0] + cantvec[0]; base.y = chip[1] + cantvec[1]; base.z = chip[2] + cantvec[2];
        tipa.x = tip[0]; tipa.y = tip[1]; tipa.z = tip[2];
        extra = {base, tipa};
        for (int i = 0; i < S; ++i)
            for (int j = 0; j < S; ++j) {
                const int i1 = i - S / 2, i2 = j - S / 2;
                Atom m;
                m.name = "CA";
                m.resName = "MIC";
                m.chain = 'M';
                m.resid = 1;
                m.occupancy = 0.0;
                m.x = m0[0] + i1 * step * r1[0] + i2 * step * r2[0];
                m.y = m0[1] + i1 * step * r1[1] + i2 * step * r2[1];
                m.z = m0[2] + i1 * step * r1[2] + i2 * step * r2[2];
                surf0.insert(surf0.end(), {(float)m.x, (float)m.y, (float)m.z});
                extra.push_back(m);
            }
        // VMD script joining the cantilever beads and the surface grid
        FILE* v = open_or_throw(g.str("indentationSurfConnectFile", "connect_mica.vmd"), "w");
        auto bond = [&](int a, const std::string& to) {
            std::fprintf(v, "set sel [atomselect top \"index %d\"]\nset bonds {%s}\n$sel setbonds [list $bonds]\n$sel delete\n",
                         a, to.c_str());
        };
        bond(n, std::to_string(n + 1));
        bond(n + 1, std::to_string(n));
        for (int i = 0; i < S; ++i)
            for (int j = 0; j < S; ++j) {
                std::string to;
                if (i != S - 1) to += std::to_string(2 + (i + 1) * S + j + n);
                if (j != S - 1) to += " " + std::to_string(2 + i * S + j + 1 + n);
                bond(2 + i * S + j + n, to);
            }
        std::fclose(v);
    }
    // files start empty; DCDs with their header (the constructors of the
    // output managers)
    for (int r = 0; r < s.ntr; ++r) {
        std::fclose(open_or_throw(dat_files[r], "w"));
        dcd_write_header(dcd_files[r], n + (int)extra.size(), (int)dcd_freq, 0.0f);
        if (pull_log) std::fclose(open_or_throw(pull_files[r], "w"));
        if (plane_log) std::fclose(open_or_throw(plane_files[r], "w"));
    }
    if (indent_log) std::fclose(open_or_throw(indent_file, "w"));
    // one event-log row per updater pass at most: a run of this many steps
    // cannot wrap the ring
    if (pull_log || indent_log || plane_log) max_run_ = (int64_t)(p.log_rows - 2) * s.stride;
}

int64_t OutputManagers::next_event(int64_t step) const {
    int64_t best = INT64_MAX;
    for (int64_t f : {dat_freq, dcd_freq, restart_freq, amino_freq}) {
        if (f <= 0) continue;
        const int64_t m = lcm64(f, sim.stride);
        best = std::min(best, (step / m + 1) * m);
    }
    return best;
}

void OutputManagers::amino_update() {
    // IndentationAminoUpdater::update (indentation.cu:553-582)
    extra[1].x = tip[0]; extra[1].y = tip[1]; extra[1].z = tip[2];
    if (sim.params.indentationMoveSurface) {
        for (size_t k = 0; k + 2 < extra.size(); ++k) {
            extra[2 + k].x = surf0[3 * k] + dx * dir[0];
            extra[2 + k].y = surf0[3 * k + 1] + dx * dir[1];
            extra[2 + k].z = surf0[3 * k + 2] + dx * dir[2];
        }
    } else {
        extra[0].x = chip[0] + cantvec[0]; extra[0].y = chip[1] + cantvec[1]; extra[0].z = chip[2] + cantvec[2];
    }
}

void OutputManagers::at_step(int64_t step) {
    const sopb_params& p = sim.params;
    if (amino_freq && step % amino_freq == 0) amino_steps.push_back(step);
    if (dat_freq > 0 && step % dat_freq == 0) {
        // OutputManager::update (output_manager.cu:73-127) and
        // printDataToFile (:339-360)
        std::vector<std::array<double, 8>> obs(sim.ntr);
        for (int r = 0; r < sim.ntr; ++r) check(sopb_job_read(sim.jobs[r], SOPB_OBSERVABLES, obs[r].data()), "observables");
        std::printf("Writing output at step %lld of %lld. ", (long long)step, (long long)sim.numsteps);
        if (sim.ntr == 1) std::printf("Run %d.\n", sim.firstrun);
        else std::printf("%d runs.\n", sim.ntr);
        std::printf("%*s%*s%*s%*s%*s%*s%*s%*s%*s", width, "Run", width, "TimeStep", width, "Temperature", width,
                    "Covalent", width, "Native", width, "Long-Range", width, "Total", width, "Native#", width, "Rg");
        if (tea) std::printf("%*s", width, "TEA-eps");
        std::printf("\n");
        // computeTemperatures (:144-155) carries its FP64 accumulator from one
        // run to the next: run r prints (T_{r-1} + sum_r) / (n nav).
        double carry = 0.0;
        const double norm = (double)n * (double)p.nav;
        for (int r = 0; r < sim.ntr; ++r) {
            carry = (carry + obs[r][0] * norm) / norm;
            const float T = (float)carry;
            const float e[3] = {(float)obs[r][1], (float)obs[r][2], (float)obs[r][3]};
            const double total = (double)e[0] + (double)e[1] + (double)e[2];
            const int contacts = (int)obs[r][5];
            const float Rg = rg ? (float)obs[r][6] : 0.0f;
            const float eps = (float)obs[r][7];
            FILE* f = open_or_throw(dat_files[r], "a");
            std::fprintf(f, "%12lld\t%8.5f\t", (long long)step, T);
            for (float v : e) std::fprintf(f, "%8.5f\t", v);
            std::fprintf(f, "%8.5f\t%8d\t%8.5f", total, contacts, Rg);
            if (tea) std::fprintf(f, "\t%2.9f", eps);
            std::fprintf(f, "\n");
            std::fclose(f);
            if (r < print_runs) {
                std::printf("%*d%*lld%*f%*f%*f%*f%*f%*d%*f", width, r + sim.firstrun, width, (long long)step, width, T,
                            width, e[0], width, e[1], width, e[2], width, total, width, contacts, width, Rg);
                if (tea) std::printf("%*f", width, eps);
                std::printf("\n");
            } else if (r == print_runs) {
                std::printf("%*s\n", width, "...");
            }
        }
    }
    const bool dcd = dcd_freq > 0 && step % dcd_freq == 0;
    const bool restart = restart_freq > 0 && step % restart_freq == 0;
    if (dcd || restart) {
        // DcdOutputManager::update (dcd_manager.cpp:72-118): coordinates now,
        // written once the tip state of this step is known
        Frame fr{step, dcd, restart, std::vector<float>((size_t)4 * n * sim.ntr)};
        check(sopb_jobs_download_coords(sim.ctx, sim.jobs.data(), (int32_t)sim.jobs.size(), fr.x.data()), "coords");
        pending.push_back(std::move(fr));
    }
}

void OutputManagers::write_frame(const Frame& fr) {
    const size_t m = (size_t)n + extra.size();
    std::vector<float> X(m), Y(m), Z(m);
    for (size_t k = 0; k < extra.size(); ++k) {
        X[n + k] = extra[k].x;
        Y[n + k] = extra[k].y;
        Z[n + k] = extra[k].z;
    }
    for (int r = 0; r < sim.ntr; ++r) {
        const float* x = fr.x.data() + (size_t)4 * n * r;
        for (int i = 0; i < n; ++i) {
            X[i] = x[4 * i];
            Y[i] = x[4 * i + 1];
            Z[i] = x[4 * i + 2];
        }
        if (fr.dcd) dcd_append_frame(dcd_files[r], X, Y, Z);
        if (fr.restart) {
            std::vector<Atom> a = atoms;
            for (int i = 0; i < n; ++i) { a[i].x = X[i]; a[i].y = Y[i]; a[i].z = Z[i]; }
            save_pdb(restart_files[r], a, extra, sim.top.bonds);
        }
    }
}

void OutputManagers::final_pdbs() {
    const std::string mask = cfg.str("finalcoord", cfg.str("name", "unnamed") + "_<run>_final.pdb");
    std::vector<float> x((size_t)4 * n);
    std::vector<Atom> a = atoms;
    for (int r = 0; r < sim.ntr; ++r) {
        check(sopb_job_read(sim.jobs[r], SOPB_COORDS, x.data()), "coords");
        for (int i = 0; i < n; ++i) {
            a[i].x = x[4 * i];
            a[i].y = x[4 * i + 1];
            a[i].z = x[4 * i + 2];
        }
        save_pdb(replace_run(mask, r + sim.firstrun), a, extra, sim.top.bonds);
    }
}

// IndentationTipUpdater::update (indentation.cu:496-534): the averages over
// the output window and one line every indentationOutputFreq steps.
void OutputManagers::tip_row(const sopb_log_row& row) {
    const float* v = row.v;
    for (int c = 0; c < 3; ++c) {
        tip[c] = v[6 + c];
        chip[c] = v[9 + c];
    }
    dx = v[5];
    tip_step = row.step;
    for (int c = 0; c < 4; ++c) fav[c] += v[c];
    kdx_av += v[4] * ks;
    if (row.step % indent_freq == 0) {
        const int factor = (int)(indent_freq / sim.params.nav);
        for (float& f : fav) f /= factor;
        kdx_av /= factor;
        const float fmod = std::sqrt(fav[0] * fav[0] + fav[1] * fav[1] + fav[2] * fav[2]);
        FILE* f = open_or_throw(indent_file, "a");
        std::fprintf(f, "%lld\t%8.5f\t%8.5f\t%8.5f\t%8.5f\t%8.5f\t%8.5f\t%8.5f\t%8.5f\t%8.5f\t%8.5f\t%8.5f\t%8.5f\t%8.5f\t%8.5f\n",
                     (long long)row.step, dx, fav[3], fmod, std::fabs(v[4] * ks), kdx_av, fav[0], fav[1], fav[2], tip[0],
                     tip[1], tip[2], chip[0], chip[1], chip[2]);
        std::fclose(f);
        for (float& q : fav) q = 0.0f;
        kdx_av = 0.0f;
    }
}

void OutputManagers::after_run(int64_t step) {
    // every row of the steps before `step` is on the device now
    std::vector<std::vector<sopb_log_row>> rows(sim.ntr);
    if (pull_log || indent_log || plane_log) {
        for (int r = 0; r < sim.ntr; ++r) {
            std::vector<sopb_log_row> buf(4096);
            for (;;) {
                int32_t got = 0;
                check(sopb_job_log(sim.jobs[r], buf.data(), (int32_t)buf.size(), &got), "event log");
                rows[r].insert(rows[r].end(), buf.begin(), buf.begin() + got);
                if (got < (int32_t)buf.size()) break;
            }
        }
    }
    if (pull_log) {
        for (int r = 0; r < sim.ntr; ++r) {
            FILE* f = open_or_throw(pull_files[r], "a");
            for (const sopb_log_row& q : rows[r])
                if (q.kind == SOPB_LOG_PULL)
                    std::fprintf(f, "%12lld\t%5.3f\t%5.3f\t%5.3f\t%5.3f\t%5.3f\t%5.3f\n", (long long)q.step, q.v[0],
                                 q.v[1], q.v[2], q.v[3], q.v[4], q.v[5]);
            std::fclose(f);
        }
    }
    if (plane_log) {
        // PullingPlaneUpdater::update's lines (pulling_plane.cu:234-246)
        for (int r = 0; r < sim.ntr; ++r) {
            FILE* f = open_or_throw(plane_files[r], "a");
            for (const sopb_log_row& q : rows[r])
                if (q.kind == SOPB_LOG_PLANE)
                    std::fprintf(f, "%12lld\t%f\t%f\t%f\t%f\t%f\n", (long long)q.step, q.v[0], q.v[1], q.v[2], q.v[3],
                                 q.v[4]);
            std::fclose(f);
        }
    }
    // tip lines and the frames / AdditionalAminos updates of the same steps,
    // in step order (the tip updater runs first at a step)
    size_t k = 0;
    const std::vector<sopb_log_row> none;
    const std::vector<sopb_log_row>& tr = indent_log ? rows[0] : none;
    auto next_row = [&]() -> int64_t {
        while (k < tr.size() && tr[k].kind != SOPB_LOG_TIP) ++k;
        return k < tr.size() ? tr[k].step : INT64_MAX;
    };
    for (;;) {
        const int64_t rs = next_row();
        const int64_t as = amino_steps.empty() ? INT64_MAX : amino_steps.front();
        const int64_t fs = pending.empty() ? INT64_MAX : pending.front().step;
        const int64_t es = std::min(as, fs);
        if (rs != INT64_MAX && rs <= es) {
            tip_row(tr[k++]);
            continue;
        }
        if (es >= step) break;             // its step's rows come with the next run
        if (as <= fs) {
            amino_update();
            amino_steps.pop_front();
        } else {
            write_frame(pending.front());
            pending.pop_front();
        }
    }
    while (k < tr.size()) {                 // rows at or after `step` cannot occur; keep order anyway
        if (tr[k].kind == SOPB_LOG_TIP) tip_row(tr[k]);
        ++k;
    }
}

// runGPU (src/gsop.cu:111-163): the updaters at every multiple of the stride
// up to (numsteps / stride) * stride, the integrator to one stride beyond,
// then the final coordinates of every run.
void Simulation::runGPU() {
    OutputManagers out(*this);
    const int64_t last = (numsteps / stride) * stride;
    const int64_t total = last + stride;
    int64_t step = 0;
    for (;;) {
        if (step <= last) out.at_step(step);
        int64_t next = std::min(out.next_event(step), total);
        if (out.max_run() < next - step) next = step + out.max_run();   // (no overflow when unbounded)
        run(next - step);
        step = next;
        out.after_run(step);
        if (step >= total) break;
    }
    out.final_pdbs();
}

}  // namespace sopb_host
