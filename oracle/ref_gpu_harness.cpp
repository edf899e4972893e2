// ref_gpu_harness.cpp — drives the reference's own CUDA path (compiled from
// the SOP-GPU source tree by oracle/build_ref.sh) for a given config and
// dumps state at chosen steps.  Run on a B200 to make golden fixtures of
// the reference itself.  TEST INFRASTRUCTURE ONLY.
//
//   ref_gpu <config.sop> <outdir> <total_steps> <dump steps...>
//
// With no dump steps it only times the loop: the wall time from the end of
// the step-0 updater pass to the device's completion of the last step
// (set-up, input reading and the step-0 list builds excluded), printed as
// "ref_gpu_time <seconds> <bead-steps/s>".
//
// The loop is runGPU's (src/gsop.cu:111-148): updaters every `stride` steps,
// then every potential's compute() and the integrator.  At a dump step s the
// files <outdir>/<what>_<s>.bin hold the state after s steps; forces_0.bin
// holds the potential forces of step 0 (after the step-0 updaters).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <set>
#include <string>
#include <vector>

#include "gsop.h"

SOP sop;  // defined by sop-gpu.cpp in the reference binary

// Layout prefixes of the reference's host-side globals (same member order).
struct HybTauView { uint4* h_seeds; uint4* d_seeds; uint4 mseed; };
struct PairsView { float pairsCutoff2, a2, el, minus6elovera2; int* d_pairs; int* d_pairsCount; float* d_energies; int max_pairs; };
struct PairListView { float pairlistCutoff; int* d_possiblePairs; int* d_possiblePairsCount; };
struct IndentView { float3 tipCoord, chipCoord, chipCoord0; };
extern HybTauView ht;
extern PairsView hc_pairs;
extern PairListView hc_pairList;
extern IndentView hc_indentation;

static void dump(const std::string& dir, const char* what, long step, const void* dev, size_t bytes, bool host = false) {
    std::vector<char> buf(bytes);
    if (host) std::memcpy(buf.data(), dev, bytes);
    else cudaMemcpy(buf.data(), dev, bytes, cudaMemcpyDeviceToHost);
    char name[512];
    std::snprintf(name, sizeof(name), "%s/%s_%ld.bin", dir.c_str(), what, step);
    FILE* f = std::fopen(name, "wb");
    std::fwrite(buf.data(), 1, bytes, f);
    std::fclose(f);
}

int main(int argc, char** argv) {
    if (argc < 4) return 2;
    const std::string dir = argv[2];
    const long total = std::atol(argv[3]);
    std::set<long> dumps;
    for (int k = 4; k < argc; ++k) dumps.insert(std::atol(argv[k]));
    // initParameters (src/sop-gpu.cpp:67-88)
    parameters::_initialize(argv[1]);
    int run = parameters::run.get();
    if (run == -1) { gsop.Ntr = parameters::runnum.get(); gsop.firstrun = parameters::firstrun.get(); }
    else { gsop.Ntr = 1; gsop.firstrun = run; }
    gsop.numsteps = total;
    gsop.nav = parameters::nav.get();
    gsop.deviceId = parameters::device.get();
    gsop.step = 0;
    sop.load(parameters::topology.get().c_str());
    initGPU();
    for (int i = 0; i < gsop.Ntr; i++) {
        readCoord(parameters::coordinates.replace("<run>", i + gsop.firstrun).c_str(), sop);
        copyCoordinatesTrajectory(i);
    }
    copyCoordinates();
    initFF();
    const size_t N = gsop.aminoCount;
    int stride = gsop.nav;
    for (int u = 0; u < updatersCount; u++) if (updaters[u]->frequency < stride) stride = updaters[u]->frequency;
    updaterByName("Pairlist")->update();
    FILE* meta = std::fopen((dir + "/meta.txt").c_str(), "w");
    std::fprintf(meta, "aminoCount %zu\nNtr %d\nstride %d\nmax_pairs %d\n", N, gsop.Ntr, stride, hc_pairs.max_pairs);
    std::fclose(meta);
    const bool timing = dumps.empty();
    auto t0 = std::chrono::steady_clock::now();
    for (long done = 0; done < total;) {
        for (int u = 0; u < updatersCount; u++) updaters[u]->update();
        if (done == 0) {
            cudaDeviceSynchronize();
            t0 = std::chrono::steady_clock::now();
        }
        for (int j = 0; j < stride && done < total; j++) {
            for (int p = 0; p < potentialsCount; p++) potentials[p]->compute();
            if (done == 0 && !timing) dump(dir, "forces", 0, gsop.d_forces, N * sizeof(float4));
            integrator->integrate();
            checkCUDAError();
            done++;
            if (dumps.count(done)) {
                cudaDeviceSynchronize();
                dump(dir, "coords", done, gsop.d_coord, N * sizeof(float4));
                dump(dir, "seeds", done, ht.d_seeds, N * sizeof(uint4));
                dump(dir, "T", done, gsop.d_T, N * sizeof(float));
                dump(dir, "paircount", done, hc_pairs.d_pairsCount, N * sizeof(int));
                dump(dir, "pairs", done, hc_pairs.d_pairs, (size_t)hc_pairs.max_pairs * N * sizeof(int));
                if (configreader::hasParameter("indentation") && configreader::getYesNoParameter("indentation")) dump(dir, "tip", done, &hc_indentation, sizeof(IndentView), true);
            }
        }
        gsop.step += stride;
    }
    cudaDeviceSynchronize();
    checkCUDAError();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("ref_gpu: %ld steps, %zu beads, stride %d\n", total, N, stride);
    if (timing) std::printf("ref_gpu_time %.6f %.6e\n", secs, (double)N * total / secs);
    return 0;
}
