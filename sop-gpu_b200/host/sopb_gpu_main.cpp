// sopb-gpu — command-line driver with the reference's usage:
//   sopb-gpu <config> [key=value ...]
// reads the config file, topology and coordinates, runs the reference's
// number of steps on the GPU and writes each run's final PDB
// (src/sop-gpu.cpp:18-65).  Library errors end the program with their status
// text instead of DIE()'s backtrace.
//   sopb-gpu --dump-config <config> <key> <str|bool|int|float|ints|float3> ...
// prints the parsed values (used to check the parser against the
// reference's own).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>

#include "sopb_mirror.h"

using namespace sopb_host;

static int dump_config(int argc, char** argv) {
    Config cfg(argv[2]);
    for (int k = 3; k + 1 < argc; k += 2) {
        const std::string key = argv[k], type = argv[k + 1];
        if (!cfg.has(key)) { std::printf("%s\tMISSING\n", key.c_str()); continue; }
        if (type == "str") std::printf("%s\t%s\n", key.c_str(), cfg.str(key).c_str());
        else if (type == "bool") std::printf("%s\t%d\n", key.c_str(), (int)cfg.boolean(key));
        else if (type == "int") std::printf("%s\t%lld\n", key.c_str(), (long long)cfg.integer(key));
        else if (type == "float") std::printf("%s\t%.9g\n", key.c_str(), cfg.real(key));
        else if (type == "ints") {
            std::printf("%s\t", key.c_str());
            const auto v = cfg.ints(key);
            for (size_t q = 0; q < v.size(); ++q) std::printf("%s%d", q ? " " : "", v[q]);
            std::printf("\n");
        } else if (type == "float3") {
            float f[3];
            cfg.float3(key, f);
            std::printf("%s\t%.9g %.9g %.9g\n", key.c_str(), f[0], f[1], f[2]);
        }
    }
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <config> [key=value ...]\n", argv[0]);
        return 2;
    }
    try {
        if (std::strcmp(argv[1], "--dump-config") == 0 && argc >= 3) return dump_config(argc, argv);
        Config cfg(argv[1]);
        for (int k = 2; k < argc; ++k) {          // argv overrides (configreader.cpp:42-57)
            const char* eq = std::strchr(argv[k], '=');
            if (eq) cfg.set(std::string(argv[k], eq - argv[k]), std::string(eq + 1));
        }
        Simulation sim(cfg);
        const int64_t total = (sim.numsteps / sim.stride + 1) * sim.stride;
        std::printf("Starting %d runs (%lld steps, stride %d, %d beads each).\n", sim.ntr, (long long)total,
                    sim.stride, sim.top.natoms);
        const auto t0 = std::chrono::steady_clock::now();
        sim.runGPU();
        const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("Done: %.3f s, %.4g bead-steps/s.\n", dt, (double)sim.ntr * sim.top.natoms * total / dt);
        return 0;
    } catch (const Error& e) {
        std::fprintf(stderr, "sopb-gpu: %s\n", e.what());
        return e.code ? e.code : 1;
    }
}
