// ref_host_harness.cpp — drives the reference's own host code (compiled from
// the SOP-GPU source tree by oracle/build_ref.sh) to produce golden vectors
// for the oracle.  TEST INFRASTRUCTURE ONLY.
//
//   ref_host seeds <seed> <count>     generateSeeds() over ran2 (ht.cu:40-56)
//   ref_host config <file> <key> <type>  configreader parse (configreader.cpp)
//   ref_host top <file.top>           SOP::load (topio.cpp:36-80)
//   ref_host coords <file.top> <file.pdb>   readCoord (pdbio.cpp:292-337)
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "Integrators/ran2.h"
#include "IO/configreader.h"
#include "IO/topio.h"
#include "IO/pdbio.h"

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    std::string mode = argv[1];
    if (mode == "seeds" && argc == 4) {
        // The loop body of generateSeeds (src/Integrators/ht.cu:40-56); ht.cu
        // itself is device code and cannot be compiled for the host.
        int seed = atoi(argv[2]);
        long count = atol(argv[3]);
        for (long i = 0; i < count; i++) {
            unsigned v[4];
            for (int c = 0; c < 4; c++) {
                do { v[c] = (unsigned)(ran2(&seed) * UINT_MAX); } while (v[c] < 128);
            }
            printf("%u %u %u %u\n", v[0], v[1], v[2], v[3]);
        }
        return 0;
    }
    if (mode == "config" && argc >= 5) {
        configreader::parseParametersFile(argv[2]);
        for (int k = 3; k + 1 < argc; k += 2) {
            const char* key = argv[k];
            std::string type = argv[k + 1];
            if (!configreader::hasParameter(key)) { printf("%s\tMISSING\n", key); continue; }
            if (type == "str") printf("%s\t%s\n", key, configreader::getMaskedParameter(key).c_str());
            else if (type == "bool") printf("%s\t%d\n", key, (int)configreader::getYesNoParameter(key));
            else if (type == "int") printf("%s\t%d\n", key, configreader::getParameterAs<int>(key));
            else if (type == "float") printf("%s\t%.9g\n", key, configreader::getParameterAs<float>(key));
            else if (type == "ints") {
                std::vector<int> v = configreader::getArrayParameter<int>(key);
                printf("%s\t", key);
                for (size_t q = 0; q < v.size(); q++) printf("%s%d", q ? " " : "", v[q]);
                printf("\n");
            } else if (type == "float3") {
                float3 f = configreader::getFloat3Parameter(key);
                printf("%s\t%.9g %.9g %.9g\n", key, f.x, f.y, f.z);
            }
        }
        return 0;
    }
    if ((mode == "top" && argc == 3) || (mode == "coords" && argc == 4)) {
        SOP sop;
        sop.load(argv[2]);
        if (mode == "coords") {
            readCoord(argv[3], sop);
            for (size_t i = 0; i < sop.aminos.size(); i++)
                printf("%.9g %.9g %.9g\n", (float)sop.aminos[i].x, (float)sop.aminos[i].y, (float)sop.aminos[i].z);
            return 0;
        }
        printf("atoms %zu\n", sop.aminos.size());
        for (size_t i = 0; i < sop.bonds.size(); i++)
            printf("bond %d %d %.9g\n", sop.bonds[i].i, sop.bonds[i].j, sop.bonds[i].r0);
        for (size_t i = 0; i < sop.natives.size(); i++)
            printf("native %d %d %.9g %.9g\n", sop.natives[i].i, sop.natives[i].j, sop.natives[i].r0, sop.natives[i].eh);
        for (size_t i = 0; i < sop.pairs.size(); i++)
            printf("pair %d %d\n", sop.pairs[i].i, sop.pairs[i].j);
        return 0;
    }
    fprintf(stderr, "usage error\n");
    return 2;
}
