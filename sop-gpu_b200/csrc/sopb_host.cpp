// sopb_host.cpp — host utilities of the C ABI that need no GPU: default
// parameters, status strings and Hybrid Taus seeding.
#include <climits>
#include <cstring>

#include "../../include/sopb.h"

extern "C" int sopb_version(void) { return SOPB_ABI_VERSION; }

extern "C" const char* sopb_status_string(int status) {
    switch (status) {
    case SOPB_OK: return "ok";
    case SOPB_ERR_INVALID: return "invalid argument or configuration";
    case SOPB_ERR_CAPACITY: return "neighbour list capacity exceeded (raise max_pairs / max_possiblePairs)";
    case SOPB_ERR_NONFINITE: return "non-finite coordinates";
    case SOPB_ERR_CUDA: return "CUDA runtime error";
    case SOPB_ERR_TIMEOUT: return "bounded device wait timed out";
    case SOPB_ERR_NOMEM: return "device memory exhausted";
    case SOPB_ERR_UNSUPPORTED: return "unsupported feature combination";
    case SOPB_ERR_HI: return "hydrodynamic tensor check failed (TEA epsilon/beta)";
    case SOPB_ERR_NODEVICE: return "no CUDA device available";
    default: return "unknown status";
    }
}

// Defaults of the PARAMETER() declarations: src/Integrators/langevin.h:12-23,
// src/Potentials/covalent.h:12-14, pairs.h:12-15, native.h:11-12,
// src/Updaters/pairlist.h:12-14, possiblepairlist.h:12-13, src/gsop.h:34,
// src/Potentials/pulling.h:15-26, indentation.h:12-47, pulling_plane.h:12-27,
// src/Integrators/bdhitea.h:15-21.  Frequencies that default to nav are 0.
extern "C" void sopb_default_params(sopb_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->zeta = 50.0f;
    p->temperature = 0.6f;
    p->kspring_cov = 20.0f;
    p->R_limit = 2.0f;
    p->R_limit_bond = 8.0f;
    p->a = 3.8f;
    p->el = 1.0f;
    p->pairs_cutoff = 20.0f;
    p->pairlist_cutoff = 20.0f;
    p->pairs_freq = 1000;
    p->pairs_threshold = 200.0f;
    p->possiblepairs_freq = 100000;
    p->max_pairs = 512;
    p->max_possiblePairs = 4096;
    p->nav = 1000;
    p->k_trans = 0.05f;
    p->pull_direction = SOPB_PULL_END_TO_END;
    p->indentationTipSigma = 1.0f;
    p->indentationTipEl = 1.0f;
    p->indentationTipA = 0.0f;
    p->indentationTipB = 1.0f;
    p->indentationSurfSigma = 1.0f;
    p->indentationSurfEl = 1.0f;
    p->indentationSurfA = 0.0f;
    p->indentationSurfB = 1.0f;
    p->indentationTipZeta = 5000.0f;
    p->indentationRetractionStep = -1;
    p->indentationSurfaceSize = 51;
    p->indentationSurfaceStep = 1.4f;
    p->indentationPairsCutoff = 40.0f;
    p->pullingPlaneKs = 0.05f;
    p->pullingPlaneKsCant = 0.05f;
    p->pullingPlaneZeta = 200.0f;
    p->hi_a = 1.8f;
    p->hi_capricious = 1;
    p->hi_unlisted = 1;
    p->hi_epsmax = 999.0f;
    p->hi_b_mode = SOPB_HI_B_CHOLESKY;
    p->hi_refresh = 1;
}

namespace {
// ran2: L'Ecuyer's two-generator combined LCG (moduli 2147483563 and
// 2147483399) with a 32-entry Bays-Durham shuffle, the published Numerical
// Recipes form the reference uses (src/Integrators/ran2.cpp:51-89).  The
// shuffle state starts as a fresh process has it: second generator at
// 123456789, table and output register zero; a non-positive seed loads the
// table after eight warm-up draws.
struct Ran2 {
    int32_t idum, idum2 = 123456789, iy = 0, iv[32] = {0};
    explicit Ran2(int32_t seed) : idum(seed) {}
    static int32_t lcg(int32_t x, int32_t a, int32_t q, int32_t r, int32_t m) {
        const int32_t k = x / q;
        x = a * (x - k * q) - k * r;
        return x < 0 ? x + m : x;
    }
    double next() {
        const int32_t m1 = 2147483563, m2 = 2147483399;
        if (idum <= 0) {
            idum = (-idum < 1) ? 1 : -idum;
            idum2 = idum;
            for (int j = 39; j >= 0; --j) {
                idum = lcg(idum, 40014, 53668, 12211, m1);
                if (j < 32) iv[j] = idum;
            }
            iy = iv[0];
        }
        idum = lcg(idum, 40014, 53668, 12211, m1);
        idum2 = lcg(idum2, 40692, 52774, 3791, m2);
        const int j = iy / (1 + (m1 - 1) / 32);
        iy = iv[j] - idum2;
        iv[j] = idum;
        if (iy < 1) iy += m1 - 1;
        const double t = (1.0 / m1) * iy;
        const double rnmx = 1.0 - 1.2e-7;
        return t > rnmx ? rnmx : t;
    }
};
}  // namespace

// generateSeeds (src/Integrators/ht.cu:40-56): every state word is
// (unsigned)(ran2 * UINT_MAX), redrawn while below 128 (Tausworthe steps
// need seeds above their shift widths).
extern "C" int sopb_generate_seeds(int32_t seed, int64_t count, uint32_t* out4) {
    if (count < 0 || (count > 0 && !out4)) return SOPB_ERR_INVALID;
    Ran2 r(seed);
    for (int64_t i = 0; i < 4 * count; ++i) {
        uint32_t v;
        do {
            v = (uint32_t)(r.next() * (double)UINT_MAX);
        } while (v < 128u);
        out4[i] = v;
    }
    return SOPB_OK;
}
