// sopb_api.cu — the C ABI: device context, job construction and the batched
// launch of the resident Langevin step kernel.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/sopb.h"
#include "sopb_device.cuh"
#include "sopb_resident.cuh"
#include "sopb_grid.cuh"
#include "sopb_hi.cuh"
#include "sopb_chol.cuh"
#include "sopb_obs.cuh"

using namespace sopb;

namespace {

constexpr int kJobSlots = 16384;
constexpr int kSideStreams = 4;   // resident launch classes run side by side
constexpr int kGridStreams = 8;   // grid-path jobs run side by side
constexpr int64_t kDefaultBeadCapacity = int64_t(1) << 22;

// First-fit allocator over index ranges [0, cap).
struct RangeAlloc {
    std::map<int64_t, int64_t> free_;  // start -> length
    void init(int64_t cap) { free_.clear(); free_[0] = cap; }
    bool alloc(int64_t n, int64_t* out) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                *out = it->first;
                const int64_t rest = it->second - n, start = it->first + n;
                free_.erase(it);
                if (rest) free_[start] = rest;
                return true;
            }
        }
        return false;
    }
    void release(int64_t start, int64_t n) {
        auto it = free_.emplace(start, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

inline size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Default skin of the near list (A): a Verlet rebuild filters the possible
// pairs within pairlist_cutoff + skin instead of all of them.
constexpr float kNearSkin = 4.0f;

inline float near_skin(const sopb_params& p) { return p.verlet_skin == 0.0f ? kNearSkin : p.verlet_skin; }

// Near-row capacity of a grid job (int32 rows): twice the Verlet rows, at
// most the possible rows.  0: no near list.
inline int64_t grid_cap_nr(const sopb_params& p, int64_t cap_pp, int64_t cap_pl) {
    return near_skin(p) > 0.02f ? std::max<int64_t>(1, std::min<int64_t>(cap_pp, 2 * cap_pl)) : 0;
}

// Default CTAs per SM that the O(N^2) TEA and D F sums are sliced for (the
// fastest of 2..32 for TEA and exact HI at 4000 beads on B200).
constexpr int32_t kHiCtasPerSm = 8;

// Shape policy of the resident kernel (see launch_shape).
struct ShapePolicy {
    int32_t lpb = 4;
    float beads_per_group = 1.0f;
    int32_t max_block = 1024;
    // grid-path HI jobs: outer-panel width of the exact-HI factorisation (tile
    // columns) and the CTAs per SM the O(N^2) sums are sliced for
    int32_t chol_panel_tiles = kCholPanelTiles;
    int32_t hi_ctas_per_sm = kHiCtasPerSm;
};

struct LaunchClass {
    int block = 0;
    int32_t max_n = 0;
    size_t smem = 0;
    std::vector<int32_t> ids;
};

// The last resident launch plan ordered on each stream of a context: its
// jobs and step counts, classes and the id/step table it uploaded.  A run
// of the same jobs with the same counts on the same stream, with no job
// created or destroyed since, reuses the plan and the device table (no
// other run writes that stream's table in between) instead of grouping and
// uploading again.
struct RunPlan {
    uint64_t generation = 0;
    std::vector<sopb_job*> jobs;
    std::vector<int64_t> steps;
    std::vector<LaunchClass> cls;
    std::vector<size_t> off;
};

}  // namespace

struct sopb_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int sm_count = 0;
    uint64_t generation = 0;      // bumped by every job creation and destruction
    std::map<cudaStream_t, RunPlan> plans;   // the last resident launch plan per stream
    int64_t bead_cap = 0;
    float4* x = nullptr;
    float4* xalt = nullptr;
    uint4* seeds = nullptr;
    float* T = nullptr;
    float4* tipF = nullptr;
    uint8_t* flags = nullptr;
    RangeAlloc beads;
    JobDev* d_jobs = nullptr;
    // job-slot tables of resident launches, one per stream runs are ordered on
    struct Ids {
        int32_t* d = nullptr;
        int64_t cap = 0;
    };
    std::map<cudaStream_t, Ids> ids;
    // bead ranges and slots of destroyed jobs, released once the work that
    // used them has finished
    struct Deferred {
        cudaEvent_t done;
        int64_t b0;
        int32_t n;
        int slot;
    };
    std::vector<Deferred> deferred;
    cudaStream_t upload = nullptr;    // job set-up copies
    cudaStream_t io = nullptr;        // reads and writes of single jobs
    float4* d_scratch4 = nullptr;
    int64_t scratch4_cap = 0;
    std::vector<sopb_job*> slots;
    std::vector<int> free_slots;
    // fork/join streams of a run, one set per stream priority so a run's
    // side work keeps the priority of the stream it was ordered on
    struct Fork {
        cudaStream_t side[kSideStreams] = {};
        cudaEvent_t join[kSideStreams] = {};
        cudaStream_t gside[kGridStreams] = {};
        cudaEvent_t gjoin[kGridStreams] = {};
        cudaEvent_t fork = nullptr;
    };
    std::map<int, Fork> forks;
    cudaStream_t capture = nullptr;   // CUDA graph capture of grid-path chunks
    int32_t last_error = SOPB_OK;
    int smem_dyn_max = 1 << 30;   // dynamic shared memory available to the resident kernel
    int smem_per_sm = 0;          // shared memory of one SM
    int smem_reserved = 0;        // shared memory the runtime reserves per CTA
    int smem_static[5] = {};      // static shared memory of k_resident_steps<64..1024>
    ShapePolicy policy;
};

struct sopb_job {
    sopb_context* ctx = nullptr;
    cudaStream_t st = nullptr;         // the stream the job's last work was ordered on
    cudaEvent_t ev = nullptr;          // recorded after every piece of the job's work
    int slot = -1;
    int64_t b0 = 0;
    int32_t n = 0;
    JobDev h{};
    void* dmem = nullptr;
    size_t dbytes = 0;
    // grid path
    GridAux aux{};
    void* amem = nullptr;
    int64_t host_step = 0;             // the device step counter, tracked on the host
    // one stride chunk (updaters + stride steps) per set of updaters due at
    // its first step (kDue* bits)
    std::map<int, cudaGraphExec_t> chunks;
    int bead_blocks = 1;               // CTAs of the per-bead grid kernels
    // exact HI: streams of the factorisation, two per stream priority level
    // (made at job creation): the single-tile chain runs two levels above
    // the caller's stream, the rest of each tile column one level above it,
    // the bulk trailing updates at the caller's level
    static constexpr int kPrioLevels = 8;
    cudaStream_t prio_st[kPrioLevels] = {};
    cudaStream_t mid_st[kPrioLevels] = {};
    bool hi_streams = false;
    cudaEvent_t la_join = nullptr, hp_fork = nullptr, hp_join = nullptr;
    // hand-offs between the chain and the tile-column stream: rings of four
    // (factor done, first tile solved, column updated, rest solved), then
    // the next-panel updates and the column stream's join
    static constexpr int kLkRing = 4;
    cudaEvent_t lk_ev[4 * kLkRing + 3] = {};
    int jsplit = 1;                    // j slices of the O(N^2) HI sums
    int chol_w = kCholPanelTiles;      // exact HI: outer-panel width of the factorisation, tile columns
    CUtensorMap tmap_ten{};            // exact HI: TMA maps of the tensor, of the diagonal tiles'
    CUtensorMap tmap_linv{};           //   inverses and of the TF32 hi and lo planes of the solved
    CUtensorMap tmap_phi{};            //   tiles (128 x 32 FP32 boxes, 128-byte swizzle)
    CUtensorMap tmap_plo{};
    uint32_t log_tail = 0;             // event-log rows drained so far
    bool ev_lazy = false;              // ev not yet recorded after the work on st (see job_ev)
};

#define CUDA_TRY(call)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            std::fprintf(stderr, "sopb: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), \
                         __FILE__, __LINE__);                                                  \
            return e_ == cudaErrorMemoryAllocation ? SOPB_ERR_NOMEM : SOPB_ERR_CUDA;           \
        }                                                                                      \
    } while (0)

#define SOPB_TRY(call)           \
    do {                         \
        const int r_ = (call);   \
        if (r_) return r_;       \
    } while (0)

namespace {

// Streams and events of an exact-HI job's factorisation.
void hi_streams_destroy(sopb_job* j) {
    for (cudaStream_t q : j->prio_st) if (q) cudaStreamDestroy(q);
    for (cudaStream_t q : j->mid_st) if (q) cudaStreamDestroy(q);
    for (cudaEvent_t e : {j->la_join, j->hp_fork, j->hp_join}) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : j->lk_ev) if (e) cudaEventDestroy(e);
}

// Opt the resident kernel in to the largest dynamic shared memory the device
// allows next to the kernel's static shared memory.
template <int B>
int set_smem_attr(int device, int* dyn_out, int* static_out) {
    int optin = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    cudaFuncAttributes fa;
    CUDA_TRY(cudaFuncGetAttributes(&fa, k_resident_steps<B>));
    const int dyn = optin - (int)fa.sharedSizeBytes;
    if (dyn < kMaxResidentBeads * kResidentSmemPerBead) return SOPB_ERR_UNSUPPORTED;
    CUDA_TRY(cudaFuncSetAttribute(k_resident_steps<B>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    if (dyn < *dyn_out) *dyn_out = dyn;
    *static_out = (int)fa.sharedSizeBytes;
    return SOPB_OK;
}

int block_index(int block) { return block == 64 ? 0 : block == 128 ? 1 : block == 256 ? 2 : block == 512 ? 3 : 4; }

// Smallest float t with sqrtf(t) >= cut: for every float r2,
// sqrtf(r2) < cut exactly when r2 < t, because a correctly rounded square
// root is monotonic (the host's sqrtf is the IEEE operation, as the
// device's __fsqrt_rn).  The list builders compare r^2 against t.
float sqrt_threshold(float cut) {
    if (!(cut > 0.0f)) return 0.0f;                         // nothing is closer than cut <= 0 (or NaN)
    if (std::isinf(cut)) return cut;
    float t = cut * cut;
    while (t > 0.0f && std::sqrt(std::nextafter(t, 0.0f)) >= cut) t = std::nextafter(t, 0.0f);
    while (std::sqrt(t) < cut) t = std::nextafter(t, INFINITY);
    return t;
}

// Lanes per bead and CTA size of a job.  A function of the job and of the
// context's shape policy only (never of the batch it runs in), so a job's
// arithmetic is identical alone and in any mix.  The CTA holds about
// n / beads_per_group lane groups of `lpb` lanes (a power of two, 64..max_block
// threads): lane groups take beads dynamically, so several beads per group
// even out the differing list lengths.  sopb_context_set_shape_policy sets
// it (the autotuner's knob).
void launch_shape(const ShapePolicy& pol, int32_t n, int32_t lpb_req, int32_t* lpb, int32_t* block) {
    int32_t l = lpb_req > 0 ? lpb_req : pol.lpb;
    int32_t p2 = 1;
    while (p2 < l && p2 < 32) p2 <<= 1;
    l = p2;
    const int32_t maxb = pol.max_block >= 64 && pol.max_block <= 1024 ? pol.max_block : 1024;
    const float bpg = pol.beads_per_group > 0.0f ? pol.beads_per_group : 1.0f;
    const float want = std::ceil((float)n / bpg) * (float)l;
    int32_t b = 64;
    while (b < maxb && (float)b < want) b <<= 1;
    while (b < 1024 && b < l) b <<= 1;
    *lpb = l;
    *block = b;
}

#define SOPB_BLOCK_SWITCH(block, LAUNCH) \
    switch (block) {                      \
    case 64: LAUNCH(64); break;           \
    case 128: LAUNCH(128); break;         \
    case 256: LAUNCH(256); break;         \
    case 512: LAUNCH(512); break;         \
    case 1024: LAUNCH(1024); break;       \
    default: return SOPB_ERR_INVALID;     \
    }

int launch_resident(int block, int grid, size_t smem, cudaStream_t st, JobDev* jobs, const int32_t* ids,
                    const int64_t* steps) {
#define L_RES(B) k_resident_steps<B><<<grid, B, smem, st>>>(jobs, ids, steps)
    SOPB_BLOCK_SWITCH(block, L_RES)
#undef L_RES
    CUDA_TRY(cudaGetLastError());
    return SOPB_OK;
}

int launch_forces(int block, int grid, cudaStream_t st, const JobDev* jobs, const int32_t* ids, float4* out) {
#define L_FRC(B) k_forces_only<B><<<grid, B, 0, st>>>(jobs, ids, out)
    SOPB_BLOCK_SWITCH(block, L_FRC)
#undef L_FRC
    CUDA_TRY(cudaGetLastError());
    return SOPB_OK;
}

int launch_rebuild(int block, int grid, cudaStream_t st, JobDev* jobs, const int32_t* ids, int possible, int verlet) {
#define L_REB(B) k_rebuild_lists<B><<<grid, B, 0, st>>>(jobs, ids, possible, verlet)
    SOPB_BLOCK_SWITCH(block, L_REB)
#undef L_REB
    CUDA_TRY(cudaGetLastError());
    return SOPB_OK;
}

// The launch table of resident launches ordered on `st`: `need` job slots
// (int32) and, after them, as many step counts (int64).  Stream-ordered, so
// a table is reused only after the launches that read it.
int ensure_ids(sopb_context* c, cudaStream_t st, int64_t need, int32_t** out, int64_t** steps = nullptr) {
    sopb_context::Ids& t = c->ids[st];
    if (need > t.cap) {
        if (t.d) cudaFreeAsync(t.d, st);
        const int64_t cap = (std::max<int64_t>(need, 1024) + 1) & ~int64_t(1);   // even: the steps stay 8-B aligned
        CUDA_TRY(cudaMallocAsync((void**)&t.d, cap * (sizeof(int32_t) + sizeof(int64_t)), st));
        t.cap = cap;
    }
    *out = t.d;
    if (steps) *steps = reinterpret_cast<int64_t*>(t.d + t.cap);
    return SOPB_OK;
}

// The fork/join streams for a run ordered on `st`, at st's priority.
int fork_set(sopb_context* c, cudaStream_t st, sopb_context::Fork** out) {
    int prio = 0;
    CUDA_TRY(cudaStreamGetPriority(st, &prio));
    auto it = c->forks.find(prio);
    if (it == c->forks.end()) {
        sopb_context::Fork f;
        for (int k = 0; k < kSideStreams; ++k) {
            CUDA_TRY(cudaStreamCreateWithPriority(&f.side[k], cudaStreamNonBlocking, prio));
            CUDA_TRY(cudaEventCreateWithFlags(&f.join[k], cudaEventDisableTiming));
        }
        for (int k = 0; k < kGridStreams; ++k) {
            CUDA_TRY(cudaStreamCreateWithPriority(&f.gside[k], cudaStreamNonBlocking, prio));
            CUDA_TRY(cudaEventCreateWithFlags(&f.gjoin[k], cudaEventDisableTiming));
        }
        CUDA_TRY(cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming));
        it = c->forks.emplace(prio, f).first;
    }
    *out = &it->second;
    return SOPB_OK;
}

// Releases the bead ranges and slots of destroyed jobs whose last work has
// finished (all of them when `wait`).
void reclaim(sopb_context* c, bool wait) {
    std::vector<sopb_context::Deferred> keep;
    for (auto& d : c->deferred) {
        if (wait) cudaEventSynchronize(d.done);
        if (cudaEventQuery(d.done) == cudaSuccess) {
            cudaEventDestroy(d.done);
            c->beads.release(d.b0, d.n);
            c->free_slots.push_back(d.slot);
        } else {
            cudaGetLastError();
            keep.push_back(d);
        }
    }
    c->deferred.swap(keep);
}

// The io stream after the job's last work (its work on other streams after
// that is unrelated); `modify`: the job's next work comes after this io.
// A job's event, recorded now on the job's stream if its last work left it
// unrecorded.  Batch operations on one stream (a run, a bulk copy) mark their
// jobs instead of recording an event per job: the event is recorded when
// something first has to wait for it, and then covers everything ordered on
// that stream so far (the job's work included).
int job_ev(sopb_job* j) {
    if (j->ev_lazy) {
        CUDA_TRY(cudaEventRecord(j->ev, j->st));
        j->ev_lazy = false;
    }
    return SOPB_OK;
}

int io_begin(sopb_job* j) {
    SOPB_TRY(job_ev(j));
    CUDA_TRY(cudaStreamWaitEvent(j->ctx->io, j->ev, 0));
    return SOPB_OK;
}
int io_end(sopb_job* j, bool modify) {
    sopb_context* c = j->ctx;
    if (modify) {
        CUDA_TRY(cudaEventRecord(j->ev, c->io));
        j->st = c->io;
        j->ev_lazy = false;
    }
    CUDA_TRY(cudaStreamSynchronize(c->io));
    return SOPB_OK;
}

int read_slot(sopb_job* j) {
    SOPB_TRY(job_ev(j));
    CUDA_TRY(cudaEventSynchronize(j->ev));
    CUDA_TRY(cudaMemcpy(&j->h, &j->ctx->d_jobs[j->slot], sizeof(JobDev), cudaMemcpyDeviceToHost));
    return SOPB_OK;
}

float f3norm(const float* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

// Updater period: the minimum over nav and the frequencies of the updaters
// that exist for this job (src/gsop.cu:117-122).  Output updaters are not
// part of the library; a caller that mirrors the reference's outputtiming
// and dcdfreq passes the full minimum in params.stride.
int32_t compute_stride(const sopb_params& p) {
    if (p.stride > 0) return p.stride;
    int32_t s = p.nav;
    auto mn = [&](int32_t v) { if (v > 0 && v < s) s = v; };
    mn(p.pairs_freq);
    mn(p.possiblepairs_freq);
    if (p.pulling && p.deltax != 0.0f) mn(p.pullFreq > 0 ? p.pullFreq : p.nav);
    if (p.heating) mn(p.tempFreq);
    if (p.hi_on && !p.hi_exact) mn(p.hi_epsilon_freq);
    if (p.hi_on && p.hi_exact && p.hi_refresh > 1) mn(p.hi_refresh);   // the factor refresh is an updater
    if (p.pullingPlane) mn(p.pullingPlaneUpdateFreq > 0 ? p.pullingPlaneUpdateFreq : p.nav);
    return s;
}

}  // namespace

extern "C" int sopb_context_create(int32_t device, void* stream, sopb_context** out) {
    if (!out) return SOPB_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return SOPB_ERR_NODEVICE;
    }
    if (device < 0 || device >= ndev) return SOPB_ERR_INVALID;
    CUDA_TRY(cudaSetDevice(device));
    sopb_context* c = new (std::nothrow) sopb_context();
    if (!c) return SOPB_ERR_NOMEM;
    c->device = device;
    CUDA_TRY(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    const char* env = std::getenv("SOPB_BEAD_CAPACITY");
    c->bead_cap = env ? std::atoll(env) : kDefaultBeadCapacity;
    if (c->bead_cap < 1024) c->bead_cap = 1024;
    const int64_t B = c->bead_cap;
    CUDA_TRY(cudaMalloc((void**)&c->x, B * sizeof(float4)));
    CUDA_TRY(cudaMalloc((void**)&c->xalt, B * sizeof(float4)));
    CUDA_TRY(cudaMalloc((void**)&c->seeds, B * sizeof(uint4)));
    CUDA_TRY(cudaMalloc((void**)&c->T, B * sizeof(float)));
    CUDA_TRY(cudaMalloc((void**)&c->tipF, B * sizeof(float4)));
    CUDA_TRY(cudaMalloc((void**)&c->flags, B));
    CUDA_TRY(cudaMalloc((void**)&c->d_jobs, kJobSlots * sizeof(JobDev)));
    CUDA_TRY(cudaMemset(c->d_jobs, 0, kJobSlots * sizeof(JobDev)));
    c->beads.init(B);
    c->slots.assign(kJobSlots, nullptr);
    for (int s = kJobSlots - 1; s >= 0; --s) c->free_slots.push_back(s);
    CUDA_TRY(cudaStreamCreateWithFlags(&c->capture, cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamCreateWithFlags(&c->upload, cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamCreateWithFlags(&c->io, cudaStreamNonBlocking));
    int rc;
    int* dm = &c->smem_dyn_max;
    int* ss = c->smem_static;
    if ((rc = set_smem_attr<64>(device, dm, &ss[0])) || (rc = set_smem_attr<128>(device, dm, &ss[1])) ||
        (rc = set_smem_attr<256>(device, dm, &ss[2])) || (rc = set_smem_attr<512>(device, dm, &ss[3])) ||
        (rc = set_smem_attr<1024>(device, dm, &ss[4])))
        return rc;
    CUDA_TRY(cudaDeviceGetAttribute(&c->smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device));
    CUDA_TRY(cudaFuncSetAttribute(k_chol_potrf64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPotrfSmem));
    CUDA_TRY(cudaFuncSetAttribute(k_chol_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    CUDA_TRY(cudaFuncSetAttribute(k_chol_factor_panels, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmallSmem));
    CUDA_TRY(cudaFuncSetAttribute(k_chol_apply_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, kCholMaxBeads * 12));
    CUDA_TRY(cudaDeviceGetAttribute(&c->smem_reserved, cudaDevAttrReservedSharedMemoryPerBlock, device));
    *out = c;
    return SOPB_OK;
}

extern "C" int sopb_context_destroy(sopb_context* c) {
    if (!c) return SOPB_ERR_INVALID;
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    reclaim(c, true);
    for (sopb_job* j : c->slots)
        if (j) {
            for (auto& g : j->chunks) if (g.second) cudaGraphExecDestroy(g.second);
            if (j->hi_streams) hi_streams_destroy(j);
            if (j->amem) cudaFree(j->amem);
            cudaFree(j->dmem);
            cudaEventDestroy(j->ev);
            delete j;
        }
    cudaFree(c->x);
    cudaFree(c->xalt);
    cudaFree(c->seeds);
    cudaFree(c->T);
    cudaFree(c->tipF);
    cudaFree(c->flags);
    cudaFree(c->d_jobs);
    for (auto& kv : c->ids)
        if (kv.second.d) cudaFree(kv.second.d);
    if (c->d_scratch4) cudaFree(c->d_scratch4);
    for (auto& kv : c->forks) {
        sopb_context::Fork& f = kv.second;
        for (int k = 0; k < kSideStreams; ++k) {
            cudaStreamDestroy(f.side[k]);
            cudaEventDestroy(f.join[k]);
        }
        for (int k = 0; k < kGridStreams; ++k) {
            cudaStreamDestroy(f.gside[k]);
            cudaEventDestroy(f.gjoin[k]);
        }
        cudaEventDestroy(f.fork);
    }
    cudaStreamDestroy(c->capture);
    cudaStreamDestroy(c->upload);
    cudaStreamDestroy(c->io);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return SOPB_OK;
}

extern "C" int sopb_context_set_shape_policy(sopb_context* c, int32_t lanes_per_bead, float beads_per_group,
                                             int32_t max_block) {
    if (!c || lanes_per_bead < 1 || lanes_per_bead > 32 || max_block < 64 || max_block > 1024) return SOPB_ERR_INVALID;
    c->policy.lpb = lanes_per_bead;
    c->policy.beads_per_group = beads_per_group;
    c->policy.max_block = max_block;
    return SOPB_OK;
}

extern "C" int sopb_context_set_hi_policy(sopb_context* c, int32_t chol_panel_tiles, int32_t hi_ctas_per_sm) {
    if (!c || chol_panel_tiles < 1 || chol_panel_tiles > 64 || hi_ctas_per_sm < 1 || hi_ctas_per_sm > 64)
        return SOPB_ERR_INVALID;
    c->policy.chol_panel_tiles = chol_panel_tiles;
    c->policy.hi_ctas_per_sm = hi_ctas_per_sm;
    return SOPB_OK;
}

extern "C" int sopb_context_sync(sopb_context* c) {
    if (!c) return SOPB_ERR_INVALID;
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (sopb_job* j : c->slots)
        if (j) {
            SOPB_TRY(job_ev(j));
            CUDA_TRY(cudaEventSynchronize(j->ev));
        }
    return SOPB_OK;
}

namespace {

struct HostMaps {
    std::vector<int32_t> cov_off, cov_j, nat_off, nat_j;
    std::vector<float> cov_r0;
    std::vector<float2> nat_par;
};

int validate_desc(const sopb_job_desc* d) {
    if (!d || d->n <= 0 || !d->xyz) return SOPB_ERR_INVALID;
    const int32_t n = d->n;
    const sopb_params& p = d->params;
    if (p.timestep <= 0.0f || p.zeta <= 0.0f) return SOPB_ERR_INVALID;
    if (p.nav <= 0 || p.pairs_freq <= 0 || p.possiblepairs_freq <= 0) return SOPB_ERR_INVALID;
    if (p.heating && p.tempFreq <= 0) return SOPB_ERR_INVALID;
    if (p.log_rows < 0 || p.log_rows > (1 << 24) || (p.log_rows & (p.log_rows - 1))) return SOPB_ERR_INVALID;
    if (!std::isfinite(p.verlet_skin) || p.verlet_skin > 1000.0f) return SOPB_ERR_INVALID;
    if (d->nbonds < 0 || d->nnatives < 0 || d->nfixed < 0 || d->npulled < 0) return SOPB_ERR_INVALID;
    if ((d->nbonds && (!d->bonds || !d->bonds_r0)) || (d->nnatives && (!d->natives || !d->natives_r0 || !d->natives_eh)))
        return SOPB_ERR_INVALID;
    for (int32_t k = 0; k < 2 * d->nbonds; ++k)
        if (d->bonds[k] < 0 || d->bonds[k] >= n) return SOPB_ERR_INVALID;
    for (int32_t k = 0; k < 2 * d->nnatives; ++k)
        if (d->natives[k] < 0 || d->natives[k] >= n) return SOPB_ERR_INVALID;
    if (p.pulling) {
        // PullingPotential ctor checks (src/Potentials/pulling.cu:54-56, 101-123)
        if (p.deltax == 0.0f && p.fconst == 0.0f) return SOPB_ERR_INVALID;
        if (p.fixedEnd < 0 || p.fixedEnd >= n || p.pulledEnd < 0 || p.pulledEnd >= n) return SOPB_ERR_INVALID;
        for (int32_t k = 0; k < d->nfixed; ++k)
            if (d->fixed[k] < 0 || d->fixed[k] >= n) return SOPB_ERR_INVALID;
        for (int32_t k = 0; k < d->npulled; ++k)
            if (d->pulled[k] < 0 || d->pulled[k] >= n) return SOPB_ERR_INVALID;
    }
    if (p.pullingPlane) {
        // PullingPlanePotential ctor checks (src/Potentials/pulling_plane.cu:60-74)
        if (p.pullingPlaneDeltax == 0.0f || f3norm(p.pullingPlaneDir) == 0.0f || p.pullingPlaneZeta == 0.0f)
            return SOPB_ERR_INVALID;
        if (d->nplane_fixed < 0 || d->nplane_pulled < 0) return SOPB_ERR_INVALID;
        if ((d->nplane_fixed && !d->plane_fixed) || (d->nplane_pulled && !d->plane_pulled)) return SOPB_ERR_INVALID;
        for (int32_t k = 0; k < d->nplane_fixed; ++k)
            if (d->plane_fixed[k] < 0 || d->plane_fixed[k] >= n) return SOPB_ERR_INVALID;
        for (int32_t k = 0; k < d->nplane_pulled; ++k)
            if (d->plane_pulled[k] < 0 || d->plane_pulled[k] >= n) return SOPB_ERR_INVALID;
    }
    if (p.indentation && p.indentationDiscreteSurf) {
        if (p.indentationSurfaceSize <= 0 || p.indentationSurfaceSize > 1024 || p.indentationPairsCutoff <= 0.0f)
            return SOPB_ERR_INVALID;
    }
    if (p.indentation) {
        if (p.indentationTipZeta == 0.0f) return SOPB_ERR_INVALID;
        if (f3norm(p.indentationDirection) == 0.0f || f3norm(p.indentationSurfaceN) == 0.0f) return SOPB_ERR_INVALID;
    }
    if (p.hi_on) {
        // TeaIntegrator ctor (src/Integrators/bdhitea.cu:30-74)
        if (p.minimization) return SOPB_ERR_INVALID;
        if (p.hi_a <= 0.0f) return SOPB_ERR_INVALID;
        if (!p.hi_exact && p.hi_epsilon_freq <= 0) return SOPB_ERR_INVALID;
        if (p.hi_exact && n > kCholMaxBeads) return SOPB_ERR_UNSUPPORTED;
        // the reference-compatible B (symmetrised upper blocks) exists for the
        // reference's own size range only
        if (p.hi_exact && n > 128 && p.hi_b_mode == SOPB_HI_B_REFCOMPAT) return SOPB_ERR_UNSUPPORTED;
    }
    return SOPB_OK;
}

// covalent.cu:126-157 and native.cu:112-146: per-bead rows in .top order.
void build_maps(const sopb_job_desc* d, HostMaps& m) {
    const int32_t n = d->n;
    std::vector<int32_t> cnt(n + 1, 0);
    for (int32_t k = 0; k < d->nbonds; ++k) { cnt[d->bonds[2 * k]]++; cnt[d->bonds[2 * k + 1]]++; }
    m.cov_off.assign(n + 1, 0);
    for (int32_t i = 0; i < n; ++i) m.cov_off[i + 1] = m.cov_off[i] + cnt[i];
    m.cov_j.assign(m.cov_off[n], 0);
    m.cov_r0.assign(m.cov_off[n], 0.0f);
    std::vector<int32_t> fill(m.cov_off.begin(), m.cov_off.end() - 1);
    for (int32_t k = 0; k < d->nbonds; ++k) {
        const int32_t a = d->bonds[2 * k], b = d->bonds[2 * k + 1];
        m.cov_j[fill[a]] = b; m.cov_r0[fill[a]++] = d->bonds_r0[k];
        m.cov_j[fill[b]] = a; m.cov_r0[fill[b]++] = d->bonds_r0[k];
    }
    std::fill(cnt.begin(), cnt.end(), 0);
    for (int32_t k = 0; k < d->nnatives; ++k) { cnt[d->natives[2 * k]]++; cnt[d->natives[2 * k + 1]]++; }
    m.nat_off.assign(n + 1, 0);
    for (int32_t i = 0; i < n; ++i) m.nat_off[i + 1] = m.nat_off[i] + cnt[i];
    m.nat_j.assign(m.nat_off[n], 0);
    m.nat_par.assign(m.nat_off[n], make_float2(0.f, 0.f));
    fill.assign(m.nat_off.begin(), m.nat_off.end() - 1);
    for (int32_t k = 0; k < d->nnatives; ++k) {
        const int32_t a = d->natives[2 * k], b = d->natives[2 * k + 1];
        const float r0 = d->natives_r0[k], eh = d->natives_eh[k];
        const float2 par = make_float2(r0 * r0, (float)(-12.0 * (double)eh / (double)(r0 * r0)));
        m.nat_j[fill[a]] = b; m.nat_par[fill[a]++] = par;
        m.nat_j[fill[b]] = a; m.nat_par[fill[b]++] = par;
    }
}

}  // namespace

namespace {

// Driver entry points the library calls through the runtime's table, so it
// needs no link against libcuda (it loads on machines without a driver).
template <typename Fn>
Fn driver_fn(const char* name, Fn* cache) {
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (!*cache) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion(name, &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            *cache = reinterpret_cast<Fn>(f);
        else
            cudaGetLastError();
    }
    return *cache;
}

// TMA map of a row-major FP32 matrix (rows x cols, leading dimension ld,
// 16-byte aligned base): 128-row x 32-column boxes, 128-byte swizzle, zero
// fill outside the matrix.  No multicast anywhere.
int encode_tmap_f32(CUtensorMap* map, float* base, int rows, int cols, int ld) {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!driver_fn("cuTensorMapEncodeTiled", &fn)) return SOPB_ERR_CUDA;
    if (((uintptr_t)base & 15) || (ld * sizeof(float)) % 16) return SOPB_ERR_INVALID;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)kTcKC, (cuuint32_t)kCT};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? SOPB_OK : SOPB_ERR_CUDA;
}

// Byte layout of a grid job's own buffer block: force partials, the HI
// buffers and the exact-HI tensor, the cell-list arrays and the near list.
// grid_alloc carves the block by these offsets and sopb_job_footprint adds
// its total, so admission and allocation cannot disagree.
struct GridLayout {
    int npart = 0, jsplit = 1, cap_nr = 0, ld = 0;
    bool cells = false, hi = false, exact = false, blocked = false;
    int plane_rows = 0, plane_ld = 0;
    size_t part = 0, rf = 0, mf = 0, xc = 0, ci = 0, eps = 0, ten = 0, linv = 0, phi = 0, plo = 0, geo = 0;
    size_t cc = 0, cs = 0, cb = 0, bc = 0, near = 0, nrj = 0, nrc = 0, xref = 0;
    size_t total = 0;
};

GridLayout grid_layout(const sopb_params& p, int64_t n, int sms, int64_t cap_pp, int64_t cap_pl,
                       int hi_cps = kHiCtasPerSm, int chol_w = kCholPanelTiles) {
    GridLayout L;
    L.npart = (int)std::min<int64_t>((n + kGridBlock - 1) / kGridBlock, (int64_t)sms * 8);
    L.cells = p.cell_list == 1 || (p.cell_list == 0 && n > 16384);
    L.hi = p.hi_on != 0;
    L.exact = L.hi && p.hi_exact;
    L.blocked = L.exact && n > 128;
    const int64_t itiles = (n + kHiTile - 1) / kHiTile;
    if ((L.hi && !p.hi_exact && p.hi_unlisted) || L.blocked)
        L.jsplit = (int)std::max<int64_t>(1, std::min<int64_t>((hi_cps * (int64_t)sms + itiles - 1) / itiles, itiles));
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off += align256(bytes); return o; };
    L.part = take(std::max<size_t>(2 * (size_t)L.npart, L.hi ? (size_t)L.jsplit * n : 0) * sizeof(float4));
    if (L.hi) {
        L.rf = take((size_t)n * 16);
        L.mf = take((size_t)n * 16);
        L.xc = take((size_t)n * 16);
        L.ci = take((size_t)n * 16);
        L.eps = take((size_t)n * 4);
        if (L.exact) {
            L.ld = L.blocked ? chol_ld((int)n) : (int)(3 * n);
            L.ten = take((size_t)3 * n * L.ld * 4);
            if (L.blocked) {
                // the inverse buffers, and the TF32 hi and lo planes of two
                // outer panels (tile rows x 128 rows each, the panel's columns)
                const int T = chol_tiles((int)(3 * n));
                L.plane_rows = T * kCT;
                L.plane_ld = std::min(std::max(1, chol_w), T) * kCT;
                L.linv = take((size_t)2 * kCT * kCT * 4);
                L.phi = take((size_t)2 * L.plane_rows * L.plane_ld * 4);
                L.plo = take((size_t)2 * L.plane_rows * L.plane_ld * 4);
            }
        }
    }
    L.geo = take(8 * sizeof(float));
    if (L.cells) {
        L.cc = take(((size_t)kCellMax + 1) * 4);
        L.cs = take(((size_t)kCellMax + 1) * 4);
        L.cb = take((size_t)n * 4);
        L.bc = take((size_t)n * 4);
    }
    L.cap_nr = (int)grid_cap_nr(p, cap_pp, cap_pl);
    L.near = take(4 * sizeof(int32_t));
    if (L.cap_nr) {
        L.nrj = take((size_t)n * L.cap_nr * 4);
        L.nrc = take((size_t)n * 4);
        L.xref = take((size_t)n * 16);
    }
    L.total = off;
    return L;
}

// Buffers of the grid path: force buffer (the context's second coordinate
// pool), reduction partials and, for large jobs, the cell list.
int grid_alloc(sopb_context* c, sopb_job* j, const sopb_params& p, int32_t n, int32_t cap_pp, int32_t cap_pl) {
    GridAux& a = j->aux;
    const GridLayout L = grid_layout(p, n, c->sm_count, cap_pp, cap_pl, c->policy.hi_ctas_per_sm,
                                     c->policy.chol_panel_tiles);
    j->bead_blocks = L.npart;
    j->jsplit = L.jsplit;
    j->chol_w = c->policy.chol_panel_tiles;
    a.npart = L.npart;
    a.use_cells = L.cells;
    a.cap_nr = L.cap_nr;
    if (L.exact) a.ld = L.ld;
    if (cudaMallocAsync(&j->amem, L.total, c->upload) != cudaSuccess) {
        cudaGetLastError();
        return SOPB_ERR_NOMEM;
    }
    char* b = (char*)j->amem;
    a.F = c->xalt + j->b0;
    a.part = (float4*)(b + L.part);
    if (L.hi) {
        a.rf = (float4*)(b + L.rf);
        a.mf = (float4*)(b + L.mf);
        a.xc = (float4*)(b + L.xc);
        a.ci4 = (float4*)(b + L.ci);
        a.eps = (float*)(b + L.eps);
        if (L.exact) a.tensor = (float*)(b + L.ten);
        if (L.blocked) {
            const int m = 3 * n;
            a.linv = (float*)(b + L.linv);
            a.plane_hi = (float*)(b + L.phi);
            a.plane_lo = (float*)(b + L.plo);
            a.plane_rows = L.plane_rows;
            a.plane_ld = L.plane_ld;
            // rows below the matrix in the planes are read (and discarded)
            // by the last tile row's updates: zero from the start
            CUDA_TRY(cudaMemsetAsync(b + L.phi, 0, L.plo + (size_t)2 * L.plane_rows * L.plane_ld * 4 - L.phi, c->upload));
            SOPB_TRY(encode_tmap_f32(&j->tmap_ten, a.tensor, m, m, a.ld));
            SOPB_TRY(encode_tmap_f32(&j->tmap_linv, a.linv, 2 * kCT, kCT, kCT));
            SOPB_TRY(encode_tmap_f32(&j->tmap_phi, a.plane_hi, 2 * L.plane_rows, L.plane_ld, L.plane_ld));
            SOPB_TRY(encode_tmap_f32(&j->tmap_plo, a.plane_lo, 2 * L.plane_rows, L.plane_ld, L.plane_ld));
            // two streams per priority level, made here rather than during
            // a stream capture
            j->hi_streams = true;
            int lo = 0, hi = 0;
            CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            for (int k = 0; k <= std::min(lo - hi, sopb_job::kPrioLevels - 1); ++k) {
                CUDA_TRY(cudaStreamCreateWithPriority(&j->prio_st[k], cudaStreamNonBlocking, lo - k));
                CUDA_TRY(cudaStreamCreateWithPriority(&j->mid_st[k], cudaStreamNonBlocking, lo - k));
            }
            for (cudaEvent_t* e : {&j->la_join, &j->hp_fork, &j->hp_join})
                CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
            for (cudaEvent_t& e : j->lk_ev) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
    }
    a.cell_geo = (float*)(b + L.geo);
    a.near = (int32_t*)(b + L.near);
    if (a.cap_nr) {
        a.nr_j = (int32_t*)(b + L.nrj);
        a.nr_cnt = (int32_t*)(b + L.nrc);
        a.x_ref = (float4*)(b + L.xref);
    }
    if (a.use_cells) {
        a.cell_count = (int32_t*)(b + L.cc);
        a.cell_start = (int32_t*)(b + L.cs);
        a.cell_beads = (int32_t*)(b + L.cb);
        a.bead_cell = (int32_t*)(b + L.bc);
    }
    CUDA_TRY(cudaMemsetAsync(j->amem, 0, L.total, c->upload));
    return SOPB_OK;
}

// Possible pairs of a grid job: brute force, or cell list + row sort.
int grid_possible(sopb_job* j, JobDev* Jp, cudaStream_t st, int force) {
    GridAux& a = j->aux;
    const int nb = j->bead_blocks;
    const int warps_blocks = (int)std::min<int64_t>((j->n + 7) / 8, (int64_t)j->ctx->sm_count * 16);
    if (!a.use_cells) {
        k_g_possible_brute<<<warps_blocks, kGridBlock, 0, st>>>(Jp, force);
        CUDA_TRY(cudaGetLastError());
        return SOPB_OK;
    }
    // cell_count is zeroed by the scan's consumer (k_cl_fill turns counts
    // into cursors); clear it for this rebuild first
    k_cl_bounds<<<nb, kGridBlock, 0, st>>>(Jp, a, force);
    k_cl_geometry<<<1, 32, 0, st>>>(Jp, a, nb, force);
    CUDA_TRY(cudaMemsetAsync(a.cell_count, 0, ((size_t)kCellMax + 1) * 4, st));
    k_cl_count<<<nb, kGridBlock, 0, st>>>(Jp, a, force);
    k_cl_scan<<<1, 1024, 0, st>>>(Jp, a, force);
    k_cl_fill<<<nb, kGridBlock, 0, st>>>(Jp, a, force);
    k_cl_possible<<<warps_blocks, kGridBlock, 0, st>>>(Jp, a, force);
    const int sort_blocks = (int)std::min<int64_t>((j->n + 3) / 4, (int64_t)j->ctx->sm_count * 16);
    k_cl_sort_rows<<<sort_blocks, 128, 4 * kSortCap * sizeof(int32_t), st>>>(Jp, force);
    CUDA_TRY(cudaGetLastError());
    return SOPB_OK;
}

// Updaters of a stride boundary (each gated on the device step), then
// `steps` Langevin steps, then the step counter moves by `steps`.
// Exact HI of a job above 128 beads: assemble D and factorise it in place in
// 128 x 128 tiles (T tile columns), outer panel by outer panel (chol_w tile
// columns each), on three streams by priority relative to the caller's:
//   hp, two levels above: the chain of single tiles.  Per tile column J: the
//     diagonal tile is brought up to date from the outer panel's earlier
//     columns, factorised in FP64 with the inverse X_J of its factor (into
//     the inverse buffer of J's parity), and the tile just below it is
//     solved (L = A X_J^T on the tensor cores);
//   ms, one level above: the rest of each tile column beside the chain --
//     the tiles below the diagonal from the panel's earlier columns, then,
//     once X_J is there, their solve;
//   la, the caller's level: after an outer panel, the trailing update with
//     K = its columns of every tile column beyond the next outer panel.
// After an outer panel, the next one's tile columns get the finished panel's
// K: the first diagonal tile on hp, the rest of the first tile column on ms
// (the first solve waits for it), then the panel's other tile columns on ms.
// Each tile receives the same updates (same tile kernel, same K ranges, same
// order) as a serial sweep of the same outer panels gives it, so the factor
// does not depend on how the streams interleave.  The caller's stream waits
// for all three at the end.
int chol_refresh(sopb_job* j, JobDev* Jp, cudaStream_t st) {
    GridAux& a = j->aux;
    const int n = j->n, m = 3 * n, T = chol_tiles(m), W = std::max(1, j->chol_w);
    // `tiles` tiles from (i0, jc0) in column order (column jc0 from row tile
    // i0, then the following tile columns from their diagonal tiles)
    auto update = [&](cudaStream_t s, int tiles, int jc0, int i0, int k0, int k1) {
        if (tiles > 0 && k1 > k0)
            k_chol_tc<<<tiles, kTcThreads, kTcSmem, s>>>(j->tmap_phi, j->tmap_plo, Jp, a, jc0, i0, k0, k1, kTcUpdate, W);
    };
    auto tiles_from = [&](int jc0, int i0, int jc1) {   // column jc0 from i0, then whole columns up to jc1
        int t = T - i0;
        for (int J = jc0 + 1; J < jc1; ++J) t += T - J;
        return t;
    };
    auto solve = [&](cudaStream_t s, int J, int i0, int i1) {
        if (i1 > i0)
            k_chol_tc<<<i1 - i0, kTcThreads, kTcSmem, s>>>(j->tmap_ten, j->tmap_linv, Jp, a, J, i0, J * kCT,
                                                           (J + 1) * kCT, kTcSolve, W);
    };
    // priorities relative to the caller's stream (numerically smaller is
    // higher)
    int lo = 0, hi = 0, p = 0;
    CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    CUDA_TRY(cudaStreamGetPriority(st, &p));
    p = std::min(lo, std::max(hi, p));
    auto idx = [&](int prio) { return std::min(sopb_job::kPrioLevels - 1, lo - std::max(hi, prio)); };
    cudaStream_t hp = j->prio_st[idx(p - 2)], ms = j->mid_st[idx(p - 1)], la = j->prio_st[idx(p)];
    if (!hp || !ms || !la) return SOPB_ERR_CUDA;
    constexpr int R = sopb_job::kLkRing;
    cudaEvent_t* e_pot = j->lk_ev;            // X_J written
    cudaEvent_t* e_s1 = j->lk_ev + R;         // tile (J + 1, J) solved
    cudaEvent_t* e_cu = j->lk_ev + 2 * R;     // tiles below (J, J) updated from the panel
    cudaEvent_t* e_sr = j->lk_ev + 3 * R;     // tiles (J + 2.., J) solved
    cudaEvent_t e_np1 = j->lk_ev[4 * R], e_np2 = j->lk_ev[4 * R + 1], ms_join = j->lk_ev[4 * R + 2];
    auto rec = [](cudaEvent_t e, cudaStream_t s) { return cudaEventRecord(e, s); };
    auto wait = [](cudaStream_t s, cudaEvent_t e) { return cudaStreamWaitEvent(s, e, 0); };

    CUDA_TRY(rec(j->hp_fork, st));
    CUDA_TRY(wait(hp, j->hp_fork));
    CUDA_TRY(wait(ms, j->hp_fork));
    k_hi_assemble<<<dim3((n + 255) / 256, n), 256, 0, hp>>>(Jp, a);
    bool rest_pending = false;   // a trailing update on la that the next outer panel must follow
    for (int P0 = 0; P0 < T; P0 += W) {
        const int P1 = std::min(T, P0 + W);
        for (int J = P0; J < P1; ++J) {
            // row J of the columns before J - 1 (solved on ms), and the
            // inverse buffer of J's parity free again
            if (J >= 2) CUDA_TRY(wait(hp, e_sr[(J - 2) % R]));
            if (J > P0) {
                if (J == P0 + 1 && P0 > 0) CUDA_TRY(wait(hp, e_np2));   // (J, J) got the last panel's K on ms
                update(hp, 1, J, J, P0 * kCT, J * kCT);
                if (J + 1 < T) {
                    CUDA_TRY(wait(ms, e_s1[(J - 1) % R]));               // row J of column J - 1
                    update(ms, T - J - 1, J, J + 1, P0 * kCT, J * kCT);
                    CUDA_TRY(rec(e_cu[J % R], ms));
                }
            }
            k_chol_potrf64<<<1, kPotrfThreads, kPotrfSmem, hp>>>(Jp, a, J);
            CUDA_TRY(rec(e_pot[J % R], hp));
            if (J + 1 < T) {
                if (J > P0) CUDA_TRY(wait(hp, e_cu[J % R]));
                else if (P0 > 0) CUDA_TRY(wait(hp, e_np1));             // (J + 1, J) got the last panel's K on ms
                solve(hp, J, J + 1, J + 2);
                CUDA_TRY(rec(e_s1[J % R], hp));
            }
            if (J + 2 < T) {
                CUDA_TRY(wait(ms, e_pot[J % R]));
                solve(ms, J, J + 2, T);
                CUDA_TRY(rec(e_sr[J % R], ms));
            }
        }
        if (P1 < T) {
            // the finished panel's K for the next panel's tile columns, the
            // earlier trailing update of those columns (on la) first
            const int Q1 = std::min(T, P1 + W);
            if (P1 >= 2) CUDA_TRY(wait(hp, e_sr[(P1 - 2) % R]));
            if (rest_pending) CUDA_TRY(wait(hp, j->la_join));
            update(hp, 1, P1, P1, P0 * kCT, P1 * kCT);
            CUDA_TRY(wait(ms, e_s1[(P1 - 1) % R]));
            if (rest_pending) CUDA_TRY(wait(ms, j->la_join));
            update(ms, T - P1 - 1, P1, P1 + 1, P0 * kCT, P1 * kCT);
            CUDA_TRY(rec(e_np1, ms));
            if (Q1 > P1 + 1) update(ms, tiles_from(P1 + 1, P1 + 1, Q1), P1 + 1, P1 + 1, P0 * kCT, P1 * kCT);
            CUDA_TRY(rec(e_np2, ms));
            if (Q1 < T) {   // the tile columns beyond the next panel, beside it
                CUDA_TRY(wait(la, e_s1[(P1 - 1) % R]));
                CUDA_TRY(wait(la, e_sr[(P1 - 1) % R]));
                update(la, tiles_from(Q1, Q1, T), Q1, Q1, P0 * kCT, P1 * kCT);
                CUDA_TRY(rec(j->la_join, la));
                rest_pending = true;
            }
        }
    }
    CUDA_TRY(rec(j->hp_join, hp));
    CUDA_TRY(rec(ms_join, ms));
    CUDA_TRY(wait(st, j->hp_join));
    CUDA_TRY(wait(st, ms_join));
    if (rest_pending) CUDA_TRY(wait(st, j->la_join));
    CUDA_TRY(cudaGetLastError());
    return SOPB_OK;
}

// Updaters due at a stride boundary, from the host's copy of the step.  The
// kernels of an updater that is not due return at once (each gates on the
// device step itself); a launch sequence leaves them out.
enum : int { kDuePossible = 1, kDueVerlet = 2, kDueTReset = 4, kDueTeaEps = 8, kDueRefresh = 16 };

int due_at(const sopb_job* j, int64_t step) {
    const JobDev& h = j->h;
    int d = 0;
    if (step % h.pp_freq == 0) d |= kDuePossible;
    if (step % h.pairs_freq == 0) d |= kDueVerlet;
    if (step % h.nav == 0) d |= kDueTReset;
    if (step % h.eps_freq == 0) d |= kDueTeaEps;
    if (h.hi && h.hi_exact && h.hi_refresh > 1 && step % h.hi_refresh == 0) d |= kDueRefresh;
    return d;
}

// Updaters (at a stride boundary, those of `due`) and `steps` Langevin steps.
int grid_launch(sopb_job* j, cudaStream_t st, bool updaters, int steps, int due = 0) {
    sopb_context* c = j->ctx;
    JobDev* Jp = &c->d_jobs[j->slot];
    GridAux& a = j->aux;
    const int nb = j->bead_blocks;
    const bool refresh_first = (due & kDueRefresh) != 0;
    if (updaters) {
        k_g_tip_partial<<<nb, kGridBlock, 0, st>>>(Jp, a);
        k_g_scalar_updaters<<<1, 32, 0, st>>>(Jp, a);
        if (j->h.indent && j->h.discrete) {
            const int sb = (int)std::min<int64_t>((j->h.nsurf + kGridBlock - 1) / kGridBlock, (int64_t)c->sm_count);
            k_g_surf_move<<<sb, kGridBlock, 0, st>>>(Jp);
            const int mb = (int)std::min<int64_t>((j->n + 7) / 8, (int64_t)c->sm_count * 16);
            k_g_mica<<<mb, kGridBlock, 0, st>>>(Jp);
        }
        if (due & kDueTReset) k_g_treset<<<nb, kGridBlock, 0, st>>>(Jp);
        if (due & kDuePossible) {
            int rc = grid_possible(j, Jp, st, 0);
            if (rc) return rc;
        }
        if (due & kDueVerlet) {
            const int wb = (int)std::min<int64_t>((j->n + 7) / 8, (int64_t)c->sm_count * 16);
            if (a.cap_nr) k_g_drift<<<nb, kGridBlock, 0, st>>>(Jp, a);
            k_g_verlet<<<wb, kGridBlock, 0, st>>>(Jp, a, 0);
        }
        if (a.cap_nr && (due & (kDuePossible | kDueVerlet))) k_g_near_commit<<<1, 32, 0, st>>>(Jp, a, -1, -1);
        if (j->h.hi && !j->h.hi_exact && (due & kDueTeaEps)) {
            // TeaUpdater (src/Integrators/bdhitea.cu:133-176), last updater
            const dim3 tg((j->n + kHiTile - 1) / kHiTile, j->jsplit);
            k_tea_eps_partial<<<tg, kHiTile, 0, st>>>(Jp, a, j->jsplit, 0);
            k_tea_eps_reduce<<<nb, kGridBlock, 0, st>>>(Jp, a, j->jsplit, 0);
            k_tea_beta<<<1, 256, 0, st>>>(Jp, a, 0);
        }
    }
    const int fb = (int)std::min<int64_t>((j->n + (kGridBlock / kGridLpb) - 1) / (kGridBlock / kGridLpb), (int64_t)c->sm_count * 8);
    for (int s = 0; s < steps; ++s) {
        if (j->h.discrete || j->h.plane) k_g_forces<true><<<fb, kGridBlock, 0, st>>>(Jp, a);
        else k_g_forces<false><<<fb, kGridBlock, 0, st>>>(Jp, a);
        if (!j->h.hi) {
            k_g_langevin<<<nb, kGridBlock, 0, st>>>(Jp, a);
        } else if (!j->h.hi_exact) {
            k_hi_prepare<<<nb, kGridBlock, 0, st>>>(Jp, a);
            const dim3 tg((j->n + kHiTile - 1) / kHiTile, j->jsplit);
            k_tea_force_partial<<<tg, kHiTile, 0, st>>>(Jp, a, j->jsplit);
            k_tea_integrate<<<nb, kGridBlock, 0, st>>>(Jp, a, j->jsplit);
        } else {
            // the factor is refreshed every step (hi_refresh 1, the
            // reference) or at the updater boundaries due for it
            const bool refresh = j->h.hi_refresh <= 1 || (s == 0 && refresh_first);
            k_hi_prepare<<<nb, kGridBlock, 0, st>>>(Jp, a);
            if (j->n <= 128) {
                k_chol_D<<<nb, kGridBlock, 0, st>>>(Jp, a, refresh ? 1 : 0);
                if (refresh && j->h.hi_bmode == SOPB_HI_B_REFCOMPAT) k_chol_factor_small<<<1, 384, 0, st>>>(Jp, a);
                else if (refresh) k_chol_factor_panels<<<1, kSmallThreads, kSmallSmem, st>>>(Jp, a);
                if (j->h.hi_bmode == SOPB_HI_B_REFCOMPAT) k_chol_apply<<<nb, kGridBlock, 0, st>>>(Jp, a);
                else k_chol_apply_warp<<<(j->n + kApplyWarps - 1) / kApplyWarps, 32 * kApplyWarps, 0, st>>>(Jp, a);
            } else {
                const dim3 tg((j->n + kHiTile - 1) / kHiTile, j->jsplit);
                k_hi_df_partial<<<tg, kHiTile, 0, st>>>(Jp, a, j->jsplit);
                if (refresh) {
                    int rc = chol_refresh(j, Jp, st);
                    if (rc) return rc;
                }
                const int ab = (int)std::min<int64_t>((j->n + 7) / 8, (int64_t)c->sm_count * 8);
                k_chol_apply_rows<<<ab, 256, (size_t)j->n * 12, st>>>(Jp, a, j->jsplit);
            }
        }
    }
    k_g_advance<<<1, 32, 0, st>>>(Jp, steps);
    CUDA_TRY(cudaGetLastError());
    return SOPB_OK;
}

// Advances a grid job: whole stride chunks by graph replay, the rest by
// direct launches.
int grid_run(sopb_job* j, cudaStream_t st, int64_t nsteps) {
    const int32_t stride = j->h.stride;
    int64_t left = nsteps;
    int rc;
    while (left > 0 && (j->host_step % stride) != 0) {   // finish a partial chunk
        if ((rc = grid_launch(j, st, false, 1))) return rc;
        j->host_step++;
        left--;
    }
    const int64_t chunks = left / stride;
    for (int64_t k = 0; k < chunks; ++k) {
        const int due = due_at(j, j->host_step);
        cudaGraphExec_t& ge = j->chunks[due];
        if (!ge) {
            cudaGraph_t g;
            cudaStream_t cap = j->ctx->capture;
            CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
            rc = grid_launch(j, cap, true, stride, due);
            cudaError_t e = cudaStreamEndCapture(cap, &g);
            if (rc) return rc;
            CUDA_TRY(e);
            CUDA_TRY(cudaGraphInstantiate(&ge, g, cudaGraphInstantiateFlagUseNodePriority));
            cudaGraphDestroy(g);
        }
        CUDA_TRY(cudaGraphLaunch(ge, st));
        j->host_step += stride;
        left -= stride;
    }
    while (left > 0) {
        const bool boundary = j->host_step % stride == 0;
        if ((rc = grid_launch(j, st, boundary, 1, boundary ? due_at(j, j->host_step) : 0))) return rc;
        j->host_step++;
        left--;
    }
    k_g_check_finite<<<j->bead_blocks, kGridBlock, 0, st>>>(&j->ctx->d_jobs[j->slot]);
    CUDA_TRY(cudaGetLastError());
    return SOPB_OK;
}

}  // namespace

extern "C" int sopb_job_footprint(const sopb_job_desc* d, size_t* bytes) {
    if (!d || !bytes || d->n <= 0) return SOPB_ERR_INVALID;
    const int64_t n = d->n;
    const int64_t cap_pp = std::max<int64_t>(1, std::min<int64_t>(d->params.max_possiblePairs > 0 ? d->params.max_possiblePairs : 4096, n - 1));
    const int64_t cap_pl = std::max<int64_t>(1, std::min<int64_t>(d->params.max_pairs > 0 ? d->params.max_pairs : 512, n - 1));
    const sopb_params& p = d->params;
    const bool grid = p.grid_path == 1 || p.hi_on || n > kMaxResidentBeads;
    size_t b = 0;
    b += align256((n + 1) * 4) * 2;                 // offsets
    b += align256(2 * (size_t)d->nbonds * 8);       // cov_j + r0
    b += align256(2 * (size_t)d->nnatives * 12);    // nat_j + par
    b += align256(n * 4) * 2;                       // counts
    if (grid) {
        b += align256(n * cap_pp * 4);              // possible-pair rows
    } else {
        const int64_t W = (n + 31) / 32;
        b += 2 * align256(n * W * 4);               // exclusion and possible-pair masks
        // near list (u16 rows) and the coordinates it was built at
        b += align256(n * std::max<int64_t>(1, std::min<int64_t>(n - 1, 2 * cap_pl)) * 2) + align256(n * 4) +
             align256(n * 16);
    }
    b += align256(n * cap_pl * 4);                  // Verlet rows
    b += n * (16 + 16 + 16 + 4 + 16 + 1);           // bead pools
    if ((p.pulling && p.deltax != 0.0f) || p.indentation || p.pullingPlane)
        b += align256((size_t)(p.log_rows > 0 ? p.log_rows : 1024) * 64);                        // event log
    if (p.indentation && p.indentationDiscreteSurf) {
        const int64_t ns = (int64_t)p.indentationSurfaceSize * p.indentationSurfaceSize;
        b += 2 * align256(ns * 16) + align256(n * ((ns + 31) / 32) * 4);                          // surface, lists
    }
    if (p.pullingPlane) b += align256(n) + 2 * align256(n * 4) + align256(n * 4 + 4);            // plane
    // a job on the grid path (HI, above the resident size, or asked for):
    // its own buffers, sized for the current device's SMs (148 without one)
    if (grid) {
        int sms = 148, dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            sms = 148;
        }
        b += grid_layout(p, n, sms, cap_pp, cap_pl).total;
    }
    *bytes = b;
    return SOPB_OK;
}

extern "C" int sopb_job_create(sopb_context* c, const sopb_job_desc* d, sopb_job** out) {
    if (!c || !out) return SOPB_ERR_INVALID;
    *out = nullptr;
    int rc = validate_desc(d);
    if (rc) return rc;
    CUDA_TRY(cudaSetDevice(c->device));
    const int32_t n = d->n;
    const sopb_params& p = d->params;
    reclaim(c, false);
    int64_t b0;
    if (c->free_slots.empty() || !c->beads.alloc(n, &b0)) {
        reclaim(c, true);   // ranges of destroyed jobs still in use: wait for them
        if (c->free_slots.empty()) return SOPB_ERR_NOMEM;
        if (!c->beads.alloc(n, &b0)) return SOPB_ERR_NOMEM;
    }

    HostMaps m;
    build_maps(d, m);
    JobDev h;
    std::memset(&h, 0, sizeof(h));
    h.n = n;
    launch_shape(c->policy, n, p.lanes_per_bead, &h.lpb, &h.block);
    h.cap_pp = (int32_t)std::max<int64_t>(1, std::min<int64_t>(p.max_possiblePairs > 0 ? p.max_possiblePairs : 4096, n - 1));
    h.cap_pl = (int32_t)std::max<int64_t>(1, std::min<int64_t>(p.max_pairs > 0 ? p.max_pairs : 512, n - 1));
    h.stride = compute_stride(p);
    h.nav = p.nav;
    h.pairs_freq = p.pairs_freq;
    h.pp_freq = p.possiblepairs_freq;
    h.pull_freq = p.pullFreq > 0 ? p.pullFreq : p.nav;
    h.temp_freq = p.heating ? p.tempFreq : 1;
    h.eps_freq = p.hi_epsilon_freq > 0 ? p.hi_epsilon_freq : 1;
    h.step = 0;
    h.retraction_step = p.indentationRetractionStep;
    // force field constants as the reference hosts compute them
    h.ks = p.kspring_cov;
    h.R2 = p.R_limit * p.R_limit;
    h.c8 = (float)(-6.0 * (double)p.el * std::pow((double)p.a, 6.0));
    h.cut2 = p.pairs_cutoff * p.pairs_cutoff;
    h.pl_cut = p.pairlist_cutoff;
    h.pp_thr = p.pairs_threshold;
    h.pl_t = sqrt_threshold(p.pairlist_cutoff);
    h.pp_t = sqrt_threshold(p.pairs_threshold);
    // near list skin: valid while no bead moved more than half of it (less
    // a margin far above the rounding of the distances); drift2 0 = no near list
    const float skin = near_skin(p);
    h.nr_t = sqrt_threshold(p.pairlist_cutoff + std::max(skin, 0.0f));
    h.rlb = p.R_limit_bond > 0.0f ? p.R_limit_bond : 8.0f;
    h.drift2 = skin > 0.02f ? (0.5f * skin - 0.01f) * (0.5f * skin - 0.01f) : 0.0f;
    h.h = p.timestep;
    h.zeta = p.zeta;
    h.hOverZeta = p.timestep / p.zeta;
    h.tempNorm = (float)(p.zeta / (6.0 * p.timestep));
    const float T0 = p.heating ? p.initialT : p.temperature;
    h.var = std::sqrt(2.0f * T0 * p.zeta / p.timestep);
    h.minimization = p.minimization ? 1 : 0;
    h.heating = p.heating ? 1 : 0;
    h.initialT = p.initialT;
    h.deltaT = p.deltaT;

    std::vector<float4> x(n);
    for (int32_t i = 0; i < n; ++i) x[i] = make_float4(d->xyz[3 * i], d->xyz[3 * i + 1], d->xyz[3 * i + 2], 0.0f);
    std::vector<uint8_t> flags(n, FLAG_FREE);
    if (p.pulling) {
        // PullingPotential ctor (src/Potentials/pulling.cu:36-146)
        h.pulling = 1;
        h.ramp = p.deltax != 0.0f ? 1 : 0;
        h.deltax = p.deltax;
        h.k_trans = p.k_trans;
        h.pulledEnd = p.pulledEnd;
        h.fixedEnd = p.fixedEnd;
        const float4 xe = x[p.pulledEnd], xf = x[p.fixedEnd];
        if (p.pull_direction == SOPB_PULL_VECTOR) {
            for (int c2 = 0; c2 < 3; ++c2) h.pullvec[c2] = p.pullVector[c2];
        } else {
            float v[3] = {xe.x - xf.x, xe.y - xf.y, xe.z - xf.z};
            const float len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            for (int c2 = 0; c2 < 3; ++c2) h.pullvec[c2] = v[c2] / len;
        }
        const float xe3[3] = {xe.x, xe.y, xe.z};
        for (int c2 = 0; c2 < 3; ++c2) {
            h.cant0[c2] = h.cant[c2] = xe3[c2];
            h.pullF[c2] = h.pullvec[c2] * p.fconst;
        }
        for (int32_t k = 0; k < d->npulled; ++k) flags[d->pulled[k]] = FLAG_PULLED;
        for (int32_t k = 0; k < d->nfixed; ++k) flags[d->fixed[k]] = FLAG_FIXED;
        // the force-ramp updater re-marks pulled beads at step 0 (pulling.cu:159-163)
        if (h.ramp)
            for (int32_t k = 0; k < d->npulled; ++k) flags[d->pulled[k]] = FLAG_PULLED;
    }
    if (p.indentation) {
        // IndentationPotential ctor (src/Potentials/indentation.cu:75-137)
        h.indent = 1;
        h.moveSurface = p.indentationMoveSurface ? 1 : 0;
        h.fixTrans = p.indentationFixTrans ? 1 : 0;
        for (int c2 = 0; c2 < 3; ++c2) {
            h.chip[c2] = h.chip0[c2] = p.indentationChip[c2];
            h.tip[c2] = p.indentationTip[c2];
            h.dir[c2] = p.indentationDirection[c2];
            h.micaR[c2] = h.micaR0[c2] = p.indentationSurfaceR0[c2];
            h.micaN[c2] = p.indentationSurfaceN[c2];
        }
        h.tipR = p.indentationTipR;
        h.cantKs = p.indentationKs;
        h.V = p.indentationDeltaX;
        h.dx = 0.0f;
        h.tipZeta = p.indentationTipZeta;
        h.tipAp = 12.0f * p.indentationTipEl * std::pow(p.indentationTipSigma, 12.0f) * p.indentationTipA;
        h.tipBp = 6.0f * p.indentationTipEl * std::pow(p.indentationTipSigma, 6.0f) * p.indentationTipB;
        h.surfAp = 12.0f * p.indentationSurfEl * std::pow(p.indentationSurfSigma, 12.0f) * p.indentationSurfA;
        h.surfBp = 6.0f * p.indentationSurfEl * std::pow(p.indentationSurfSigma, 6.0f) * p.indentationSurfB;
        float nd = f3norm(h.dir);
        for (int c2 = 0; c2 < 3; ++c2) h.dir[c2] /= nd;
        nd = f3norm(h.micaN);
        for (int c2 = 0; c2 < 3; ++c2) h.micaN[c2] /= nd;
    }
    // discrete surface: the square of surface beads IndentationAminoUpdater
    // builds from the configured (unnormalised) surface normal
    // (indentation.cu:311-362); lists are rebuilt at every tip update
    std::vector<float4> surf0;
    if (p.indentation && p.indentationDiscreteSurf) {
        const int32_t S = p.indentationSurfaceSize;
        const float* nn = p.indentationSurfaceN;
        const float* r0 = p.indentationSurfaceR0;
        float r1[3];
        if (nn[0] == 0.0f) { r1[0] = 1.0f; r1[1] = 0.0f; r1[2] = 0.0f; }
        else if (nn[1] == 0.0f) { r1[0] = 0.0f; r1[1] = 1.0f; r1[2] = 0.0f; }
        else if (nn[2] == 0.0f) { r1[0] = 0.0f; r1[1] = 0.0f; r1[2] = 1.0f; }
        else { r1[0] = 0.0f; r1[1] = 1.0f; r1[2] = -(nn[1] / nn[2]) * r1[1]; }
        const float nr = std::sqrt(r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2]);
        for (float& v : r1) v /= nr;
        const float r2[3] = {nn[1] * r1[2] - nn[2] * r1[1], nn[2] * r1[0] - nn[0] * r1[2], nn[0] * r1[1] - nn[1] * r1[0]};
        const float displ = p.indentationSurfaceStep;
        for (int32_t a = 0; a < S; ++a)
            for (int32_t b = 0; b < S; ++b) {
                const int32_t i1 = a - S / 2, i2 = b - S / 2;
                float q[3];
                for (int c2 = 0; c2 < 3; ++c2) q[c2] = r0[c2] + i1 * displ * r1[c2] + i2 * displ * r2[c2];
                surf0.push_back(make_float4(q[0], q[1], q[2], 0.0f));
            }
        h.discrete = 1;
        h.nsurf = S * S;
        h.Wm = (h.nsurf + 31) / 32;
        h.mica_cut2 = p.indentationPairsCutoff * p.indentationPairsCutoff;
    }
    // pulling plane (PullingPlanePotential ctor, pulling_plane.cu:35-135):
    // the masks (pulled, then fixed over them), each bead's distance from
    // the plane at step 0, and the masked beads in bead order
    std::vector<uint8_t> plane_mask;
    std::vector<float> plane_r0;
    std::vector<int32_t> plane_idx;
    if (p.pullingPlane) {
        h.plane = 1;
        const float t = std::sqrt(p.pullingPlaneDir[0] * p.pullingPlaneDir[0] + p.pullingPlaneDir[1] * p.pullingPlaneDir[1] +
                                  p.pullingPlaneDir[2] * p.pullingPlaneDir[2]);
        for (int c2 = 0; c2 < 3; ++c2) {
            h.plane_n[c2] = p.pullingPlaneDir[c2] / t;
            h.plane_p0[c2] = p.pullingPlanePos[c2];
        }
        h.plane_ks = p.pullingPlaneKs;
        h.plane_kscant = p.pullingPlaneKsCant;
        h.plane_zeta = p.pullingPlaneZeta;
        h.plane_deltax = p.pullingPlaneDeltax;
        h.plane_freq = p.pullingPlaneUpdateFreq > 0 ? p.pullingPlaneUpdateFreq : p.nav;
        h.plane_ofreq = p.pullingPlaneOutputFreq > 0 ? p.pullingPlaneOutputFreq : p.nav;
        plane_mask.assign(n, 0);
        plane_r0.resize(n);
        for (int32_t i = 0; i < n; ++i) {
            const float dr[3] = {x[i].x - h.plane_p0[0], x[i].y - h.plane_p0[1], x[i].z - h.plane_p0[2]};
            plane_r0[i] = dr[0] * h.plane_n[0] + dr[1] * h.plane_n[1] + dr[2] * h.plane_n[2];
        }
        for (int32_t k = 0; k < d->nplane_pulled; ++k) plane_mask[d->plane_pulled[k]] = 2;
        for (int32_t k = 0; k < d->nplane_fixed; ++k) plane_mask[d->plane_fixed[k]] = 1;
        for (int want = 1; want <= 2; ++want)
            for (int32_t i = 0; i < n; ++i)
                if (plane_mask[i] == want) plane_idx.push_back(i);
        h.nplane_fixed = 0;
        for (int32_t i = 0; i < n; ++i) h.nplane_fixed += plane_mask[i] == 1;
        h.nplane_pulled = (int32_t)plane_idx.size() - h.nplane_fixed;
    }
    std::vector<uint32_t> seeds(4 * (size_t)n);
    if (d->seeds) std::memcpy(seeds.data(), d->seeds, seeds.size() * 4);
    else sopb_generate_seeds(d->seed, n, seeds.data());

    // path: the resident kernel while a job fits one CTA, else per-step
    // grid kernels; list representation: bitmasks when the Verlet masks fit
    // in shared memory
    h.grid = (p.grid_path == 1 || p.hi_on || n > kMaxResidentBeads) ? 1 : 0;
    if (p.hi_on) {
        h.hi = 1;
        h.hi_exact = p.hi_exact ? 1 : 0;
        h.hi_unlisted = p.hi_unlisted ? 1 : 0;
        h.hi_capricious = p.hi_capricious ? 1 : 0;
        h.hi_bmode = p.hi_b_mode;
        h.hi_refresh = p.hi_refresh > 0 ? p.hi_refresh : 1;
        h.hi_a = p.hi_a;
        h.hi_epsmax = p.hi_epsmax;
        h.beta = 0.5f;
    }
    h.W = (n + 31) / 32;
    h.mask = h.grid ? 0 : 1;
    h.ncov = m.cov_off[n];
    h.nnat = m.nat_off[n];
    if (!h.grid) {
        // bonded maps in shared memory when they fit beside the per-bead
        // state; then a cache of the Verlet list: the list at the initial
        // coordinates plus 10% and 4 entries per bead, as far as it fits
        h.bsm = resident_layout(n, h.ncov, h.nnat, 1, 0).total <= (size_t)c->smem_dyn_max ? 1 : 0;
        const float cut = std::min(p.pairlist_cutoff, p.pairs_threshold);
        std::vector<uint8_t> bonded((size_t)n * n, 0);
        for (int32_t i = 0; i < n; ++i) {
            for (int32_t k = m.cov_off[i]; k < m.cov_off[i + 1]; ++k) bonded[(size_t)i * n + m.cov_j[k]] = 1;
            for (int32_t k = m.nat_off[i]; k < m.nat_off[i + 1]; ++k) bonded[(size_t)i * n + m.nat_j[k]] = 1;
        }
        int64_t total = 0;
        for (int32_t i = 0; i < n; ++i)
            for (int32_t q = i + 1; q < n; ++q) {
                const float dx = d->xyz[3 * q] - d->xyz[3 * i], dy = d->xyz[3 * q + 1] - d->xyz[3 * i + 1],
                            dz = d->xyz[3 * q + 2] - d->xyz[3 * i + 2];
                if (!bonded[(size_t)i * n + q] && std::sqrt(dx * dx + dy * dy + dz * dz) < cut) total += 2;
            }
        int64_t want = (int64_t)std::ceil(1.10 * (double)total) + 4 * (int64_t)n;
        want = std::min<int64_t>(want, (int64_t)n * h.cap_pl);
        const int64_t fit =
            ((int64_t)c->smem_dyn_max - (int64_t)resident_layout(n, h.ncov, h.nnat, h.bsm, 0).total - 16) / 2;
        h.lcache = (int32_t)std::max<int64_t>(0, std::min(want, fit));
    }
    if (h.grid) {
        h.lpb = kGridLpb;
        h.block = 1024;
    }
    h.max_pp = p.max_possiblePairs > 0 ? p.max_possiblePairs : 4096;
    h.max_pl = p.max_pairs > 0 ? p.max_pairs : 512;
    // exclusion mask: self, covalent and native partners (the linear scans of
    // possiblepairlist_kernel.cu:47-59, precomputed)
    // (grid jobs scan their partners' rows instead: n^2 bits would not fit)
    std::vector<uint32_t> ex(h.grid ? 0 : (size_t)n * h.W, 0u);
    auto excl = [&](int32_t i, int32_t q) { ex[(size_t)i * h.W + (q >> 5)] |= 1u << (q & 31); };
    if (!h.grid) {
        for (int32_t i = 0; i < n; ++i) excl(i, i);
        for (int32_t i = 0; i < n; ++i) {
            for (int32_t k = m.cov_off[i]; k < m.cov_off[i + 1]; ++k) excl(i, m.cov_j[k]);
            for (int32_t k = m.nat_off[i]; k < m.nat_off[i + 1]; ++k) excl(i, m.nat_j[k]);
        }
    }

    // device block for the maps and lists
    const size_t mask_bytes = h.grid ? 0 : (size_t)n * h.W * 4;
    const size_t o_covoff = 0;
    const size_t o_covj = o_covoff + align256((n + 1) * 4);
    const size_t o_covr0 = o_covj + align256(m.cov_j.size() * 4 + 4);
    const size_t o_natoff = o_covr0 + align256(m.cov_r0.size() * 4 + 4);
    const size_t o_natj = o_natoff + align256((n + 1) * 4);
    const size_t o_natpar = o_natj + align256(m.nat_j.size() * 4 + 4);
    const size_t o_ex = o_natpar + align256(m.nat_par.size() * 8 + 8);
    const size_t o_ppm = o_ex + align256(mask_bytes);
    const size_t o_ppcnt = o_ppm + (h.mask ? align256(mask_bytes) : 0);
    const size_t o_plcnt = o_ppcnt + align256((size_t)n * 4);
    const size_t o_ppj = o_plcnt + align256((size_t)n * 4);
    const size_t o_plj = o_ppj + (h.mask ? 0 : align256((size_t)n * h.cap_pp * 4));
    // resident jobs: the near list (pairs within pairlist_cutoff + skin,
    // u16) and the coordinates it was built at
    h.cap_nr = h.mask ? std::max<int32_t>(1, std::min<int32_t>(n - 1, 2 * h.cap_pl)) : 0;
    const size_t o_nrj = o_plj + align256((size_t)n * h.cap_pl * 4);
    const size_t o_nrc = o_nrj + (h.mask ? align256((size_t)n * h.cap_nr * 2) : 0);
    const size_t o_xref = o_nrc + (h.mask ? align256((size_t)n * 4) : 0);
    const size_t o_log = o_xref + (h.mask ? align256((size_t)n * 16) : 0);
    // event-log ring of the jobs whose updaters print per-update lines
    h.log_cap = (h.ramp || h.indent || h.plane) ? (p.log_rows > 0 ? p.log_rows : 1024) : 0;
    const size_t o_surf = o_log + align256((size_t)h.log_cap * 64);
    const size_t o_surf0 = o_surf + align256((size_t)h.nsurf * 16);
    const size_t o_mica = o_surf0 + align256((size_t)h.nsurf * 16);
    const size_t o_pmask = o_mica + align256((size_t)n * h.Wm * 4);
    const size_t o_pr0 = o_pmask + (h.plane ? align256((size_t)n) : 0);
    const size_t o_pf = o_pr0 + (h.plane ? align256((size_t)n * 4) : 0);
    const size_t o_pidx = o_pf + (h.plane ? align256((size_t)n * 4) : 0);
    const size_t total = o_pidx + (h.plane ? align256(plane_idx.size() * 4 + 4) : 0);
    sopb_job* j = new (std::nothrow) sopb_job();
    if (!j) { c->beads.release(b0, n); return SOPB_ERR_NOMEM; }
    // stream-ordered allocation: a destroyed job's memory returns to the
    // pool after its last work, without stalling other streams
    cudaError_t e = cudaMallocAsync(&j->dmem, total, c->upload);
    if (e != cudaSuccess) {
        cudaGetLastError();
        c->beads.release(b0, n);
        delete j;
        return SOPB_ERR_NOMEM;
    }
    char* base = (char*)j->dmem;
    h.cov_off = (int32_t*)(base + o_covoff);
    h.cov_j = (int32_t*)(base + o_covj);
    h.cov_r0 = (float*)(base + o_covr0);
    h.nat_off = (int32_t*)(base + o_natoff);
    h.nat_j = (int32_t*)(base + o_natj);
    h.nat_par = (float2*)(base + o_natpar);
    h.ex_mask = h.grid ? nullptr : (uint32_t*)(base + o_ex);
    h.pp_mask = h.mask ? (uint32_t*)(base + o_ppm) : nullptr;
    h.pp_cnt = (int32_t*)(base + o_ppcnt);
    h.pl_cnt = (int32_t*)(base + o_plcnt);
    h.pp_j = h.mask ? nullptr : (int32_t*)(base + o_ppj);
    h.pl_j = (int32_t*)(base + o_plj);
    h.nr_j = h.mask ? (uint16_t*)(base + o_nrj) : nullptr;
    h.nr_cnt = h.mask ? (int32_t*)(base + o_nrc) : nullptr;
    h.x_ref = h.mask ? (float4*)(base + o_xref) : nullptr;
    h.log = h.log_cap ? (float*)(base + o_log) : nullptr;
    h.log_head = 0;
    h.surf = h.nsurf ? (float4*)(base + o_surf) : nullptr;
    h.surf0 = h.nsurf ? (float4*)(base + o_surf0) : nullptr;
    h.mica = h.nsurf ? (uint32_t*)(base + o_mica) : nullptr;
    h.plane_mask = h.plane ? (uint8_t*)(base + o_pmask) : nullptr;
    h.plane_r0 = h.plane ? (float*)(base + o_pr0) : nullptr;
    h.plane_f = h.plane ? (float*)(base + o_pf) : nullptr;
    h.plane_idx = h.plane ? (int32_t*)(base + o_pidx) : nullptr;
    h.nr_valid = 0;
    h.x = c->x + b0;
    h.xalt = c->xalt + b0;
    h.seeds = c->seeds + b0;
    h.T = c->T + b0;
    h.tipF = c->tipF + b0;
    h.flags = c->flags + b0;
    cudaStream_t st = c->upload;   // set-up copies do not wait for running work
    CUDA_TRY(cudaMemsetAsync(base + o_ppm, 0, o_ppj - o_ppm, st));   // mask and counts
    if (!h.grid) CUDA_TRY(cudaMemcpyAsync(h.ex_mask, ex.data(), mask_bytes, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(h.cov_off, m.cov_off.data(), (n + 1) * 4, cudaMemcpyHostToDevice, st));
    if (!m.cov_j.empty()) {
        CUDA_TRY(cudaMemcpyAsync(h.cov_j, m.cov_j.data(), m.cov_j.size() * 4, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(h.cov_r0, m.cov_r0.data(), m.cov_r0.size() * 4, cudaMemcpyHostToDevice, st));
    }
    CUDA_TRY(cudaMemcpyAsync(h.nat_off, m.nat_off.data(), (n + 1) * 4, cudaMemcpyHostToDevice, st));
    if (!m.nat_j.empty()) {
        CUDA_TRY(cudaMemcpyAsync(h.nat_j, m.nat_j.data(), m.nat_j.size() * 4, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(h.nat_par, m.nat_par.data(), m.nat_par.size() * 8, cudaMemcpyHostToDevice, st));
    }
    CUDA_TRY(cudaMemcpyAsync(h.x, x.data(), (size_t)n * 16, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(h.seeds, seeds.data(), (size_t)n * 16, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(h.flags, flags.data(), (size_t)n, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemsetAsync(h.T, 0, (size_t)n * 4, st));
    CUDA_TRY(cudaMemsetAsync(h.tipF, 0, (size_t)n * 16, st));
    if (h.nsurf) {
        CUDA_TRY(cudaMemcpyAsync(h.surf, surf0.data(), (size_t)h.nsurf * 16, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(h.surf0, surf0.data(), (size_t)h.nsurf * 16, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemsetAsync(h.mica, 0, (size_t)n * h.Wm * 4, st));   // lists built at the first tip update
    }
    if (h.plane) {
        CUDA_TRY(cudaMemcpyAsync(h.plane_mask, plane_mask.data(), (size_t)n, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(h.plane_r0, plane_r0.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemsetAsync(h.plane_f, 0, (size_t)n * 4, st));
        if (!plane_idx.empty())
            CUDA_TRY(cudaMemcpyAsync(h.plane_idx, plane_idx.data(), plane_idx.size() * 4, cudaMemcpyHostToDevice, st));
    }
    j->b0 = b0;   // the grid buffers are views of the job's bead range
    j->n = n;
    if (h.grid) {
        int rc2 = grid_alloc(c, j, p, n, h.cap_pp, h.cap_pl);
        if (rc2) {
            cudaFreeAsync(j->dmem, c->upload);
            c->beads.release(b0, n);
            delete j;
            return rc2;
        }
    }
    c->generation++;
    const int slot = c->free_slots.back();
    c->free_slots.pop_back();
    CUDA_TRY(cudaMemcpyAsync(&c->d_jobs[slot], &h, sizeof(JobDev), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaStreamSynchronize(st));   // host staging vectors go out of scope
    CUDA_TRY(cudaEventCreateWithFlags(&j->ev, cudaEventDisableTiming));
    CUDA_TRY(cudaEventRecord(j->ev, st));
    j->st = st;
    j->ctx = c;
    j->slot = slot;
    j->b0 = b0;
    j->n = n;
    j->h = h;
    j->dbytes = total;
    c->slots[slot] = j;
    *out = j;
    return SOPB_OK;
}

extern "C" int sopb_job_destroy(sopb_job* j) {
    if (!j) return SOPB_ERR_INVALID;
    sopb_context* c = j->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    // nothing waits here: graphs and memory are released after the job's
    // last work on its stream, the bead range and slot once it has finished
    for (auto& g : j->chunks) if (g.second) cudaGraphExecDestroy(g.second);
    if (j->hi_streams) hi_streams_destroy(j);   // released by the runtime once their work is done
    SOPB_TRY(job_ev(j));
    CUDA_TRY(cudaStreamWaitEvent(c->io, j->ev, 0));
    if (j->amem) CUDA_TRY(cudaFreeAsync(j->amem, c->io));
    CUDA_TRY(cudaFreeAsync(j->dmem, c->io));
    CUDA_TRY(cudaEventRecord(j->ev, c->io));
    c->slots[j->slot] = nullptr;
    c->generation++;
    c->deferred.push_back({j->ev, j->b0, j->n, j->slot});
    delete j;
    return SOPB_OK;
}

namespace {
// Groups jobs by CTA size class; returns (block, ids) per class, largest
// jobs' class first so the longest CTAs start first.

// CTAs of a job's resident launch that fit one SM: 1024 threads' worth of
// registers (the kernel's launch bound) and the SM's shared memory.
int ctas_per_sm(const sopb_context* c, int block, size_t smem) {
    const int by_regs = 1024 / block;
    const size_t per_cta = smem + (size_t)c->smem_static[block_index(block)] + (size_t)c->smem_reserved;
    const int by_smem = (int)((size_t)c->smem_per_sm / per_cta);
    return std::max(1, std::min(by_regs, by_smem));
}
// Jobs of one class share a CTA size and the number of CTAs an SM holds, so
// the class's largest shared-memory request never lowers the residency of
// its smaller jobs.
void group_jobs(const sopb_context* c, sopb_job* const* jobs, int32_t njobs, std::vector<LaunchClass>& out) {
    std::map<int, LaunchClass> cls;   // key: block * 64 + CTAs per SM
    std::vector<int32_t> order(njobs);
    for (int32_t k = 0; k < njobs; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return jobs[a]->n > jobs[b]->n; });
    for (int32_t k : order) {
        const JobDev& h = jobs[k]->h;
        const size_t smem = resident_smem_bytes(h);
        LaunchClass& L = cls[h.block * 64 + ctas_per_sm(c, h.block, smem)];
        L.block = h.block;
        L.max_n = std::max(L.max_n, jobs[k]->n);
        L.smem = std::max(L.smem, smem);
        L.ids.push_back(jobs[k]->slot);
    }
    out.clear();
    for (auto& kv : cls) out.push_back(kv.second);
    std::sort(out.begin(), out.end(), [](const LaunchClass& a, const LaunchClass& b) { return a.max_n > b.max_n; });
}
int run_ordered(sopb_context* c, sopb_job* const* jobs, int32_t njobs, const int64_t* nsteps, cudaStream_t st);
}  // namespace

extern "C" int sopb_run_ragged(sopb_context* c, sopb_job* const* jobs, int32_t njobs, const int64_t* nsteps,
                               void* stream) {
    if (!c || (njobs > 0 && (!jobs || !nsteps)) || njobs < 0) return SOPB_ERR_INVALID;
    if (njobs == 0) return SOPB_OK;
    for (int32_t k = 0; k < njobs; ++k)
        if (!jobs[k] || jobs[k]->ctx != c || nsteps[k] < 0) return SOPB_ERR_INVALID;
    CUDA_TRY(cudaSetDevice(c->device));
    const cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    // a job that last ran on another stream: this run starts after that work
    for (int32_t k = 0; k < njobs; ++k) {
        sopb_job* j = jobs[k];
        if (j->st != st) {
            SOPB_TRY(job_ev(j));
            CUDA_TRY(cudaStreamWaitEvent(st, j->ev, 0));
            j->st = st;
        }
    }
    // jobs with no steps take no part
    std::vector<sopb_job*> act;
    std::vector<int64_t> n;
    for (int32_t k = 0; k < njobs; ++k)
        if (nsteps[k] > 0) {
            act.push_back(jobs[k]);
            n.push_back(nsteps[k]);
        }
    int rc = act.empty() ? SOPB_OK : run_ordered(c, act.data(), (int32_t)act.size(), n.data(), st);
    // the jobs' last work is this run (their events are recorded on demand)
    for (int32_t k = 0; k < njobs; ++k) jobs[k]->ev_lazy = true;
    return rc;
}

extern "C" int sopb_run_on(sopb_context* c, sopb_job* const* jobs, int32_t njobs, int64_t nsteps, void* stream) {
    if (nsteps < 0 || njobs < 0) return SOPB_ERR_INVALID;
    std::vector<int64_t> n((size_t)std::max(njobs, 0), nsteps);
    return sopb_run_ragged(c, jobs, njobs, n.data(), stream);
}

namespace {
int run_ordered(sopb_context* c, sopb_job* const* jobs, int32_t njobs, const int64_t* nsteps, cudaStream_t st) {
    std::vector<sopb_job*> resident, grid;
    std::vector<int64_t> rsteps, gsteps;
    for (int32_t k = 0; k < njobs; ++k) {
        if (jobs[k]->h.grid) {
            grid.push_back(jobs[k]);
            gsteps.push_back(nsteps[k]);
        } else {
            resident.push_back(jobs[k]);
            rsteps.push_back(nsteps[k]);
        }
    }
    // resident jobs: one launch per class; the class table goes up first
    int32_t* d_ids = nullptr;
    int64_t* d_steps = nullptr;
    int rc;
    RunPlan& plan = c->plans[st];
    const std::vector<LaunchClass>& cls = plan.cls;
    const std::vector<size_t>& off = plan.off;
    if (!resident.empty()) {
        const bool same = plan.generation == c->generation && plan.jobs == resident && plan.steps == rsteps;
        if (!same) {
            plan.generation = c->generation;
            plan.jobs = resident;
            plan.steps = rsteps;
            plan.cls.clear();
            plan.off.clear();
            group_jobs(c, resident.data(), (int32_t)resident.size(), plan.cls);
        }
        std::vector<int64_t> slot_steps(c->slots.size(), 0);
        for (size_t k = 0; k < resident.size(); ++k) slot_steps[resident[k]->slot] = rsteps[k];
        int64_t total = 0;
        for (auto& L : cls) total += (int64_t)L.ids.size();
        if ((rc = ensure_ids(c, st, total, &d_ids, &d_steps))) return rc;
        if (!same) {
            std::vector<int32_t> ids;
            std::vector<int64_t> steps;
            for (auto& L : cls) {
                plan.off.push_back(ids.size());
                ids.insert(ids.end(), L.ids.begin(), L.ids.end());
                for (int32_t slot : L.ids) steps.push_back(slot_steps[slot]);
            }
            // (a copy from pageable memory is staged before the call returns)
            CUDA_TRY(cudaMemcpyAsync(d_ids, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaMemcpyAsync(d_steps, steps.data(), steps.size() * 8, cudaMemcpyHostToDevice, st));
        }
        if (grid.empty() && cls.size() == 1)
            return launch_resident(cls[0].block, (int)cls[0].ids.size(), cls[0].smem, st, c->d_jobs, d_ids, d_steps);
    } else {
        // no resident jobs in this run: no classes to launch, and the table
        // on this stream is no longer the plan's
        plan.jobs.clear();
        plan.steps.clear();
        plan.cls.clear();
        plan.off.clear();
        plan.generation = ~uint64_t(0);
    }
    // one grid job alone: straight on the stream
    if (resident.empty() && grid.size() == 1) return grid_run(grid[0], st, gsteps[0]);
    // otherwise fork: classes on the side streams, grid jobs (each a chain
    // of small launches) round-robin on their own streams, then join
    sopb_context::Fork* f = nullptr;
    if ((rc = fork_set(c, st, &f))) return rc;
    CUDA_TRY(cudaEventRecord(f->fork, st));
    for (size_t k = 0; k < cls.size(); ++k) {
        cudaStream_t s = f->side[k % kSideStreams];
        CUDA_TRY(cudaStreamWaitEvent(s, f->fork, 0));
        rc = launch_resident(cls[k].block, (int)cls[k].ids.size(), cls[k].smem, s, c->d_jobs, d_ids + off[k],
                             d_steps + off[k]);
        if (rc) return rc;
    }
    for (size_t g = 0; g < grid.size(); ++g) {
        cudaStream_t s = f->gside[g % kGridStreams];
        if (g < (size_t)kGridStreams) CUDA_TRY(cudaStreamWaitEvent(s, f->fork, 0));
        if ((rc = grid_run(grid[g], s, gsteps[g]))) return rc;
    }
    for (int k = 0; k < kSideStreams && k < (int)cls.size(); ++k) {
        CUDA_TRY(cudaEventRecord(f->join[k], f->side[k]));
        CUDA_TRY(cudaStreamWaitEvent(st, f->join[k], 0));
    }
    for (int k = 0; k < kGridStreams && k < (int)grid.size(); ++k) {
        CUDA_TRY(cudaEventRecord(f->gjoin[k], f->gside[k]));
        CUDA_TRY(cudaStreamWaitEvent(st, f->gjoin[k], 0));
    }
    return SOPB_OK;
}
}  // namespace

extern "C" int sopb_run(sopb_context* c, sopb_job* const* jobs, int32_t njobs, int64_t nsteps) {
    return sopb_run_on(c, jobs, njobs, nsteps, nullptr);
}

extern "C" int sopb_job_status(sopb_job* j) {
    if (!j) return SOPB_ERR_INVALID;
    int rc = read_slot(j);
    if (rc) return rc;
    return j->h.status;
}

extern "C" int sopb_job_step(sopb_job* j, int64_t* step) {
    if (!j || !step) return SOPB_ERR_INVALID;
    int rc = read_slot(j);
    if (rc) return rc;
    *step = j->h.step;
    return SOPB_OK;
}

extern "C" int sopb_job_size(sopb_job* j, int32_t* n) {
    if (!j || !n) return SOPB_ERR_INVALID;
    *n = j->n;
    return SOPB_OK;
}

extern "C" int sopb_job_shape(sopb_job* j, int32_t* lpb, int32_t* block) {
    if (!j || !lpb || !block) return SOPB_ERR_INVALID;
    *lpb = j->h.lpb;
    *block = j->h.block;
    return SOPB_OK;
}

extern "C" int sopb_job_read(sopb_job* j, int32_t what, void* out) {
    if (!j || !out) return SOPB_ERR_INVALID;
    sopb_context* c = j->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    SOPB_TRY(io_begin(j));
    const size_t n = j->n;
    switch (what) {
    case SOPB_COORDS:
        CUDA_TRY(cudaMemcpyAsync(out, c->x + j->b0, n * 16, cudaMemcpyDeviceToHost, c->io));
        break;
    case SOPB_SEEDS:
        CUDA_TRY(cudaMemcpyAsync(out, c->seeds + j->b0, n * 16, cudaMemcpyDeviceToHost, c->io));
        break;
    case SOPB_TEMP:
        CUDA_TRY(cudaMemcpyAsync(out, c->T + j->b0, n * 4, cudaMemcpyDeviceToHost, c->io));
        break;
    case SOPB_TIPFORCES:
        CUDA_TRY(cudaMemcpyAsync(out, c->tipF + j->b0, n * 16, cudaMemcpyDeviceToHost, c->io));
        break;
    case SOPB_FORCES: {
        if ((int64_t)n > c->scratch4_cap) {
            if (c->d_scratch4) cudaFreeAsync(c->d_scratch4, c->io);
            CUDA_TRY(cudaMallocAsync((void**)&c->d_scratch4, n * 16, c->io));
            c->scratch4_cap = (int64_t)n;
        }
        int32_t* d_ids = nullptr;
        int rc = ensure_ids(c, c->io, 1, &d_ids);
        c->plans.erase(c->io);   // the io stream's table no longer holds a run plan
        if (rc) return rc;
        const int32_t id = j->slot;
        CUDA_TRY(cudaMemcpyAsync(d_ids, &id, 4, cudaMemcpyHostToDevice, c->io));
        rc = launch_forces(j->h.block, 1, c->io, c->d_jobs, d_ids, c->d_scratch4);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(out, c->d_scratch4, n * 16, cudaMemcpyDeviceToHost, c->io));
        break;
    }
    case SOPB_PULLSTATE: {
        int rc = read_slot(j);
        if (rc) return rc;
        float* o = (float*)out;
        std::memcpy(o, j->h.pullF, 12);
        std::memcpy(o + 3, j->h.cant, 12);
        std::memcpy(o + 6, j->h.cant0, 12);
        std::memcpy(o + 9, j->h.pullvec, 12);
        return SOPB_OK;
    }
    case SOPB_HISTATE: {
        int rc = read_slot(j);
        if (rc) return rc;
        float* o = (float*)out;
        o[0] = j->h.beta;
        o[1] = j->h.epsilon;
        o[2] = o[3] = 0.0f;
        return SOPB_OK;
    }
    case SOPB_HIFACTOR: {
        if (!j->h.hi || !j->h.hi_exact || !j->aux.tensor) return SOPB_ERR_INVALID;
        const size_t m = 3 * (size_t)n;
        CUDA_TRY(cudaMemcpy2DAsync(out, m * 4, j->aux.tensor, (size_t)j->aux.ld * 4, m * 4, m,
                                   cudaMemcpyDeviceToHost, c->io));
        break;
    }
    case SOPB_OBSERVABLES: {
        // per-CTA partials and the 8 results, stream-ordered scratch on io
        const int nb = (int)std::min<int64_t>(((int64_t)n + kObsBlock - 1) / kObsBlock, (int64_t)c->sm_count * 4);
        double* d = nullptr;
        CUDA_TRY(cudaMallocAsync((void**)&d, ((size_t)nb * kObsTerms + 8) * sizeof(double), c->io));
        JobDev* Jp = &c->d_jobs[j->slot];
        k_obs_partial<<<nb, kObsBlock, 0, c->io>>>(Jp, d);
        k_obs_final<<<1, 32, 0, c->io>>>(Jp, d, nb, d + (size_t)nb * kObsTerms);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(out, d + (size_t)nb * kObsTerms, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->io));
        CUDA_TRY(cudaFreeAsync(d, c->io));
        break;
    }
    case SOPB_TIPSTATE: {
        int rc = read_slot(j);
        if (rc) return rc;
        float* o = (float*)out;
        std::memset(o, 0, 64);
        std::memcpy(o, j->h.tip, 12);
        std::memcpy(o + 3, j->h.chip, 12);
        std::memcpy(o + 6, j->h.micaR, 12);
        o[9] = j->h.V;
        o[10] = j->h.dx;
        std::memcpy(o + 11, j->h.fav, 16);
        return SOPB_OK;
    }
    default: return SOPB_ERR_INVALID;
    }
    SOPB_TRY(io_end(j, false));
    return SOPB_OK;
}

extern "C" int sopb_job_log(sopb_job* j, sopb_log_row* rows, int32_t max_rows, int32_t* nrows) {
    if (!j || !nrows || max_rows < 0 || (max_rows > 0 && !rows)) return SOPB_ERR_INVALID;
    *nrows = 0;
    sopb_context* c = j->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    SOPB_TRY(read_slot(j));
    const uint32_t cap = (uint32_t)j->h.log_cap;
    if (cap == 0) return SOPB_OK;
    const uint32_t head = j->h.log_head;
    int rc = SOPB_OK;
    if (head - j->log_tail > cap) {        // the ring wrapped: keep the newest cap rows
        j->log_tail = head - cap;
        rc = SOPB_ERR_CAPACITY;
    }
    const uint32_t take = std::min<uint32_t>(head - j->log_tail, (uint32_t)max_rows);
    const uint32_t r0 = j->log_tail & (cap - 1);
    const uint32_t first = std::min<uint32_t>(take, cap - r0);
    const float* ring = j->h.log;
    if (first)
        CUDA_TRY(cudaMemcpyAsync(rows, ring + (size_t)r0 * 16, (size_t)first * 64, cudaMemcpyDeviceToHost, c->io));
    if (take > first)
        CUDA_TRY(cudaMemcpyAsync(rows + first, ring, (size_t)(take - first) * 64, cudaMemcpyDeviceToHost, c->io));
    CUDA_TRY(cudaStreamSynchronize(c->io));
    j->log_tail += take;
    *nrows = (int32_t)take;
    return rc;
}

extern "C" int sopb_job_write(sopb_job* j, int32_t what, const void* in) {
    if (!j || !in) return SOPB_ERR_INVALID;
    sopb_context* c = j->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    SOPB_TRY(io_begin(j));
    const size_t n = j->n;
    switch (what) {
    case SOPB_COORDS: CUDA_TRY(cudaMemcpyAsync(c->x + j->b0, in, n * 16, cudaMemcpyHostToDevice, c->io)); break;
    case SOPB_SEEDS: CUDA_TRY(cudaMemcpyAsync(c->seeds + j->b0, in, n * 16, cudaMemcpyHostToDevice, c->io)); break;
    case SOPB_TEMP: CUDA_TRY(cudaMemcpyAsync(c->T + j->b0, in, n * 4, cudaMemcpyHostToDevice, c->io)); break;
    case SOPB_TIPFORCES: CUDA_TRY(cudaMemcpyAsync(c->tipF + j->b0, in, n * 16, cudaMemcpyHostToDevice, c->io)); break;
    default: return SOPB_ERR_INVALID;
    }
    SOPB_TRY(io_end(j, true));
    return SOPB_OK;
}

extern "C" int sopb_job_pairlist(sopb_job* j, int32_t possible, int32_t* counts, int32_t* rows, int32_t cap) {
    if (!j || !counts || !rows || cap <= 0) return SOPB_ERR_INVALID;
    sopb_context* c = j->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    SOPB_TRY(io_begin(j));
    const int32_t n = j->n;
    if (j->h.mask && possible) {
        const int32_t W = j->h.W;
        std::vector<uint32_t> msk((size_t)n * W);
        CUDA_TRY(cudaMemcpyAsync(msk.data(), j->h.pp_mask, msk.size() * 4, cudaMemcpyDeviceToHost, c->io));
        SOPB_TRY(io_end(j, false));
        for (int32_t i = 0; i < n; ++i) {
            int32_t k = 0;
            for (int32_t q = 0; q < n; ++q)
                if ((msk[(size_t)i * W + (q >> 5)] >> (q & 31)) & 1u) {
                    if (k < cap) rows[(size_t)i * cap + k] = q;
                    ++k;
                }
            counts[i] = k;
            for (int32_t r = k; r < cap; ++r) rows[(size_t)i * cap + r] = -1;
        }
        return SOPB_OK;
    }
    const int32_t lcap = possible ? j->h.cap_pp : j->h.cap_pl;
    std::vector<int32_t> cnt(n), lst((size_t)n * lcap);
    CUDA_TRY(cudaMemcpyAsync(cnt.data(), possible ? j->h.pp_cnt : j->h.pl_cnt, (size_t)n * 4, cudaMemcpyDeviceToHost, c->io));
    CUDA_TRY(cudaMemcpyAsync(lst.data(), possible ? j->h.pp_j : j->h.pl_j, lst.size() * 4, cudaMemcpyDeviceToHost, c->io));
    SOPB_TRY(io_end(j, false));
    for (int32_t i = 0; i < n; ++i) {
        counts[i] = cnt[i];
        for (int32_t k = 0; k < cap; ++k) rows[(size_t)i * cap + k] = (k < cnt[i] && k < lcap) ? lst[(size_t)i * lcap + k] : -1;
    }
    return SOPB_OK;
}

extern "C" int sopb_job_rebuild_lists(sopb_job* j, int32_t possible, int32_t verlet) {
    if (!j) return SOPB_ERR_INVALID;
    sopb_context* c = j->ctx;
    CUDA_TRY(cudaSetDevice(c->device));
    SOPB_TRY(io_begin(j));
    if (j->h.grid) {
        JobDev* Jp = &c->d_jobs[j->slot];
        int rc = SOPB_OK;
        if (possible) rc = grid_possible(j, Jp, c->io, 1);
        if (rc) return rc;
        if (verlet) {
            const int wb = (int)std::min<int64_t>((j->n + 7) / 8, (int64_t)c->sm_count * 16);
            k_g_verlet<<<wb, kGridBlock, 0, c->io>>>(Jp, j->aux, 1);
        }
        if (j->aux.cap_nr && (possible || verlet))
            k_g_near_commit<<<1, 32, 0, c->io>>>(Jp, j->aux, possible ? 1 : 0, verlet ? 1 : 0);
        CUDA_TRY(cudaGetLastError());
        SOPB_TRY(io_end(j, true));
        return SOPB_OK;
    }
    int32_t* d_ids = nullptr;
    int rc = ensure_ids(c, c->io, 1, &d_ids);
    c->plans.erase(c->io);   // the io stream's table no longer holds a run plan
    if (rc) return rc;
    const int32_t id = j->slot;
    CUDA_TRY(cudaMemcpyAsync(d_ids, &id, 4, cudaMemcpyHostToDevice, c->io));
    rc = launch_rebuild(j->h.block, 1, c->io, c->d_jobs, d_ids, possible, verlet);
    if (rc) return rc;
    SOPB_TRY(io_end(j, true));
    return SOPB_OK;
}

namespace {
// One copy when the jobs' bead ranges are contiguous and in order, else one
// copy per job.
int bulk_coords(sopb_context* c, sopb_job* const* jobs, int32_t njobs, void* host, bool up) {
    if (!c || (njobs && !jobs) || !host) return SOPB_ERR_INVALID;
    CUDA_TRY(cudaSetDevice(c->device));
    // the copies go on the context stream, after each job's last work
    for (int32_t k = 0; k < njobs; ++k) {
        sopb_job* j = jobs[k];
        if (j->st != c->stream) {
            SOPB_TRY(job_ev(j));
            CUDA_TRY(cudaStreamWaitEvent(c->stream, j->ev, 0));
            j->st = c->stream;
        }
    }
    bool contiguous = true;
    for (int32_t k = 1; k < njobs; ++k)
        if (jobs[k]->b0 != jobs[k - 1]->b0 + jobs[k - 1]->n) contiguous = false;
    if (contiguous && njobs) {
        int64_t total = 0;
        for (int32_t k = 0; k < njobs; ++k) total += jobs[k]->n;
        if (up) CUDA_TRY(cudaMemcpyAsync(c->x + jobs[0]->b0, host, total * 16, cudaMemcpyHostToDevice, c->stream));
        else CUDA_TRY(cudaMemcpyAsync(host, c->x + jobs[0]->b0, total * 16, cudaMemcpyDeviceToHost, c->stream));
    } else {
        char* h = (char*)host;
        for (int32_t k = 0; k < njobs; ++k) {
            const size_t b = (size_t)jobs[k]->n * 16;
            if (up) CUDA_TRY(cudaMemcpyAsync(c->x + jobs[k]->b0, h, b, cudaMemcpyHostToDevice, c->stream));
            else CUDA_TRY(cudaMemcpyAsync(h, c->x + jobs[k]->b0, b, cudaMemcpyDeviceToHost, c->stream));
            h += b;
        }
    }
    if (up)   // the jobs' next work comes after the upload (events on demand)
        for (int32_t k = 0; k < njobs; ++k) jobs[k]->ev_lazy = true;
    return SOPB_OK;
}
}  // namespace

extern "C" int sopb_jobs_upload_coords(sopb_context* c, sopb_job* const* jobs, int32_t njobs, const float* host_xyzw) {
    return bulk_coords(c, jobs, njobs, (void*)host_xyzw, true);
}

extern "C" int sopb_jobs_download_coords(sopb_context* c, sopb_job* const* jobs, int32_t njobs, float* host_xyzw) {
    int rc = bulk_coords(c, jobs, njobs, host_xyzw, false);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return SOPB_OK;
}

// ===========================================================================
// No-allocation entry point: TEA coupling coefficients of one system.
//
// Some callers cannot call cudaMalloc: a host program that owns every byte of
// device memory through its own pool and forbids libraries to allocate
// behind it (a molecular-dynamics engine or a plugin host), or code that runs
// where an allocation would stall or break the stream it is ordering work on.
// This entry point serves them.  It runs the same kernels as the TEA updater
// of sopb_run (the O(N^2) epsilon sums in j slices, the per-bead reduction
// and the FP64 beta') on caller-owned inputs and outputs, and keeps its slice
// partials in the file-scope array below instead of allocated scratch.
//
// The array is a fixed part of the library image: every GPU that loads the
// library holds its 4 MiB until the process exits.  Every call shares it and
// it keeps the last call's contents; each call overwrites every slot it reads
// before reading it, so nothing has to start at zero.  Calls that overlap on
// the GPU (two streams, or two host threads) race on the array and must be
// ordered by the caller.  The first call in each CUDA context does the set-up
// (it looks up the array's device address in that context with
// cudaGetSymbolAddress); make that first call before any stream capture.  A
// context is told apart by its driver-assigned id, unique for the life of the
// process, so a context made with cuCtxCreate, or the new primary context
// after a cudaDeviceReset, gets its own look-up instead of a stale address.
// ===========================================================================

namespace {

// Slice partials: at most kNoAllocSlots float4, i.e. n x (number of j slices).
constexpr int kNoAllocSlots = 1 << 18;   // 4 MiB
static __device__ __align__(256) float4 s_tea_partials[kNoAllocSlots];

// Set-up cache: the device address of s_tea_partials and the SM count, per
// CUDA context.  Host code cannot use the symbol itself as a device address.
struct NoAllocSetup {
    unsigned long long ctx_id;   // 0 = empty slot (driver ids start at 1)
    float4* part;
    int sms;
};
constexpr int kNoAllocContexts = 64;
std::mutex g_mutex;
NoAllocSetup g_setup[kNoAllocContexts] = {};
int g_setup_next = 0;             // slot to reuse once all are taken
PFN_cuCtxGetId_v12000 g_ctx_get_id = nullptr;

// Id of the current CUDA context (cuCtxGetId through the runtime's driver
// entry-point table, so the library needs no link against libcuda).  With
// no context current yet, the current device's primary context is made
// current first.  Called with g_mutex held.
int current_context_id(unsigned long long* id) {
    if (!g_ctx_get_id) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            cudaGetLastError();
            return SOPB_ERR_CUDA;
        }
        g_ctx_get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(fn);
    }
    if (g_ctx_get_id(nullptr, id) == CUDA_SUCCESS && *id != 0) return SOPB_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaSetDevice(dev) != cudaSuccess) {
        cudaGetLastError();
        return SOPB_ERR_NODEVICE;
    }
    if (g_ctx_get_id(nullptr, id) == CUDA_SUCCESS && *id != 0) return SOPB_OK;
    return SOPB_ERR_CUDA;
}

// Unlisted branch of k_tea_eps_partial on plain pointers.
__global__ void __launch_bounds__(kHiTile)
k_tea_eps_partial_raw(const float4* __restrict__ x, int n, float a, int jsplit, float4* __restrict__ part) {
    __shared__ float4 xs[kHiTile];
    const int i = blockIdx.x * kHiTile + threadIdx.x, s = blockIdx.y;
    const float4 xi = x[i < n ? i : 0];
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    const int span = ((n + jsplit - 1) / jsplit + kHiTile - 1) / kHiTile * kHiTile;
    const int j0 = s * span, j1 = min(n, j0 + span);
    for (int t0 = j0; t0 < j1; t0 += kHiTile) {
        __syncthreads();
        if (t0 + threadIdx.x < j1) xs[threadIdx.x] = x[t0 + threadIdx.x];
        __syncthreads();
        const int cnt = min(kHiTile, j1 - t0);
        if (i < n)
            for (int q = 0; q < cnt; ++q)
                if (t0 + q != i) eps_stats(xi, xs[q], a, acc);
    }
    if (i < n) part[(size_t)s * n + i] = acc;
}

__global__ void __launch_bounds__(kGridBlock)
k_tea_eps_reduce_raw(const float4* __restrict__ part, int n, int jsplit, float4* __restrict__ ci4) {
    for (int i = blockIdx.x * kGridBlock + threadIdx.x; i < n; i += gridDim.x * kGridBlock) {
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int s = 0; s < jsplit; ++s) {
            const float4 p = part[(size_t)s * n + i];
            a.x += p.x; a.y += p.y; a.z += p.z; a.w += p.w;
        }
        ci4[i] = a;
    }
}

// k_tea_beta's arithmetic: epsilon averaged over the 3N(3N-3) off-diagonal
// entries in FP64, beta' = (1 - sqrt(1 - a)) / a, 0.5 when |a| < 1e-7.
__global__ void __launch_bounds__(256)
k_tea_beta_raw(const float4* __restrict__ ci4, int n, float* __restrict__ out) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) s += (double)ci4[i].w;
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double eps = red[0];
        if (n > 1) eps /= 3. * n * (3. * n - 3.);
        if (eps > 1.0) eps = 1.0;
        const double a = (3. * n - 1.) * eps * eps - (3. * n - 2.) * eps;
        const double beta = fabs(a) < 1e-7 ? 0.5 : (1. - sqrt(1. - a)) / a;
        out[0] = (float)beta;
        out[1] = (float)eps;
    }
}

}  // namespace

// TEA coupling coefficients of one system, allocating nothing.  See the
// declaration in include/sopb.h.
extern "C" int sopb_tea_coefficients_noalloc(const float* d_xyzw, int32_t n, float hi_a, float* d_ci4,
                                             float* d_beta_eps, void* stream) {
    if (!d_xyzw || !d_ci4 || !d_beta_eps || n < 1 || !(hi_a > 0.0f)) return SOPB_ERR_INVALID;
    // float4 loads and stores need 16-byte alignment, the two floats 4 bytes
    if ((((uintptr_t)d_xyzw | (uintptr_t)d_ci4) & 15) || ((uintptr_t)d_beta_eps & 3)) return SOPB_ERR_INVALID;
    if (n > kNoAllocSlots) return SOPB_ERR_CAPACITY;   // one slice of n partials must fit the array
    float4* part = nullptr;
    int sms = 0;
    {
        // set-up, once per CUDA context, with that context current
        std::lock_guard<std::mutex> lock(g_mutex);
        unsigned long long id = 0;
        const int rc = current_context_id(&id);
        if (rc != SOPB_OK) return rc;
        const NoAllocSetup* hit = nullptr;
        for (const NoAllocSetup& e : g_setup)
            if (e.ctx_id == id) { hit = &e; break; }
        if (!hit) {
            void* p = nullptr;
            int dev = 0, nsm = 0;
            if (cudaGetSymbolAddress(&p, s_tea_partials) != cudaSuccess || !p || cudaGetDevice(&dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 1) {
                cudaGetLastError();
                return SOPB_ERR_CUDA;
            }
            int slot = -1;
            for (int k = 0; k < kNoAllocContexts && slot < 0; ++k)
                if (g_setup[k].ctx_id == 0) slot = k;
            if (slot < 0) slot = g_setup_next++ % kNoAllocContexts;
            g_setup[slot] = NoAllocSetup{id, static_cast<float4*>(p), nsm};
            hit = &g_setup[slot];
        }
        part = hit->part;
        sms = hit->sms;
    }
    // the TEA updater's slicing (4 CTAs per SM), capped by the array
    const int itiles = (n + kHiTile - 1) / kHiTile;
    int jsplit = std::max(1, std::min((4 * sms + itiles - 1) / itiles, itiles));
    jsplit = std::min(jsplit, kNoAllocSlots / n);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float4* x = reinterpret_cast<const float4*>(d_xyzw);
    float4* ci4 = reinterpret_cast<float4*>(d_ci4);
    k_tea_eps_partial_raw<<<dim3(itiles, jsplit), kHiTile, 0, st>>>(x, n, hi_a, jsplit, part);
    const int rb = std::max(1, std::min((n + kGridBlock - 1) / kGridBlock, sms * 8));
    k_tea_eps_reduce_raw<<<rb, kGridBlock, 0, st>>>(part, n, jsplit, ci4);
    k_tea_beta_raw<<<1, 256, 0, st>>>(ci4, n, d_beta_eps);
    if (cudaGetLastError() != cudaSuccess) return SOPB_ERR_CUDA;
    return SOPB_OK;
}
