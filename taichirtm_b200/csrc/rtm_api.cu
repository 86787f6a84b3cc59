// Host side of librtm_b200: plans, time loops and the extern "C" entry
// points declared in include/rtm_b200.h.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rtm_b200.h"
#include "adjoint_kernels.cuh"
#include "checkpoint_kernels.cuh"
#include "aux_kernels.cuh"
#include "step2_kernels.cuh"
#include "adjoint2_kernels.cuh"
#include "plan_host.h"
#include "step_kernels.cuh"

using namespace rtm;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (expr);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail(e_ == cudaErrorMemoryAllocation ? RTM_E_NOMEM : RTM_E_CUDA,     \
                        "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                      \
    } while (0)

template <typename T>
int dalloc(T **p, size_t n) {
    *p = nullptr;
    if (n == 0) return 0;
    CUDA_TRY(cudaMalloc((void **)p, n * sizeof(T)));
    return 0;
}

// NVTX range around an entry point: the phases show up by name in Nsight
// Systems; without a profiler attached it costs a call that returns.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

}  // namespace

struct rtm_plan {
    rtm_grid g{};
    int nshots = 0;
    int vec = 4, rows = 32, warps = 4, prefetch = 1;
    int tsteps = 1;  // time steps per launch of the propagation loops (1 or 2)
    int pitch = 0;
    int nstrips = 0;
    std::vector<ShotDev> shots_h;
    ShotDev *d_shots = nullptr;
    int4 *d_work = nullptr;
    int n_work = 0;
    int *d_src_ptr = nullptr, *d_rec_ptr = nullptr;
    int2 *d_src_ent = nullptr, *d_rec_ent = nullptr;
    int nsrc_total = 0, nrec_total = 0;
    size_t n_src_ptr = 0, n_rec_ptr = 0, n_src_ent = 0, n_rec_ent = 0;  // table lengths
    long long rows_total = 0;  // sum of nx over shots
    size_t state_floats = 0;   // per field, per buffer
    float *d_state[2][NFIELD] = {};
    float *d_mat[NMAT] = {};
    float *d_surface = nullptr;
    bool has_surface = false;
    float *d_sponge = nullptr;
    float *d_img[3] = {}, *d_imgc[3] = {};
    float *d_seis_t = nullptr, *d_obs_t = nullptr;
    int *d_flags = nullptr;
    int *d_fail_seq = nullptr;  // per shot: first failing launch of the current loop
    // Scratch of the checkpointed entry points (rtm_adjoint,
    // rtm_backward_checkpointed): kept and reused from call to call, grown
    // when a call needs more, freed with the plan.  A cudaMalloc / cudaFree
    // pair of several GB per call costs a device-wide synchronisation and
    // page mapping on every gradient.
    float *d_scratch = nullptr;
    size_t scratch_floats = 0;
    bool model_set = false;
    long long launches = 0;
    // CUDA-graph replay of time loops (tune.graphs): one cached executable per
    // loop kind, keyed by every pointer and schedule value it bakes in.
    struct GraphCache {
        std::vector<unsigned long long> key;
        cudaGraphExec_t exec = nullptr;
    };
    bool use_graphs = false;
    cudaStream_t gstream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    GraphCache g_fwd, g_bwd, g_ckpt;
    // Host step callback (rtm_plan_set_callback) and the ping-pong buffer that
    // holds the latest state of rtm_forward / rtm_backward (-1: none).
    rtm_step_callback cb = nullptr;
    void *cb_user = nullptr;
    int cb_every = 0;
    int live = -1;
};

namespace {

bool field_active(int modes, int f) {
    if (f == F_U || f == F_W || f == F_SXX || f == F_SZZ || f == F_SXZ) return modes & RTM_PSV;
    return modes & RTM_SH;
}
bool comp_active(int modes, int c) { return c == 1 ? (modes & RTM_SH) : (modes & RTM_PSV); }

// The plan's scratch, at least n floats (contents undefined).
int plan_scratch(rtm_plan *p, size_t n, float **out) {
    if (p->scratch_floats < n) {
        if (p->d_scratch) cudaFree(p->d_scratch);
        p->d_scratch = nullptr;
        p->scratch_floats = 0;
        if (int rc = dalloc(&p->d_scratch, n)) return rc;
        p->scratch_floats = n;
    }
    *out = p->d_scratch;
    return 0;
}

void plan_free(rtm_plan *p) {
    auto F = [](void *q) { if (q) cudaFree(q); };
    F(p->d_shots); F(p->d_work); F(p->d_src_ptr); F(p->d_rec_ptr); F(p->d_src_ent); F(p->d_rec_ent);
    for (int b = 0; b < 2; ++b) for (int f = 0; f < NFIELD; ++f) F(p->d_state[b][f]);
    for (int m = 0; m < NMAT; ++m) F(p->d_mat[m]);
    F(p->d_surface); F(p->d_sponge);
    for (int c = 0; c < 3; ++c) { F(p->d_img[c]); F(p->d_imgc[c]); }
    F(p->d_seis_t); F(p->d_obs_t); F(p->d_flags); F(p->d_fail_seq); F(p->d_scratch);
    for (auto *gc : {&p->g_fwd, &p->g_bwd, &p->g_ckpt})
        if (gc->exec) cudaGraphExecDestroy(gc->exec);
    if (p->ev_in) cudaEventDestroy(p->ev_in);
    if (p->ev_out) cudaEventDestroy(p->ev_out);
    if (p->gstream) cudaStreamDestroy(p->gstream);
}

// Buffers one call may touch, for the bounds-checking build (debug_bounds.cuh):
// the plan's allocations and the caller's buffers, with their sizes.  In the
// normal build every method is empty.
struct BoundsScope {
#ifdef RTM_BOUNDS_CHECK
    std::vector<std::pair<unsigned long long, unsigned long long>> r;
    void add(const void *ptr, size_t bytes) {
        if (ptr && bytes) r.push_back({(unsigned long long)(uintptr_t)ptr, (unsigned long long)(uintptr_t)ptr + bytes});
    }
    int begin(cudaStream_t s) {
        DbgTable t{};
        if (r.size() > (size_t)DBG_MAX_RANGES) return fail(RTM_E_STATE, "bounds check: %zu buffers > %d", r.size(), DBG_MAX_RANGES);
        for (size_t k = 0; k < r.size(); ++k) {
            t.begin[k] = r[k].first;
            t.end[k] = r[k].second;
        }
        t.n = (int)r.size();
        const unsigned long long zero = 0;
        CUDA_TRY(cudaMemcpyToSymbolAsync(g_dbg_table, &t, sizeof t, 0, cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaMemcpyToSymbolAsync(g_dbg_bad, &zero, sizeof zero, 0, cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaStreamSynchronize(s));  // the table is a stack object's copy: upload before returning
        return 0;
    }
    int end(cudaStream_t s) {
        unsigned long long bad = 0, first = 0;
        CUDA_TRY(cudaMemcpyFromSymbolAsync(&bad, g_dbg_bad, sizeof bad, 0, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaMemcpyFromSymbolAsync(&first, g_dbg_first, sizeof first, 0, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        DbgTable none{};
        CUDA_TRY(cudaMemcpyToSymbol(g_dbg_table, &none, sizeof none));  // later calls of other entry points: unchecked until set
        if (bad) return fail(RTM_E_CUDA, "bounds check: %llu accesses outside every buffer (first at 0x%llx)", bad, first);
        return 0;
    }
#else
    void add(const void *, size_t) {}
    int begin(cudaStream_t) { return 0; }
    int end(cudaStream_t) { return 0; }
#endif
    void add_plan(const rtm_plan *p) {
        const size_t F = sizeof(float);
        add(p->d_shots, p->shots_h.size() * sizeof(ShotDev));
        add(p->d_work, (size_t)p->n_work * sizeof(int4));
        add(p->d_src_ptr, p->n_src_ptr * sizeof(int));
        add(p->d_rec_ptr, p->n_rec_ptr * sizeof(int));
        add(p->d_src_ent, p->n_src_ent * sizeof(int2));
        add(p->d_rec_ent, p->n_rec_ent * sizeof(int2));
        add(p->d_flags, p->nshots * sizeof(int));
        add(p->d_fail_seq, p->nshots * sizeof(int));
        add(p->d_sponge, (size_t)std::max(p->g.absorbing_frame, 1) * F);
        for (int b = 0; b < 2; ++b)
            for (int f = 0; f < NFIELD; ++f) add(p->d_state[b][f], p->state_floats * F);
        const size_t mat = (size_t)(p->g.nx + 2) * p->pitch * F;
        for (int m = 0; m < NMAT; ++m) add(p->d_mat[m], mat);
        add(p->d_surface, mat);
        for (int c = 0; c < 3; ++c) {
            add(p->d_img[c], (size_t)p->rows_total * p->pitch * F);
            add(p->d_imgc[c], (size_t)p->rows_total * p->pitch * F);
        }
        const size_t seis = std::max<size_t>((size_t)3 * p->g.nt * p->nrec_total, 1) * F;
        add(p->d_seis_t, seis);
        add(p->d_obs_t, seis);
    }
};

// Run a time loop: directly on s, or (use_graphs) as a CUDA graph captured on
// the plan's own stream the first time this key is seen and replayed after.
// The caller's stream and the plan stream are ordered by two events.
template <typename Body>
int run_loop(rtm_plan *p, rtm_plan::GraphCache &gc, const std::vector<unsigned long long> &key,
             cudaStream_t s, Body &&body) {
    if (!p->use_graphs) return body(s);
    if (!p->gstream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&p->gstream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&p->ev_out, cudaEventDisableTiming));
    }
    if (!gc.exec || gc.key != key) {
        if (gc.exec) {
            cudaGraphExecDestroy(gc.exec);
            gc.exec = nullptr;
        }
        CUDA_TRY(cudaStreamBeginCapture(p->gstream, cudaStreamCaptureModeThreadLocal));
        const int rc = body(p->gstream);
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(p->gstream, &graph);
        if (rc || e != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            return rc ? rc : fail(RTM_E_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
        }
        const cudaError_t e2 = cudaGraphInstantiate(&gc.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e2 != cudaSuccess) {
            gc.exec = nullptr;
            return fail(RTM_E_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e2));
        }
        gc.key = key;
    }
    CUDA_TRY(cudaEventRecord(p->ev_in, s));
    CUDA_TRY(cudaStreamWaitEvent(p->gstream, p->ev_in, 0));
    CUDA_TRY(cudaGraphLaunch(gc.exec, p->gstream));
    CUDA_TRY(cudaEventRecord(p->ev_out, p->gstream));
    CUDA_TRY(cudaStreamWaitEvent(s, p->ev_out, 0));
    return 0;
}

unsigned long long U(const void *ptr) { return (unsigned long long)(uintptr_t)ptr; }

template <int DIR, int MODE, int VEC, int PFM>
cudaError_t launch_step(const StepParams &sp, int warps, cudaStream_t s) {
    const int threads = 32 * warps;
    const int blocks = (sp.n_work + warps - 1) / warps;
    size_t smem = 0;
    if constexpr (PFM == 3) {
        constexpr size_t kMaxSmem = 227 * 1024;  // per-block opt-in limit
        smem = (size_t)warps * async_smem_per_warp<MODE, VEC>();
        if (smem > kMaxSmem) return cudaErrorInvalidConfiguration;
        static bool attr_set = false;  // per instantiation; raises the 48 KB default
        if (!attr_set) {
            const size_t want = std::min<size_t>(8 * async_smem_per_warp<MODE, VEC>(), kMaxSmem);
            cudaError_t e = cudaFuncSetAttribute(step_kernel<DIR, MODE, VEC, PFM>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)want);
            if (e != cudaSuccess) return e;
            attr_set = true;
        }
    }
    step_kernel<DIR, MODE, VEC, PFM><<<blocks, threads, smem, s>>>(sp);
    return cudaGetLastError();
}

template <int DIR, int MODE, int VEC>
cudaError_t launch_pf(const StepParams &sp, int pfm, int warps, cudaStream_t s) {
    switch (pfm) {
        case 0: return launch_step<DIR, MODE, VEC, 0>(sp, warps, s);
        case 1: return launch_step<DIR, MODE, VEC, 1>(sp, warps, s);
        case 2: return launch_step<DIR, MODE, VEC, 2>(sp, warps, s);
        default: return launch_step<DIR, MODE, VEC, 3>(sp, warps, s);
    }
}

// vec: columns per lane in bits 0-7, prefetch mode (0/1/2) in bits 8-9
template <int DIR, int MODE>
cudaError_t launch_vec(const StepParams &sp, int vec, int warps, cudaStream_t s) {
    const int pfm = (vec >> 8) & 3;
    switch (vec & 0xff) {
        case 1: return launch_pf<DIR, MODE, 1>(sp, pfm, warps, s);
        case 2: return launch_pf<DIR, MODE, 2>(sp, pfm, warps, s);
        default: return launch_pf<DIR, MODE, 4>(sp, pfm, warps, s);
    }
}

template <int DIR>
cudaError_t launch_mode(const StepParams &sp, int modes, int vec, int warps, cudaStream_t s) {
    switch (modes) {
        case RTM_PSV: return launch_vec<DIR, RTM_PSV>(sp, vec, warps, s);
        case RTM_SH: return launch_vec<DIR, RTM_SH>(sp, vec, warps, s);
        default: return launch_vec<DIR, RTM_BOTH>(sp, vec, warps, s);
    }
}

template <int DIR, int MODE, int VEC, bool RING, bool STOREA = false, bool CKPT = false, bool UNI = false>
cudaError_t launch_step2(const StepParams &sp, int warps, cudaStream_t s) {
    size_t smem = 0;
    if constexpr (RING) {
        constexpr size_t kMaxSmem = 227 * 1024;  // per-block opt-in limit
        smem = (size_t)warps * ring2_smem_per_warp<MODE, VEC>();
        if (smem > kMaxSmem) return cudaErrorInvalidConfiguration;
        static bool attr_set = false;  // per instantiation; raises the 48 KB default
        if (!attr_set) {
            const size_t want = std::min<size_t>(8 * ring2_smem_per_warp<MODE, VEC>(), kMaxSmem);
            cudaError_t e = cudaFuncSetAttribute(step2_kernel<DIR, MODE, VEC, RING, STOREA, CKPT, UNI>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)want);
            if (e != cudaSuccess) return e;
            attr_set = true;
        }
    }
    step2_kernel<DIR, MODE, VEC, RING, STOREA, CKPT, UNI><<<(sp.n_work + warps - 1) / warps, 32 * warps, smem, s>>>(sp);
    return cudaGetLastError();
}

// Checkpoint-storing forward P-SV launches (sp.ck set): one step or two
// steps, the output state also packed into the compressed slot.
template <int VEC, int PFM>
cudaError_t launch_step_ckpt(const StepParams &sp, int warps, cudaStream_t s) {
    const int threads = 32 * warps;
    const int blocks = (sp.n_work + warps - 1) / warps;
    size_t smem = 0;
    if constexpr (PFM == 3) {
        constexpr size_t kMaxSmem = 227 * 1024;
        smem = (size_t)warps * async_smem_per_warp<RTM_PSV, VEC>();
        if (smem > kMaxSmem) return cudaErrorInvalidConfiguration;
        static bool attr_set = false;
        if (!attr_set) {
            const size_t want = std::min<size_t>(8 * async_smem_per_warp<RTM_PSV, VEC>(), kMaxSmem);
            cudaError_t e = cudaFuncSetAttribute(step_kernel<0, RTM_PSV, VEC, PFM, true>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)want);
            if (e != cudaSuccess) return e;
            attr_set = true;
        }
    }
    step_kernel<0, RTM_PSV, VEC, PFM, true><<<blocks, threads, smem, s>>>(sp);
    return cudaGetLastError();
}
template <int VEC>
cudaError_t launch_pf_ckpt(const StepParams &sp, int pfm, int warps, cudaStream_t s) {
    switch (pfm) {
        case 0: return launch_step_ckpt<VEC, 0>(sp, warps, s);
        case 1: return launch_step_ckpt<VEC, 1>(sp, warps, s);
        case 2: return launch_step_ckpt<VEC, 2>(sp, warps, s);
        default: return launch_step_ckpt<VEC, 3>(sp, warps, s);
    }
}
cudaError_t launch_ckpt(const StepParams &sp, bool two, int vec, int prefetch, int warps, cudaStream_t s) {
    if (two) {
        const bool ring = prefetch >= 3;
        if (vec == 2)
            return ring ? launch_step2<0, RTM_PSV, 2, true, false, true>(sp, warps, s)
                        : launch_step2<0, RTM_PSV, 2, false, false, true>(sp, warps, s);
        return ring ? launch_step2<0, RTM_PSV, 4, true, false, true>(sp, warps, s)
                    : launch_step2<0, RTM_PSV, 4, false, false, true>(sp, warps, s);
    }
    switch (vec) {
        case 1: return launch_pf_ckpt<1>(sp, prefetch, warps, s);
        case 2: return launch_pf_ckpt<2>(sp, prefetch, warps, s);
        default: return launch_pf_ckpt<4>(sp, prefetch, warps, s);
    }
}

// uni (prefetch 4): the ring kernel with the task taken from blockIdx.x,
// one warp per CTA (the plan forces warps = 1).
template <int DIR, int MODE>
cudaError_t launch_vec2(const StepParams &sp, int vec, bool ring, bool uni, int warps, cudaStream_t s) {
    if (uni) {
        if (warps != 1) return cudaErrorInvalidConfiguration;
        return vec == 2 ? launch_step2<DIR, MODE, 2, true, false, false, true>(sp, 1, s)
                        : launch_step2<DIR, MODE, 4, true, false, false, true>(sp, 1, s);
    }
    if (vec == 2) return ring ? launch_step2<DIR, MODE, 2, true>(sp, warps, s) : launch_step2<DIR, MODE, 2, false>(sp, warps, s);
    return ring ? launch_step2<DIR, MODE, 4, true>(sp, warps, s) : launch_step2<DIR, MODE, 4, false>(sp, warps, s);
}

// Forward recompute of the adjoint, P-SV: steps sp.it and sp.it2 in one
// launch, storing the state after each (sp.souta, sp.sout).
cudaError_t launch_recompute2(const StepParams &sp, int vec, int prefetch, int warps, cudaStream_t s) {
    const bool ring = prefetch >= 3;
    if (vec == 2)
        return ring ? launch_step2<0, RTM_PSV, 2, true, true>(sp, warps, s) : launch_step2<0, RTM_PSV, 2, false, true>(sp, warps, s);
    return ring ? launch_step2<0, RTM_PSV, 4, true, true>(sp, warps, s) : launch_step2<0, RTM_PSV, 4, false, true>(sp, warps, s);
}

// Two steps (sp.it, sp.it2) in one launch; vec is 2 or 4 (checked at plan
// creation); prefetch 3 selects the shared-memory material ring.
template <int DIR>
cudaError_t launch_mode2(const StepParams &sp, int modes, int vec, int prefetch, int warps, cudaStream_t s) {
    const bool ring = prefetch >= 3, uni = prefetch == 4;
    switch (modes) {
        case RTM_PSV: return launch_vec2<DIR, RTM_PSV>(sp, vec, ring, uni, warps, s);
        case RTM_SH: return launch_vec2<DIR, RTM_SH>(sp, vec, ring, uni, warps, s);
        default: return launch_vec2<DIR, RTM_BOTH>(sp, vec, ring, uni, warps, s);
    }
}

// The launches of a time loop over loop steps 0 .. nt-1: step `it` alone, or
// steps it and it+1 together when the plan runs two steps per launch and
// step `it` may be the first of a pair (pairable(it): it is not checked and
// its state need not be stored).
struct LoopLaunch {
    int it;
    bool two;
};
template <typename Pairable>
std::vector<LoopLaunch> loop_schedule(int first, int end, int tsteps, Pairable &&pairable) {
    std::vector<LoopLaunch> out;
    for (int it = first; it < end;) {
        const bool two = tsteps == 2 && it + 1 < end && pairable(it);
        out.push_back({it, two});
        it += two ? 2 : 1;
    }
    return out;
}

// The host callback after launch number `seq` (1-based) at step `step`:
// waits for the stream, skips the call once every shot stopped in an earlier
// launch (a failed check ends the reference's loop before its next
// callback), and turns a non-zero return into RTM_E_CALLBACK.
int call_back(rtm_plan *p, int seq, int step, cudaStream_t s) {
    CUDA_TRY(cudaStreamSynchronize(s));
    std::vector<int> fs(p->nshots);
    CUDA_TRY(cudaMemcpy(fs.data(), p->d_fail_seq, p->nshots * sizeof(int), cudaMemcpyDeviceToHost));
    bool alive = false;
    for (int v : fs) alive = alive || v >= seq;
    if (!alive) return 0;
    if (int rc = p->cb(p->cb_user, step))
        return fail(RTM_E_CALLBACK, "the step callback returned %d at step %d", rc, step);
    return 0;
}

void fill_common(const rtm_plan *p, StepParams &sp) {
    std::memset(&sp, 0, sizeof sp);
    const double dt = 1.0 / p->g.fs;
    sp.nz = p->g.nz;
    sp.pitch = p->pitch;
    sp.nt = p->g.nt;
    sp.fw = p->g.absorbing_frame;
    sp.dt = (float)dt;
    sp.inv_dx = (float)(1.0 / p->g.dx);
    sp.inv_dz = (float)(1.0 / p->g.dz);
    sp.src_factor = (float)(dt * p->g.dx * p->g.dz);  // forward_modeling.py:430
    sp.sponge = p->d_sponge;
    sp.work = p->d_work;
    sp.n_work = p->n_work;
    sp.shots = p->d_shots;
    for (int m = 0; m < NMAT; ++m) sp.mat[m] = p->d_mat[m];
    sp.surface = p->has_surface ? p->d_surface : nullptr;
    sp.src_ptr = p->d_src_ptr;
    sp.src_ent = p->d_src_ent;
    sp.rec_ptr = p->d_rec_ptr;
    sp.rec_ent = p->d_rec_ent;
    sp.nrec_total = p->nrec_total;
    sp.flags = p->d_flags;
    sp.fail_seq = p->d_fail_seq;
    sp.snap_k = -1;
}

int zero_state(rtm_plan *p, cudaStream_t s) {
    for (int b = 0; b < 2; ++b)
        for (int f = 0; f < NFIELD; ++f)
            if (p->d_state[b][f])
                CUDA_TRY(cudaMemsetAsync(p->d_state[b][f], 0, p->state_floats * sizeof(float), s));
    CUDA_TRY(cudaMemsetAsync(p->d_flags, 0, p->nshots * sizeof(int), s));
    CUDA_TRY(cudaMemsetAsync(p->d_fail_seq, 0x7f, p->nshots * sizeof(int), s));  // 0x7f7f7f7f: none
    return 0;
}

}  // namespace

extern "C" {

const char *rtm_version(void) {
#ifdef RTM_BOUNDS_CHECK
    return "rtm_b200 1.0 (sm_100a, bounds-checking build)";
#else
    return "rtm_b200 1.0 (sm_100a)";
#endif
}

int rtm_bounds_probe(const rtm_plan *p, const void *buf, size_t buf_bytes, const void *ptr, size_t bytes,
                     int32_t *inside) {
#ifdef RTM_BOUNDS_CHECK
    if (!p || !inside) return fail(RTM_E_ARG, "null argument");
    BoundsScope bs;
    bs.add_plan(p);
    bs.add(buf, buf_bytes);
    if (int rc = bs.begin(0)) return rc;
    bounds_probe_kernel<<<1, 1>>>(ptr, (unsigned)bytes);
    CUDA_TRY(cudaGetLastError());
    int v = 0;
    CUDA_TRY(cudaMemcpyFromSymbol(&v, g_dbg_probe, sizeof v));
    *inside = v;
    const unsigned long long zero = 0;
    CUDA_TRY(cudaMemcpyToSymbol(g_dbg_bad, &zero, sizeof zero));  // the probe's own count
    DbgTable none{};
    CUDA_TRY(cudaMemcpyToSymbol(g_dbg_table, &none, sizeof none));
    return RTM_OK;
#else
    (void)p; (void)buf; (void)buf_bytes; (void)ptr; (void)bytes; (void)inside;
    return fail(RTM_E_STATE, "rtm_bounds_probe needs the bounds-checking build (-DRTM_BOUNDS_CHECK)");
#endif
}
const char *rtm_last_error(void) { return g_err.c_str(); }

int rtm_plan_create(const rtm_grid *grid, int nshots, const rtm_shot *shots, const rtm_tune *tune,
                    rtm_plan **out) {
    if (!grid || !shots || !out || nshots <= 0) return fail(RTM_E_ARG, "null argument or nshots <= 0");
    *out = nullptr;
    const rtm_grid g = *grid;
    if (const char *bad = check_grid(g))
        return fail(RTM_E_ARG, "%s (nx=%d nz=%d nt=%d absorbing_frame=%d)", bad, g.nx, g.nz, g.nt, g.absorbing_frame);
    rtm_plan *p = new rtm_plan();
    p->g = g;
    p->nshots = nshots;
    if (tune) {
        if (tune->vec == 1 || tune->vec == 2 || tune->vec == 4) p->vec = tune->vec;
        if (tune->rows > 0) p->rows = tune->rows;
        if (tune->warps > 0 && tune->warps <= 8) p->warps = tune->warps;
        if (tune->prefetch >= 0 && tune->prefetch <= 4) p->prefetch = tune->prefetch;
        if (p->prefetch == 4) p->warps = 1;  // the uniform-task kernel runs one warp per CTA
        p->use_graphs = tune->graphs == 1;
        if (tune->tsteps == 2) {
            if (p->vec == 1) {
                delete p;
                return fail(RTM_E_ARG, "two steps per launch need vec 2 or 4");
            }
            p->tsteps = 2;
        }
    }
    const int W = 30 * p->vec;
    p->nstrips = (g.nz + W - 1) / W;
    p->pitch = layout_pitch(g.nz);

    // shots, row tables, work list
    std::vector<int> src_ptr, rec_ptr;
    std::vector<int2> src_ent, rec_ent;
    std::vector<int4> work;
    long long state_rows = 0;
    for (int s = 0; s < nshots; ++s) {
        const rtm_shot &sh = shots[s];
        if (sh.nx < 3 || sh.x0 < 0 || sh.x0 + sh.nx > g.nx) {
            delete p;
            return fail(RTM_E_ARG, "shot %d window [%d, %d) outside grid nx=%d", s, sh.x0, sh.x0 + sh.nx, g.nx);
        }
        if (g.absorbing_frame > sh.nx) {
            delete p;
            return fail(RTM_E_ARG, "absorbing_frame %d wider than shot %d window (%d rows)", g.absorbing_frame, s, sh.nx);
        }
        if ((sh.nsrc > 0 && !sh.src_ij) || (sh.nrec > 0 && !sh.rec_ij) || sh.nsrc < 0 || sh.nrec < 0) {
            delete p;
            return fail(RTM_E_ARG, "shot %d: bad source/receiver arrays", s);
        }
        ShotDev d{};
        d.nx = sh.nx;
        d.x0 = sh.x0;
        d.state_off = state_rows * p->pitch;
        d.row_off = p->rows_total;
        d.src_row0 = (int)src_ptr.size();
        d.rec_row0 = (int)rec_ptr.size();
        // per-row CSR, stable in the given order (duplicates accumulate in order)
        auto build = [&](int n, const int32_t *ij, int base, std::vector<int> &ptr,
                         std::vector<int2> &ent, const char *what) -> int {
            const int k = append_row_table(sh.nx, g.nz, n, ij, base, ptr, ent);
            if (k >= 0)
                return fail(RTM_E_ARG, "shot %d: %s %d at (%d, %d) outside the %dx%d window", s, what, k, ij[2 * k],
                            ij[2 * k + 1], sh.nx, g.nz);
            return 0;
        };
        if (build(sh.nsrc, sh.src_ij, p->nsrc_total, src_ptr, src_ent, "source") ||
            build(sh.nrec, sh.rec_ij, p->nrec_total, rec_ptr, rec_ent, "receiver")) {
            delete p;
            return RTM_E_ARG;
        }
        p->nsrc_total += sh.nsrc;
        p->nrec_total += sh.nrec;
        p->shots_h.push_back(d);
        state_rows += sh.nx + 2;
        p->rows_total += sh.nx;
        // Per task: bit 20 / 21 of the strip word = no source / no receiver in
        // rows [ia-2, ib+1] (every row a one- or two-step launch updates) and
        // the lanes' columns [j0 - vec, j0 + 31 vec).
        auto none_in = [&](const std::vector<int> &ptr, const std::vector<int2> &ent, int row0, int r0, int r1,
                           int c_lo, int c_hi) {
            for (int r = std::max(r0, 0); r <= std::min(r1, sh.nx - 1); ++r)
                for (int e = ptr[row0 + r]; e < ptr[row0 + r + 1]; ++e)
                    if (ent[e].x >= c_lo && ent[e].x < c_hi) return false;
            return true;
        };
        for (int ia = 0; ia < sh.nx; ia += p->rows)
            for (int st = 0; st < p->nstrips; ++st) {
                const int ib = std::min(ia + p->rows, sh.nx);
                const int j0 = st * W, c_lo = j0 - p->vec, c_hi = j0 + 31 * p->vec;
                int word = st;
                if (none_in(src_ptr, src_ent, d.src_row0, ia - 2, ib + 1, c_lo, c_hi)) word |= 1 << 20;
                if (none_in(rec_ptr, rec_ent, d.rec_row0, ia - 2, ib + 1, c_lo, c_hi)) word |= 1 << 21;
                work.push_back(make_int4(s, word, ia, ib));
            }
    }
    // Order tasks by global row so that concurrently running shots that
    // overlap read the same material rows while they are in L2.
    std::stable_sort(work.begin(), work.end(), [&](const int4 &a, const int4 &b) {
        const int ga = p->shots_h[a.x].x0 + a.z, gb = p->shots_h[b.x].x0 + b.z;
        if (ga != gb) return ga < gb;
        if (a.y != b.y) return a.y < b.y;
        return a.x < b.x;
    });
    // Tail split: the last tasks of the list (the last blocks a launch
    // dispatches) are cut into two halves of rows, so the final wave of a
    // launch is made of short tasks and the SMs run out of work closer
    // together.  Any partition of a shot's rows into tasks gives the same
    // results; a half keeps its parent's no-source / no-receiver flags, which
    // hold for any sub-range of rows.
    {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            sms = 148;
        split_tail(work, tail_split_tasks(work.size(), sms));
    }
    p->n_work = (int)work.size();
    p->state_floats = (size_t)state_rows * p->pitch;
    const size_t mat_floats = (size_t)(g.nx + 2) * p->pitch;
    const size_t img_floats = (size_t)p->rows_total * p->pitch;
    int rc = 0;
    rc |= dalloc(&p->d_shots, p->shots_h.size());
    rc |= dalloc(&p->d_work, work.size());
    rc |= dalloc(&p->d_src_ptr, src_ptr.size());
    rc |= dalloc(&p->d_rec_ptr, rec_ptr.size());
    rc |= dalloc(&p->d_src_ent, std::max<size_t>(src_ent.size(), 1));
    rc |= dalloc(&p->d_rec_ent, std::max<size_t>(rec_ent.size(), 1));
    p->n_src_ptr = src_ptr.size();
    p->n_rec_ptr = rec_ptr.size();
    p->n_src_ent = std::max<size_t>(src_ent.size(), 1);
    p->n_rec_ent = std::max<size_t>(rec_ent.size(), 1);
    rc |= dalloc(&p->d_flags, nshots);
    rc |= dalloc(&p->d_fail_seq, nshots);
    rc |= dalloc(&p->d_sponge, std::max(g.absorbing_frame, 1));
    for (int b = 0; b < 2 && !rc; ++b)
        for (int f = 0; f < NFIELD && !rc; ++f)
            if (field_active(g.modes, f)) rc |= dalloc(&p->d_state[b][f], p->state_floats);
    for (int m = 0; m < NMAT && !rc; ++m) {
        const bool need = (m <= M_MXZ) ? (g.modes & RTM_PSV) : (g.modes & RTM_SH);
        if (need) rc |= dalloc(&p->d_mat[m], mat_floats);
    }
    rc |= dalloc(&p->d_surface, mat_floats);
    for (int c = 0; c < 3 && !rc; ++c)
        if (comp_active(g.modes, c)) {
            rc |= dalloc(&p->d_img[c], img_floats);
            rc |= dalloc(&p->d_imgc[c], img_floats);
        }
    rc |= dalloc(&p->d_seis_t, std::max<size_t>((size_t)3 * g.nt * p->nrec_total, 1));
    rc |= dalloc(&p->d_obs_t, std::max<size_t>((size_t)3 * g.nt * p->nrec_total, 1));
    if (rc) {
        plan_free(p);
        delete p;
        return rc < 0 ? rc : RTM_E_NOMEM;
    }
    const std::vector<float> prof = sponge_profile(g.absorbing_frame);
    auto H2D = [](void *dst, const void *src, size_t bytes) {
        return bytes ? cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
    };
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = H2D(p->d_shots, p->shots_h.data(), p->shots_h.size() * sizeof(ShotDev));
    if (e == cudaSuccess) e = H2D(p->d_work, work.data(), work.size() * sizeof(int4));
    if (e == cudaSuccess) e = H2D(p->d_src_ptr, src_ptr.data(), src_ptr.size() * sizeof(int));
    if (e == cudaSuccess) e = H2D(p->d_rec_ptr, rec_ptr.data(), rec_ptr.size() * sizeof(int));
    if (e == cudaSuccess) e = H2D(p->d_src_ent, src_ent.data(), src_ent.size() * sizeof(int2));
    if (e == cudaSuccess) e = H2D(p->d_rec_ent, rec_ent.data(), rec_ent.size() * sizeof(int2));
    if (e == cudaSuccess) e = H2D(p->d_sponge, prof.data(), prof.size() * sizeof(float));
    if (e != cudaSuccess) {
        plan_free(p);
        delete p;
        return fail(RTM_E_CUDA, "plan upload failed: %s", cudaGetErrorString(e));
    }
    *out = p;
    return RTM_OK;
}

int rtm_plan_destroy(rtm_plan *p) {
    if (!p) return RTM_OK;
    plan_free(p);
    delete p;
    return RTM_OK;
}

int rtm_plan_pitch(const rtm_plan *p) { return p ? p->pitch : 0; }

size_t rtm_plan_snapshot_floats(const rtm_plan *p, int nsnap) {
    if (!p || nsnap <= 0) return 0;
    return (size_t)nsnap * (size_t)p->rows_total * (size_t)p->pitch;
}

long long rtm_plan_launch_count(const rtm_plan *p) { return p ? p->launches : 0; }

int rtm_plan_set_callback(rtm_plan *p, int forward_every, rtm_step_callback cb, void *user) {
    if (!p) return fail(RTM_E_ARG, "null plan");
    if (cb && forward_every < 0) return fail(RTM_E_ARG, "forward_every < 0");
    p->cb = cb;
    p->cb_user = cb ? user : nullptr;
    p->cb_every = cb ? forward_every : 0;
    return RTM_OK;
}

int rtm_plan_wavefield(const rtm_plan *p, int shot, float *u, float *v, float *w, rtm_stream_t stream) {
    if (!p) return fail(RTM_E_ARG, "null plan");
    if (shot < 0 || shot >= p->nshots) return fail(RTM_E_ARG, "shot %d outside [0, %d)", shot, p->nshots);
    if (p->live < 0) return fail(RTM_E_STATE, "no wavefield: rtm_forward / rtm_backward has not run");
    cudaStream_t s = (cudaStream_t)stream;
    const ShotDev &d = p->shots_h[shot];
    const int nz = p->g.nz;
    float *dst[3] = {u, v, w};
    const int field[3] = {F_U, F_V, F_W};
    for (int c = 0; c < 3; ++c) {
        if (!dst[c]) continue;
        const float *src = p->d_state[p->live][field[c]];
        if (!src) {  // a mode the plan does not propagate: zero
            CUDA_TRY(cudaMemsetAsync(dst[c], 0, (size_t)d.nx * nz * sizeof(float), s));
            continue;
        }
        CUDA_TRY(cudaMemcpy2DAsync(dst[c], (size_t)nz * sizeof(float), src + d.state_off + p->pitch + COL_OFF,
                                   (size_t)p->pitch * sizeof(float), (size_t)nz * sizeof(float), (size_t)d.nx,
                                   cudaMemcpyDeviceToDevice, s));
    }
    return RTM_OK;
}

int rtm_plan_set_model(rtm_plan *p, const float *mu, const float *lam, const float *rho,
                       const float *surface, rtm_stream_t stream) {
    NvtxRange nvtx_range("rtm_plan_set_model");
    if (!p || !mu || !lam || !rho) return fail(RTM_E_ARG, "null model pointer");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t mat_floats = (size_t)(p->g.nx + 2) * p->pitch;
    for (int m = 0; m < NMAT; ++m)
        if (p->d_mat[m]) CUDA_TRY(cudaMemsetAsync(p->d_mat[m], 0, mat_floats * sizeof(float), s));
    CUDA_TRY(cudaMemsetAsync(p->d_surface, 0, mat_floats * sizeof(float), s));
    const long long n = (long long)p->g.nx * p->g.nz;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    setup_material_kernel<<<blocks, 256, 0, s>>>(
        mu, lam, rho, surface, p->g.nx, p->g.nz, p->pitch, p->d_mat[M_IRU], p->d_mat[M_IRW],
        p->d_mat[M_LAM], p->d_mat[M_MU], p->d_mat[M_MXZ], p->d_mat[M_IR], p->d_mat[M_MYX],
        p->d_mat[M_MYZ], surface ? p->d_surface : nullptr);
    CUDA_TRY(cudaGetLastError());
    p->has_surface = surface != nullptr;
    p->model_set = true;
    return RTM_OK;
}

static int transpose(const float *in, float *out, int planes, int rows, int cols, cudaStream_t s) {
    if (rows == 0 || cols == 0) return 0;
    dim3 grid((cols + 31) / 32, (rows + 31) / 32, planes);
    transpose_kernel<<<grid, dim3(32, 8), 0, s>>>(in, out, rows, cols);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

int rtm_forward(rtm_plan *p, const float *wavelets, float *seis, int save, int isnap, float *snap_u,
                float *snap_v, float *snap_w, int32_t *isnaps_out, int check_interval,
                int32_t *flags, rtm_stream_t stream) {
    NvtxRange nvtx_range("rtm_forward");
    if (!p) return fail(RTM_E_ARG, "null plan");
    if (!p->model_set) return fail(RTM_E_STATE, "rtm_plan_set_model has not been called");
    if (p->nsrc_total > 0 && !wavelets) return fail(RTM_E_ARG, "null wavelets");
    if (check_interval < 0) return fail(RTM_E_ARG, "check_interval < 0");
    const int nt = p->g.nt;
    int nsnap = 0;
    if (save) {
        if (isnap <= 0) return fail(RTM_E_ARG, "isnap must be positive");
        nsnap = nt / isnap;  // forward_modeling.py:531
        float *sp[3] = {snap_u, snap_v, snap_w};
        for (int c = 0; c < 3; ++c)
            if (comp_active(p->g.modes, c) && nsnap > 0 && !sp[c])
                return fail(RTM_E_ARG, "snapshot buffer %d is null", c);
    }
    cudaStream_t s = (cudaStream_t)stream;
    BoundsScope bs;
    bs.add_plan(p);
    bs.add(wavelets, (size_t)3 * p->nsrc_total * nt * sizeof(float));
    bs.add(seis, (size_t)3 * p->nrec_total * nt * sizeof(float));
    if (save)
        for (float *b : {snap_u, snap_v, snap_w}) bs.add(b, rtm_plan_snapshot_floats(p, nsnap) * sizeof(float));
    if (int rc = bs.begin(s)) return rc;
    if (int rc = zero_state(p, s)) return rc;
    // Snapshot slots the time loop never reaches ((k+1)*isnap > nt-1) stay
    // zero, like the reference's zero-initialised fields (fm:533-535).
    if (save)
        for (int k = 0; k < nsnap; ++k) {
            if ((long long)(k + 1) * isnap <= nt - 1) continue;
            float *sp3[3] = {snap_u, snap_v, snap_w};
            for (int c = 0; c < 3; ++c) {
                if (!comp_active(p->g.modes, c) || !sp3[c]) continue;
                for (const ShotDev &d : p->shots_h) {
                    const size_t off = ((size_t)nsnap * d.row_off + (size_t)k * d.nx) * p->pitch;
                    CUDA_TRY(cudaMemsetAsync(sp3[c] + off, 0, (size_t)d.nx * p->pitch * sizeof(float), s));
                }
            }
        }
    const size_t nseis = (size_t)3 * nt * p->nrec_total;
    if (nseis) CUDA_TRY(cudaMemsetAsync(p->d_seis_t, 0, nseis * sizeof(float), s));
    StepParams sp;
    fill_common(p, sp);
    sp.code_base = 1;
    const size_t plane = (size_t)nt * p->nrec_total;
    for (int c = 0; c < 3; ++c) {
        sp.wav[c] = wavelets ? wavelets + (size_t)c * p->nsrc_total * nt : nullptr;
        sp.seis[c] = p->d_seis_t + c * plane;
    }
    sp.snap[0] = snap_u;
    sp.snap[1] = snap_v;
    sp.snap[2] = snap_w;
    sp.nsnap = nsnap;
    p->launches = 0;
    auto check_at = [&](int it) { return check_interval > 0 && it % check_interval == 0; };
    auto snap_at = [&](int it) {
        const int k = (save && it % isnap == 0 && it != 0) ? it / isnap - 1 : -1;  // fm:569-570
        return k < nsnap ? k : -1;
    };
    // display_callback steps, it % every == 0 (forward_modeling.py:553-559):
    // a launch ends at each of them
    auto cb_at = [&](int it) { return p->cb && p->cb_every > 0 && it % p->cb_every == 0; };
    const std::vector<LoopLaunch> sched =
        loop_schedule(0, nt, p->tsteps, [&](int it) { return !check_at(it) && !cb_at(it); });
    auto loop = [&](cudaStream_t ls) -> int {
        for (size_t L = 0; L < sched.size(); ++L) {
            const int it = sched[L].it;
            for (int f = 0; f < NFIELD; ++f) {
                sp.sin[f] = p->d_state[L & 1][f];
                sp.sout[f] = p->d_state[(L + 1) & 1][f];
            }
            sp.it = it;
            sp.seq = it + 1;
            sp.snap_k = snap_at(it);
            const int last = sched[L].two ? it + 1 : it;
            if (sched[L].two) {
                sp.it2 = it + 1;
                sp.snap_k2 = snap_at(it + 1);
                sp.check = check_at(it + 1);
                CUDA_TRY((launch_mode2<0>(sp, p->g.modes, p->vec, p->prefetch, p->warps, ls)));
            } else {
                sp.check = check_at(it);
                CUDA_TRY((launch_mode<0>(sp, p->g.modes, p->vec | (std::min(p->prefetch, 3) << 8), p->warps, ls)));
            }
            p->live = (int)((L + 1) & 1);
            if (cb_at(last))
                if (int rc = call_back(p, it + 1, last, ls)) return rc;
        }
        return 0;
    };
    const std::vector<unsigned long long> key = {U(wavelets), U(snap_u), U(snap_v), U(snap_w),
                                                 (unsigned long long)save, (unsigned long long)isnap,
                                                 (unsigned long long)check_interval};
    if (p->cb) {  // host callbacks in the loop: direct launches
        if (int rc = loop(s)) return rc;
    } else if (int rc = run_loop(p, p->g_fwd, key, s, loop)) {
        return rc;
    }
    p->live = (int)(sched.size() & 1);  // also when a replayed graph ran the loop
    p->launches += (long long)sched.size();
    if (seis && p->nrec_total) {
        if (int rc = transpose(p->d_seis_t, seis, 3, nt, p->nrec_total, s)) return rc;
        ++p->launches;
    }
    if (isnaps_out)
        for (int k = 0; k < nsnap; ++k) {
            const int it = (k + 1) * isnap;
            isnaps_out[k] = it <= nt - 1 ? it : 0;  // fm:572; slots never reached stay 0
        }
    if (flags) {
        CUDA_TRY(cudaMemcpyAsync(flags, p->d_flags, p->nshots * sizeof(int), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (int rc = bs.end(s)) return rc;
    return RTM_OK;
}

// rtm_backward; norm_eps >= 0 adds the source-illumination normalisation of
// rtm_backward_normalized.
static int backward_impl(rtm_plan *p, const float *obs, const float *snap_u, const float *snap_v,
                         const float *snap_w, const int32_t *isnaps, int num_snaps, int isnap, float *image,
                         double *stack, int check_interval, int32_t *flags, rtm_stream_t stream,
                         double norm_eps) {
    NvtxRange nvtx_range("rtm_backward");
    if (!p) return fail(RTM_E_ARG, "null plan");
    if (!p->model_set) return fail(RTM_E_STATE, "rtm_plan_set_model has not been called");
    if (p->nrec_total > 0 && !obs) return fail(RTM_E_ARG, "null observed data");
    if (check_interval < 0) return fail(RTM_E_ARG, "check_interval < 0");
    if (isnap <= 0) return fail(RTM_E_ARG, "isnap must be positive");
    if (num_snaps < 0 || (num_snaps > 0 && !isnaps)) return fail(RTM_E_ARG, "bad snapshot table");
    if (image && p->nshots != 1) return fail(RTM_E_ARG, "image output needs a single-shot plan; use stack");
    const float *sp3[3] = {snap_u, snap_v, snap_w};
    for (int c = 0; c < 3; ++c)
        if (comp_active(p->g.modes, c) && num_snaps > 0 && !sp3[c])
            return fail(RTM_E_ARG, "snapshot buffer %d is null", c);
    const int nt = p->g.nt;
    cudaStream_t s = (cudaStream_t)stream;
    BoundsScope bs;
    bs.add_plan(p);
    bs.add(obs, (size_t)3 * p->nrec_total * nt * sizeof(float));
    for (const float *b : sp3) bs.add(b, rtm_plan_snapshot_floats(p, num_snaps) * sizeof(float));
    bs.add(image, (size_t)3 * p->g.nx * p->g.nz * sizeof(float));
    bs.add(stack, (size_t)3 * p->g.nx * p->g.nz * sizeof(double));
    if (int rc = bs.begin(s)) return rc;
    if (int rc = zero_state(p, s)) return rc;
    const size_t img_floats = (size_t)p->rows_total * p->pitch;
    for (int c = 0; c < 3; ++c)
        if (p->d_img[c]) {
            CUDA_TRY(cudaMemsetAsync(p->d_img[c], 0, img_floats * sizeof(float), s));
            CUDA_TRY(cudaMemsetAsync(p->d_imgc[c], 0, img_floats * sizeof(float), s));
        }
    if (p->nrec_total) {
        if (int rc = transpose(obs, p->d_obs_t, 3, p->nrec_total, nt, s)) return rc;
    }
    StepParams sp;
    fill_common(p, sp);
    sp.code_base = 4;
    const size_t plane = (size_t)nt * p->nrec_total;
    for (int c = 0; c < 3; ++c) {
        sp.obs[c] = p->d_obs_t + c * plane;
        sp.snap[c] = const_cast<float *>(sp3[c]);
        sp.img[c] = p->d_img[c];
        sp.imgc[c] = p->d_imgc[c];
    }
    sp.nsnap = num_snaps;
    p->launches = 1;
    // imaging schedule, known on the host (replaces _check_isnap_match, bm:490-496)
    std::vector<int> snap_of(nt, -1);
    for (int it = 0; it < nt; ++it) {
        const int t = (nt - 1) - it;
        if (t > 0 && t % isnap == 0) {  // backward_modeling.py:558-564
            const int k = t / isnap - 1;
            if (k >= 0 && k < num_snaps && isnaps[k] == t) snap_of[it] = k;
        }
    }
    auto check_at = [&](int it) { return check_interval > 0 && it % check_interval == 0; };
    // display_callback at every imaging step, after the correlation
    // (backward_modeling.py:565-569): a launch ends at each of them
    auto cb_at = [&](int it) { return p->cb && snap_of[it] >= 0; };
    const std::vector<LoopLaunch> sched =
        loop_schedule(0, nt, p->tsteps, [&](int it) { return !check_at(it) && !cb_at(it); });
    auto loop = [&](cudaStream_t ls) -> int {
        for (size_t L = 0; L < sched.size(); ++L) {
            const int it = sched[L].it;
            for (int f = 0; f < NFIELD; ++f) {
                sp.sin[f] = p->d_state[L & 1][f];
                sp.sout[f] = p->d_state[(L + 1) & 1][f];
            }
            sp.it = (nt - 1) - it;  // backward_modeling.py:549
            sp.seq = it + 1;
            sp.snap_k = snap_of[it];
            const int last = sched[L].two ? it + 1 : it;
            if (sched[L].two) {
                sp.it2 = (nt - 1) - (it + 1);
                sp.snap_k2 = snap_of[it + 1];
                sp.check = check_at(it + 1);
                CUDA_TRY((launch_mode2<1>(sp, p->g.modes, p->vec, p->prefetch, p->warps, ls)));
            } else {
                sp.check = check_at(it);
                CUDA_TRY((launch_mode<1>(sp, p->g.modes, p->vec | (std::min(p->prefetch, 3) << 8), p->warps, ls)));
            }
            p->live = (int)((L + 1) & 1);
            if (cb_at(last))
                if (int rc = call_back(p, it + 1, (nt - 1) - last, ls)) return rc;
        }
        return 0;
    };
    std::vector<unsigned long long> key = {U(snap_u), U(snap_v), U(snap_w), (unsigned long long)num_snaps,
                                           (unsigned long long)isnap, (unsigned long long)check_interval};
    for (int it = 0; it < nt; ++it)
        if (snap_of[it] >= 0) key.push_back(((unsigned long long)it << 32) | (unsigned)snap_of[it]);
    if (p->cb) {  // host callbacks in the loop: direct launches
        if (int rc = loop(s)) return rc;
    } else if (int rc = run_loop(p, p->g_bwd, key, s, loop)) {
        return rc;
    }
    p->live = (int)(sched.size() & 1);  // also when a replayed graph ran the loop
    p->launches += (long long)sched.size();
    const int blocks = 148 * 8;
    const size_t n = (size_t)p->g.nx * p->g.nz;
    // source illumination (rtm_backward_normalized): FP64 per cell, one
    // component at a time, over the snapshot slots the correlation used
    struct Scratch {
        double *illum = nullptr;
        unsigned long long *imax = nullptr;
        int *slots = nullptr;
        ~Scratch() {
            if (illum) cudaFree(illum);
            if (imax) cudaFree(imax);
            if (slots) cudaFree(slots);
        }
    } sc;
    std::vector<int> slots;
    const bool norm = norm_eps >= 0.0;
    if (norm) {
        for (int it = 0; it < nt; ++it)
            if (snap_of[it] >= 0) slots.push_back(snap_of[it]);
        if (int rc = dalloc(&sc.illum, img_floats)) return rc;
        if (int rc = dalloc(&sc.imax, (size_t)p->nshots)) return rc;
        if (!slots.empty()) {
            if (int rc = dalloc(&sc.slots, slots.size())) return rc;
            CUDA_TRY(cudaMemcpyAsync(sc.slots, slots.data(), slots.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        }
    }
    for (int c = 0; c < 3; ++c) {
        IllumNorm nm;
        if (norm && p->d_img[c]) {
            CUDA_TRY(cudaMemsetAsync(sc.imax, 0, (size_t)p->nshots * sizeof(unsigned long long), s));
            illum_kernel<<<dim3(64, p->nshots), 256, 0, s>>>(sp3[c], sc.slots, (int)slots.size(), num_snaps,
                                                             p->d_shots, p->g.nz, p->pitch, sc.illum, sc.imax);
            CUDA_TRY(cudaGetLastError());
            ++p->launches;
            nm.illum = sc.illum;
            nm.imax = sc.imax;
            nm.eps = norm_eps;
        }
        if (image) {
            float *dst = image + c * n;
            if (p->d_img[c]) {
                image_out_kernel<<<blocks, 256, 0, s>>>(p->d_img[c], p->d_imgc[c], dst, 0, p->shots_h[0].nx,
                                                        p->g.nz, p->pitch, nm);
                CUDA_TRY(cudaGetLastError());
                ++p->launches;
            } else {
                CUDA_TRY(cudaMemsetAsync(dst, 0, n * sizeof(float), s));
            }
        }
        if (stack && p->d_img[c]) {
            stack_kernel<<<blocks, 256, 0, s>>>(p->d_img[c], p->d_imgc[c], stack + c * n, p->d_shots, p->nshots,
                                                p->g.nx, p->g.nz, p->pitch, nm);
            CUDA_TRY(cudaGetLastError());
            ++p->launches;
        }
    }
    if (flags) CUDA_TRY(cudaMemcpyAsync(flags, p->d_flags, p->nshots * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (flags || norm) CUDA_TRY(cudaStreamSynchronize(s));  // scratch is freed on return
    if (int rc = bs.end(s)) return rc;
    return RTM_OK;
}

int rtm_backward(rtm_plan *p, const float *obs, const float *snap_u, const float *snap_v,
                 const float *snap_w, const int32_t *isnaps, int num_snaps, int isnap, float *image,
                 double *stack, int check_interval, int32_t *flags, rtm_stream_t stream) {
    return backward_impl(p, obs, snap_u, snap_v, snap_w, isnaps, num_snaps, isnap, image, stack, check_interval,
                         flags, stream, -1.0);
}

int rtm_backward_normalized(rtm_plan *p, const float *obs, const float *snap_u, const float *snap_v,
                            const float *snap_w, const int32_t *isnaps, int num_snaps, int isnap, float eps,
                            float *image, double *stack, int check_interval, int32_t *flags,
                            rtm_stream_t stream) {
    if (!(eps >= 0.0f) || !std::isfinite(eps)) return fail(RTM_E_ARG, "eps must be finite and >= 0");
    return backward_impl(p, obs, snap_u, snap_v, snap_w, isnaps, num_snaps, isnap, image, stack, check_interval,
                         flags, stream, (double)eps);
}

size_t rtm_plan_state_floats(const rtm_plan *p) { return p ? p->state_floats : 0; }

int rtm_plan_num_checkpoints(const rtm_plan *p, int ckpt_every) {
    if (!p || ckpt_every <= 0) return 0;
    const int nseg = (p->g.nt + ckpt_every - 1) / ckpt_every;
    return nseg - 1;
}

static bool ckpt_dtype_ok(int dtype) { return dtype >= RTM_CKPT_F32 && dtype <= RTM_CKPT_I16; }
static size_t ckpt_elem(int dtype) { return dtype == RTM_CKPT_F32 ? 4 : 2; }
static size_t ckpt_data_bytes(const rtm_plan *p, int dtype) {
    return ((size_t)NADJ * p->state_floats * ckpt_elem(dtype) + 255) & ~size_t(255);
}
// Block exponents of a compressed slot: one int32 per (field, padded state
// row, block of ckpt_block_cols(vec) columns).
static int ckpt_blocks_per_row(const rtm_plan *p) { return p->nstrips * 30 * p->vec / ckpt_block_cols(p->vec); }
static long long ckpt_shifts_per_field(const rtm_plan *p) {
    return (long long)(p->state_floats / (size_t)p->pitch) * ckpt_blocks_per_row(p);
}
static size_t ckpt_shift_bytes(const rtm_plan *p) {
    return ((size_t)NADJ * (size_t)ckpt_shifts_per_field(p) * sizeof(int) + 255) & ~size_t(255);
}
static size_t ckpt_slot_total(const rtm_plan *p, int dtype) {
    return ckpt_data_bytes(p, dtype) + (dtype == RTM_CKPT_F32 ? 0 : ckpt_shift_bytes(p));
}

size_t rtm_plan_checkpoint_bytes(const rtm_plan *p, int ckpt_every, int ckpt_dtype) {
    const int n = rtm_plan_num_checkpoints(p, ckpt_every);
    if (n <= 0 || !ckpt_dtype_ok(ckpt_dtype)) return 0;
    return (size_t)n * ckpt_slot_total(p, ckpt_dtype);
}

namespace {

// Checkpoint slot c: data, then (compressed dtypes) its block-exponent table.
unsigned char *ckpt_slot(const rtm_plan *p, void *ckpt, int dtype, int c) {
    return static_cast<unsigned char *>(ckpt) + (size_t)c * ckpt_slot_total(p, dtype);
}

// The compressed slot c as the storing step launch writes it.
CkptOut ckpt_out(const rtm_plan *p, void *ckpt, int dtype, int c) {
    unsigned char *slot = ckpt_slot(p, ckpt, dtype, c);
    CkptOut o{};
    o.data = slot;
    o.shift = reinterpret_cast<int *>(slot + ckpt_data_bytes(p, dtype));
    o.field_elems = (long long)p->state_floats;
    o.shift_per_field = ckpt_shifts_per_field(p);
    o.dtype = dtype;
    o.nblk = ckpt_blocks_per_row(p);
    return o;
}

// Restore compressed slot c into the 5 FP32 fields `dst` (their pad rows and
// pad columns are left as they are: zero).
int ckpt_load(rtm_plan *p, const void *ckpt, int dtype, int c, float *const *dst, cudaStream_t s) {
    const CkptOut o = ckpt_out(p, const_cast<void *>(ckpt), dtype, c);
    CkptIn ci{};
    ci.data = o.data;
    ci.shift = o.shift;
    for (int f = 0; f < NADJ; ++f) ci.dst[f] = dst[f];
    ci.field_elems = o.field_elems;
    ci.shift_per_field = o.shift_per_field;
    ci.shots = p->d_shots;
    ci.pitch = p->pitch;
    ci.ncols = p->nstrips * 30 * p->vec;
    ci.nblk = ckpt_blocks_per_row(p);
    ci.block_w = ckpt_block_cols(p->vec);
    ci.dtype = dtype;
    ckpt_unpack_kernel<<<dim3(64, p->nshots, NADJ), 256, 0, s>>>(ci);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

// Where segment sgi's start state (after step sgi*K - 1) lives: the zero
// state for sgi = 0, the FP32 slot itself, or `stage` after unpacking.
int segment_start(rtm_plan *p, const void *ckpt, int dtype, int sgi, float *zero, float *stage,
                  float **out, cudaStream_t s) {
    if (sgi == 0) {
        *out = zero;
        return 0;
    }
    if (dtype == RTM_CKPT_F32) {
        *out = reinterpret_cast<float *>(ckpt_slot(p, const_cast<void *>(ckpt), dtype, sgi - 1));
        return 0;
    }
    float *dst[NADJ];
    for (int f = 0; f < NADJ; ++f) dst[f] = stage + (size_t)f * p->state_floats;
    if (int rc = ckpt_load(p, ckpt, dtype, sgi - 1, dst, s)) return rc;
    *out = stage;
    return 0;
}

}  // namespace

int rtm_forward_checkpointed(rtm_plan *p, const float *wavelets, float *seis, int ckpt_every, int ckpt_dtype,
                             void *ckpt, int check_interval, int32_t *flags, rtm_stream_t stream) {
    NvtxRange nvtx_range("rtm_forward_checkpointed");
    if (!p) return fail(RTM_E_ARG, "null plan");
    if (!p->model_set) return fail(RTM_E_STATE, "rtm_plan_set_model has not been called");
    if (p->g.modes != RTM_PSV) return fail(RTM_E_ARG, "checkpointed propagation supports the P-SV mode");
    if (ckpt_every <= 0) return fail(RTM_E_ARG, "ckpt_every must be positive");
    if (!ckpt_dtype_ok(ckpt_dtype)) return fail(RTM_E_ARG, "bad ckpt_dtype");
    if (p->nsrc_total > 0 && !wavelets) return fail(RTM_E_ARG, "null wavelets");
    const int nt = p->g.nt;
    const int nck = rtm_plan_num_checkpoints(p, ckpt_every);
    if (nck > 0 && !ckpt) return fail(RTM_E_ARG, "null checkpoint buffer");
    cudaStream_t s = (cudaStream_t)stream;
    BoundsScope bs;
    bs.add_plan(p);
    bs.add(wavelets, (size_t)3 * p->nsrc_total * nt * sizeof(float));
    bs.add(seis, (size_t)3 * p->nrec_total * nt * sizeof(float));
    bs.add(ckpt, rtm_plan_checkpoint_bytes(p, ckpt_every, ckpt_dtype));
    if (int rc = bs.begin(s)) return rc;
    if (int rc = zero_state(p, s)) return rc;
    // every slot starts at zero: pad rows / columns of FP32 slots, and the
    // slots of a shot that stops before reaching them
    if (nck > 0) CUDA_TRY(cudaMemsetAsync(ckpt, 0, rtm_plan_checkpoint_bytes(p, ckpt_every, ckpt_dtype), s));
    const size_t nseis = (size_t)3 * nt * p->nrec_total;
    if (nseis) CUDA_TRY(cudaMemsetAsync(p->d_seis_t, 0, nseis * sizeof(float), s));
    StepParams sp;
    fill_common(p, sp);
    sp.code_base = 1;
    const size_t plane = (size_t)nt * p->nrec_total;
    for (int c = 0; c < 3; ++c) {
        sp.wav[c] = wavelets ? wavelets + (size_t)c * p->nsrc_total * nt : nullptr;
        sp.seis[c] = p->d_seis_t + c * plane;
    }
    float *in[NFIELD] = {}, *out[NFIELD] = {};
    for (int f = 0; f < NADJ; ++f) in[f] = p->d_state[0][f];
    p->launches = 0;
    p->live = -1;
    auto check_at = [&](int it) { return check_interval > 0 && it % check_interval == 0; };
    auto save_at = [&](int it) { return (it + 1) % ckpt_every == 0 && it + 1 < nt; };
    const std::vector<LoopLaunch> sched =
        loop_schedule(0, nt, p->tsteps, [&](int it) { return !check_at(it) && !save_at(it); });
    for (const LoopLaunch &ln : sched) {
        const int last = ln.two ? ln.it + 1 : ln.it;  // the step whose state the launch writes
        const bool save = save_at(last);
        const int c = (last + 1) / ckpt_every - 1;
        for (int f = 0; f < NADJ; ++f) {
            if (save && ckpt_dtype == RTM_CKPT_F32)  // the step writes its output into the slot
                out[f] = reinterpret_cast<float *>(ckpt_slot(p, ckpt, ckpt_dtype, c)) + (size_t)f * p->state_floats;
            else
                out[f] = (in[f] == p->d_state[0][f]) ? p->d_state[1][f] : p->d_state[0][f];
            sp.sin[f] = in[f];
            sp.sout[f] = out[f];
        }
        sp.it = ln.it;
        sp.seq = ln.it + 1;
        sp.check = check_at(last);
        if (ln.two) {
            sp.it2 = last;
            sp.snap_k2 = -1;
        }
        if (save && ckpt_dtype != RTM_CKPT_F32) {
            // the launch also packs its output state into compressed slot c
            sp.ck = ckpt_out(p, ckpt, ckpt_dtype, c);
            CUDA_TRY(launch_ckpt(sp, ln.two, p->vec, p->prefetch, p->warps, s));
            sp.ck = CkptOut{};
        } else if (ln.two) {
            CUDA_TRY((launch_mode2<0>(sp, p->g.modes, p->vec, p->prefetch, p->warps, s)));
        } else {
            CUDA_TRY((launch_mode<0>(sp, p->g.modes, p->vec | (std::min(p->prefetch, 3) << 8), p->warps, s)));
        }
        ++p->launches;
        for (int f = 0; f < NADJ; ++f) in[f] = out[f];
    }
    if (seis && p->nrec_total) {
        if (int rc = transpose(p->d_seis_t, seis, 3, nt, p->nrec_total, s)) return rc;
        ++p->launches;
    }
    if (flags) {
        CUDA_TRY(cudaMemcpyAsync(flags, p->d_flags, p->nshots * sizeof(int), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (int rc = bs.end(s)) return rc;
    return RTM_OK;
}

int rtm_adjoint(rtm_plan *p, const float *wavelets, const float *resid, int ckpt_every, int ckpt_dtype,
                const void *ckpt, double *grad, float *grad_wavelet, rtm_stream_t stream) {
    NvtxRange nvtx_range("rtm_adjoint");
    if (!p) return fail(RTM_E_ARG, "null plan");
    if (!p->model_set) return fail(RTM_E_STATE, "rtm_plan_set_model has not been called");
    if (p->g.modes != RTM_PSV) return fail(RTM_E_ARG, "the adjoint supports the P-SV mode");
    if (ckpt_every <= 0) return fail(RTM_E_ARG, "ckpt_every must be positive");
    if (!ckpt_dtype_ok(ckpt_dtype)) return fail(RTM_E_ARG, "bad ckpt_dtype");
    if (!grad) return fail(RTM_E_ARG, "null gradient output");
    if (p->nrec_total > 0 && !resid) return fail(RTM_E_ARG, "null residual");
    if (p->nsrc_total > 0 && !wavelets) return fail(RTM_E_ARG, "null wavelets");
    const int nt = p->g.nt;
    const int K = ckpt_every;
    const int nseg = (nt + K - 1) / K;
    if (nseg > 1 && !ckpt) return fail(RTM_E_ARG, "null checkpoint buffer");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t sf = p->state_floats;
    const size_t slot = (size_t)NADJ * sf;
    const size_t gfl = (size_t)p->rows_total * p->pitch;
    // scratch: K-1 recompute slots, zero state, 2 adjoint states, unpack stage;
    // Kahan gradients; wavelet gradient
    // (the plan's scratch, subdivided; every piece starts on a 128-byte
    // boundary since state_floats and gfl are multiples of the pitch)
    const size_t nrec_slots = (size_t)std::max(K - 1, 1);
    const size_t nslots = nrec_slots + 1 + 2 + (ckpt_dtype == RTM_CKPT_F32 ? 0 : 1);
    const size_t n_gsum = (size_t)3 * NGRAD * gfl;  // Kahan sums, compensations, partials
    const size_t n_gwt = grad_wavelet && p->nsrc_total ? (size_t)3 * nt * p->nsrc_total : 0;
    float *scratch = nullptr;
    if (int rc = plan_scratch(p, nslots * slot + n_gsum + n_gwt, &scratch)) return rc;
    float *seg = scratch, *gsum = seg + nslots * slot, *gwt = n_gwt ? gsum + n_gsum : nullptr;
    BoundsScope bs;
    bs.add_plan(p);
    bs.add(wavelets, (size_t)3 * p->nsrc_total * nt * sizeof(float));
    bs.add(ckpt, rtm_plan_checkpoint_bytes(p, ckpt_every, ckpt_dtype));
    bs.add(seg, nslots * slot * sizeof(float));
    bs.add(gsum, (size_t)3 * NGRAD * gfl * sizeof(float));
    bs.add(gwt, (size_t)3 * nt * p->nsrc_total * sizeof(float));
    p->live = -1;
    auto body = [&]() -> int {
        if (int r = bs.begin(s)) return r;
        CUDA_TRY(cudaMemsetAsync(p->d_flags, 0, p->nshots * sizeof(int), s));
        CUDA_TRY(cudaMemsetAsync(p->d_fail_seq, 0x7f, p->nshots * sizeof(int), s));
        CUDA_TRY(cudaMemsetAsync(seg, 0, nslots * slot * sizeof(float), s));
        CUDA_TRY(cudaMemsetAsync(gsum, 0, (size_t)3 * NGRAD * gfl * sizeof(float), s));
        if (gwt) CUDA_TRY(cudaMemsetAsync(gwt, 0, (size_t)3 * nt * p->nsrc_total * sizeof(float), s));
        if (p->nrec_total) {
            if (int r = transpose(resid, p->d_obs_t, 3, p->nrec_total, nt, s)) return r;
        }
        float *zero = seg + nrec_slots * slot;
        float *adj[2] = {zero + slot, zero + 2 * slot};
        float *stage = zero + 3 * slot;
        auto fld = [&](float *base, int f) { return base + (size_t)f * sf; };
        // a_{nt-1} = R^T g_{nt-1}
        if (p->nrec_total) {
            int max_nx = 1;
            for (const ShotDev &d : p->shots_h) max_nx = std::max(max_nx, d.nx);
            inject_last_resid_kernel<<<dim3((max_nx + 127) / 128, p->nshots), 128, 0, s>>>(
                p->d_shots, p->nshots, p->d_rec_ptr, p->d_rec_ent, p->d_obs_t, nt, p->nrec_total,
                p->g.nz, p->pitch, fld(adj[0], A_U), fld(adj[0], A_W));
            CUDA_TRY(cudaGetLastError());
        }
        StepParams sp;
        fill_common(p, sp);
        sp.check = 0;
        const size_t plane = (size_t)nt * p->nrec_total;
        for (int c = 0; c < 3; ++c) {
            sp.wav[c] = wavelets ? wavelets + (size_t)c * p->nsrc_total * nt : nullptr;
            sp.seis[c] = p->d_seis_t + c * plane;  // recompute records here; not returned
        }
        AdjParams ap;
        std::memset(&ap, 0, sizeof ap);
        ap.nz = p->g.nz;
        ap.pitch = p->pitch;
        ap.nt = nt;
        ap.fw = p->g.absorbing_frame;
        ap.dt = sp.dt;
        ap.inv_dx = sp.inv_dx;
        ap.inv_dz = sp.inv_dz;
        ap.src_factor = sp.src_factor;
        ap.sponge = p->d_sponge;
        ap.work = p->d_work;
        ap.n_work = p->n_work;
        ap.shots = p->d_shots;
        for (int m = 0; m < NMAT; ++m) ap.mat[m] = p->d_mat[m];
        ap.surface = p->has_surface ? p->d_surface : nullptr;
        ap.src_ptr = p->d_src_ptr;
        ap.src_ent = p->d_src_ent;
        ap.rec_ptr = p->d_rec_ptr;
        ap.rec_ent = p->d_rec_ent;
        ap.nrec_total = p->nrec_total;
        ap.nsrc_total = p->nsrc_total;
        for (int c = 0; c < 3; ++c) {
            ap.wav[c] = sp.wav[c];
            ap.resid[c] = p->d_obs_t + c * plane;
            ap.gwav[c] = gwt ? gwt + (size_t)c * nt * p->nsrc_total : nullptr;
        }
        GradFold fold;
        fold.n = (long long)gfl;
        for (int g = 0; g < NGRAD; ++g) {
            fold.sum[g] = gsum + (size_t)g * gfl;
            fold.comp[g] = gsum + (size_t)(NGRAD + g) * gfl;
            fold.part[g] = gsum + (size_t)(2 * NGRAD + g) * gfl;
            ap.gpart[g] = fold.part[g];
        }
        int cur = 0;
        const int warps = p->warps;
        const int blocks = (p->n_work + warps - 1) / warps;
        p->launches = 1;
        for (int sgi = nseg - 1; sgi >= 0; --sgi) {
            const int start = sgi * K, end = std::min(start + K, nt);
            float *s0 = nullptr;
            if (int r = segment_start(p, ckpt, ckpt_dtype, sgi, zero, stage, &s0, s)) return r;
            // recompute forward states start .. end-2 into seg slots 0 .. len-2,
            // two steps per launch (each state stored) where the plan runs two
            for (int it = start; it <= end - 2;) {
                float *src = it == start ? s0 : seg + (size_t)(it - 1 - start) * slot;
                float *dst = seg + (size_t)(it - start) * slot;
                const bool two = p->tsteps == 2 && p->vec >= 2 && it + 1 <= end - 2;
                for (int f = 0; f < NADJ; ++f) {
                    sp.sin[f] = fld(src, f);
                    sp.souta[f] = two ? fld(dst, f) : nullptr;
                    sp.sout[f] = two ? fld(dst + slot, f) : fld(dst, f);
                }
                sp.it = it;
                sp.seq = it + 1;
                if (two) {
                    sp.it2 = it + 1;
                    sp.snap_k2 = -1;
                    CUDA_TRY(launch_recompute2(sp, p->vec, p->prefetch, warps, s));
                    it += 2;
                } else {
                    CUDA_TRY((launch_mode<0>(sp, RTM_PSV, p->vec | (std::min(p->prefetch, 3) << 8), warps, s)));
                    it += 1;
                }
                ++p->launches;
            }
            // reverse steps end-1 .. start; with two steps per launch, steps n and
            // n-1 together unless the partials are folded after step n
            auto fwd_state = [&](int m) { return m == start ? s0 : seg + (size_t)(m - 1 - start) * slot; };
            for (int n = end - 1; n >= start;) {
                float *fs = fwd_state(n);
                for (int f = 0; f < NADJ; ++f) {
                    ap.fwd[f] = fld(fs, f);
                    ap.ain[f] = fld(adj[cur], f);
                    ap.aout[f] = fld(adj[1 - cur], f);
                }
                ap.n = n;
                if (p->tsteps == 2 && p->vec >= 2 && n - 1 >= start && n % GRAD_FOLD_STEPS != 0) {
                    float *fs2 = fwd_state(n - 1);
                    for (int f = 0; f < NADJ; ++f) ap.fwd2[f] = fld(fs2, f);
                    // one warp per CTA: the uniform-task instantiation (same task, same arithmetic)
                    if (p->vec == 2) {
                        if (warps == 1) adjoint2_kernel<2, true><<<blocks, 32, 0, s>>>(ap);
                        else adjoint2_kernel<2><<<blocks, 32 * warps, 0, s>>>(ap);
                    } else {
                        adjoint2_kernel<4><<<blocks, 32 * warps, 0, s>>>(ap);
                    }
                    CUDA_TRY(cudaGetLastError());
                    ++p->launches;
                    cur = 1 - cur;
                    n -= 2;
                    if ((n + 1) % GRAD_FOLD_STEPS == 0) {  // after step n+1 (the pair's second)
                        grad_fold_kernel<<<148 * 8, 256, 0, s>>>(fold);
                        CUDA_TRY(cudaGetLastError());
                        ++p->launches;
                    }
                    continue;
                }
                switch (p->vec) {
                    case 1: adjoint_step_kernel<1><<<blocks, 32 * warps, 0, s>>>(ap); break;
                    case 2:
                        if (warps == 1) adjoint_step_kernel<2, true><<<blocks, 32, 0, s>>>(ap);
                        else adjoint_step_kernel<2><<<blocks, 32 * warps, 0, s>>>(ap);
                        break;
                    default: adjoint_step_kernel<4><<<blocks, 32 * warps, 0, s>>>(ap); break;
                }
                CUDA_TRY(cudaGetLastError());
                ++p->launches;
                cur = 1 - cur;
                if (n % GRAD_FOLD_STEPS == 0) {  // n = 0 is the last step: everything is folded
                    grad_fold_kernel<<<148 * 8, 256, 0, s>>>(fold);
                    CUDA_TRY(cudaGetLastError());
                    ++p->launches;
                }
                --n;
            }
        }
        const size_t n2 = (size_t)p->g.nx * p->g.nz;
        for (int g = 0; g < NGRAD; ++g) {
            stack_kernel<<<148 * 8, 256, 0, s>>>(fold.sum[g], fold.comp[g], grad + g * n2, p->d_shots, p->nshots,
                                                 p->g.nx, p->g.nz, p->pitch);
            CUDA_TRY(cudaGetLastError());
        }
        if (gwt) {
            if (int r = transpose(gwt, grad_wavelet, 3, nt, p->nsrc_total, s)) return r;
        }
        CUDA_TRY(cudaStreamSynchronize(s));
        if (int r = bs.end(s)) return r;
        return RTM_OK;
    };
    return body();
}

int rtm_backward_checkpointed(rtm_plan *p, const float *wavelets, const float *obs, int ckpt_every,
                              int ckpt_dtype, const void *ckpt, int isnap, float *image, double *stack,
                              int check_interval, int32_t *flags, rtm_stream_t stream) {
    NvtxRange nvtx_range("rtm_backward_checkpointed");
    if (!p) return fail(RTM_E_ARG, "null plan");
    if (!p->model_set) return fail(RTM_E_STATE, "rtm_plan_set_model has not been called");
    if (p->g.modes != RTM_PSV) return fail(RTM_E_ARG, "checkpointed RTM supports the P-SV mode");
    if (ckpt_every <= 0 || isnap <= 0) return fail(RTM_E_ARG, "ckpt_every and isnap must be positive");
    if (!ckpt_dtype_ok(ckpt_dtype)) return fail(RTM_E_ARG, "bad ckpt_dtype");
    if (p->nrec_total > 0 && !obs) return fail(RTM_E_ARG, "null observed data");
    if (p->nsrc_total > 0 && !wavelets) return fail(RTM_E_ARG, "null wavelets");
    if (image && p->nshots != 1) return fail(RTM_E_ARG, "image output needs a single-shot plan; use stack");
    const int nt = p->g.nt;
    const int K = ckpt_every;
    const int nseg = (nt + K - 1) / K;
    if (nseg > 1 && !ckpt) return fail(RTM_E_ARG, "null checkpoint buffer");
    const int num_snaps = nt / isnap;  // the snapshot slots the reference would allocate (fm:531)
    cudaStream_t s = (cudaStream_t)stream;
    const size_t sf = p->state_floats;
    const size_t slot = (size_t)NADJ * sf;
    const int seg_snaps = K / isnap + 1;
    const size_t snap_comp = (size_t)seg_snaps * p->rows_total * p->pitch;
    // scratch: recompute ping-pong (2 states), zero state, unpack stage, segment snapshots (u, w)
    float *buf = nullptr;
    const size_t nbuf = 4 * slot + 2 * snap_comp;
    if (int rc = plan_scratch(p, nbuf, &buf)) return rc;
    BoundsScope bs;
    bs.add_plan(p);
    bs.add(wavelets, (size_t)3 * p->nsrc_total * nt * sizeof(float));
    bs.add(obs, (size_t)3 * p->nrec_total * nt * sizeof(float));
    bs.add(ckpt, rtm_plan_checkpoint_bytes(p, ckpt_every, ckpt_dtype));
    bs.add(image, (size_t)3 * p->g.nx * p->g.nz * sizeof(float));
    bs.add(stack, (size_t)3 * p->g.nx * p->g.nz * sizeof(double));
    bs.add(buf, nbuf * sizeof(float));
    p->live = -1;
    auto body = [&]() -> int {
        if (int rc = bs.begin(s)) return rc;
        if (int rc = zero_state(p, s)) return rc;
        CUDA_TRY(cudaMemsetAsync(buf, 0, nbuf * sizeof(float), s));
        const size_t img_floats = (size_t)p->rows_total * p->pitch;
        for (int c = 0; c < 3; ++c)
            if (p->d_img[c]) {
                CUDA_TRY(cudaMemsetAsync(p->d_img[c], 0, img_floats * sizeof(float), s));
                CUDA_TRY(cudaMemsetAsync(p->d_imgc[c], 0, img_floats * sizeof(float), s));
            }
        if (p->nrec_total) {
            if (int r = transpose(obs, p->d_obs_t, 3, p->nrec_total, nt, s)) return r;
        }
        float *rec[2] = {buf, buf + slot};
        float *zero = buf + 2 * slot, *stage = buf + 3 * slot;
        float *snapu = buf + 4 * slot, *snapw = snapu + snap_comp;
        const size_t plane = (size_t)nt * p->nrec_total;
        StepParams fp;  // forward recompute
        fill_common(p, fp);
        fp.check = 0;
        fp.nsnap = seg_snaps;
        fp.snap[0] = snapu;
        fp.snap[2] = snapw;
        for (int c = 0; c < 3; ++c) {
            fp.wav[c] = wavelets ? wavelets + (size_t)c * p->nsrc_total * nt : nullptr;
            fp.seis[c] = p->d_seis_t + c * plane;  // not returned
        }
        StepParams bp;  // backward with imaging
        fill_common(p, bp);
        bp.code_base = 4;
        bp.nsnap = seg_snaps;
        bp.snap[0] = snapu;
        bp.snap[2] = snapw;
        for (int c = 0; c < 3; ++c) {
            bp.obs[c] = p->d_obs_t + c * plane;
            bp.img[c] = p->d_img[c];
            bp.imgc[c] = p->d_imgc[c];
        }
        // imaging at t > 0, t % isnap == 0 with a snapshot slot t/isnap - 1 < nt/isnap
        // that the forward fills (t <= nt-1): backward_modeling.py:556-564, fm:569-572
        auto images_at = [&](int t) { return t > 0 && t % isnap == 0 && t / isnap - 1 < num_snaps && t <= nt - 1; };
        auto check_at = [&](int it) { return check_interval > 0 && it % check_interval == 0; };
        p->launches = 1;
        long long nb = 0;  // backward launches so far: the ping-pong parity
        for (int sgi = nseg - 1; sgi >= 0; --sgi) {
            const int start = sgi * K, end = std::min(start + K, nt);
            float *s0 = nullptr;
            if (int r = segment_start(p, ckpt, ckpt_dtype, sgi, zero, stage, &s0, s)) return r;
            // recompute forward steps start .. end-1, keeping u, w at imaging steps
            const int first = ((start + isnap - 1) / isnap) * isnap;  // first multiple of isnap >= start
            auto slot_at = [&](int t) { return images_at(t) ? (t - first) / isnap : -1; };
            const std::vector<LoopLaunch> fsched = loop_schedule(start, end, p->tsteps, [](int) { return true; });
            for (size_t L = 0; L < fsched.size(); ++L) {
                const int it = fsched[L].it;
                float *src = L == 0 ? s0 : rec[(L - 1) & 1];
                float *dst = rec[L & 1];
                for (int f = 0; f < NADJ; ++f) {
                    fp.sin[f] = src + (size_t)f * sf;
                    fp.sout[f] = dst + (size_t)f * sf;
                }
                fp.it = it;
                fp.seq = it + 1;
                fp.snap_k = slot_at(it);
                if (fsched[L].two) {
                    fp.it2 = it + 1;
                    fp.snap_k2 = slot_at(it + 1);
                    CUDA_TRY((launch_mode2<0>(fp, RTM_PSV, p->vec, p->prefetch, p->warps, s)));
                } else {
                    CUDA_TRY((launch_mode<0>(fp, RTM_PSV, p->vec | (std::min(p->prefetch, 3) << 8), p->warps, s)));
                }
                ++p->launches;
            }
            // backward iterations it whose reversed time t = nt-1-it falls in [start, end)
            const std::vector<LoopLaunch> bsched =
                loop_schedule(nt - end, nt - start, p->tsteps, [&](int it) { return !check_at(it); });
            for (const LoopLaunch &ln : bsched) {
                const int it = ln.it, t = (nt - 1) - it;
                for (int f = 0; f < NFIELD; ++f) {
                    bp.sin[f] = p->d_state[nb & 1][f];
                    bp.sout[f] = p->d_state[(nb + 1) & 1][f];
                }
                bp.it = t;
                bp.seq = it + 1;
                bp.snap_k = slot_at(t);
                if (ln.two) {
                    bp.it2 = t - 1;
                    bp.snap_k2 = slot_at(t - 1);
                    bp.check = check_at(it + 1);
                    CUDA_TRY((launch_mode2<1>(bp, RTM_PSV, p->vec, p->prefetch, p->warps, s)));
                } else {
                    bp.check = check_at(it);
                    CUDA_TRY((launch_mode<1>(bp, RTM_PSV, p->vec | (std::min(p->prefetch, 3) << 8), p->warps, s)));
                }
                ++p->launches;
                ++nb;
            }
        }
        const int blocks = 148 * 8;
        if (image) {
            const size_t n = (size_t)p->g.nx * p->g.nz;
            for (int c = 0; c < 3; ++c) {
                float *dst = image + c * n;
                if (p->d_img[c]) {
                    image_out_kernel<<<blocks, 256, 0, s>>>(p->d_img[c], p->d_imgc[c], dst, 0, p->shots_h[0].nx,
                                                            p->g.nz, p->pitch);
                    CUDA_TRY(cudaGetLastError());
                } else {
                    CUDA_TRY(cudaMemsetAsync(dst, 0, n * sizeof(float), s));
                }
            }
        }
        if (stack) {
            const size_t n = (size_t)p->g.nx * p->g.nz;
            for (int c = 0; c < 3; ++c)
                if (p->d_img[c]) {
                    stack_kernel<<<blocks, 256, 0, s>>>(p->d_img[c], p->d_imgc[c], stack + c * n, p->d_shots,
                                                        p->nshots, p->g.nx, p->g.nz, p->pitch);
                    CUDA_TRY(cudaGetLastError());
                }
        }
        if (flags) CUDA_TRY(cudaMemcpyAsync(flags, p->d_flags, p->nshots * sizeof(int), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        if (int rc = bs.end(s)) return rc;
        return RTM_OK;
    };
    return body();
}

}  // extern "C"
