// rtm_forward_noalloc: forward propagation of one shot that allocates no
// device memory.
//
// Some callers cannot call cudaMalloc once they are running: a plugin inside a
// host processing system that hands it a device, a stream and its input /
// output buffers, and owns every byte of device memory itself (an allocation
// behind its back would either fail against its reserved budget or break its
// accounting).  This entry point serves them: the caller passes inputs and
// outputs; every intermediate -- the ping-pong wavefield, the derived material,
// the source/receiver row tables, the time-major seismogram staging -- lives
// in one file-scope __device__ array of fixed size (RTM_NOALLOC_SCRATCH_BYTES,
// 64 MiB).  Every GPU that loads this library's device code holds that array
// until the process exits.
//
// When the array is reserved.  With lazy module loading (the CUDA default
// since 12.2) the device code -- the array included -- is loaded on a
// device the first time host code touches it there.  rtm_noalloc_prepare()
// does that on the current device: it looks up the array's device address
// and loads every kernel rtm_forward_noalloc launches, so that a caller can
// take the reservation in its set-up phase.  A call of rtm_forward_noalloc
// on a device that was not prepared does the same set-up first.
//
// It runs the same fused step kernel as rtm_forward (one launch per time
// step, launch shape vec 2, 16 rows, 4 warps), and the same host-side table
// construction (plan_host.h), so its results equal rtm_forward's bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rtm_b200.h"
#include "aux_kernels.cuh"
#include "plan_host.h"
#include "step_kernels.cuh"

using namespace rtm;

#define RTM_NOALLOC_SCRATCH_BYTES (64ull << 20)

// The scratch.  In host code its name is only a stand-in for the device
// symbol: its device address is obtained with cudaGetSymbolAddress (below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[RTM_NOALLOC_SCRATCH_BYTES];

namespace {

thread_local std::string g_na_err;

int na_fail(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int na_fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_na_err = buf;
    return code;
}

#define NA_TRY(expr)                                                                         \
    do {                                                                                     \
        cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return na_fail(RTM_E_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_));       \
    } while (0)

// Device address of the scratch on the current device.  cudaGetSymbolAddress
// is a host-side table lookup once the module is loaded, so it is done on
// every call rather than cached: a device reset between calls reloads the
// module at a new address, and a cached pointer would be stale.
int scratch_address(void **out) {
    int dev = -1;
    NA_TRY(cudaGetDevice(&dev));
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return na_fail(RTM_E_CUDA, "cudaGetSymbolAddress(scratch) failed on device %d: %s", dev,
                       cudaGetErrorString(e));
    *out = p;
    return RTM_OK;
}

template <int DIR, int MODE, int VEC>
cudaError_t na_launch(const StepParams &sp, int warps, cudaStream_t s) {
    step_kernel<DIR, MODE, VEC><<<(sp.n_work + warps - 1) / warps, 32 * warps, 0, s>>>(sp);
    return cudaGetLastError();
}

cudaError_t na_launch_mode(const StepParams &sp, int modes, cudaStream_t s) {
    constexpr int warps = 4;
    switch (modes) {
        case RTM_PSV: return na_launch<0, RTM_PSV, 2>(sp, warps, s);
        case RTM_SH: return na_launch<0, RTM_SH, 2>(sp, warps, s);
        default: return na_launch<0, RTM_BOTH, 2>(sp, warps, s);
    }
}

// Scratch layout, in 256-byte aligned pieces.
struct Layout {
    size_t state[2][NFIELD], mat[NMAT], sponge, shot, work, src_ptr, rec_ptr, src_ent, rec_ent,
        seis_t, flags, total;
};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

constexpr int kPitchVec = 2;  // launch shape: vec 2, 16 rows per task, 4 warps
constexpr int kRows = 16;

Layout layout_for(const rtm_grid &g, int nsrc, int nrec, int n_work) {
    Layout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += align256(bytes);
        return o;
    };
    const int P = layout_pitch(g.nz);
    const size_t grid_f = (size_t)(g.nx + 2) * P * sizeof(float);
    for (int b = 0; b < 2; ++b)
        for (int f = 0; f < NFIELD; ++f) {
            const bool psv_field = f <= F_SXZ;
            L.state[b][f] = ((psv_field && (g.modes & RTM_PSV)) || (!psv_field && (g.modes & RTM_SH)))
                                ? take(grid_f) : SIZE_MAX;
        }
    for (int m = 0; m < NMAT; ++m) {
        const bool psv_mat = m <= M_MXZ;
        L.mat[m] = ((psv_mat && (g.modes & RTM_PSV)) || (!psv_mat && (g.modes & RTM_SH))) ? take(grid_f) : SIZE_MAX;
    }
    L.sponge = take(sizeof(float) * (size_t)(g.absorbing_frame > 0 ? g.absorbing_frame : 1));
    L.shot = take(sizeof(ShotDev));
    L.work = take(sizeof(int4) * (size_t)n_work);
    L.src_ptr = take(sizeof(int) * (size_t)(g.nx + 1));
    L.rec_ptr = take(sizeof(int) * (size_t)(g.nx + 1));
    L.src_ent = take(sizeof(int2) * (size_t)(nsrc > 0 ? nsrc : 1));
    L.rec_ent = take(sizeof(int2) * (size_t)(nrec > 0 ? nrec : 1));
    L.seis_t = take(sizeof(float) * (size_t)3 * g.nt * (nrec > 0 ? nrec : 1));
    L.flags = take(2 * sizeof(int));  // status flag, then the first failing launch
    L.total = off;
    return L;
}

int n_work_for(const rtm_grid &g) {
    const int strips = (g.nz + 30 * kPitchVec - 1) / (30 * kPitchVec);
    return ((g.nx + kRows - 1) / kRows) * strips;
}

// The checks of rtm_plan_create for one shot on the whole grid: the grid,
// then the shot (absorbing_frame no wider than its rows, positions inside).
int validate(const rtm_grid *g, int nsrc, const int32_t *src_ij, int nrec, const int32_t *rec_ij) {
    if (!g) return na_fail(RTM_E_ARG, "null grid");
    if (const char *bad = check_grid(*g))
        return na_fail(RTM_E_ARG, "%s (nx=%d nz=%d nt=%d absorbing_frame=%d)", bad, g->nx, g->nz, g->nt,
                       g->absorbing_frame);
    if (g->absorbing_frame > g->nx)
        return na_fail(RTM_E_ARG, "absorbing_frame %d wider than the %d rows of the grid", g->absorbing_frame, g->nx);
    if (nsrc < 0 || nrec < 0 || (nsrc && !src_ij) || (nrec && !rec_ij))
        return na_fail(RTM_E_ARG, "bad source/receiver arrays");
    for (int k = 0; k < nsrc; ++k)
        if (src_ij[2 * k] < 0 || src_ij[2 * k] >= g->nx || src_ij[2 * k + 1] < 0 || src_ij[2 * k + 1] >= g->nz)
            return na_fail(RTM_E_ARG, "source %d at (%d, %d) outside the grid", k, src_ij[2 * k], src_ij[2 * k + 1]);
    for (int k = 0; k < nrec; ++k)
        if (rec_ij[2 * k] < 0 || rec_ij[2 * k] >= g->nx || rec_ij[2 * k + 1] < 0 || rec_ij[2 * k + 1] >= g->nz)
            return na_fail(RTM_E_ARG, "receiver %d at (%d, %d) outside the grid", k, rec_ij[2 * k], rec_ij[2 * k + 1]);
    return RTM_OK;
}

// Loads every kernel rtm_forward_noalloc launches on the current device
// (cudaFuncGetAttributes makes the driver load a lazily loaded function), so
// that no module load -- which reserves device memory -- happens later.
int load_kernels() {
    cudaFuncAttributes a;
    NA_TRY(cudaFuncGetAttributes(&a, step_kernel<0, RTM_PSV, 2>));
    NA_TRY(cudaFuncGetAttributes(&a, step_kernel<0, RTM_SH, 2>));
    NA_TRY(cudaFuncGetAttributes(&a, step_kernel<0, RTM_BOTH, 2>));
    NA_TRY(cudaFuncGetAttributes(&a, setup_material_kernel));
    NA_TRY(cudaFuncGetAttributes(&a, transpose_kernel));
    return RTM_OK;
}

// The set-up: the scratch's device address on the current device and every
// kernel loaded.  Both are host-side lookups once the module is loaded, so
// every call repeats them instead of caching: a device reset between calls
// reloads the module (at a new address), and this finds it again.
int prepare_current_device(void **scratch) {
    if (int rc = scratch_address(scratch)) return rc;
    return load_kernels();
}

}  // namespace

extern "C" {

size_t rtm_noalloc_scratch_bytes(void) { return (size_t)RTM_NOALLOC_SCRATCH_BYTES; }

size_t rtm_noalloc_required_bytes(const rtm_grid *grid, int nsrc, int nrec) {
    if (!grid || grid->nx < 3 || grid->nz < 3 || grid->nt <= 0) return 0;
    return layout_for(*grid, nsrc, nrec, n_work_for(*grid)).total;
}

const char *rtm_noalloc_last_error(void) { return g_na_err.c_str(); }

int rtm_noalloc_prepare(void) {
    void *p = nullptr;
    return prepare_current_device(&p);
}

int rtm_forward_noalloc(const rtm_grid *grid, int nsrc, const int32_t *src_ij, int nrec,
                        const int32_t *rec_ij, const float *mu, const float *lam, const float *rho,
                        const float *wavelets, float *seis, int check_interval, int32_t *flag,
                        rtm_stream_t stream) {
    if (int rc = validate(grid, nsrc, src_ij, nrec, rec_ij)) return rc;
    if (!mu || !lam || !rho || (nsrc && !wavelets) || (nrec && !seis) || !flag || check_interval < 0)
        return na_fail(RTM_E_ARG, "null input/output pointer or negative check_interval");
    const rtm_grid g = *grid;
    const int n_work = n_work_for(g);
    const Layout L = layout_for(g, nsrc, nrec, n_work);
    if (L.total > RTM_NOALLOC_SCRATCH_BYTES)
        return na_fail(RTM_E_RANGE,
                       "problem needs %zu bytes of scratch, above the fixed %llu-byte limit of "
                       "rtm_forward_noalloc (nx=%d nz=%d nt=%d nrec=%d); use rtm_forward",
                       L.total, (unsigned long long)RTM_NOALLOC_SCRATCH_BYTES, g.nx, g.nz, g.nt, nrec);
    void *base_v = nullptr;
    if (int rc = prepare_current_device(&base_v)) return rc;  // loads the module on a device's first call
    unsigned char *base = static_cast<unsigned char *>(base_v);
    cudaStream_t s = (cudaStream_t)stream;
    const int P = layout_pitch(g.nz);

    // host-side tables: the construction of rtm_plan_create (plan_host.h)
    std::vector<int> src_ptr, rec_ptr;
    std::vector<int2> src_ent, rec_ent;
    append_row_table(g.nx, g.nz, nsrc, src_ij, 0, src_ptr, src_ent);  // positions checked by validate()
    append_row_table(g.nx, g.nz, nrec, rec_ij, 0, rec_ptr, rec_ent);
    std::vector<int4> work;
    const int strips = (g.nz + 30 * kPitchVec - 1) / (30 * kPitchVec);
    for (int ia = 0; ia < g.nx; ia += kRows)
        for (int st = 0; st < strips; ++st) work.push_back(make_int4(0, st, ia, std::min(ia + kRows, g.nx)));
    ShotDev shot{};
    shot.nx = g.nx;
    shot.x0 = 0;
    shot.state_off = 0;
    shot.row_off = 0;
    shot.src_row0 = 0;
    shot.rec_row0 = 0;
    const std::vector<float> prof = sponge_profile(g.absorbing_frame);
    // The tables live in pageable host memory that goes out of scope when this
    // call returns, so these copies complete before it does.
    NA_TRY(cudaMemcpyAsync(base + L.sponge, prof.data(), prof.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    NA_TRY(cudaMemcpyAsync(base + L.shot, &shot, sizeof shot, cudaMemcpyHostToDevice, s));
    NA_TRY(cudaMemcpyAsync(base + L.work, work.data(), work.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
    NA_TRY(cudaMemcpyAsync(base + L.src_ptr, src_ptr.data(), src_ptr.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    NA_TRY(cudaMemcpyAsync(base + L.rec_ptr, rec_ptr.data(), rec_ptr.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    if (!src_ent.empty())
        NA_TRY(cudaMemcpyAsync(base + L.src_ent, src_ent.data(), src_ent.size() * sizeof(int2), cudaMemcpyHostToDevice, s));
    if (!rec_ent.empty())
        NA_TRY(cudaMemcpyAsync(base + L.rec_ent, rec_ent.data(), rec_ent.size() * sizeof(int2), cudaMemcpyHostToDevice, s));

    // The array keeps the previous call's contents: clear everything that
    // must start at zero (wavefield incl. padding, material padding, staging, flag).
    const size_t grid_f = (size_t)(g.nx + 2) * P * sizeof(float);
    auto F = [&](size_t off) { return off == SIZE_MAX ? nullptr : reinterpret_cast<float *>(base + off); };
    for (int b = 0; b < 2; ++b)
        for (int f = 0; f < NFIELD; ++f)
            if (L.state[b][f] != SIZE_MAX) NA_TRY(cudaMemsetAsync(base + L.state[b][f], 0, grid_f, s));
    for (int m = 0; m < NMAT; ++m)
        if (L.mat[m] != SIZE_MAX) NA_TRY(cudaMemsetAsync(base + L.mat[m], 0, grid_f, s));
    NA_TRY(cudaMemsetAsync(base + L.seis_t, 0, sizeof(float) * (size_t)3 * g.nt * (nrec > 0 ? nrec : 1), s));
    NA_TRY(cudaMemsetAsync(base + L.flags, 0, sizeof(int), s));
    NA_TRY(cudaMemsetAsync(base + L.flags + sizeof(int), 0x7f, sizeof(int), s));  // no failing launch yet

    const long long n = (long long)g.nx * g.nz;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    setup_material_kernel<<<blocks, 256, 0, s>>>(mu, lam, rho, nullptr, g.nx, g.nz, P, F(L.mat[M_IRU]),
                                                 F(L.mat[M_IRW]), F(L.mat[M_LAM]), F(L.mat[M_MU]),
                                                 F(L.mat[M_MXZ]), F(L.mat[M_IR]), F(L.mat[M_MYX]),
                                                 F(L.mat[M_MYZ]), nullptr);
    NA_TRY(cudaGetLastError());

    StepParams sp;
    std::memset(&sp, 0, sizeof sp);
    const double dt = 1.0 / g.fs;
    sp.nz = g.nz;
    sp.pitch = P;
    sp.nt = g.nt;
    sp.fw = g.absorbing_frame;
    sp.dt = (float)dt;
    sp.inv_dx = (float)(1.0 / g.dx);
    sp.inv_dz = (float)(1.0 / g.dz);
    sp.src_factor = (float)(dt * g.dx * g.dz);
    sp.sponge = F(L.sponge);
    sp.work = reinterpret_cast<const int4 *>(base + L.work);
    sp.n_work = n_work;
    sp.shots = reinterpret_cast<const ShotDev *>(base + L.shot);
    for (int m = 0; m < NMAT; ++m) sp.mat[m] = F(L.mat[m]);
    sp.surface = nullptr;
    sp.src_ptr = reinterpret_cast<const int *>(base + L.src_ptr);
    sp.src_ent = reinterpret_cast<const int2 *>(base + L.src_ent);
    sp.rec_ptr = reinterpret_cast<const int *>(base + L.rec_ptr);
    sp.rec_ent = reinterpret_cast<const int2 *>(base + L.rec_ent);
    sp.nrec_total = nrec;
    sp.flags = reinterpret_cast<int *>(base + L.flags);
    sp.fail_seq = reinterpret_cast<int *>(base + L.flags) + 1;
    sp.code_base = 1;
    sp.snap_k = -1;
    float *seis_t = F(L.seis_t);
    const size_t plane = (size_t)g.nt * nrec;
    for (int c = 0; c < 3; ++c) {
        sp.wav[c] = wavelets ? wavelets + (size_t)c * nsrc * g.nt : nullptr;
        sp.seis[c] = seis_t + c * plane;
    }
    for (int it = 0; it < g.nt; ++it) {
        for (int f = 0; f < NFIELD; ++f) {
            sp.sin[f] = F(L.state[it & 1][f]);
            sp.sout[f] = F(L.state[(it + 1) & 1][f]);
        }
        sp.it = it;
        sp.seq = it + 1;
        sp.check = check_interval > 0 && it % check_interval == 0;
        NA_TRY(na_launch_mode(sp, g.modes, s));
    }
    if (nrec > 0) {
        dim3 tg((nrec + 31) / 32, (g.nt + 31) / 32, 3);
        transpose_kernel<<<tg, dim3(32, 8), 0, s>>>(seis_t, seis, g.nt, nrec);
        NA_TRY(cudaGetLastError());
    }
    NA_TRY(cudaMemcpyAsync(flag, base + L.flags, sizeof(int), cudaMemcpyDeviceToHost, s));
    NA_TRY(cudaStreamSynchronize(s));
    return RTM_OK;
}

}  // extern "C"
