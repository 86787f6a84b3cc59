/* rtm_b200.h -- C ABI of the B200-native elastic RTM hot path.
 *
 * One library (taichirtm_b200/lib/librtm_b200.so) replaces the Taichi kernels
 * and host time loops of TaichiRTM's src/forward_modeling.py and
 * src/backward_modeling.py.  The reference has no FFI: its boundary is the
 * Python classes ForwardModeling / BackwardModeling (exported from
 * src/__init__.py:24-38).  Each entry point below names the reference code it
 * replaces; the Python package taichirtm_b200 binds them with ctypes and keeps
 * the reference's class and function names.
 *
 * Conventions
 *   - Grid index i = x (rows), j = z (contiguous), arrays (nx, nz) row-major,
 *     exactly the reference's field layout.
 *   - All array pointers are DEVICE pointers unless the comment says "host".
 *   - Every call is asynchronous on the given stream unless it returns
 *     results in host memory (those synchronise the stream).
 *   - Return value: 0 = success, negative = RTM_E_* error.  Per-shot
 *     propagation status uses the reference's codes: 0 ok, 1/2/3 forward
 *     non-finite u/v/w, 4/5/6 backward (forward_modeling.py:455-488,
 *     backward_modeling.py:417-450); the highest code wins.
 *   - A plan is not thread-safe; use one plan per host thread.
 */
#ifndef RTM_B200_H
#define RTM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *rtm_stream_t; /* = cudaStream_t */
typedef struct rtm_plan rtm_plan;

enum {
    RTM_OK = 0,
    RTM_E_ARG = -1,      /* invalid argument (sizes, indices, null pointers) */
    RTM_E_CUDA = -2,     /* a CUDA runtime call failed (see rtm_last_error) */
    RTM_E_STATE = -3,    /* call out of order (e.g. propagate before set_model) */
    RTM_E_NOMEM = -4,    /* device allocation failed */
    RTM_E_RANGE = -5,    /* size above a fixed limit of the entry point */
    RTM_E_CALLBACK = -6  /* the step callback (rtm_plan_set_callback) asked to stop */
};

enum { RTM_PSV = 1, RTM_SH = 2, RTM_BOTH = 3 };

/* Global grid and time axis: the kwargs nx, nz, dx, dz, nt, fs,
 * absorbing_frame of ForwardModeling.__init__ (forward_modeling.py:126-135). */
typedef struct {
    int nx, nz;
    double dx, dz;
    double fs;            /* dt = 1 / fs (forward_modeling.py:135) */
    int nt;
    int absorbing_frame;  /* sponge width FW (forward_modeling.py:133, 237-241) */
    int modes;            /* RTM_PSV | RTM_SH; RTM_BOTH is what the reference runs */
} rtm_grid;

/* One shot on a window of the global model: rows [x0, x0 + nx) (all columns).
 * Source and receiver positions are LOCAL grid indices (i, j) in host memory,
 * the contents of src_loc_field / recv_loc_field (forward_modeling.py:142-143).
 * A window equal to the whole grid (x0 = 0, nx = grid nx) is the reference's
 * single-shot run. */
typedef struct {
    int x0, nx;
    int nsrc;
    const int32_t *src_ij;  /* host, nsrc x 2 */
    int nrec;
    const int32_t *rec_ij;  /* host, nrec x 2 */
} rtm_shot;

/* Kernel launch shape (autotuned by the Python layer; 0 = default). */
typedef struct {
    int vec;        /* columns per lane: 1, 2 or 4 */
    int rows;       /* rows per warp task (the tasks a launch dispatches last get half as many) */
    int warps;      /* warps per CTA */
    int prefetch;   /* 1: software-pipelined row loads; 3: cp.async pipeline, rows 3 ahead in a
                       per-warp shared-memory ring (with tsteps 2: the material and 1/rho rows
                       through a 4-row ring, the state in registers); 2: row loads plus L2 cache
                       policies (state evict-first, material evict-last); 4: as 3 with tsteps 2, one
                       warp per CTA and the task taken from the block index (warps is set to 1);
                       0: plain; other values = default (1) */
    int graphs;     /* 1: capture each time loop as a CUDA graph on first use and replay it
                       while its pointers and schedule stay the same; 0 = direct launches */
    int tsteps;     /* time steps per launch of rtm_forward, rtm_backward and the
                       checkpointed entry points: 2 = temporal blocking (needs vec 2 or 4;
                       bit-identical results), 1 or 0 = one step per launch */
} rtm_tune;

/* Create a plan for nshots shots on one grid: validates geometry, builds the
 * per-row source/receiver tables and the work list, allocates the
 * ping-pong wavefield state.  Replaces ForwardModeling/BackwardModeling
 * _init_fields (forward_modeling.py:155-190, backward_modeling.py:153-193). */
int rtm_plan_create(const rtm_grid *grid, int nshots, const rtm_shot *shots,
                    const rtm_tune *tune, rtm_plan **out);
int rtm_plan_destroy(rtm_plan *plan);

/* Floats per padded row of the internal layout (row i at (i+1)*pitch + 4). */
int rtm_plan_pitch(const rtm_plan *plan);
/* Floats of ONE snapshot component for all shots of the plan and nsnap
 * snapshots (layout per shot: [nsnap][nx_shot][pitch], shots back to back). */
size_t rtm_plan_snapshot_floats(const rtm_plan *plan, int nsnap);

/* Material set-up: derived fields (harmonic shear averages, arithmetic
 * density averages, inverses) of ForwardModeling._init_material_from_fields,
 * _compute_shear_avg, _compute_rho_avg, _compute_inv_rho
 * (forward_modeling.py:192-201, 243-307) and the sponge profile of
 * _init_absorbing (forward_modeling.py:203-241).  mu, lam, rho: (nx, nz)
 * float32.  surface: (nx, nz) 0/1 topography mask or NULL
 * (surface_matrix_field, forward_modeling.py:149, 412-419).  The averages are
 * evaluated in double and rounded once to float. */
int rtm_plan_set_model(rtm_plan *plan, const float *mu, const float *lam, const float *rho,
                       const float *surface, rtm_stream_t stream);

/* Forward propagation of every shot: ForwardModeling.run
 * (forward_modeling.py:504-575), fused per time step.
 *   wavelets: (3, nsrc_total, nt) u, v, w source wavelets, shots' sources in
 *             plan order (wavelet_{u,v,w}_field).
 *   seis:     (3, nrec_total, nt) output seismograms (seismogram_{u,v,w}).
 *   save != 0: snapshots every isnap steps (it % isnap == 0, it != 0) into
 *             snap_u/v/w (rtm_plan_snapshot_floats(plan, nt / isnap) floats
 *             each; NULL for a component the plan does not propagate);
 *             isnaps_out (host, nt / isnap) receives the saved step numbers.
 *   check_interval: finite check every that many steps (0 = never).
 *   flags:    host, nshots status codes (0 / 1..3). */
int rtm_forward(rtm_plan *plan, const float *wavelets, float *seis, int save, int isnap,
                float *snap_u, float *snap_v, float *snap_w, int32_t *isnaps_out,
                int check_interval, int32_t *flags, rtm_stream_t stream);

/* Backward (time-reversed) propagation with the zero-lag cross-correlation
 * imaging condition: BackwardModeling.run_calc (backward_modeling.py:498-579)
 * with _add_observed_data_kernel and _correlate_with_snapshot fused into the
 * step.
 *   obs:      (3, nrec_total, nt) observed data (obsdata_{u,v,w}_field).
 *   snap_*:   forward snapshots (layout of rtm_forward), isnaps (host,
 *             num_snaps) their step numbers, isnap the interval.
 *   image:    (3, nx, nz) float32 per-shot image of shot 0 when nshots == 1
 *             (result_{u,v,w}); may be NULL.
 *   stack:    (3, grid nx, nz) float64; every shot's image is ADDED at its
 *             window (the cross-shot sum of imaging.stack_rtm_images,
 *             imaging.py:81-93); may be NULL.
 *   flags:    host, nshots status codes (0 / 4..6). */
int rtm_backward(rtm_plan *plan, const float *obs, const float *snap_u, const float *snap_v,
                 const float *snap_w, const int32_t *isnaps, int num_snaps, int isnap,
                 float *image, double *stack, int check_interval, int32_t *flags,
                 rtm_stream_t stream);

/* Source-normalised zero-lag cross-correlation: the imaging condition that
 * the reference advertises beside plain cross-correlation but leaves
 * unimplemented (it accepts and ignores run_calc's `method`,
 * backward_modeling.py:505).  rtm_backward, then each shot's image is divided,
 * component by component, by that shot's source illumination
 *     I_c(i, j) = sum over the imaging steps of snapshot_c(i, j)^2
 * (the snapshots and steps the correlation used), stabilised by eps times
 * the shot's maximum illumination:
 *     image_c = xcorr_c / (I_c + eps * max I_c)      (0 where the divisor is 0).
 * Shots are normalised one by one before the stack.  Arguments as
 * rtm_backward, plus eps >= 0.  No reference counterpart (extension). */
int rtm_backward_normalized(rtm_plan *plan, const float *obs, const float *snap_u,
                            const float *snap_v, const float *snap_w, const int32_t *isnaps,
                            int num_snaps, int isnap, float eps, float *image, double *stack,
                            int check_interval, int32_t *flags, rtm_stream_t stream);

/* ---- Exact adjoint (FWI gradients).  No counterpart in the reference, whose
 * backward propagation (backward_modeling.py:312-380) is not the adjoint of
 * its forward; these differentiate the forward step of
 * forward_modeling.py:309-453 exactly.  P-SV plans only. */

/* Floats of one wavefield component buffer of the plan (all shots, padded);
 * a checkpoint slot holds 5 of them (u, w, sxx, szz, sxz). */
size_t rtm_plan_state_floats(const rtm_plan *plan);
/* Checkpoint slots for interval ckpt_every: ceil(nt / ckpt_every) - 1. */
int rtm_plan_num_checkpoints(const rtm_plan *plan, int ckpt_every);

/* Checkpoint storage: FP32 (exact), or 16 bits per value with one shared
 * exponent S per block, a block being one row of one shot's field over 60
 * columns (30 for plans with vec 1), S chosen so that the block's largest
 * magnitude times 2^S lies in [2^14, 2^15):
 *   RTM_CKPT_F16 / RTM_CKPT_BF16: half / bfloat16 of x * 2^S;
 *   RTM_CKPT_I16: round(x * 2^S) as int16 (block floating point: values to
 *                 within 2^-15 of the block maximum, against 2^-11 of each
 *                 value for F16).
 * The compressed copy is written by the step launch that produces the
 * checkpointed state (no extra pass over the wavefield). */
enum { RTM_CKPT_F32 = 0, RTM_CKPT_F16 = 1, RTM_CKPT_BF16 = 2, RTM_CKPT_I16 = 3 };
/* Bytes of the checkpoint buffer (data and scale tables) for this interval/dtype. */
size_t rtm_plan_checkpoint_bytes(const rtm_plan *plan, int ckpt_every, int ckpt_dtype);

/* ForwardModeling.run without snapshots (forward_modeling.py:504-575) that
 * also stores the full state after every step it with (it+1) % ckpt_every == 0
 * (rtm_plan_num_checkpoints slots) into ckpt (rtm_plan_checkpoint_bytes).
 * FP32 storage costs no extra traffic (the step writes its output into the
 * slot); the 16-bit formats cost the step's extra 10 bytes per cell written
 * (plus one scale per block) at checkpoint steps only. */
int rtm_forward_checkpointed(rtm_plan *plan, const float *wavelets, float *seis, int ckpt_every,
                             int ckpt_dtype, void *ckpt, int check_interval, int32_t *flags,
                             rtm_stream_t stream);

/* Adjoint sweep: given resid = dJ/d(seis) (3, nrec_total, nt) and the
 * checkpoints of rtm_forward_checkpointed, recompute each segment forward and
 * run the exact adjoint step backward through it.  Adds, per shot window, the
 * gradients dJ/d(lam, mu, mxz, inv_rho_u, inv_rho_w) into grad
 * ((5, nx, nz) float64, global grid; the caller zeroes it) and, if non-NULL,
 * writes dJ/d(wavelets) into grad_wavelet (3, nsrc_total, nt).  Image-style
 * Kahan FP32 accumulation per shot, FP64 sum over shots.  Synchronises.
 * With two steps per launch (rtm_tune.tsteps 2) the segment recompute and
 * the reverse sweep run steps in pairs; the gradient is bit-identical.
 * Its scratch (ckpt_every + 3 states plus the gradient sums) is allocated on
 * the first call and kept by the plan, grown when a later call needs more,
 * and freed by rtm_plan_destroy; rtm_backward_checkpointed shares it. */
int rtm_adjoint(rtm_plan *plan, const float *wavelets, const float *resid, int ckpt_every,
                int ckpt_dtype, const void *ckpt, double *grad, float *grad_wavelet,
                rtm_stream_t stream);

/* Checkpointed RTM backward: BackwardModeling.run_calc (backward_modeling.py:
 * 498-579) imaging against forward wavefields RECOMPUTED segment by segment
 * from the checkpoints of rtm_forward_checkpointed instead of stored
 * snapshots (forward_modeling.py:530-537, 569-572).  Images at the same steps
 * as the snapshot path with interval isnap (t > 0, t % isnap == 0); with FP32
 * checkpoints the result equals rtm_backward bit for bit.  Outputs as
 * rtm_backward.  Synchronises. */
int rtm_backward_checkpointed(rtm_plan *plan, const float *wavelets, const float *obs, int ckpt_every,
                              int ckpt_dtype, const void *ckpt, int isnap, float *image, double *stack,
                              int check_interval, int32_t *flags, rtm_stream_t stream);

/* Forward propagation of ONE shot on the whole grid that allocates no device
 * memory.  No counterpart in the reference: it exists for callers that cannot
 * call cudaMalloc while running, such as a plugin inside a host processing
 * system that owns all device memory and hands the plugin only a stream and
 * its buffers.  Inputs and outputs are the caller's: mu, lam, rho (nx, nz),
 * wavelets (3, nsrc, nt), seis (3, nrec, nt), all device pointers; src_ij /
 * rec_ij and *flag (status 0 / 1..3) are host memory.  Every intermediate
 * lives in one static device array of rtm_noalloc_scratch_bytes() bytes
 * (64 MiB); a problem needing more (rtm_noalloc_required_bytes) is rejected
 * with RTM_E_RANGE and a message.
 *   Set-up: the array belongs to this library's device code, which the CUDA
 * driver loads on a device the first time it is used there (lazy module
 * loading): that load reserves the 64 MiB on that device until the process
 * exits.  rtm_noalloc_prepare() does it for the current device (it looks up
 * the array's device address and loads every kernel the call launches); call
 * it once per device in the host's set-up phase, before any stream capture.
 * A call on a device that was not prepared does the same set-up first, so
 * that first call is the one that reserves memory.  Later calls allocate
 * nothing.  After a device reset, prepare again.
 *   All calls share the array and each clears what must start at zero: calls
 * that overlap on the GPU (other streams, other host threads) race and must
 * not be issued.  The call synchronises the stream.  Results equal
 * rtm_forward's bit for bit on a one-shot full-grid plan (same step kernel
 * and tables; launch shape vec 2, 16 rows, 4 warps).
 * Errors: rtm_noalloc_last_error(). */
int rtm_forward_noalloc(const rtm_grid *grid, int nsrc, const int32_t *src_ij, int nrec,
                        const int32_t *rec_ij, const float *mu, const float *lam, const float *rho,
                        const float *wavelets, float *seis, int check_interval, int32_t *flag,
                        rtm_stream_t stream);
int rtm_noalloc_prepare(void);
size_t rtm_noalloc_scratch_bytes(void);
size_t rtm_noalloc_required_bytes(const rtm_grid *grid, int nsrc, int nrec);
const char *rtm_noalloc_last_error(void);

/* Host step callback of rtm_forward and rtm_backward: the display_callback
 * of ForwardModeling.run (forward_modeling.py:553-559) and
 * BackwardModeling.run_calc (backward_modeling.py:565-569).  With a callback
 * set, rtm_forward calls cb(user, it) after step it for every it with
 * it % forward_every == 0 (it = 0 included), and rtm_backward calls cb(user, t)
 * after every imaging step t (t > 0, t % isnap == 0, a matching snapshot),
 * after its correlation -- the reference's steps and order.  Each call comes
 * after the stream has finished that step; rtm_plan_wavefield then gives the
 * live wavefield.  As in the reference, no callback follows a failed finite
 * check (the one at the failing step itself is made: the reference calls
 * back before it checks).  A non-zero return stops the loop: the entry
 * point returns RTM_E_CALLBACK.  The time loop then runs as direct launches
 * (no CUDA-graph replay) that end at every callback step.  cb = NULL clears
 * it.  No reference counterpart as a C function. */
typedef int (*rtm_step_callback)(void *user, int step);
int rtm_plan_set_callback(rtm_plan *plan, int forward_every, rtm_step_callback cb, void *user);
/* The velocity wavefield of one shot as the last step of rtm_forward /
 * rtm_backward left it (during a step callback: after that step), copied to
 * dense (nx_shot, nz) DEVICE arrays u, v, w (any may be NULL; a component the
 * plan does not propagate is written as zeros).  RTM_E_STATE before any
 * rtm_forward / rtm_backward, or after a checkpointed entry point. */
int rtm_plan_wavefield(const rtm_plan *plan, int shot, float *u, float *v, float *w, rtm_stream_t stream);

/* Diagnostics: kernels launched by the last propagate call, and the last
 * error message of this thread. */
long long rtm_plan_launch_count(const rtm_plan *plan);
const char *rtm_last_error(void);
const char *rtm_version(void);

/* Bounds-checking build (librtm_b200_debug.so, compiled with
 * -DRTM_BOUNDS_CHECK).  In that build every global access of the propagation
 * and adjoint kernels is checked against the device buffers of the current
 * call.  An access outside all of them is skipped and counted, and the entry
 * point returns RTM_E_CUDA.
 * rtm_bounds_probe says whether [ptr, ptr + bytes) lies inside one of the
 * plan's buffers or the caller buffer [buf, buf + buf_bytes), as the kernels'
 * checks see it (nothing is read at ptr); *inside (host) receives 1 or 0.
 * The normal build returns RTM_E_STATE.  No reference counterpart (a test
 * aid standing in for a memory checker). */
int rtm_bounds_probe(const rtm_plan *plan, const void *buf, size_t buf_bytes, const void *ptr, size_t bytes,
                     int32_t *inside);

#ifdef __cplusplus
}
#endif
#endif /* RTM_B200_H */
