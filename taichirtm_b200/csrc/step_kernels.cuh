// Fused time-step kernels of the elastic O(2,2) staggered-grid propagator.
//
// One launch advances every shot of a plan by one time step.  It fuses the
// reference's per-step kernel sequence
//   forward  (src/forward_modeling.py:539-572):
//     _set_free_surface/_set_surface_boundary, _update_velocity,
//     _add_source_kernel, _update_stress, _apply_absorbing,
//     _record_seismogram_kernel, _check_finite, _save_snapshot_kernel
//   backward (src/backward_modeling.py:539-577):
//     surface, _update_velocity_backward, _add_observed_data_kernel,
//     _update_stress_backward, _apply_absorbing, _correlate_with_snapshot,
//     _check_finite
// into a single pass over the wavefield: state is read once from buffer A
// and written once to buffer B (ping-pong), material is read once.
//
// Work decomposition.  Storage is (rows i = x) x (columns j = z, contiguous)
// with a padded pitch; element (i, j) of a shot sits at
// state_off + (i + 1) * pitch + (j + 4), so row -1 / row nx and columns
// -4..-1 / nz.. are zero padding that halo reads may touch.  A warp owns a
// strip of W = 30*VEC columns and a range of rows [ia, ib): lane L holds
// columns c0 .. c0+VEC-1 with c0 = j0 - VEC + VEC*L, so lanes 1..30 own the
// strip and lanes 0 / 31 carry the column halo.  The warp streams down the
// rows; the stress row lags the velocity row by one, so every neighbour a
// stencil needs is either in registers (previous row) or one warp shuffle
// away (adjacent column).
//
// Semantics kept exactly (see the reference lines cited):
//   * stencils update the interior only (1 <= i <= nx-2, 1 <= j <= nz-2);
//     edge velocities change only by injection, edge stresses stay
//     c * previous (they are zero);
//   * sponge c(i, j) from the reference's loop order left -> right -> bottom
//     (forward_modeling.py:211-235), evaluated from a 1-D profile;
//   * the topography mask of the NEXT step's S0 multiplies sxz, szz, syz as
//     they are written (nothing reads stress between S4 and the next S0);
//   * sources add wavelet * (dt dx dz) * inv_rho at the source cell, with
//     inv_rho_u / inv_rho_w = +inf on the shot's edge cells like the
//     reference's 1 / 0 (forward_modeling.py:291-307, 421-443);
//   * recorded, snapshotted, imaged and checked values are the velocities
//     after absorbing (forward_modeling.py:550-572).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ckpt_pack.cuh"
#include "debug_bounds.cuh"

namespace rtm {

constexpr int COL_OFF = 4;
constexpr unsigned FULL = 0xffffffffu;

enum Field { F_U = 0, F_W, F_SXX, F_SZZ, F_SXZ, F_V, F_SYX, F_SYZ, NFIELD };
enum Mat { M_IRU = 0, M_IRW, M_LAM, M_MU, M_MXZ, M_IR, M_MYX, M_MYZ, NMAT };

struct ShotDev {
    int nx, x0;          // rows of the window, first global row
    long long state_off; // floats: the shot's padded block in each state field
    long long row_off;   // sum of nx of earlier shots (compact per-shot blocks)
    int src_row0;        // first entry of this shot's row table in src_ptr (nx+1 entries)
    int rec_row0;        // same for rec_ptr
};

struct StepParams {
    int nz, pitch, nt, fw;
    float dt, inv_dx, inv_dz, src_factor;
    const float *sponge;   // fw floats, profile by distance d = 0..fw-1
    const int4 *work;      // (shot, strip, ia, ib) per warp task
    int n_work;
    const ShotDev *shots;
    const float *sin[NFIELD];
    float *sout[NFIELD];
    const float *mat[NMAT];  // global model, padded like the state
    const float *surface;    // global padded 0/1 mask, or nullptr
    const int *src_ptr;
    const int2 *src_ent;     // (j, source index)
    const float *wav[3];     // (nsrc_total, nt) per component u, v, w
    const int *rec_ptr;
    const int2 *rec_ent;     // (j, receiver index)
    int nrec_total;
    float *seis[3];          // time-major (nt, nrec_total) per component
    const float *obs[3];     // time-major (nt, nrec_total) per component
    float *snap[3];          // per component: shots back to back, [nsnap][nx][pitch]
    int nsnap, snap_k;       // snapshot slot written (forward) / read (backward); -1 none
    float *img[3];           // per component Kahan sum, [row_off + i][pitch]
    float *imgc[3];          // Kahan compensation
    int check;               // run the finite check this step
    int code_base;           // 1 forward, 4 backward
    int *flags;              // per shot status
    int *fail_seq;           // per shot: seq of the launch whose check first failed (INT_MAX: none)
    int seq;                 // this launch's number in its time loop (increasing)
    int it;                  // forward: step it; backward: reversed time t
    int it2, snap_k2;        // two-step launches: time and snapshot slot of the second step
    float *souta[NFIELD];    // two-step launches storing the first step's state too (recompute)
    CkptOut ck;              // CKPT launches: the compressed checkpoint slot of the output state
};

template <int VEC>
__device__ __forceinline__ void ldv(float (&v)[VEC], const float *__restrict__ p) {
    if constexpr (VEC == 4) {
        float4 t = ldg_chk(reinterpret_cast<const float4 *>(p));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (VEC == 2) {
        float2 t = ldg_chk(reinterpret_cast<const float2 *>(p));
        v[0] = t.x; v[1] = t.y;
    } else {
        v[0] = ldg_chk(p);
    }
}

template <int VEC>
__device__ __forceinline__ void stv(float *__restrict__ p, const float (&v)[VEC]) {
    if (!RTM_DBG_OK(p, VEC * sizeof(float))) return;
    if constexpr (VEC == 4) {
        *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else if constexpr (VEC == 2) {
        *reinterpret_cast<float2 *>(p) = make_float2(v[0], v[1]);
    } else {
        *p = v[0];
    }
}

// L2 cache policies: wavefield state is streamed once per step (evict first),
// the shared material is re-read by every overlapping shot (evict last).
__device__ __forceinline__ unsigned long long l2_policy_evict_first() {
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ unsigned long long l2_policy_evict_last() {
    unsigned long long p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Read-only vector load with an L2 cache policy.
template <int VEC>
__device__ __forceinline__ void ldv_pol(float (&v)[VEC], const float *__restrict__ p, unsigned long long pol) {
    if (!RTM_DBG_OK(p, VEC * sizeof(float))) {
#pragma unroll
        for (int q = 0; q < VEC; ++q) v[q] = 0.f;
        return;
    }
    if constexpr (VEC == 4) {
        asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
            : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3])
            : "l"(p), "l"(pol));
    } else if constexpr (VEC == 2) {
        asm("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v[0]), "=f"(v[1]) : "l"(p), "l"(pol));
    } else {
        asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v[0]) : "l"(p), "l"(pol));
    }
}

// Vector store with an L2 cache policy.
template <int VEC>
__device__ __forceinline__ void stv_pol(float *p, const float (&v)[VEC], unsigned long long pol) {
    if (!RTM_DBG_OK(p, VEC * sizeof(float))) return;
    if constexpr (VEC == 4) {
        asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;"
                     :: "l"(p), "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "l"(pol) : "memory");
    } else if constexpr (VEC == 2) {
        asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;"
                     :: "l"(p), "f"(v[0]), "f"(v[1]), "l"(pol) : "memory");
    } else {
        asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" :: "l"(p), "f"(v[0]), "l"(pol) : "memory");
    }
}

// Asynchronous global -> shared copies of one lane's VEC floats (cp.async,
// completion tracked per thread by commit / wait groups: no spinning).
template <int VEC>
__device__ __forceinline__ void cp_async_vec(float *smem, const float *gmem) {
    if (!RTM_DBG_OK(gmem, VEC * sizeof(float))) return;
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (VEC == 4) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
    } else if constexpr (VEC == 2) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Rows in flight per warp in the asynchronous pipeline, and the fields one row
// brings in (P-SV: sxx szz sxz u w + inv_rho_u inv_rho_w lam mu mxz; SH: syx
// syz v + inv_rho myx myz).
constexpr int ASYNC_DEPTH = 4;
template <int MODE>
__host__ __device__ constexpr int async_fields() { return ((MODE & 1) ? 10 : 0) + ((MODE & 2) ? 6 : 0); }
template <int MODE, int VEC>
__host__ __device__ constexpr size_t async_smem_per_warp() {
    return (size_t)ASYNC_DEPTH * async_fields<MODE>() * 32 * VEC * sizeof(float);
}

// forward_modeling.py:203-235: 1 everywhere, then left, right, bottom strips,
// later strips overwriting earlier ones.
__device__ __forceinline__ float sponge_coef(const StepParams &p, int nx, int i, int j) {
    const int fw = p.fw, db = p.nz - 1 - j, dr = nx - 1 - i;
    int d = -1;
    if (i >= 0 && i < fw && db > i) d = i;
    if (dr >= 0 && dr < fw && db > dr) d = dr;
    if (db >= 0 && db < fw && i >= db && dr >= db) d = db;
    return d >= 0 ? ldg_chk(p.sponge + d) : 1.0f;
}

__device__ __forceinline__ bool interior(int i, int j, int nx, int nz) {
    return (unsigned)(i - 1) < (unsigned)(nx - 2) && (unsigned)(j - 1) < (unsigned)(nz - 2);
}

// A shot whose finite check failed in an EARLIER launch is stopped.  Warps of
// the failing launch itself all finish, whatever order they run in, so every
// row is updated, recorded and imaged at the failing step, as the reference
// does before it returns (forward_modeling.py:562-566).
__device__ __forceinline__ bool shot_stopped(const StepParams &p, int shot) {
    if (p.fail_seq && !RTM_DBG_OK(p.fail_seq + shot, sizeof(int))) return true;
    return p.fail_seq ? p.fail_seq[shot] < p.seq : ldg_chk(p.flags + shot) != 0;
}

// Record a failed check of this launch: the highest code wins, the first
// failing launch stops the shot for the launches after it.
__device__ __forceinline__ void report_failure(const StepParams &p, int shot, int code) {
    if (!RTM_DBG_OK(p.flags + shot, sizeof(int)) || (p.fail_seq && !RTM_DBG_OK(p.fail_seq + shot, sizeof(int)))) return;
    atomicMax(p.flags + shot, code);
    if (p.fail_seq) atomicMin(p.fail_seq + shot, p.seq);
}

__device__ __forceinline__ int bad_code(float x, int code) {
    return (isnan(x) || fabsf(x) > 1e30f) ? code : 0;
}

// Kahan update of one image cell: sum += prod with compensation comp.
__device__ __forceinline__ void kahan_add(float &sum, float &comp, float prod) {
    float y = __fsub_rn(prod, comp);
    float t = __fadd_rn(sum, y);
    comp = __fsub_rn(__fsub_rn(t, sum), y);
    sum = t;
}

// PF = true software-pipelines the row loop: the loads of the next row (stress,
// velocity, inverse density, material) are issued before the current row is
// computed, so each warp keeps about twice as many bytes in flight.  The
// arithmetic is unchanged (bit-identical results).
// PFM: 0 plain, 1 prefetch, 2 prefetch + L2 cache policies (state evict-first,
// material evict-last), 3 asynchronous pipeline (every field of the row
// ASYNC_DEPTH-1 ahead copied by cp.async into a per-warp shared-memory ring;
// launch with async_smem_per_warp() bytes of dynamic shared memory per warp).
// None of them changes a result bit.
// CKPT (forward P-SV only): the launch's output state is also stored, block-
// scaled to 16 bits, into the checkpoint slot p.ck (ckpt_pack.cuh).
template <int DIR, int MODE, int VEC, int PFM = 0, bool CKPT = false>
__global__ void __launch_bounds__(256) step_kernel(const StepParams p) {
    static_assert(!CKPT || (DIR == 0 && MODE == 1), "checkpoint stores are forward P-SV");
    constexpr bool PF = PFM == 1 || PFM == 2;
    constexpr bool HINT = PFM == 2;
    constexpr bool ASYNC = PFM == 3;
    unsigned long long pol_s = 0, pol_m = 0;
    if constexpr (HINT) {
        pol_s = l2_policy_evict_first();
        pol_m = l2_policy_evict_last();
    }
    auto LS = [&](float (&v)[VEC], const float *ptr) {
        if constexpr (HINT) ldv_pol<VEC>(v, ptr, pol_s); else ldv<VEC>(v, ptr);
    };
    auto LM = [&](float (&v)[VEC], const float *ptr) {
        if constexpr (HINT) ldv_pol<VEC>(v, ptr, pol_m); else ldv<VEC>(v, ptr);
    };
    auto SS = [&](float *ptr, const float (&v)[VEC]) {
        if constexpr (HINT) stv_pol<VEC>(ptr, v, pol_s); else stv<VEC>(ptr, v);
    };
    constexpr bool PSV = (MODE & 1) != 0;
    constexpr bool SH = (MODE & 2) != 0;
    constexpr int W = 30 * VEC;
    const int lane = threadIdx.x & 31;
    const int task = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (task >= p.n_work) return;
    const int4 wk = p.work[task];
    if (shot_stopped(p, wk.x)) return;
    const ShotDev sh = p.shots[wk.x];
    const int nx = sh.nx, nz = p.nz, P = p.pitch;
    // wk.y: strip in bits 0-19; bit 20 / 21 set = no source / no receiver in
    // this task's rows and columns (the row-table lookups can be skipped)
    const int j0 = (wk.y & 0xFFFFF) * W;
    const bool no_src = (wk.y >> 20) & 1, no_rec = (wk.y >> 21) & 1;
    const int c0 = j0 - VEC + VEC * lane;
    const bool owner = lane >= 1 && lane <= 30;
    const int ia = wk.z, ib = wk.w;
    // warp-uniform-per-row fast paths: a lane whose columns are all interior
    // and at least FW above the bottom edge needs the per-cell interior and
    // sponge logic only on rows near the left/right edges
    const bool lane_in = c0 >= 1 && c0 + VEC - 1 <= nz - 2;
    const bool lane_far = nz - 1 - (c0 + VEC - 1) >= p.fw;
    auto all_in = [&](int i) { return lane_in && i >= 1 && i <= nx - 2; };
    auto all_far = [&](int i) { return lane_far && i >= p.fw && nx - 1 - i >= p.fw; };
    const long long soff = sh.state_off + (long long)(c0 + COL_OFF);
    const long long moff = (long long)sh.x0 * P + (long long)(c0 + COL_OFF);
    const float dt = p.dt, idx = p.inv_dx, idz = p.inv_dz;
    const float sdt = DIR == 0 ? dt : -dt;
    // CKPT: scale block of row -1 of this task's strip (padded row 0 of the shot)
    long long ck_blk0 = 0;
    if constexpr (CKPT) ck_blk0 = (sh.state_off / P) * p.ck.nblk + (wk.y & 0xFFFFF) * (W / ckpt_block_cols(VEC));
    auto S = [&](int f, int i) { return p.sin[f] + soff + (long long)(i + 1) * P; };
    auto M = [&](int m, int i) { return p.mat[m] + moff + (long long)(i + 1) * P; };

    // stress of the previous and current row, velocities of the previous and
    // current row (after the velocity update, before absorbing), sponge
    float sxx_p[VEC], szz_p[VEC], sxz_p[VEC], syx_p[VEC], syz_p[VEC];
    float sxx_c[VEC], szz_c[VEC], sxz_c[VEC], syx_c[VEC], syz_c[VEC];
    float u_p[VEC], w_p[VEC], v_p[VEC], u_c[VEC], w_c[VEC], v_c[VEC];
    float vs_u[VEC], vs_w[VEC], vs_v[VEC], ir_u[VEC], ir_w[VEC], ir_v[VEC];
    float cc[VEC];
    int code = 0;
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
        u_p[q] = w_p[q] = v_p[q] = 0.f;
        u_c[q] = w_c[q] = v_c[q] = 0.f;
    }

    auto load_sigma = [&](int i, float (&xx)[VEC], float (&zz)[VEC], float (&xz)[VEC],
                          float (&yx)[VEC], float (&yz)[VEC]) {
        if constexpr (PSV) {
            LS(xx, S(F_SXX, i));
            LS(zz, S(F_SZZ, i));
            LS(xz, S(F_SXZ, i));
        }
        if constexpr (SH) {
            LS(yx, S(F_SYX, i));
            LS(yz, S(F_SYZ, i));
        }
    };
    auto load_vel_into = [&](int i, float (&a_u)[VEC], float (&a_w)[VEC], float (&a_v)[VEC],
                             float (&b_u)[VEC], float (&b_w)[VEC], float (&b_v)[VEC]) {
        if constexpr (PSV) {
            LS(a_u, S(F_U, i));
            LS(a_w, S(F_W, i));
            LM(b_u, M(M_IRU, i));
            LM(b_w, M(M_IRW, i));
        }
        if constexpr (SH) {
            LS(a_v, S(F_V, i));
            LM(b_v, M(M_IR, i));
        }
    };
    auto load_vel = [&](int i) { load_vel_into(i, vs_u, vs_w, vs_v, ir_u, ir_w, ir_v); };
    // stress-update material of the row being finished (lam, mu, mxz / myx,
    // myz) and the surface mask
    float lam[VEC], mu[VEC], mxz[VEC], myx[VEC], myz[VEC], sm[VEC];
    float n_lam[VEC], n_mu[VEC], n_mxz[VEC], n_myx[VEC], n_myz[VEC], n_sm[VEC];
    auto load_mat = [&](int r, float (&a)[VEC], float (&b)[VEC], float (&c)[VEC], float (&d)[VEC],
                        float (&e)[VEC], float (&s)[VEC]) {
        if constexpr (PSV) {
            LM(a, M(M_LAM, r));
            LM(b, M(M_MU, r));
            LM(c, M(M_MXZ, r));
        }
        if constexpr (SH) {
            LM(d, M(M_MYX, r));
            LM(e, M(M_MYZ, r));
        }
        if (p.surface) {
            ldv<VEC>(s, p.surface + moff + (long long)(r + 1) * P);
        } else {
#pragma unroll
            for (int q = 0; q < VEC; ++q) s[q] = 1.f;
        }
    };
    auto take_mat = [&]() {
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            lam[q] = n_lam[q]; mu[q] = n_mu[q]; mxz[q] = n_mxz[q];
            myx[q] = n_myx[q]; myz[q] = n_myz[q]; sm[q] = n_sm[q];
        }
    };
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
        lam[q] = mu[q] = mxz[q] = myx[q] = myz[q] = sm[q] = 0.f;
        n_lam[q] = n_mu[q] = n_mxz[q] = n_myx[q] = n_myz[q] = n_sm[q] = 0.f;
    }
    // Point injection into the velocities of row i (held in u_c/w_c/v_c):
    // forward sources (forward_modeling.py:421-443) or backward observed data
    // (backward_modeling.py:452-460).  Every lane that computes a column does
    // it, halo lanes included, so halo velocities are exact.
    auto inject = [&](int i) {
        if (i < 0 || i >= nx) return;
        if ((DIR == 0 && no_src) || (DIR == 1 && no_rec)) return;
        if constexpr (DIR == 0) {
            const int e0 = ldg_chk(p.src_ptr + sh.src_row0 + i), e1 = ldg_chk(p.src_ptr + sh.src_row0 + i + 1);
            for (int e = e0; e < e1; ++e) {
                const int2 en = ldg_chk(p.src_ent + e);
                const int q = en.x - c0;
                if (q < 0 || q >= VEC) continue;
                const bool in = interior(i, en.x, nx, nz);
                const float f = p.src_factor;
                const size_t t = (size_t)en.y * p.nt + p.it;
#pragma unroll
                for (int qq = 0; qq < VEC; ++qq) {
                    if (qq != q) continue;
                    if constexpr (PSV) {
                        u_c[qq] += ldg_chk(p.wav[0] + t) * f * (in ? ir_u[qq] : __int_as_float(0x7f800000));
                        w_c[qq] += ldg_chk(p.wav[2] + t) * f * (in ? ir_w[qq] : __int_as_float(0x7f800000));
                    }
                    if constexpr (SH) v_c[qq] += ldg_chk(p.wav[1] + t) * f * ir_v[qq];
                }
            }
        } else {
            const int e0 = ldg_chk(p.rec_ptr + sh.rec_row0 + i), e1 = ldg_chk(p.rec_ptr + sh.rec_row0 + i + 1);
            for (int e = e0; e < e1; ++e) {
                const int2 en = ldg_chk(p.rec_ent + e);
                const int q = en.x - c0;
                if (q < 0 || q >= VEC) continue;
                const size_t t = (size_t)p.it * p.nrec_total + en.y;
#pragma unroll
                for (int qq = 0; qq < VEC; ++qq) {
                    if (qq != q) continue;
                    if constexpr (PSV) {
                        u_c[qq] += ldg_chk(p.obs[0] + t);
                        w_c[qq] += ldg_chk(p.obs[2] + t);
                    }
                    if constexpr (SH) v_c[qq] += ldg_chk(p.obs[1] + t);
                }
            }
        }
    };
    // Stress update of row r from the velocities of rows r and r+1 (forward)
    // or r-1 and r (backward); writes stress and absorbed velocity of row r,
    // then records / snapshots / images / checks it.
    auto finish_row = [&](int r, const float (&cr)[VEC], const float (&va_u)[VEC],
                          const float (&va_w)[VEC], const float (&va_v)[VEC],
                          const float (&vb_u)[VEC], const float (&vb_w)[VEC],
                          const float (&vb_v)[VEC]) {
        // va = velocities of row r, vb = the other row (r+1 forward, r-1 backward);
        // lam/mu/mxz/myx/myz/sm hold row r's material (loaded by the caller)
        if constexpr (!PF && !ASYNC) load_mat(r, lam, mu, mxz, myx, myz, sm);
        // column neighbour of row r's velocities: j+1 (forward) or j-1 (backward)
        float nu = 0.f, nw = 0.f, nv = 0.f;
        if constexpr (DIR == 0) {
            if constexpr (PSV) { nu = __shfl_down_sync(FULL, va_u[0], 1); nw = __shfl_down_sync(FULL, va_w[0], 1); }
            if constexpr (SH) nv = __shfl_down_sync(FULL, va_v[0], 1);
        } else {
            if constexpr (PSV) { nu = __shfl_up_sync(FULL, va_u[VEC - 1], 1); nw = __shfl_up_sync(FULL, va_w[VEC - 1], 1); }
            if constexpr (SH) nv = __shfl_up_sync(FULL, va_v[VEC - 1], 1);
        }
        float o_sxx[VEC], o_szz[VEC], o_sxz[VEC], o_syx[VEC], o_syz[VEC];
        float o_u[VEC], o_w[VEC], o_v[VEC];
        const bool rin = all_in(r);
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            const int j = c0 + q;
            const bool in = rin || interior(r, j, nx, nz);
            if constexpr (PSV) {
                float u_x, u_z, w_x, w_z;
                if constexpr (DIR == 0) {
                    const float uj = q < VEC - 1 ? va_u[q + 1] : nu;
                    const float wj = q < VEC - 1 ? va_w[q + 1] : nw;
                    u_x = (vb_u[q] - va_u[q]) * idx;   // fm:369
                    u_z = (uj - va_u[q]) * idz;        // fm:370
                    w_x = (vb_w[q] - va_w[q]) * idx;   // fm:371
                    w_z = (wj - va_w[q]) * idz;        // fm:372
                } else {
                    const float uj = q > 0 ? va_u[q - 1] : nu;
                    const float wj = q > 0 ? va_w[q - 1] : nw;
                    u_x = (va_u[q] - vb_u[q]) * idx;   // bm:366
                    u_z = (va_u[q] - uj) * idz;        // bm:367
                    w_x = (va_w[q] - vb_w[q]) * idx;   // bm:368
                    w_z = (va_w[q] - wj) * idz;        // bm:369
                }
                const float div = u_x + w_z;
                float sxx = sxx_p[q] + sdt * (lam[q] * div + 2.0f * mu[q] * u_x);
                float szz = szz_p[q] + sdt * (lam[q] * div + 2.0f * mu[q] * w_z);
                float sxz = sxz_p[q] + sdt * mxz[q] * (u_z + w_x);
                sxx = in ? sxx : sxx_p[q];
                szz = in ? szz : szz_p[q];
                sxz = in ? sxz : sxz_p[q];
                o_sxx[q] = cr[q] * sxx;
                o_szz[q] = (cr[q] * szz) * sm[q];
                o_sxz[q] = (cr[q] * sxz) * sm[q];
                o_u[q] = cr[q] * va_u[q];
                o_w[q] = cr[q] * va_w[q];
            }
            if constexpr (SH) {
                float v_x, v_z;
                if constexpr (DIR == 0) {
                    const float vj = q < VEC - 1 ? va_v[q + 1] : nv;
                    v_x = (vb_v[q] - va_v[q]) * idx;   // fm:381
                    v_z = (vj - va_v[q]) * idz;        // fm:382
                } else {
                    const float vj = q > 0 ? va_v[q - 1] : nv;
                    v_x = (va_v[q] - vb_v[q]) * idx;   // bm:377
                    v_z = (va_v[q] - vj) * idz;        // bm:378
                }
                float syx = syx_p[q] + sdt * myx[q] * v_x;
                float syz = syz_p[q] + sdt * myz[q] * v_z;
                syx = in ? syx : syx_p[q];
                syz = in ? syz : syz_p[q];
                o_syx[q] = cr[q] * syx;
                o_syz[q] = (cr[q] * syz) * sm[q];
                o_v[q] = cr[q] * va_v[q];
            }
        }
        if constexpr (CKPT)
            ckpt_pack_row<VEC>(p.ck, soff + (long long)(r + 1) * P, ck_blk0 + (long long)(r + 1) * p.ck.nblk, lane,
                               owner, o_u, o_w, o_sxx, o_szz, o_sxz);
        if (!owner) return;
        const long long so = soff + (long long)(r + 1) * P;
        if constexpr (PSV) {
            SS(p.sout[F_SXX] + so, o_sxx);
            SS(p.sout[F_SZZ] + so, o_szz);
            SS(p.sout[F_SXZ] + so, o_sxz);
            SS(p.sout[F_U] + so, o_u);
            SS(p.sout[F_W] + so, o_w);
        }
        if constexpr (SH) {
            SS(p.sout[F_SYX] + so, o_syx);
            SS(p.sout[F_SYZ] + so, o_syz);
            SS(p.sout[F_V] + so, o_v);
        }
        if constexpr (DIR == 0) {
            // _record_seismogram_kernel (forward_modeling.py:445-453)
            const int e0 = no_rec ? 0 : ldg_chk(p.rec_ptr + sh.rec_row0 + r);
            const int e1 = no_rec ? 0 : ldg_chk(p.rec_ptr + sh.rec_row0 + r + 1);
            for (int e = e0; e < e1; ++e) {
                const int2 en = ldg_chk(p.rec_ent + e);
                const int q = en.x - c0;
                if (q < 0 || q >= VEC) continue;
                const size_t t = (size_t)p.it * p.nrec_total + en.y;
#pragma unroll
                for (int qq = 0; qq < VEC; ++qq) {
                    if (qq != q) continue;
                    if constexpr (PSV) { st_chk(p.seis[0] + t, o_u[qq]); st_chk(p.seis[2] + t, o_w[qq]); }
                    if constexpr (SH) st_chk(p.seis[1] + t, o_v[qq]);
                }
            }
            // _save_snapshot_kernel (forward_modeling.py:490-497, 569-572)
            if (p.snap_k >= 0) {
                const long long o = ((long long)p.nsnap * sh.row_off + (long long)p.snap_k * nx + r) * P + c0 + COL_OFF;
                if constexpr (PSV) { stv<VEC>(p.snap[0] + o, o_u); stv<VEC>(p.snap[2] + o, o_w); }
                if constexpr (SH) stv<VEC>(p.snap[1] + o, o_v);
            }
        } else {
            // _correlate_with_snapshot (backward_modeling.py:481-488), Kahan-compensated
            if (p.snap_k >= 0) {
                const long long o = ((long long)p.nsnap * sh.row_off + (long long)p.snap_k * nx + r) * P + c0 + COL_OFF;
                const long long io = (sh.row_off + r) * (long long)P + c0 + COL_OFF;
                auto image = [&](int c, const float (&ov)[VEC]) {
                    float s[VEC], sum[VEC], cmp[VEC];
                    ldv<VEC>(s, p.snap[c] + o);
                    ldv<VEC>(sum, p.img[c] + io);
                    ldv<VEC>(cmp, p.imgc[c] + io);
#pragma unroll
                    for (int q = 0; q < VEC; ++q) kahan_add(sum[q], cmp[q], __fmul_rn(s[q], ov[q]));
                    stv<VEC>(p.img[c] + io, sum);
                    stv<VEC>(p.imgc[c] + io, cmp);
                };
                if constexpr (PSV) { image(0, o_u); image(2, o_w); }
                if constexpr (SH) image(1, o_v);
            }
        }
        // _check_finite (forward_modeling.py:455-488, backward_modeling.py:417-450)
        if (p.check) {
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                if constexpr (PSV) {
                    code = max(code, bad_code(o_u[q], p.code_base));
                    code = max(code, bad_code(o_w[q], p.code_base + 2));
                }
                if constexpr (SH) code = max(code, bad_code(o_v[q], p.code_base + 1));
            }
        }
    };

    // ---- asynchronous pipeline (PFM 3): per-warp ring of ASYNC_DEPTH rows in
    // shared memory; each lane copies and later reads back only its own VEC
    // columns, so the only synchronisation is the lane's own wait_group.
    constexpr int NLF = async_fields<MODE>();
    extern __shared__ float step_smem[];
    float *ring = step_smem + (size_t)(threadIdx.x >> 5) * (ASYNC_DEPTH * (NLF > 0 ? NLF : 1) * 32 * VEC);
    auto slot = [&](int row, int f) {
        const int s = (row + ASYNC_DEPTH) % ASYNC_DEPTH;  // rows start at -1
        return ring + ((size_t)(s * NLF + f) * 32 + lane) * VEC;
    };
    auto issue_row = [&](int row) {
        if (row <= ib) {
            if constexpr (PSV) {
                cp_async_vec<VEC>(slot(row, 0), S(F_SXX, row));
                cp_async_vec<VEC>(slot(row, 1), S(F_SZZ, row));
                cp_async_vec<VEC>(slot(row, 2), S(F_SXZ, row));
                cp_async_vec<VEC>(slot(row, 3), S(F_U, row));
                cp_async_vec<VEC>(slot(row, 4), S(F_W, row));
                cp_async_vec<VEC>(slot(row, 5), M(M_IRU, row));
                cp_async_vec<VEC>(slot(row, 6), M(M_IRW, row));
                cp_async_vec<VEC>(slot(row, 7), M(M_LAM, row));
                cp_async_vec<VEC>(slot(row, 8), M(M_MU, row));
                cp_async_vec<VEC>(slot(row, 9), M(M_MXZ, row));
            }
            if constexpr (SH) {
                constexpr int o = PSV ? 10 : 0;
                cp_async_vec<VEC>(slot(row, o + 0), S(F_SYX, row));
                cp_async_vec<VEC>(slot(row, o + 1), S(F_SYZ, row));
                cp_async_vec<VEC>(slot(row, o + 2), S(F_V, row));
                cp_async_vec<VEC>(slot(row, o + 3), M(M_IR, row));
                cp_async_vec<VEC>(slot(row, o + 4), M(M_MYX, row));
                cp_async_vec<VEC>(slot(row, o + 5), M(M_MYZ, row));
            }
        }
        cp_async_commit();  // one group per row, empty past ib, so the counts stay aligned
    };
    auto rd = [&](int row, int f, float (&v)[VEC]) {
        const float *s = slot(row, f);
#pragma unroll
        for (int q = 0; q < VEC; ++q) v[q] = s[q];
    };
    auto rd_sigma = [&](int row, float (&xx)[VEC], float (&zz)[VEC], float (&xz)[VEC], float (&yx)[VEC],
                        float (&yz)[VEC]) {
        if constexpr (PSV) { rd(row, 0, xx); rd(row, 1, zz); rd(row, 2, xz); }
        if constexpr (SH) { constexpr int o = PSV ? 10 : 0; rd(row, o + 0, yx); rd(row, o + 1, yz); }
    };
    auto rd_vel = [&](int row) {
        if constexpr (PSV) { rd(row, 3, vs_u); rd(row, 4, vs_w); rd(row, 5, ir_u); rd(row, 6, ir_w); }
        if constexpr (SH) { constexpr int o = PSV ? 10 : 0; rd(row, o + 2, vs_v); rd(row, o + 3, ir_v); }
    };
    auto rd_mat = [&](int row) {
        if constexpr (PSV) { rd(row, 7, lam); rd(row, 8, mu); rd(row, 9, mxz); }
        if constexpr (SH) { constexpr int o = PSV ? 10 : 0; rd(row, o + 4, myx); rd(row, o + 5, myz); }
        if (p.surface) {
            ldv<VEC>(sm, p.surface + moff + (long long)(row + 1) * P);
        } else {
#pragma unroll
            for (int q = 0; q < VEC; ++q) sm[q] = 1.f;
        }
    };
    // prologue: rows ia-1 .. ia+DEPTH-3 in flight, then row ia-1's stress in registers
    if constexpr (ASYNC) {
#pragma unroll
        for (int t = 0; t < ASYNC_DEPTH - 1; ++t) issue_row(ia - 1 + t);
        cp_async_wait<ASYNC_DEPTH - 2>();
        rd_sigma(ia - 1, sxx_p, szz_p, sxz_p, syx_p, syz_p);
        if constexpr (DIR == 1) rd_vel(ia - 1);
        issue_row(ia + ASYNC_DEPTH - 2);
    }

    if constexpr (DIR == 0) {
        // ---------------- forward: velocity row k, stress row k-1 ----------------
        if constexpr (!ASYNC) load_sigma(ia - 1, sxx_p, szz_p, sxz_p, syx_p, syz_p);
        float c_prev[VEC];
        float n_sxx[VEC], n_szz[VEC], n_sxz[VEC], n_syx[VEC], n_syz[VEC];
        float n_vu[VEC], n_vw[VEC], n_vv[VEC], n_iu[VEC], n_iw[VEC], n_iv[VEC];
#pragma unroll
        for (int q = 0; q < VEC; ++q) c_prev[q] = 1.f;
        if constexpr (PF) {
            load_sigma(ia, n_sxx, n_szz, n_sxz, n_syx, n_syz);
            load_vel_into(ia, n_vu, n_vw, n_vv, n_iu, n_iw, n_iv);
        }
        for (int k = ia; k <= ib; ++k) {
            if constexpr (ASYNC) {
                cp_async_wait<ASYNC_DEPTH - 2>();  // row k has landed
                rd_sigma(k, sxx_c, szz_c, sxz_c, syx_c, syz_c);
                rd_vel(k);
                if (k > ia) rd_mat(k - 1);
                issue_row(k + ASYNC_DEPTH - 1);   // reuses row k-1's slot, read above
            } else if constexpr (PF) {
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    sxx_c[q] = n_sxx[q]; szz_c[q] = n_szz[q]; sxz_c[q] = n_sxz[q];
                    syx_c[q] = n_syx[q]; syz_c[q] = n_syz[q];
                    vs_u[q] = n_vu[q]; vs_w[q] = n_vw[q]; vs_v[q] = n_vv[q];
                    ir_u[q] = n_iu[q]; ir_w[q] = n_iw[q]; ir_v[q] = n_iv[q];
                }
                if (k > ia) take_mat();  // row k-1, prefetched one iteration ago
                if (k < ib) {
                    load_sigma(k + 1, n_sxx, n_szz, n_sxz, n_syx, n_syz);
                    load_vel_into(k + 1, n_vu, n_vw, n_vv, n_iu, n_iw, n_iv);
                    load_mat(k, n_lam, n_mu, n_mxz, n_myx, n_myz, n_sm);
                }
            } else {
                load_sigma(k, sxx_c, szz_c, sxz_c, syx_c, syz_c);
                load_vel(k);
            }
            float szz_m = 0.f, sxz_m = 0.f, syz_m = 0.f;  // column j-1 of row k
            if constexpr (PSV) {
                szz_m = __shfl_up_sync(FULL, szz_c[VEC - 1], 1);
                sxz_m = __shfl_up_sync(FULL, sxz_c[VEC - 1], 1);
            }
            if constexpr (SH) syz_m = __shfl_up_sync(FULL, syz_c[VEC - 1], 1);
            const bool kin = all_in(k), kfar = all_far(k);
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                const int j = c0 + q;
                const bool in = kin || interior(k, j, nx, nz);
                cc[q] = kfar ? 1.0f : sponge_coef(p, nx, k, j);
                if constexpr (PSV) {
                    const float sxz_jm = q > 0 ? sxz_c[q - 1] : sxz_m;
                    const float szz_jm = q > 0 ? szz_c[q - 1] : szz_m;
                    const float sxx_x = (sxx_c[q] - sxx_p[q]) * idx;  // fm:332
                    const float szz_z = (szz_c[q] - szz_jm) * idz;    // fm:333
                    const float sxz_x = (sxz_c[q] - sxz_p[q]) * idx;  // fm:334
                    const float sxz_z = (sxz_c[q] - sxz_jm) * idz;    // fm:335
                    const float du = (sxx_x + sxz_z) * dt * ir_u[q];  // fm:339
                    const float dw = (sxz_x + szz_z) * dt * ir_w[q];  // fm:340
                    u_c[q] = in ? vs_u[q] + du : vs_u[q];
                    w_c[q] = in ? vs_w[q] + dw : vs_w[q];
                }
                if constexpr (SH) {
                    const float syz_jm = q > 0 ? syz_c[q - 1] : syz_m;
                    const float syx_x = (syx_c[q] - syx_p[q]) * idx;  // fm:343
                    const float syz_z = (syz_c[q] - syz_jm) * idz;    // fm:344
                    const float dv = (syx_x + syz_z) * dt * ir_v[q];  // fm:347
                    v_c[q] = in ? vs_v[q] + dv : vs_v[q];
                }
            }
            inject(k);
            if (k > ia) finish_row(k - 1, c_prev, u_p, w_p, v_p, u_c, w_c, v_c);
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                sxx_p[q] = sxx_c[q]; szz_p[q] = szz_c[q]; sxz_p[q] = sxz_c[q];
                syx_p[q] = syx_c[q]; syz_p[q] = syz_c[q];
                u_p[q] = u_c[q]; w_p[q] = w_c[q]; v_p[q] = v_c[q];
                c_prev[q] = cc[q];
            }
        }
    } else {
        // ------------- backward: velocity row k-1 (needs stress row k) -------------
        if constexpr (!ASYNC) {
            load_sigma(ia - 1, sxx_p, szz_p, sxz_p, syx_p, syz_p);
            load_vel(ia - 1);
        }
        float n_sxx[VEC], n_szz[VEC], n_sxz[VEC], n_syx[VEC], n_syz[VEC];
        float n_vu[VEC], n_vw[VEC], n_vv[VEC], n_iu[VEC], n_iw[VEC], n_iv[VEC];
        if constexpr (PF) load_sigma(ia, n_sxx, n_szz, n_sxz, n_syx, n_syz);
        for (int k = ia; k <= ib; ++k) {
            const int r = k - 1;
            if constexpr (ASYNC) {
                cp_async_wait<ASYNC_DEPTH - 2>();  // row k has landed
                rd_sigma(k, sxx_c, szz_c, sxz_c, syx_c, syz_c);
                if (k > ia) {
                    rd_vel(r);  // row r's velocity inputs (row ia-1's came in the prologue)
                    rd_mat(r);
                }
                issue_row(k + ASYNC_DEPTH - 1);   // reuses row r's slot, read above
            } else if constexpr (PF) {
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    sxx_c[q] = n_sxx[q]; szz_c[q] = n_szz[q]; sxz_c[q] = n_sxz[q];
                    syx_c[q] = n_syx[q]; syz_c[q] = n_syz[q];
                }
                if (k > ia) take_mat();  // row r, prefetched one iteration ago
                if (k < ib) {
                    load_sigma(k + 1, n_sxx, n_szz, n_sxz, n_syx, n_syz);
                    load_vel_into(k, n_vu, n_vw, n_vv, n_iu, n_iw, n_iv);
                    load_mat(k, n_lam, n_mu, n_mxz, n_myx, n_myz, n_sm);
                }
            } else {
                load_sigma(k, sxx_c, szz_c, sxz_c, syx_c, syz_c);
            }
            float szz_n = 0.f, sxz_n = 0.f, syz_n = 0.f;  // column j+1 of row r
            if constexpr (PSV) {
                szz_n = __shfl_down_sync(FULL, szz_p[0], 1);
                sxz_n = __shfl_down_sync(FULL, sxz_p[0], 1);
            }
            if constexpr (SH) syz_n = __shfl_down_sync(FULL, syz_p[0], 1);
            const bool rin = all_in(r), rfar = all_far(r);
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                const int j = c0 + q;
                const bool in = rin || interior(r, j, nx, nz);
                cc[q] = rfar ? 1.0f : sponge_coef(p, nx, r, j);
                if constexpr (PSV) {
                    const float sxz_jp = q < VEC - 1 ? sxz_p[q + 1] : sxz_n;
                    const float szz_jp = q < VEC - 1 ? szz_p[q + 1] : szz_n;
                    const float sxx_x = (sxx_c[q] - sxx_p[q]) * idx;  // bm:333
                    const float szz_z = (szz_jp - szz_p[q]) * idz;    // bm:334
                    const float sxz_x = (sxz_c[q] - sxz_p[q]) * idx;  // bm:335
                    const float sxz_z = (sxz_jp - sxz_p[q]) * idz;    // bm:336
                    const float du = -(sxx_x + sxz_z) * dt * ir_u[q]; // bm:340
                    const float dw = -(sxz_x + szz_z) * dt * ir_w[q]; // bm:341
                    u_c[q] = in ? vs_u[q] + du : vs_u[q];
                    w_c[q] = in ? vs_w[q] + dw : vs_w[q];
                }
                if constexpr (SH) {
                    const float syz_jp = q < VEC - 1 ? syz_p[q + 1] : syz_n;
                    const float syx_x = (syx_c[q] - syx_p[q]) * idx;  // bm:343
                    const float syz_z = (syz_jp - syz_p[q]) * idz;    // bm:344
                    const float dv = -(syx_x + syz_z) * dt * ir_v[q]; // bm:345
                    v_c[q] = in ? vs_v[q] + dv : vs_v[q];
                }
            }
            inject(r);
            if (k > ia) finish_row(r, cc, u_c, w_c, v_c, u_p, w_p, v_p);
            if constexpr (PF) {
                if (k < ib) {
#pragma unroll
                    for (int q = 0; q < VEC; ++q) {
                        vs_u[q] = n_vu[q]; vs_w[q] = n_vw[q]; vs_v[q] = n_vv[q];
                        ir_u[q] = n_iu[q]; ir_w[q] = n_iw[q]; ir_v[q] = n_iv[q];
                    }
                }
            } else if constexpr (!ASYNC) {
                if (k < ib) load_vel(k);
            }
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                sxx_p[q] = sxx_c[q]; szz_p[q] = szz_c[q]; sxz_p[q] = sxz_c[q];
                syx_p[q] = syx_c[q]; syz_p[q] = syz_c[q];
                u_p[q] = u_c[q]; w_p[q] = w_c[q]; v_p[q] = v_c[q];
            }
        }
    }
    if (p.check) {
        code = __reduce_max_sync(FULL, code);
        if (lane == 0 && code > 0) report_failure(p, wk.x, code);
    }
}

}  // namespace rtm
