// Two time steps per launch (temporal blocking) of the fused elastic step.
//
// step2_kernel advances every shot by steps A (time p.it) and B (time p.it2)
// in one pass over the wavefield: the state is read once (before A) and
// written once (after B), the material once, so a launch costs the HBM
// traffic of one single step for two steps of work.  Every cell's
// arithmetic is the single-step kernel's, operation by operation, so the
// result is bit-identical to two launches of step_kernel.
//
// Dependencies.  One step reaches one row and one column in each direction:
// forward, the velocity of row i reads the stress of rows i-1, i and the
// stress of row i reads the new velocity of rows i, i+1; backward the other
// way round (backward_modeling.py:312-380).  A warp streaming down rows k
// therefore runs four row updates per iteration:
//   forward:  A velocity k, A stress k-1, B velocity k-1, B stress k-2
//   backward: A velocity k-1, A stress k-1, B velocity k-2, B stress k-2
// and a task that writes rows [ia, ib) recomputes step A on one extra row
// above and below (rows ia-1 .. ib) from the old state of rows ia-2 .. ib+1.
// Row indices are clamped to the pad rows -1 .. nx of the shot block: rows -2
// and nx+1 read the zero pad state (no update touches a non-interior cell, so
// pad rows stay zero), and the material read there feeds only updates of
// non-interior cells, which the interior selects discard.  The loads need no
// per-row branch.
//
// Columns.  Lanes 0 and 31 carry VEC halo columns.  After step A only their
// outermost column is wrong (its neighbour is outside the warp); after step
// B the two outermost ones.  With VEC >= 2 every column that an owner lane
// (1..30) reads is still exact, so the single-step decomposition is kept.
//
// Epilogues.  Step A's values are recorded (forward receivers,
// _record_seismogram_kernel), snapshotted (forward) or correlated (backward
// imaging) for rows [ia, ib) exactly like a single step; they are not
// written back.  The finite check runs on step B only: the host never pairs
// a step that is checked as step A, so a shot that fails stops at the step
// where the reference stops.
#pragma once
#include <type_traits>

#include "step_kernels.cuh"

namespace rtm {

template <int VEC>
struct SigRow { float xx[VEC], zz[VEC], xz[VEC], yx[VEC], yz[VEC]; };
template <int VEC>
struct VelRow { float u[VEC], w[VEC], v[VEC]; };
template <int VEC>
struct MatRow { float lam[VEC], mu[VEC], mxz[VEC], myx[VEC], myz[VEC], sm[VEC]; };

template <int VEC>
__device__ __forceinline__ void zero_arr(float (&a)[VEC]) {
#pragma unroll
    for (int q = 0; q < VEC; ++q) a[q] = 0.f;
}

template <int VEC>
__device__ __forceinline__ void copy_arr(float (&d)[VEC], const float (&s)[VEC]) {
#pragma unroll
    for (int q = 0; q < VEC; ++q) d[q] = s[q];
}

// Plain (coherent) vector load for the Kahan image: one thread may read a
// cell again after writing it in the same launch (steps A and B both
// imaging), which the read-only path (ld.global.nc) does not allow.
template <int VEC>
__device__ __forceinline__ void ldv_coherent(float (&v)[VEC], float *p) {
    if (!RTM_DBG_OK(p, VEC * sizeof(float))) {
#pragma unroll
        for (int q = 0; q < VEC; ++q) v[q] = 0.f;
        return;
    }
    if constexpr (VEC == 4) {
        const float4 t = *reinterpret_cast<float4 *>(p);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (VEC == 2) {
        const float2 t = *reinterpret_cast<float2 *>(p);
        v[0] = t.x; v[1] = t.y;
    } else {
        v[0] = *p;
    }
}

// Material ring (RING = true): the material and inverse-density rows reach a
// warp through a per-warp shared-memory ring of RING2_ROWS rows, filled by
// cp.async one iteration ahead, instead of rolling through registers.  Each
// lane copies and reads back only its own VEC columns, so its own
// wait_group is the only synchronisation.  It frees about 30 registers per
// thread, i.e. more resident warps.  Fields per ring row: P-SV lam, mu, mxz,
// 1/rho_u, 1/rho_w; SH myx, myz, 1/rho; the surface mask.
constexpr int RING2_ROWS = 4;
template <int MODE>
__host__ __device__ constexpr int ring2_fields() { return ((MODE & 1) ? 5 : 0) + ((MODE & 2) ? 3 : 0) + 1; }
template <int MODE, int VEC>
__host__ __device__ constexpr size_t ring2_smem_per_warp() {
    return (size_t)RING2_ROWS * ring2_fields<MODE>() * 32 * VEC * sizeof(float);
}

// STOREA: also store step A's state (rows [ia, ib), into p.souta), for the
// forward recompute of the FWI adjoint, which needs the state after every step.
// CKPT: step B's state is also stored, block-scaled to 16 bits, into the
// checkpoint slot p.ck (ckpt_pack.cuh); forward P-SV only.
// UNI: launched with one warp per CTA, the task is blockIdx.x.  Everything
// derived from the task (shot, strip, row range, loop bounds, fast-path
// choices) is then provably the same for the whole warp, so the compiler
// keeps it in uniform registers and branches on it without divergence
// bookkeeping; the arithmetic of every cell is unchanged.
template <int DIR, int MODE, int VEC, bool RING = false, bool STOREA = false, bool CKPT = false, bool UNI = false>
__global__ void __launch_bounds__(UNI ? 32 : 256) step2_kernel(const StepParams p) {
    static_assert(VEC >= 2, "two steps per launch need two halo columns per side");
    static_assert(!STOREA || DIR == 0, "only the forward recompute stores step A");
    static_assert(!CKPT || (DIR == 0 && MODE == 1), "checkpoint stores are forward P-SV");
    constexpr bool PSV = (MODE & 1) != 0;
    constexpr bool SH = (MODE & 2) != 0;
    constexpr int W = 30 * VEC;
    using Sig = SigRow<VEC>;
    using Vel = VelRow<VEC>;
    using Mat = MatRow<VEC>;
    const int lane = threadIdx.x & 31;
    const int task = UNI ? (int)blockIdx.x : (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (task >= p.n_work) return;
    const int4 wk = p.work[task];
    if (shot_stopped(p, wk.x)) return;
    const ShotDev sh = p.shots[wk.x];
    const int nx = sh.nx, nz = p.nz, P = p.pitch;
    const int j0 = (wk.y & 0xFFFFF) * W;
    const bool no_src = (wk.y >> 20) & 1, no_rec = (wk.y >> 21) & 1;
    const int c0 = j0 - VEC + VEC * lane;
    const bool owner = lane >= 1 && lane <= 30;
    const int ia = wk.z, ib = wk.w;
    // The fast paths are chosen per warp (one uniform branch): a warp whose
    // columns are not all interior / outside the sponge runs the general path
    // on every lane instead of both paths.
    const bool strip_in = __all_sync(FULL, c0 >= 1 && c0 + VEC - 1 <= nz - 2);
    const bool strip_far = __all_sync(FULL, nz - 1 - (c0 + VEC - 1) >= p.fw);
    auto all_in = [&](int i) { return strip_in && i >= 1 && i <= nx - 2; };
    auto all_far = [&](int i) { return strip_far && i >= p.fw && nx - 1 - i >= p.fw; };
    // The general path's per-cell interior test and sponge coefficient,
    // factored into a column part fixed for the task (here, once per lane)
    // and a warp-uniform row part (ColRow below): the same cells are interior
    // and the same sponge entry is chosen as by interior() and sponge_coef().
    bool col_in[VEC], col_sp[VEC];
    int col_db[VEC];
    float col_cr[VEC];
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
        const int j = c0 + q;
        col_in[q] = (unsigned)(j - 1) < (unsigned)(nz - 2);
        col_db[q] = nz - 1 - j;  // distance to the bottom edge
        col_sp[q] = col_db[q] >= 0 && col_db[q] < p.fw;
        col_cr[q] = col_sp[q] ? ldg_chk(p.sponge + col_db[q]) : 1.0f;
    }
    const long long soff = sh.state_off + (long long)(c0 + COL_OFF);
    const long long moff = (long long)sh.x0 * P + (long long)(c0 + COL_OFF);
    const float dt = p.dt, idx = p.inv_dx, idz = p.inv_dz;
    const float sdt = DIR == 0 ? dt : -dt;
    // CKPT: scale block of row -1 of this task's strip (padded row 0 of the shot)
    long long ck_blk0 = 0;
    if constexpr (CKPT) ck_blk0 = (sh.state_off / P) * p.ck.nblk + (wk.y & 0xFFFFF) * (W / ckpt_block_cols(VEC));
    // rows -1 and nx are the zero pad rows of the shot block (and of the
    // material window); rows beyond them read the pad row (header comment)
    auto rowc = [&](int i) { return min(max(i, -1), nx); };
    auto LSt = [&](float (&v)[VEC], int f, int i) { ldv<VEC>(v, p.sin[f] + soff + (long long)(rowc(i) + 1) * P); };
    auto LMt = [&](float (&v)[VEC], int m, int i) { ldv<VEC>(v, p.mat[m] + moff + (long long)(rowc(i) + 1) * P); };
    auto load_sig = [&](int i, Sig &s) {
        if constexpr (PSV) { LSt(s.xx, F_SXX, i); LSt(s.zz, F_SZZ, i); LSt(s.xz, F_SXZ, i); }
        if constexpr (SH) { LSt(s.yx, F_SYX, i); LSt(s.yz, F_SYZ, i); }
    };
    auto load_vel = [&](int i, Vel &v) {
        if constexpr (PSV) { LSt(v.u, F_U, i); LSt(v.w, F_W, i); }
        if constexpr (SH) LSt(v.v, F_V, i);
    };
    auto load_ir = [&](int i, Vel &v) {
        if constexpr (PSV) { LMt(v.u, M_IRU, i); LMt(v.w, M_IRW, i); }
        if constexpr (SH) LMt(v.v, M_IR, i);
    };
    auto load_mat = [&](int i, Mat &m) {
        if constexpr (PSV) { LMt(m.lam, M_LAM, i); LMt(m.mu, M_MU, i); LMt(m.mxz, M_MXZ, i); }
        if constexpr (SH) { LMt(m.myx, M_MYX, i); LMt(m.myz, M_MYZ, i); }
        if (p.surface) {
            ldv<VEC>(m.sm, p.surface + moff + (long long)(rowc(i) + 1) * P);
        } else {
#pragma unroll
            for (int q = 0; q < VEC; ++q) m.sm[q] = 1.f;
        }
    };
    // ---- material ring (RING): slot of a row, copy-in, read-back
    constexpr int NRF = ring2_fields<MODE>();
    constexpr int RF_LAM = 0, RF_MU = 1, RF_MXZ = 2, RF_IRU = 3, RF_IRW = 4;
    constexpr int RF_MYX = PSV ? 5 : 0, RF_MYZ = RF_MYX + 1, RF_IR = RF_MYX + 2;
    constexpr int RF_SM = NRF - 1;
    extern __shared__ float step2_smem[];
    static_assert((RING2_ROWS & (RING2_ROWS - 1)) == 0, "the ring slot is the row modulo a power of two");
    // this lane's VEC floats of slot 0, field 0; a (slot, field) is a fixed
    // 32-bit offset from it (rows >= -2: row & (RING2_ROWS - 1) is the slot)
    float *const ring = step2_smem + (UNI ? 0 : (int)(threadIdx.x >> 5) * (RING2_ROWS * NRF * 32 * VEC)) + lane * VEC;
    auto rslot = [&](int row, int f) { return ring + ((row & (RING2_ROWS - 1)) * NRF + f) * (32 * VEC); };
    auto ring_issue = [&](int row) {
        auto put = [&](int f, const float *src) {
            cp_async_vec<VEC>(rslot(row, f), src + moff + (long long)(rowc(row) + 1) * P);
        };
        if constexpr (PSV) {
            put(RF_LAM, p.mat[M_LAM]); put(RF_MU, p.mat[M_MU]); put(RF_MXZ, p.mat[M_MXZ]);
            put(RF_IRU, p.mat[M_IRU]); put(RF_IRW, p.mat[M_IRW]);
        }
        if constexpr (SH) { put(RF_MYX, p.mat[M_MYX]); put(RF_MYZ, p.mat[M_MYZ]); put(RF_IR, p.mat[M_IR]); }
        if (p.surface) put(RF_SM, p.surface);
        cp_async_commit();  // one group per issued row, so the group counts stay aligned
    };
    auto rd_ring = [&](int row, int f, float (&v)[VEC]) {
        const float *s = rslot(row, f);
#pragma unroll
        for (int q = 0; q < VEC; ++q) v[q] = s[q];
    };
    auto ring_ir = [&](int row, Vel &v) {
        if constexpr (PSV) { rd_ring(row, RF_IRU, v.u); rd_ring(row, RF_IRW, v.w); }
        if constexpr (SH) rd_ring(row, RF_IR, v.v);
    };
    auto ring_mat = [&](int row, Mat &m) {
        if constexpr (PSV) { rd_ring(row, RF_LAM, m.lam); rd_ring(row, RF_MU, m.mu); rd_ring(row, RF_MXZ, m.mxz); }
        if constexpr (SH) { rd_ring(row, RF_MYX, m.myx); rd_ring(row, RF_MYZ, m.myz); }
        if (p.surface) {
            rd_ring(row, RF_SM, m.sm);
        } else {
#pragma unroll
            for (int q = 0; q < VEC; ++q) m.sm[q] = 1.f;
        }
    };
    (void)ring_issue; (void)ring_ir; (void)ring_mat;

    auto cp_sig = [&](Sig &d, const Sig &s) {
        if constexpr (PSV) { copy_arr<VEC>(d.xx, s.xx); copy_arr<VEC>(d.zz, s.zz); copy_arr<VEC>(d.xz, s.xz); }
        if constexpr (SH) { copy_arr<VEC>(d.yx, s.yx); copy_arr<VEC>(d.yz, s.yz); }
    };
    auto cp_vel = [&](Vel &d, const Vel &s) {
        if constexpr (PSV) { copy_arr<VEC>(d.u, s.u); copy_arr<VEC>(d.w, s.w); }
        if constexpr (SH) copy_arr<VEC>(d.v, s.v);
    };
    auto cp_mat = [&](Mat &d, const Mat &s) {
        if constexpr (PSV) { copy_arr<VEC>(d.lam, s.lam); copy_arr<VEC>(d.mu, s.mu); copy_arr<VEC>(d.mxz, s.mxz); }
        if constexpr (SH) { copy_arr<VEC>(d.myx, s.myx); copy_arr<VEC>(d.myz, s.myz); }
        copy_arr<VEC>(d.sm, s.sm);
    };
    auto zero_sig = [&](Sig &s) {
        if constexpr (PSV) { zero_arr<VEC>(s.xx); zero_arr<VEC>(s.zz); zero_arr<VEC>(s.xz); }
        if constexpr (SH) { zero_arr<VEC>(s.yx); zero_arr<VEC>(s.yz); }
    };
    auto zero_vel = [&](Vel &v) {
        if constexpr (PSV) { zero_arr<VEC>(v.u); zero_arr<VEC>(v.w); }
        if constexpr (SH) zero_arr<VEC>(v.v);
    };

    // Velocity update of row r (step time t), the arithmetic of step_kernel.
    // Forward: sc = stress row r, sp = row r-1.  Backward: sc = row r+1,
    // sp = row r.  vo = velocity of row r before the update.  FAST (every
    // column of the lane interior) drops the interior select, nothing else.
    auto vel_cells = [&](auto fast_tag, int r, const Sig &sc, const Sig &sp, const Vel &vo, const Vel &ir,
                         Vel &out, float zz_nb, float xz_nb, float yz_nb) {
        constexpr bool FAST = decltype(fast_tag)::value;
        const bool row_in = (unsigned)(r - 1) < (unsigned)(nx - 2);
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            bool in = true;
            if constexpr (!FAST) in = row_in && col_in[q];
            if constexpr (PSV) {
                float du, dw;
                if constexpr (DIR == 0) {
                    const float sxz_jm = q > 0 ? sc.xz[q - 1] : xz_nb;
                    const float szz_jm = q > 0 ? sc.zz[q - 1] : zz_nb;
                    const float sxx_x = (sc.xx[q] - sp.xx[q]) * idx;  // fm:332
                    const float szz_z = (sc.zz[q] - szz_jm) * idz;    // fm:333
                    const float sxz_x = (sc.xz[q] - sp.xz[q]) * idx;  // fm:334
                    const float sxz_z = (sc.xz[q] - sxz_jm) * idz;    // fm:335
                    du = (sxx_x + sxz_z) * dt * ir.u[q];              // fm:339
                    dw = (sxz_x + szz_z) * dt * ir.w[q];              // fm:340
                } else {
                    const float sxz_jp = q < VEC - 1 ? sp.xz[q + 1] : xz_nb;
                    const float szz_jp = q < VEC - 1 ? sp.zz[q + 1] : zz_nb;
                    const float sxx_x = (sc.xx[q] - sp.xx[q]) * idx;  // bm:333
                    const float szz_z = (szz_jp - sp.zz[q]) * idz;    // bm:334
                    const float sxz_x = (sc.xz[q] - sp.xz[q]) * idx;  // bm:335
                    const float sxz_z = (sxz_jp - sp.xz[q]) * idz;    // bm:336
                    du = -(sxx_x + sxz_z) * dt * ir.u[q];             // bm:340
                    dw = -(sxz_x + szz_z) * dt * ir.w[q];             // bm:341
                }
                if constexpr (FAST) {
                    out.u[q] = vo.u[q] + du;
                    out.w[q] = vo.w[q] + dw;
                } else {
                    out.u[q] = in ? vo.u[q] + du : vo.u[q];
                    out.w[q] = in ? vo.w[q] + dw : vo.w[q];
                }
            }
            if constexpr (SH) {
                float dv;
                if constexpr (DIR == 0) {
                    const float syz_jm = q > 0 ? sc.yz[q - 1] : yz_nb;
                    const float syx_x = (sc.yx[q] - sp.yx[q]) * idx;  // fm:343
                    const float syz_z = (sc.yz[q] - syz_jm) * idz;    // fm:344
                    dv = (syx_x + syz_z) * dt * ir.v[q];              // fm:347
                } else {
                    const float syz_jp = q < VEC - 1 ? sp.yz[q + 1] : yz_nb;
                    const float syx_x = (sc.yx[q] - sp.yx[q]) * idx;  // bm:343
                    const float syz_z = (syz_jp - sp.yz[q]) * idz;    // bm:344
                    dv = -(syx_x + syz_z) * dt * ir.v[q];             // bm:345
                }
                if constexpr (FAST) out.v[q] = vo.v[q] + dv;
                else out.v[q] = in ? vo.v[q] + dv : vo.v[q];
            }
        }
    };
    auto vel_update = [&](int r, int t, const Sig &sc, const Sig &sp, const Vel &vo, const Vel &ir, Vel &out) {
        // column neighbour: j-1 of row r (forward), j+1 of row r (backward)
        float zz_nb = 0.f, xz_nb = 0.f, yz_nb = 0.f;
        if constexpr (DIR == 0) {
            if constexpr (PSV) {
                zz_nb = __shfl_up_sync(FULL, sc.zz[VEC - 1], 1);
                xz_nb = __shfl_up_sync(FULL, sc.xz[VEC - 1], 1);
            }
            if constexpr (SH) yz_nb = __shfl_up_sync(FULL, sc.yz[VEC - 1], 1);
        } else {
            if constexpr (PSV) {
                zz_nb = __shfl_down_sync(FULL, sp.zz[0], 1);
                xz_nb = __shfl_down_sync(FULL, sp.xz[0], 1);
            }
            if constexpr (SH) yz_nb = __shfl_down_sync(FULL, sp.yz[0], 1);
        }
        if (all_in(r)) vel_cells(std::true_type{}, r, sc, sp, vo, ir, out, zz_nb, xz_nb, yz_nb);
        else vel_cells(std::false_type{}, r, sc, sp, vo, ir, out, zz_nb, xz_nb, yz_nb);
        // point injection at time t: forward sources (fm:421-443), backward
        // observed data (bm:452-460); halo lanes too, so halo cells are exact
        if (r < 0 || r >= nx) return;
        if constexpr (DIR == 0) {
            if (no_src) return;
            const int e0 = ldg_chk(p.src_ptr + sh.src_row0 + r), e1 = ldg_chk(p.src_ptr + sh.src_row0 + r + 1);
            for (int e = e0; e < e1; ++e) {
                const int2 en = ldg_chk(p.src_ent + e);
                const int q = en.x - c0;
                if (q < 0 || q >= VEC) continue;
                const bool in = interior(r, en.x, nx, nz);
                const float f = p.src_factor;
                const size_t ti = (size_t)en.y * p.nt + t;
#pragma unroll
                for (int qq = 0; qq < VEC; ++qq) {
                    if (qq != q) continue;
                    if constexpr (PSV) {
                        out.u[qq] += ldg_chk(p.wav[0] + ti) * f * (in ? ir.u[qq] : __int_as_float(0x7f800000));
                        out.w[qq] += ldg_chk(p.wav[2] + ti) * f * (in ? ir.w[qq] : __int_as_float(0x7f800000));
                    }
                    if constexpr (SH) out.v[qq] += ldg_chk(p.wav[1] + ti) * f * ir.v[qq];
                }
            }
        } else {
            if (no_rec) return;
            const int e0 = ldg_chk(p.rec_ptr + sh.rec_row0 + r), e1 = ldg_chk(p.rec_ptr + sh.rec_row0 + r + 1);
            for (int e = e0; e < e1; ++e) {
                const int2 en = ldg_chk(p.rec_ent + e);
                const int q = en.x - c0;
                if (q < 0 || q >= VEC) continue;
                const size_t ti = (size_t)t * p.nrec_total + en.y;
#pragma unroll
                for (int qq = 0; qq < VEC; ++qq) {
                    if (qq != q) continue;
                    if constexpr (PSV) {
                        out.u[qq] += ldg_chk(p.obs[0] + ti);
                        out.w[qq] += ldg_chk(p.obs[2] + ti);
                    }
                    if constexpr (SH) out.v[qq] += ldg_chk(p.obs[1] + ti);
                }
            }
        }
    };

    // Stress update of row r, then absorbing and the surface mask of the
    // next step: va = new velocity of row r, vb = of row r+1 (forward) or
    // r-1 (backward), base = stress of row r before the step.  FAST (every
    // column of the lane interior, outside the sponge, no topography mask)
    // drops the interior select and the multiplications by a coefficient of
    // exactly 1.0, which leave every value unchanged.
    auto stress_cells = [&](auto fast_tag, int r, const Vel &va, const Vel &vb, const Sig &base, const Mat &m,
                            Sig &os, Vel &ov, float nu, float nw, float nv) {
        constexpr bool FAST = decltype(fast_tag)::value;
        // row part of the sponge choice (sponge_coef): d = r if the row is in
        // the left sponge and the cell is farther from the bottom, d = nx-1-r
        // likewise for the right sponge, d = the bottom distance if that is
        // in the sponge and no larger than both row distances (last wins)
        bool row_in = true, ra = false, rb = false;
        int dr = 0;
        float cr_i = 1.0f, cr_dr = 1.0f;
        if constexpr (!FAST) {
            row_in = (unsigned)(r - 1) < (unsigned)(nx - 2);
            dr = nx - 1 - r;
            ra = r >= 0 && r < p.fw;
            rb = dr >= 0 && dr < p.fw;
            if (ra) cr_i = ldg_chk(p.sponge + r);
            if (rb) cr_dr = ldg_chk(p.sponge + dr);
        }
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            bool in = true;
            float cr = 1.0f;
            if constexpr (!FAST) {
                in = row_in && col_in[q];
                if (ra && col_db[q] > r) cr = cr_i;
                if (rb && col_db[q] > dr) cr = cr_dr;
                if (col_sp[q] && r >= col_db[q] && dr >= col_db[q]) cr = col_cr[q];
            }
            if constexpr (PSV) {
                float u_x, u_z, w_x, w_z;
                if constexpr (DIR == 0) {
                    const float uj = q < VEC - 1 ? va.u[q + 1] : nu;
                    const float wj = q < VEC - 1 ? va.w[q + 1] : nw;
                    u_x = (vb.u[q] - va.u[q]) * idx;   // fm:369
                    u_z = (uj - va.u[q]) * idz;        // fm:370
                    w_x = (vb.w[q] - va.w[q]) * idx;   // fm:371
                    w_z = (wj - va.w[q]) * idz;        // fm:372
                } else {
                    const float uj = q > 0 ? va.u[q - 1] : nu;
                    const float wj = q > 0 ? va.w[q - 1] : nw;
                    u_x = (va.u[q] - vb.u[q]) * idx;   // bm:366
                    u_z = (va.u[q] - uj) * idz;        // bm:367
                    w_x = (va.w[q] - vb.w[q]) * idx;   // bm:368
                    w_z = (va.w[q] - wj) * idz;        // bm:369
                }
                const float div = u_x + w_z;
                const float sxx = base.xx[q] + sdt * (m.lam[q] * div + 2.0f * m.mu[q] * u_x);
                const float szz = base.zz[q] + sdt * (m.lam[q] * div + 2.0f * m.mu[q] * w_z);
                const float sxz = base.xz[q] + sdt * m.mxz[q] * (u_z + w_x);
                if constexpr (FAST) {
                    os.xx[q] = sxx;
                    os.zz[q] = szz;
                    os.xz[q] = sxz;
                    ov.u[q] = va.u[q];
                    ov.w[q] = va.w[q];
                } else {
                    os.xx[q] = cr * (in ? sxx : base.xx[q]);
                    os.zz[q] = (cr * (in ? szz : base.zz[q])) * m.sm[q];
                    os.xz[q] = (cr * (in ? sxz : base.xz[q])) * m.sm[q];
                    ov.u[q] = cr * va.u[q];
                    ov.w[q] = cr * va.w[q];
                }
            }
            if constexpr (SH) {
                float v_x, v_z;
                if constexpr (DIR == 0) {
                    const float vj = q < VEC - 1 ? va.v[q + 1] : nv;
                    v_x = (vb.v[q] - va.v[q]) * idx;   // fm:381
                    v_z = (vj - va.v[q]) * idz;        // fm:382
                } else {
                    const float vj = q > 0 ? va.v[q - 1] : nv;
                    v_x = (va.v[q] - vb.v[q]) * idx;   // bm:377
                    v_z = (va.v[q] - vj) * idz;        // bm:378
                }
                const float syx = base.yx[q] + sdt * m.myx[q] * v_x;
                const float syz = base.yz[q] + sdt * m.myz[q] * v_z;
                if constexpr (FAST) {
                    os.yx[q] = syx;
                    os.yz[q] = syz;
                    ov.v[q] = va.v[q];
                } else {
                    os.yx[q] = cr * (in ? syx : base.yx[q]);
                    os.yz[q] = (cr * (in ? syz : base.yz[q])) * m.sm[q];
                    ov.v[q] = cr * va.v[q];
                }
            }
        }
    };
    auto stress_update = [&](int r, const Vel &va, const Vel &vb, const Sig &base, const Mat &m, Sig &os,
                             Vel &ov) {
        float nu = 0.f, nw = 0.f, nv = 0.f;
        if constexpr (DIR == 0) {
            if constexpr (PSV) { nu = __shfl_down_sync(FULL, va.u[0], 1); nw = __shfl_down_sync(FULL, va.w[0], 1); }
            if constexpr (SH) nv = __shfl_down_sync(FULL, va.v[0], 1);
        } else {
            if constexpr (PSV) { nu = __shfl_up_sync(FULL, va.u[VEC - 1], 1); nw = __shfl_up_sync(FULL, va.w[VEC - 1], 1); }
            if constexpr (SH) nv = __shfl_up_sync(FULL, va.v[VEC - 1], 1);
        }
        if (all_in(r) && all_far(r) && p.surface == nullptr)
            stress_cells(std::true_type{}, r, va, vb, base, m, os, ov, nu, nw, nv);
        else
            stress_cells(std::false_type{}, r, va, vb, base, m, os, ov, nu, nw, nv);
    };

    // Per-step outputs of an absorbed velocity row r (owner lanes, r in
    // [ia, ib)): forward receivers at time t and snapshot slot k, backward
    // Kahan imaging against snapshot slot k.
    auto epilogue = [&](int r, int t, int k, const Vel &v) {
        if constexpr (DIR == 0) {
            const int e0 = no_rec ? 0 : ldg_chk(p.rec_ptr + sh.rec_row0 + r);
            const int e1 = no_rec ? 0 : ldg_chk(p.rec_ptr + sh.rec_row0 + r + 1);
            for (int e = e0; e < e1; ++e) {
                const int2 en = ldg_chk(p.rec_ent + e);
                const int q = en.x - c0;
                if (q < 0 || q >= VEC) continue;
                const size_t ti = (size_t)t * p.nrec_total + en.y;
#pragma unroll
                for (int qq = 0; qq < VEC; ++qq) {
                    if (qq != q) continue;
                    if constexpr (PSV) { st_chk(p.seis[0] + ti, v.u[qq]); st_chk(p.seis[2] + ti, v.w[qq]); }
                    if constexpr (SH) st_chk(p.seis[1] + ti, v.v[qq]);
                }
            }
            if (k >= 0) {
                const long long o = ((long long)p.nsnap * sh.row_off + (long long)k * nx + r) * P + c0 + COL_OFF;
                if constexpr (PSV) { stv<VEC>(p.snap[0] + o, v.u); stv<VEC>(p.snap[2] + o, v.w); }
                if constexpr (SH) stv<VEC>(p.snap[1] + o, v.v);
            }
        } else {
            if (k >= 0) {
                const long long o = ((long long)p.nsnap * sh.row_off + (long long)k * nx + r) * P + c0 + COL_OFF;
                const long long io = (sh.row_off + r) * (long long)P + c0 + COL_OFF;
                auto image = [&](int c, const float (&ov)[VEC]) {
                    float s[VEC], sum[VEC], cmp[VEC];
                    ldv<VEC>(s, p.snap[c] + o);
                    ldv_coherent<VEC>(sum, p.img[c] + io);
                    ldv_coherent<VEC>(cmp, p.imgc[c] + io);
#pragma unroll
                    for (int q = 0; q < VEC; ++q) kahan_add(sum[q], cmp[q], __fmul_rn(s[q], ov[q]));
                    stv<VEC>(p.img[c] + io, sum);
                    stv<VEC>(p.imgc[c] + io, cmp);
                };
                if constexpr (PSV) { image(0, v.u); image(2, v.w); }
                if constexpr (SH) image(1, v.v);
            }
        }
    };

    int code = 0;
    auto check_row = [&](const Vel &v) {
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            if constexpr (PSV) {
                code = max(code, bad_code(v.u[q], p.code_base));
                code = max(code, bad_code(v.w[q], p.code_base + 2));
            }
            if constexpr (SH) code = max(code, bad_code(v.v[q], p.code_base + 1));
        }
    };
    // step A's stress and absorbed velocity of row r (STOREA)
    auto store_a = [&](int r, const Sig &os, const Vel &ov) {
        const long long so = soff + (long long)(r + 1) * P;
        if constexpr (PSV) {
            stv<VEC>(p.souta[F_SXX] + so, os.xx);
            stv<VEC>(p.souta[F_SZZ] + so, os.zz);
            stv<VEC>(p.souta[F_SXZ] + so, os.xz);
            stv<VEC>(p.souta[F_U] + so, ov.u);
            stv<VEC>(p.souta[F_W] + so, ov.w);
        }
        if constexpr (SH) {
            stv<VEC>(p.souta[F_SYX] + so, os.yx);
            stv<VEC>(p.souta[F_SYZ] + so, os.yz);
            stv<VEC>(p.souta[F_V] + so, ov.v);
        }
    };
    (void)store_a;
    // step B's stress and absorbed velocity of row r: store, outputs, check
    auto finish_b = [&](int r, const Sig &os, const Vel &ov) {
        if constexpr (CKPT)
            ckpt_pack_row<VEC>(p.ck, soff + (long long)(r + 1) * P, ck_blk0 + (long long)(r + 1) * p.ck.nblk, lane,
                               owner, ov.u, ov.w, os.xx, os.zz, os.xz);
        if (!owner) return;
        const long long so = soff + (long long)(r + 1) * P;
        if constexpr (PSV) {
            stv<VEC>(p.sout[F_SXX] + so, os.xx);
            stv<VEC>(p.sout[F_SZZ] + so, os.zz);
            stv<VEC>(p.sout[F_SXZ] + so, os.xz);
            stv<VEC>(p.sout[F_U] + so, ov.u);
            stv<VEC>(p.sout[F_W] + so, ov.w);
        }
        if constexpr (SH) {
            stv<VEC>(p.sout[F_SYX] + so, os.yx);
            stv<VEC>(p.sout[F_SYZ] + so, os.yz);
            stv<VEC>(p.sout[F_V] + so, ov.v);
        }
        epilogue(r, p.it2, p.snap_k2, ov);
        if (p.check) check_row(ov);
    };

    const int tA = p.it, tB = p.it2;
    if constexpr (RING) {
        // rolling rows as in the register version below, minus 1/rho and the
        // material, which come from the ring at the point of use
        Sig so_p, so_c, sa_p, sa_c, s_out, n_so;
        Vel va_p, va_c, vb_p, vb_c, vo, vabs_c, vabs_p, v_out, n_vo;
        zero_sig(sa_p); zero_sig(sa_c);
        zero_vel(va_p); zero_vel(vb_p); zero_vel(vabs_c); zero_vel(vabs_p);
        load_sig(ia - 2, so_p);
        if constexpr (DIR == 0) {
            // iteration k: A velocity k, A stress k-1, B velocity k-1, B stress k-2;
            // ring rows read: k (1/rho), k-1 (1/rho, material), k-2 (material);
            // issued: row k+1 into the slot of row k-3
            load_sig(ia - 1, n_so);
            load_vel(ia - 1, n_vo);
            ring_issue(ia - 2);
            ring_issue(ia - 1);
            for (int k = ia - 1; k <= ib + 1; ++k) {
                cp_sig(so_c, n_so);
                cp_vel(vo, n_vo);
                if (k <= ib) {
                    load_sig(k + 1, n_so);
                    load_vel(k + 1, n_vo);
                }
                ring_issue(k + 1);
                cp_async_wait<1>();  // every row up to k has landed
                {
                    Vel ir;
                    ring_ir(k, ir);
                    vel_update(k, tA, so_c, so_p, vo, ir, va_c);
                }
                if (k >= ia) {
                    Mat m;
                    ring_mat(k - 1, m);
                    stress_update(k - 1, va_p, va_c, so_p, m, sa_c, vabs_c);
                    if (owner && k - 1 >= ia && k - 1 < ib) {
                        epilogue(k - 1, tA, p.snap_k, vabs_c);
                        if constexpr (STOREA) store_a(k - 1, sa_c, vabs_c);
                    }
                }
                if (k >= ia + 1) {
                    Vel ir;
                    ring_ir(k - 1, ir);
                    vel_update(k - 1, tB, sa_c, sa_p, vabs_c, ir, vb_c);
                }
                if (k >= ia + 2) {
                    Mat m;
                    ring_mat(k - 2, m);
                    stress_update(k - 2, vb_p, vb_c, sa_p, m, s_out, v_out);
                    finish_b(k - 2, s_out, v_out);
                }
                cp_sig(so_p, so_c);
                cp_vel(va_p, va_c);
                cp_sig(sa_p, sa_c);
                cp_vel(vb_p, vb_c);
            }
        } else {
            // iteration k: A velocity k-1, A stress k-1, B velocity k-2, B stress k-2;
            // ring rows read: k-1, k-2; issued: row k into the slot of row k-4
            load_sig(ia - 1, n_so);
            load_vel(ia - 2, n_vo);
            ring_issue(ia - 2);
            for (int k = ia - 1; k <= ib + 1; ++k) {
                cp_sig(so_c, n_so);   // row k
                cp_vel(vo, n_vo);     // row k-1
                if (k <= ib) {
                    load_sig(k + 1, n_so);
                    load_vel(k, n_vo);
                }
                ring_issue(k);
                cp_async_wait<1>();  // every row up to k-1 has landed
                {
                    Vel ir;
                    ring_ir(k - 1, ir);
                    vel_update(k - 1, tA, so_c, so_p, vo, ir, va_c);
                }
                if (k >= ia) {
                    Mat m;
                    ring_mat(k - 1, m);
                    stress_update(k - 1, va_c, va_p, so_p, m, sa_c, vabs_c);
                    if (owner && k - 1 >= ia && k - 1 < ib) epilogue(k - 1, tA, p.snap_k, vabs_c);
                }
                if (k >= ia + 1) {
                    Vel ir;
                    ring_ir(k - 2, ir);
                    vel_update(k - 2, tB, sa_c, sa_p, vabs_p, ir, vb_c);
                }
                if (k >= ia + 2) {
                    Mat m;
                    ring_mat(k - 2, m);
                    stress_update(k - 2, vb_c, vb_p, sa_p, m, s_out, v_out);
                    finish_b(k - 2, s_out, v_out);
                }
                cp_sig(so_p, so_c);
                cp_vel(va_p, va_c);
                cp_sig(sa_p, sa_c);
                cp_vel(vabs_p, vabs_c);
                cp_vel(vb_p, vb_c);
            }
        }
        cp_async_wait<0>();  // no copy outlives the kernel
    } else {
        // rolling rows (see the header comment for which row each holds)
        Sig so_p, so_c, sa_p, sa_c, s_out, n_so;
        Vel va_p, va_c, vb_p, vb_c, vo, ir_p, ir_c, vabs_c, v_out, n_vo, n_ir;
        Mat m_p, m_c, n_m;
        zero_sig(sa_p); zero_sig(sa_c);
        zero_vel(va_p); zero_vel(vb_p); zero_vel(vabs_c);
        load_sig(ia - 2, so_p);

        if constexpr (DIR == 0) {
            // iteration k: A velocity k, A stress k-1, B velocity k-1, B stress k-2
            // prefetched per iteration: old stress, old velocity, 1/rho of row k+1; material of row k
            load_sig(ia - 1, n_so);
            load_vel(ia - 1, n_vo);
            load_ir(ia - 1, n_ir);
            load_mat(ia - 2, n_m);
            for (int k = ia - 1; k <= ib + 1; ++k) {
                cp_sig(so_c, n_so);
                cp_vel(vo, n_vo);
                cp_vel(ir_c, n_ir);
                cp_mat(m_c, n_m);  // row k-1
                if (k <= ib) {
                    load_sig(k + 1, n_so);
                    load_vel(k + 1, n_vo);
                    load_ir(k + 1, n_ir);
                    load_mat(k, n_m);
                }
                vel_update(k, tA, so_c, so_p, vo, ir_c, va_c);
                if (k >= ia) {
                    stress_update(k - 1, va_p, va_c, so_p, m_c, sa_c, vabs_c);
                    if (owner && k - 1 >= ia && k - 1 < ib) {
                        epilogue(k - 1, tA, p.snap_k, vabs_c);
                        if constexpr (STOREA) store_a(k - 1, sa_c, vabs_c);
                    }
                }
                if (k >= ia + 1) vel_update(k - 1, tB, sa_c, sa_p, vabs_c, ir_p, vb_c);
                if (k >= ia + 2) {
                    stress_update(k - 2, vb_p, vb_c, sa_p, m_p, s_out, v_out);
                    finish_b(k - 2, s_out, v_out);
                }
                cp_sig(so_p, so_c);
                cp_vel(va_p, va_c);
                cp_sig(sa_p, sa_c);
                cp_vel(vb_p, vb_c);
                cp_vel(ir_p, ir_c);
                cp_mat(m_p, m_c);
            }
        } else {
            // iteration k: A velocity k-1, A stress k-1, B velocity k-2, B stress k-2
            // prefetched per iteration: old stress of row k+1; old velocity, 1/rho, material of row k
            Vel vabs_p;
            zero_vel(vabs_p);
            load_sig(ia - 1, n_so);
            load_vel(ia - 2, n_vo);
            load_ir(ia - 2, n_ir);
            load_mat(ia - 2, n_m);
            for (int k = ia - 1; k <= ib + 1; ++k) {
                cp_sig(so_c, n_so);   // row k
                cp_vel(vo, n_vo);     // row k-1
                cp_vel(ir_c, n_ir);   // row k-1
                cp_mat(m_c, n_m);     // row k-1
                if (k <= ib) {
                    load_sig(k + 1, n_so);
                    load_vel(k, n_vo);
                    load_ir(k, n_ir);
                    load_mat(k, n_m);
                }
                vel_update(k - 1, tA, so_c, so_p, vo, ir_c, va_c);
                if (k >= ia) {
                    stress_update(k - 1, va_c, va_p, so_p, m_c, sa_c, vabs_c);
                    if (owner && k - 1 >= ia && k - 1 < ib) epilogue(k - 1, tA, p.snap_k, vabs_c);
                }
                if (k >= ia + 1) vel_update(k - 2, tB, sa_c, sa_p, vabs_p, ir_p, vb_c);
                if (k >= ia + 2) {
                    stress_update(k - 2, vb_c, vb_p, sa_p, m_p, s_out, v_out);
                    finish_b(k - 2, s_out, v_out);
                }
                cp_sig(so_p, so_c);
                cp_vel(va_p, va_c);
                cp_sig(sa_p, sa_c);
                cp_vel(vabs_p, vabs_c);
                cp_vel(vb_p, vb_c);
                cp_vel(ir_p, ir_c);
                cp_mat(m_p, m_c);
            }
        }
    }
    if (p.check) {
        code = __reduce_max_sync(FULL, code);
        if (lane == 0 && code > 0) report_failure(p, wk.x, code);
    }
}

}  // namespace rtm
