// Two reversed steps per launch of the exact adjoint (temporal blocking).
//
// adjoint2_kernel reverses forward steps n and n-1 in one pass: the adjoint
// state a_n, b_n is read once and a_{n-2}, b_{n-2} written once, and each
// cell's gradient partials are read and written once for both steps.  Every
// value is computed by the operations of adjoint_step_kernel in the same
// order (the partials get d_n added, then d_{n-1}), so gradients are
// bit-identical to two launches of it.
//
// Rows.  Output row r of one reversed step reads input rows r-1 .. r+1, so a
// task writing rows [ia, ib) computes the first step on rows ia-1 .. ib (one
// extra row each side; those are kept in registers, never stored) from input
// rows ia-2 .. ib+1.  Row indices are clamped to the pad rows -1 .. nx: the
// state there is zero, and the first step's output on a pad row is forced to
// zero, which is what the pad rows hold between two single-step launches.
// Iteration k: first step pointwise row k and finish row k-1, second step
// pointwise row k-1 and finish row k-2.
//
// Columns.  As in the forward two-step kernel, the halo lanes' outermost
// column is wrong after the first step and every column an owner lane reads
// in the second step is exact (VEC >= 2).  The first step's receiver
// injection therefore runs on the halo lanes too.
//
// The host never pairs a step n after which the gradient partials are folded
// (n % GRAD_FOLD_STEPS == 0), nor two steps of different checkpoint segments.
#pragma once
#include "adjoint_kernels.cuh"

namespace rtm {

template <int VEC>
struct AdjIn {  // one row's inputs of one reversed step
    float sxx[VEC], szz[VEC], sxz[VEC], u[VEC], w[VEC];    // forward state before the step
    float bxx[VEC], bzz[VEC], bxz[VEC], au[VEC], aw[VEC];  // adjoint state after it
};
template <int VEC>
struct AdjMat {
    float lam[VEC], mu[VEC], mxz[VEC], sm[VEC], bu[VEC], bw[VEC];
};
template <int VEC>
struct AdjRow {  // one row's pointwise quantities (adjoint_step_kernel's row k-1 registers)
    float sxx[VEC], sxz[VEC], szz[VEC];
    float uxb[VEC], wzb[VEC], xzb[VEC];
    float bxx[VEC], bzz[VEC], bxz[VEC];
    float ins[VEC];
    float up[VEC], wp[VEC], au[VEC], aw[VEC], gu[VEC], gw[VEC], dvu[VEC], dvw[VEC];
};
template <int VEC>
struct AdjOut {
    float xx[VEC], zz[VEC], xz[VEC], u[VEC], w[VEC];
};

// UNI: launched with one warp per CTA, the task is blockIdx.x (the same
// task as the general form computes then), so task-derived values are
// provably warp-uniform; the arithmetic is unchanged.
template <int VEC, bool UNI = false>
__global__ void __launch_bounds__(UNI ? 32 : 256) adjoint2_kernel(const AdjParams p) {
    static_assert(VEC >= 2, "two steps per launch need two halo columns per side");
    constexpr int W = 30 * VEC;
    const int lane = threadIdx.x & 31;
    const int task = UNI ? (int)blockIdx.x : (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (task >= p.n_work) return;
    const int4 wk = p.work[task];
    const ShotDev sh = p.shots[wk.x];
    const int nx = sh.nx, nz = p.nz, P = p.pitch;
    const int c0 = (wk.y & 0xFFFFF) * W - VEC + VEC * lane;
    const bool no_src = (wk.y >> 20) & 1, no_rec = (wk.y >> 21) & 1;
    const bool owner = lane >= 1 && lane <= 30;
    const int ia = wk.z, ib = wk.w;
    const long long soff = sh.state_off + (long long)(c0 + COL_OFF);
    const long long moff = (long long)sh.x0 * P + (long long)(c0 + COL_OFF);
    const float dt = p.dt, idx = p.inv_dx, idz = p.inv_dz;
    const int n1 = p.n, n2 = p.n - 1;  // the forward steps reversed, in order
    auto rowc = [&](int i) { return min(max(i, -1), nx); };
    auto F1 = [&](int f, int i) { return p.fwd[f] + soff + (long long)(rowc(i) + 1) * P; };
    auto F2 = [&](int f, int i) { return p.fwd2[f] + soff + (long long)(rowc(i) + 1) * P; };
    auto A = [&](int f, int i) { return p.ain[f] + soff + (long long)(rowc(i) + 1) * P; };
    auto M = [&](int m, int i) { return p.mat[m] + moff + (long long)(rowc(i) + 1) * P; };

    auto load_mat = [&](int i, AdjMat<VEC> &m, bool vel) {
        ldv<VEC>(m.lam, M(M_LAM, i));
        ldv<VEC>(m.mu, M(M_MU, i));
        ldv<VEC>(m.mxz, M(M_MXZ, i));
        if (p.surface) {
            ldv<VEC>(m.sm, p.surface + moff + (long long)(rowc(i) + 1) * P);
        } else {
#pragma unroll
            for (int q = 0; q < VEC; ++q) m.sm[q] = 1.f;
        }
        if (vel) {
            ldv<VEC>(m.bu, M(M_IRU, i));
            ldv<VEC>(m.bw, M(M_IRW, i));
        } else {
#pragma unroll
            for (int q = 0; q < VEC; ++q) m.bu[q] = m.bw[q] = 0.f;
        }
    };
    auto load_fwd = [&](auto Fp, int i, AdjIn<VEC> &x, bool vel) {
        ldv<VEC>(x.sxx, Fp(A_SXX, i));
        ldv<VEC>(x.szz, Fp(A_SZZ, i));
        ldv<VEC>(x.sxz, Fp(A_SXZ, i));
        if (vel) {
            ldv<VEC>(x.u, Fp(A_U, i));
            ldv<VEC>(x.w, Fp(A_W, i));
        } else {
#pragma unroll
            for (int q = 0; q < VEC; ++q) x.u[q] = x.w[q] = 0.f;
        }
    };
    auto load_adj = [&](int i, AdjIn<VEC> &x, bool vel) {
        ldv<VEC>(x.bxx, A(A_SXX, i));
        ldv<VEC>(x.bzz, A(A_SZZ, i));
        ldv<VEC>(x.bxz, A(A_SXZ, i));
        if (vel) {
            ldv<VEC>(x.au, A(A_U, i));
            ldv<VEC>(x.aw, A(A_W, i));
        } else {
#pragma unroll
            for (int q = 0; q < VEC; ++q) x.au[q] = x.aw[q] = 0.f;
        }
    };

    // Pointwise quantities of row k for reversed step nstep (adjoint_step_kernel,
    // "pointwise quantities of row k"); pr = row k-1; vel = row >= the task's
    // first finished row (the velocity part is not needed above it).
    auto pointwise = [&](int k, int nstep, const AdjIn<VEC> &in, const AdjMat<VEC> &mt, const AdjRow<VEC> &pr,
                         bool vel, AdjRow<VEC> &o) {
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            o.sxx[q] = in.sxx[q]; o.szz[q] = in.szz[q]; o.sxz[q] = in.sxz[q];
            o.bxx[q] = in.bxx[q]; o.bzz[q] = in.bzz[q]; o.bxz[q] = in.bxz[q];
        }
        float cc[VEC];
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            const int j = c0 + q;
            cc[q] = adj_sponge(p.sponge, p.fw, nz, nx, k, j);
            o.ins[q] = interior(k, j, nx, nz) ? 1.f : 0.f;
            o.bxx[q] = cc[q] * o.bxx[q];
            o.bzz[q] = (cc[q] * o.bzz[q]) * mt.sm[q];
            o.bxz[q] = (cc[q] * o.bxz[q]) * mt.sm[q];
            const float Bxx = o.ins[q] != 0.f ? o.bxx[q] : 0.f;
            const float Bzz = o.ins[q] != 0.f ? o.bzz[q] : 0.f;
            const float Bxz = o.ins[q] != 0.f ? o.bxz[q] : 0.f;
            const float l2m = mt.lam[q] + 2.0f * mt.mu[q];
            o.uxb[q] = dt * (l2m * Bxx + mt.lam[q] * Bzz);
            o.wzb[q] = dt * (mt.lam[q] * Bxx + l2m * Bzz);
            o.xzb[q] = dt * (mt.mxz[q] * Bxz);
        }
#pragma unroll
        for (int q = 0; q < VEC; ++q) o.up[q] = o.wp[q] = o.au[q] = o.aw[q] = o.gu[q] = o.gw[q] = o.dvu[q] = o.dvw[q] = 0.f;
        const float sxz_m = __shfl_up_sync(FULL, o.sxz[VEC - 1], 1);
        const float szz_m = __shfl_up_sync(FULL, o.szz[VEC - 1], 1);
        const float xzb_m = __shfl_up_sync(FULL, o.xzb[VEC - 1], 1);
        const float wzb_m = __shfl_up_sync(FULL, o.wzb[VEC - 1], 1);
        if (!vel) return;
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            const float sxz_jm = q > 0 ? o.sxz[q - 1] : sxz_m;
            const float szz_jm = q > 0 ? o.szz[q - 1] : szz_m;
            const float xzb_jm = q > 0 ? o.xzb[q - 1] : xzb_m;
            const float wzb_jm = q > 0 ? o.wzb[q - 1] : wzb_m;
            o.dvu[q] = (o.sxx[q] - pr.sxx[q]) * idx + (o.sxz[q] - sxz_jm) * idz;
            o.dvw[q] = (o.sxz[q] - pr.sxz[q]) * idx + (o.szz[q] - szz_jm) * idz;
            const bool in_ = o.ins[q] != 0.f;
            o.up[q] = in_ ? in.u[q] + o.dvu[q] * dt * mt.bu[q] : in.u[q];
            o.wp[q] = in_ ? in.w[q] + o.dvw[q] * dt * mt.bw[q] : in.w[q];
            o.au[q] = cc[q] * in.au[q] + (pr.uxb[q] - o.uxb[q]) * idx + (xzb_jm - o.xzb[q]) * idz;
            o.aw[q] = cc[q] * in.aw[q] + (pr.xzb[q] - o.xzb[q]) * idx + (wzb_jm - o.wzb[q]) * idz;
            o.gu[q] = in_ ? dt * mt.bu[q] * o.au[q] : 0.f;
            o.gw[q] = in_ ? dt * mt.bw[q] * o.aw[q] : 0.f;
        }
        // sources of row k: recompute injection (fm:421-443)
        if (!no_src && k >= 0 && k < nx && nstep < p.nt) {
            const int e0 = ldg_chk(p.src_ptr + sh.src_row0 + k), e1 = ldg_chk(p.src_ptr + sh.src_row0 + k + 1);
            for (int e = e0; e < e1; ++e) {
                const int2 en = ldg_chk(p.src_ent + e);
                const int q = en.x - c0;
                if (q < 0 || q >= VEC) continue;
                const bool in_ = interior(k, en.x, nx, nz);
                const size_t t = (size_t)en.y * p.nt + nstep;
#pragma unroll
                for (int qq = 0; qq < VEC; ++qq) {
                    if (qq != q) continue;
                    o.up[qq] += ldg_chk(p.wav[0] + t) * p.src_factor * (in_ ? mt.bu[qq] : __int_as_float(0x7f800000));
                    o.wp[qq] += ldg_chk(p.wav[2] + t) * p.src_factor * (in_ ? mt.bw[qq] : __int_as_float(0x7f800000));
                }
            }
        }
    };

    // Finish row r of reversed step nstep from its pointwise row pr and row
    // r+1's cr (adjoint_step_kernel, "finish row r = k-1"): the adjoint state
    // before the step and the gradient contributions.  own: an owner lane on
    // a row the task writes (source gradients there); the receiver injection
    // runs on every lane of a row inside the shot.
    auto finish = [&](int r, int nstep, const AdjRow<VEC> &pr, const AdjRow<VEC> &cr, bool own, AdjOut<VEC> &o,
                      float (&d)[NGRAD][VEC]) {
        const float gu_n = __shfl_down_sync(FULL, pr.gu[0], 1);
        const float gw_n = __shfl_down_sync(FULL, pr.gw[0], 1);
        const float up_n = __shfl_down_sync(FULL, pr.up[0], 1);
        const float wp_n = __shfl_down_sync(FULL, pr.wp[0], 1);
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            const float gu_j = q < VEC - 1 ? pr.gu[q + 1] : gu_n;
            const float gw_j = q < VEC - 1 ? pr.gw[q + 1] : gw_n;
            const float up_j = q < VEC - 1 ? pr.up[q + 1] : up_n;
            const float wp_j = q < VEC - 1 ? pr.wp[q + 1] : wp_n;
            o.xx[q] = pr.bxx[q] + (pr.gu[q] - cr.gu[q]) * idx;
            o.xz[q] = pr.bxz[q] + (pr.gu[q] - gu_j) * idz + (pr.gw[q] - cr.gw[q]) * idx;
            o.zz[q] = pr.bzz[q] + (pr.gw[q] - gw_j) * idz;
            o.u[q] = pr.au[q];
            o.w[q] = pr.aw[q];
            const float u_x = (cr.up[q] - pr.up[q]) * idx;
            const float u_z = (up_j - pr.up[q]) * idz;
            const float w_x = (cr.wp[q] - pr.wp[q]) * idx;
            const float w_z = (wp_j - pr.wp[q]) * idz;
            const bool in_ = pr.ins[q] != 0.f;
            const float Bxx = in_ ? pr.bxx[q] : 0.f, Bzz = in_ ? pr.bzz[q] : 0.f, Bxz = in_ ? pr.bxz[q] : 0.f;
            d[G_LAM][q] = dt * ((Bxx + Bzz) * (u_x + w_z));
            d[G_MU][q] = dt * (2.0f * (Bxx * u_x + Bzz * w_z));
            d[G_MXZ][q] = dt * (Bxz * (u_z + w_x));
            d[G_BU][q] = in_ ? pr.au[q] * (dt * pr.dvu[q]) : 0.f;
            d[G_BW][q] = in_ ? pr.aw[q] * (dt * pr.dvw[q]) : 0.f;
        }
        if (own) {
            const int e0 = !no_src && nstep < p.nt ? ldg_chk(p.src_ptr + sh.src_row0 + r) : 0;
            const int e1 = !no_src && nstep < p.nt ? ldg_chk(p.src_ptr + sh.src_row0 + r + 1) : 0;
            for (int e = e0; e < e1; ++e) {
                const int2 en = ldg_chk(p.src_ent + e);
                const int q = en.x - c0;
                if (q < 0 || q >= VEC) continue;
                const bool in_ = interior(r, en.x, nx, nz);
                const size_t t = (size_t)en.y * p.nt + nstep;
                const float f = p.src_factor;
#pragma unroll
                for (int qq = 0; qq < VEC; ++qq) {
                    if (qq != q || !in_) continue;
                    d[G_BU][qq] += pr.au[qq] * (ldg_chk(p.wav[0] + t) * f);
                    d[G_BW][qq] += pr.aw[qq] * (ldg_chk(p.wav[2] + t) * f);
                    if (p.gwav[0]) {
                        const float bu_r = ldg_chk(M(M_IRU, r) + qq), bw_r = ldg_chk(M(M_IRW, r) + qq);
                        const size_t g = (size_t)nstep * p.nsrc_total + en.y;
                        if (RTM_DBG_OK(p.gwav[0] + g, 4) && RTM_DBG_OK(p.gwav[2] + g, 4)) {
                            p.gwav[0][g] += pr.au[qq] * f * bu_r;
                            p.gwav[2][g] += pr.aw[qq] * f * bw_r;
                        }
                    }
                }
            }
        }
        // R^T g_{nstep-1}: adjoint source at the receivers (fm:445-453 transposed)
        if (!no_rec && nstep >= 1 && r >= 0 && r < nx) {
            const int e0r = ldg_chk(p.rec_ptr + sh.rec_row0 + r), e1r = ldg_chk(p.rec_ptr + sh.rec_row0 + r + 1);
            for (int e = e0r; e < e1r; ++e) {
                const int2 en = ldg_chk(p.rec_ent + e);
                const int q = en.x - c0;
                if (q < 0 || q >= VEC) continue;
                const size_t t = (size_t)(nstep - 1) * p.nrec_total + en.y;
#pragma unroll
                for (int qq = 0; qq < VEC; ++qq) {
                    if (qq != q) continue;
                    o.u[qq] += ldg_chk(p.resid[0] + t);
                    o.w[qq] += ldg_chk(p.resid[2] + t);
                }
            }
        }
    };

    auto zero_row = [&](AdjRow<VEC> &x) {
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            x.sxx[q] = x.sxz[q] = x.szz[q] = x.uxb[q] = x.wzb[q] = x.xzb[q] = 0.f;
            x.bxx[q] = x.bzz[q] = x.bxz[q] = x.ins[q] = 0.f;
            x.up[q] = x.wp[q] = x.au[q] = x.aw[q] = x.gu[q] = x.gw[q] = x.dvu[q] = x.dvw[q] = 0.f;
        }
    };
    AdjRow<VEC> r1p, r2p;  // first / second step: pointwise row k-1 / k-2
    zero_row(r1p);
    zero_row(r2p);
    AdjMat<VEC> m_prev;    // material of row k-1 (the second step's row this iteration)
    float s1[NGRAD][VEC];  // row k-2: partial sums after the first step's contribution
#pragma unroll
    for (int gi = 0; gi < NGRAD; ++gi)
#pragma unroll
        for (int q = 0; q < VEC; ++q) s1[gi][q] = 0.f;
    AdjIn<VEC> in_nxt;
    AdjMat<VEC> m_nxt;
    load_fwd(F1, ia - 2, in_nxt, false);
    load_adj(ia - 2, in_nxt, false);
    load_mat(ia - 2, m_nxt, false);
    for (int k = ia - 2; k <= ib + 1; ++k) {
        const AdjIn<VEC> in1 = in_nxt;
        const AdjMat<VEC> mt = m_nxt;
        if (k <= ib) {
            const bool vn = k + 1 >= ia - 1;
            load_fwd(F1, k + 1, in_nxt, vn);
            load_adj(k + 1, in_nxt, vn);
            load_mat(k + 1, m_nxt, vn);
        }
        AdjIn<VEC> in2;  // the second step's row k-1: forward state n-2 (the adjoint part comes from step 1)
        if (k >= ia) load_fwd(F2, k - 1, in2, k - 1 >= ia);
        // gradient partials of row k-1 (its first-step contribution is added below)
        const long long go1 = (sh.row_off + (k - 1)) * (long long)P + c0 + COL_OFF;
        const bool own1 = owner && k - 1 >= ia && k - 1 < ib;
        float gp[NGRAD][VEC];
        if (own1) {
#pragma unroll
            for (int gi = 0; gi < NGRAD; ++gi) ldv<VEC>(gp[gi], p.gpart[gi] + go1);
        }
        // ---- first step: pointwise row k, finish row k-1
        AdjRow<VEC> r1c;
        pointwise(k, n1, in1, mt, r1p, k >= ia - 1, r1c);
        if (k >= ia) {
            const int r = k - 1;
            AdjOut<VEC> o1;
            float d1[NGRAD][VEC];
            finish(r, n1, r1p, r1c, own1, o1, d1);
            if (r < 0 || r >= nx) {  // pad rows stay zero
#pragma unroll
                for (int q = 0; q < VEC; ++q) o1.xx[q] = o1.zz[q] = o1.xz[q] = o1.u[q] = o1.w[q] = 0.f;
            }
            if (own1) {
#pragma unroll
                for (int gi = 0; gi < NGRAD; ++gi)
#pragma unroll
                    for (int q = 0; q < VEC; ++q) gp[gi][q] = __fadd_rn(gp[gi][q], d1[gi][q]);
            }
            // ---- second step: pointwise row k-1 (adjoint state = the first step's output)
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                in2.bxx[q] = o1.xx[q]; in2.bzz[q] = o1.zz[q]; in2.bxz[q] = o1.xz[q];
                in2.au[q] = o1.u[q]; in2.aw[q] = o1.w[q];
            }
            AdjRow<VEC> r2c;
            pointwise(r, n2, in2, m_prev, r2p, r >= ia, r2c);
            if (k >= ia + 2) {
                // ---- second step: finish row k-2
                const int r2 = k - 2;
                const bool own2 = owner && r2 < ib;
                AdjOut<VEC> o2;
                float d2[NGRAD][VEC];
                finish(r2, n2, r2p, r2c, own2, o2, d2);
                if (own2) {
                    const long long so = soff + (long long)(r2 + 1) * P;
                    stv<VEC>(p.aout[A_U] + so, o2.u);
                    stv<VEC>(p.aout[A_W] + so, o2.w);
                    stv<VEC>(p.aout[A_SXX] + so, o2.xx);
                    stv<VEC>(p.aout[A_SZZ] + so, o2.zz);
                    stv<VEC>(p.aout[A_SXZ] + so, o2.xz);
                    const long long go2 = (sh.row_off + r2) * (long long)P + c0 + COL_OFF;
#pragma unroll
                    for (int gi = 0; gi < NGRAD; ++gi) {
                        float s[VEC];
#pragma unroll
                        for (int q = 0; q < VEC; ++q) s[q] = __fadd_rn(s1[gi][q], d2[gi][q]);
                        stv<VEC>(p.gpart[gi] + go2, s);
                    }
                }
            }
            r2p = r2c;
        }
        // shift: row k-1 becomes row k-2 for the second step's partial sums
        // (read next iteration exactly when own1 holds now)
        if (own1) {
#pragma unroll
            for (int gi = 0; gi < NGRAD; ++gi)
#pragma unroll
                for (int q = 0; q < VEC; ++q) s1[gi][q] = gp[gi][q];
        }
        r1p = r1c;
        m_prev = mt;
    }
}

}  // namespace rtm
