// Exact discrete adjoint of the P-SV forward step (no counterpart in the
// reference, whose backward propagation is neither the adjoint nor the time
// reverse of its forward: it uses -dt with transposed difference directions,
// src/backward_modeling.py:312-380).
//
// Forward step n in stored quantities (V = (u, w), S = (sxx, szz, sxz), I =
// interior mask, c = sponge, m = surface mask on sxz/szz, B = (inv_rho_u,
// inv_rho_w), Dv = backward differences of the velocity update, Ds = forward
// differences of the stress update, C = (lam, mu, mxz)):
//   v'_n = V_{n-1} + I dt B Dv(S_{n-1}) + src_n                      (fm:330-347, 421-443)
//   s'_n = S_{n-1} + I dt C(Ds(v'_n))                                (fm:367-384)
//   V_n  = c v'_n,   S_n = c m s'_n                                  (fm:386-419)
//   d_n  = R V_n                                                     (fm:445-453)
// Its adjoint, with a_n = dJ/dV_n and b_n = dJ/dS_n:
//   beta'  = c m b_n,      beta = I beta'
//   ubar   = dt C^T beta   (adjoint strain rates u_x, w_z and u_z = w_x)
//   alpha' = c a_n + Ds^T ubar                    (= dJ/dv'_n)
//   gamma  = I dt B alpha'
//   b_{n-1} = beta' + Dv^T gamma,   a_{n-1} = alpha' + R^T g_{n-1}
// and the model gradients accumulated over n (FP32 partials folded into
// Kahan pairs every GRAD_FOLD_STEPS steps):
//   dJ/dlam += dt (beta_xx + beta_zz) div(v'_n),  dJ/dmu += 2 dt (beta_xx u_x + beta_zz w_z),
//   dJ/dmxz += dt beta_xz (u_z + w_x),            dJ/dB   += alpha' I dt Dv(S_{n-1})
//                                                           (+ alpha' w_n f at interior sources),
// and dJ/dw_n = alpha'(src) f B(src) for the wavelets.
//
// One launch reverses step n for every shot.  Rows stream like the forward
// kernel: lanes 1..30 own VEC columns each, lanes 0 / 31 are the column halo,
// and row r = k-1 is finished while row k streams in, so every neighbour is in
// a register or one shuffle away.  v'_n is recomputed on the fly from the
// stored forward state n-1.
#pragma once
#include "step_kernels.cuh"

namespace rtm {

enum AdjField { A_U = 0, A_W, A_SXX, A_SZZ, A_SXZ, NADJ };
enum Grad { G_LAM = 0, G_MU, G_MXZ, G_BU, G_BW, NGRAD };

struct AdjParams {
    int nz, pitch, nt, fw;
    float dt, inv_dx, inv_dz, src_factor;
    const float *sponge;
    const int4 *work;
    int n_work;
    const ShotDev *shots;
    const float *fwd[NADJ];   // forward state n-1 (stored, absorbed): u, w, sxx, szz, sxz
    const float *fwd2[NADJ];  // forward state n-2 (adjoint2_kernel: the second step reversed)
    const float *ain[NADJ];   // adjoint state n
    float *aout[NADJ];        // adjoint state n-1
    const float *mat[NMAT];
    const float *surface;
    const int *src_ptr;
    const int2 *src_ent;
    const float *wav[3];      // (nsrc_total, nt)
    const int *rec_ptr;
    const int2 *rec_ent;
    int nrec_total;
    const float *resid[3];    // time-major (nt, nrec_total): dJ/d(seismogram)
    float *gpart[NGRAD];      // per shot [row_off + i][pitch]: FP32 partial sums since the last fold
    float *gwav[3];           // time-major (nt, nsrc_total) dJ/d(wavelet), or null
    int nsrc_total;
    int n;                    // forward step reversed by this launch
};

// Initial adjoint state a_{nt-1} = R^T g_{nt-1}: the last residual sample is
// added at the receivers.  One thread per (row, shot = blockIdx.y) walks its
// row's receivers in order, so duplicates at one cell accumulate in receiver
// order (deterministic); different rows are different cells.  resid_t is
// time-major, 3 planes of (nt, nrec_total).
static __global__ void inject_last_resid_kernel(const ShotDev *__restrict__ shots, int nshots,
                                                const int *__restrict__ rec_ptr, const int2 *__restrict__ rec_ent,
                                                const float *__restrict__ resid_t, int nt, int nrec_total,
                                                int nz, int pitch, float *au, float *aw) {
    const int s = blockIdx.y;
    if (s >= nshots) return;
    (void)nz;
    const ShotDev sh = shots[s];
    const size_t plane = (size_t)nt * nrec_total;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < sh.nx; i += gridDim.x * blockDim.x)
        for (int e = rec_ptr[sh.rec_row0 + i]; e < rec_ptr[sh.rec_row0 + i + 1]; ++e) {
            const int2 en = rec_ent[e];
            const long long o = sh.state_off + (long long)(i + 1) * pitch + en.x + COL_OFF;
            const size_t t = (size_t)(nt - 1) * nrec_total + en.y;
            if (!RTM_DBG_OK(au + o, 4) || !RTM_DBG_OK(aw + o, 4) || !RTM_DBG_OK(resid_t + t, 4) ||
                !RTM_DBG_OK(resid_t + 2 * plane + t, 4))
                continue;
            au[o] += resid_t[t];
            aw[o] += resid_t[2 * plane + t];
        }
}

// Gradient accumulation: every adjoint step adds its contribution to a plain
// FP32 partial sum (one read and one write per cell and gradient); every
// GRAD_FOLD_STEPS reversed steps, counted on the global step number n (so
// the grouping does not depend on the checkpoint interval), the partials are
// folded into a Kahan pair (sum, comp) and cleared.  A partial holds at most
// 64 terms, so its relative rounding error stays below 64 x 2^-24.
constexpr int GRAD_FOLD_STEPS = 64;

struct GradFold {
    float *part[NGRAD], *sum[NGRAD], *comp[NGRAD];
    long long n;  // floats per array
};

static __global__ void grad_fold_kernel(const GradFold f) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < f.n;
         i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int g = 0; g < NGRAD; ++g) {
            float s = f.sum[g][i], c = f.comp[g][i];
            kahan_add(s, c, f.part[g][i]);
            f.sum[g][i] = s;
            f.comp[g][i] = c;
            f.part[g][i] = 0.f;
        }
    }
}

// Same coefficient as sponge_coef (forward_modeling.py:203-235 loop order).
__device__ __forceinline__ float adj_sponge(const float *prof, int fw, int nz, int nx, int i, int j) {
    const int db = nz - 1 - j, dr = nx - 1 - i;
    int d = -1;
    if (i >= 0 && i < fw && db > i) d = i;
    if (dr >= 0 && dr < fw && db > dr) d = dr;
    if (db >= 0 && db < fw && i >= db && dr >= db) d = db;
    return d >= 0 ? ldg_chk(prof + d) : 1.0f;
}

// UNI: launched with one warp per CTA, the task is blockIdx.x (the same
// task as the general form computes then), so task-derived values are
// provably warp-uniform; the arithmetic is unchanged.
template <int VEC, bool UNI = false>
__global__ void __launch_bounds__(UNI ? 32 : 256) adjoint_step_kernel(const AdjParams p) {
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
    const int n = p.n;
    auto F = [&](int f, int i) { return p.fwd[f] + soff + (long long)(i + 1) * P; };
    auto A = [&](int f, int i) { return p.ain[f] + soff + (long long)(i + 1) * P; };
    auto M = [&](int m, int i) { return p.mat[m] + moff + (long long)(i + 1) * P; };

    // row k-1 registers
    float sxx_p[VEC], sxz_p[VEC], szz_p[VEC];  // forward stress
    float uxb_p[VEC], wzb_p[VEC], xzb_p[VEC];  // adjoint strain rates
    float bxx_p[VEC], bzz_p[VEC], bxz_p[VEC];  // beta'
    float ins_p[VEC];                          // interior mask (1/0)
    float up_p[VEC], wp_p[VEC];                // v'_n
    float au_p[VEC], aw_p[VEC];                // alpha'
    float gu_p[VEC], gw_p[VEC];                // gamma
    float dvu_p[VEC], dvw_p[VEC];              // Dv(S_{n-1})
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
        sxx_p[q] = sxz_p[q] = szz_p[q] = 0.f;
        uxb_p[q] = wzb_p[q] = xzb_p[q] = 0.f;
        bxx_p[q] = bzz_p[q] = bxz_p[q] = 0.f;
        ins_p[q] = 0.f;
        up_p[q] = wp_p[q] = au_p[q] = aw_p[q] = gu_p[q] = gw_p[q] = dvu_p[q] = dvw_p[q] = 0.f;
    }

    // Inputs of one row, loaded one iteration ahead (software pipelining:
    // the loads of row k+1 are in flight while row k is computed).
    struct Row {
        float sxx[VEC], szz[VEC], sxz[VEC], bxx[VEC], bzz[VEC], bxz[VEC];
        float lam[VEC], mu[VEC], mxz[VEC], sm[VEC];
        float u[VEC], w[VEC], au[VEC], aw[VEC], bu[VEC], bw[VEC];  // rows >= ia only
    };
    auto load_row = [&](int i, Row &x, bool vel) {
        ldv<VEC>(x.sxx, F(A_SXX, i));
        ldv<VEC>(x.szz, F(A_SZZ, i));
        ldv<VEC>(x.sxz, F(A_SXZ, i));
        ldv<VEC>(x.bxx, A(A_SXX, i));
        ldv<VEC>(x.bzz, A(A_SZZ, i));
        ldv<VEC>(x.bxz, A(A_SXZ, i));
        ldv<VEC>(x.lam, M(M_LAM, i));
        ldv<VEC>(x.mu, M(M_MU, i));
        ldv<VEC>(x.mxz, M(M_MXZ, i));
        if (p.surface) {
            ldv<VEC>(x.sm, p.surface + moff + (long long)(i + 1) * P);
        } else {
#pragma unroll
            for (int q = 0; q < VEC; ++q) x.sm[q] = 1.f;
        }
        if (vel) {
            ldv<VEC>(x.u, F(A_U, i));
            ldv<VEC>(x.w, F(A_W, i));
            ldv<VEC>(x.au, A(A_U, i));
            ldv<VEC>(x.aw, A(A_W, i));
            ldv<VEC>(x.bu, M(M_IRU, i));
            ldv<VEC>(x.bw, M(M_IRW, i));
        } else {
#pragma unroll
            for (int q = 0; q < VEC; ++q) x.u[q] = x.w[q] = x.au[q] = x.aw[q] = x.bu[q] = x.bw[q] = 0.f;
        }
    };
    Row nxt;
    load_row(ia - 1, nxt, false);  // row ia-1 needs no velocity inputs
    for (int k = ia - 1; k <= ib; ++k) {
        // ---- pointwise quantities of row k
        const Row cur = nxt;
        if (k < ib) load_row(k + 1, nxt, true);
        // gradient partial sums of row k-1 (finished below): issued here so
        // that their latency overlaps the arithmetic of row k (at VEC 4 the
        // registers are not there: loaded where they are used)
        constexpr bool HOIST = VEC <= 2;
        float gp[NGRAD][VEC];
        const long long go = (sh.row_off + (k - 1)) * (long long)P + c0 + COL_OFF;
        if (HOIST && k >= ia + 1 && owner) {
#pragma unroll
            for (int gi = 0; gi < NGRAD; ++gi) ldv<VEC>(gp[gi], p.gpart[gi] + go);
        }
        float sxx[VEC], szz[VEC], sxz[VEC], bxx[VEC], bzz[VEC], bxz[VEC];
        float lam[VEC], mu[VEC], mxz[VEC], sm[VEC];
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            sxx[q] = cur.sxx[q]; szz[q] = cur.szz[q]; sxz[q] = cur.sxz[q];
            bxx[q] = cur.bxx[q]; bzz[q] = cur.bzz[q]; bxz[q] = cur.bxz[q];
            lam[q] = cur.lam[q]; mu[q] = cur.mu[q]; mxz[q] = cur.mxz[q]; sm[q] = cur.sm[q];
        }
        float cc[VEC], ins[VEC], uxb[VEC], wzb[VEC], xzb[VEC];
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            const int j = c0 + q;
            cc[q] = adj_sponge(p.sponge, p.fw, nz, nx, k, j);
            ins[q] = interior(k, j, nx, nz) ? 1.f : 0.f;
            bxx[q] = cc[q] * bxx[q];                 // beta' = c m b
            bzz[q] = (cc[q] * bzz[q]) * sm[q];
            bxz[q] = (cc[q] * bxz[q]) * sm[q];
            const float Bxx = ins[q] != 0.f ? bxx[q] : 0.f;  // beta = I beta'
            const float Bzz = ins[q] != 0.f ? bzz[q] : 0.f;
            const float Bxz = ins[q] != 0.f ? bxz[q] : 0.f;
            const float l2m = lam[q] + 2.0f * mu[q];
            uxb[q] = dt * (l2m * Bxx + lam[q] * Bzz);
            wzb[q] = dt * (lam[q] * Bxx + l2m * Bzz);
            xzb[q] = dt * (mxz[q] * Bxz);
        }
        float up[VEC], wp[VEC], au[VEC], aw[VEC], gu[VEC], gw[VEC], dvu[VEC], dvw[VEC];
#pragma unroll
        for (int q = 0; q < VEC; ++q) up[q] = wp[q] = au[q] = aw[q] = gu[q] = gw[q] = dvu[q] = dvw[q] = 0.f;
        // column j-1 neighbours of row k
        const float sxz_m = __shfl_up_sync(FULL, sxz[VEC - 1], 1);
        const float szz_m = __shfl_up_sync(FULL, szz[VEC - 1], 1);
        const float xzb_m = __shfl_up_sync(FULL, xzb[VEC - 1], 1);
        const float wzb_m = __shfl_up_sync(FULL, wzb[VEC - 1], 1);
        if (k >= ia) {
            const float(&u)[VEC] = cur.u;
            const float(&w)[VEC] = cur.w;
            const float(&au_in)[VEC] = cur.au;
            const float(&aw_in)[VEC] = cur.aw;
            const float(&bu)[VEC] = cur.bu;
            const float(&bw)[VEC] = cur.bw;
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                const float sxz_jm = q > 0 ? sxz[q - 1] : sxz_m;
                const float szz_jm = q > 0 ? szz[q - 1] : szz_m;
                const float xzb_jm = q > 0 ? xzb[q - 1] : xzb_m;
                const float wzb_jm = q > 0 ? wzb[q - 1] : wzb_m;
                // forward recompute of v'_n (fm:332-340)
                dvu[q] = (sxx[q] - sxx_p[q]) * idx + (sxz[q] - sxz_jm) * idz;
                dvw[q] = (sxz[q] - sxz_p[q]) * idx + (szz[q] - szz_jm) * idz;
                const bool in = ins[q] != 0.f;
                up[q] = in ? u[q] + dvu[q] * dt * bu[q] : u[q];
                wp[q] = in ? w[q] + dvw[q] * dt * bw[q] : w[q];
                // alpha' = c a + Ds^T ubar
                au[q] = cc[q] * au_in[q] + (uxb_p[q] - uxb[q]) * idx + (xzb_jm - xzb[q]) * idz;
                aw[q] = cc[q] * aw_in[q] + (xzb_p[q] - xzb[q]) * idx + (wzb_jm - wzb[q]) * idz;
                gu[q] = in ? dt * bu[q] * au[q] : 0.f;
                gw[q] = in ? dt * bw[q] * aw[q] : 0.f;
            }
            // sources of row k: recompute injection (fm:421-443)
            if (!no_src && k < nx && n < p.nt) {
                const int e0 = ldg_chk(p.src_ptr + sh.src_row0 + k), e1 = ldg_chk(p.src_ptr + sh.src_row0 + k + 1);
                for (int e = e0; e < e1; ++e) {
                    const int2 en = ldg_chk(p.src_ent + e);
                    const int q = en.x - c0;
                    if (q < 0 || q >= VEC) continue;
                    const bool in = interior(k, en.x, nx, nz);
                    const size_t t = (size_t)en.y * p.nt + n;
#pragma unroll
                    for (int qq = 0; qq < VEC; ++qq) {
                        if (qq != q) continue;
                        up[qq] += ldg_chk(p.wav[0] + t) * p.src_factor * (in ? bu[qq] : __int_as_float(0x7f800000));
                        wp[qq] += ldg_chk(p.wav[2] + t) * p.src_factor * (in ? bw[qq] : __int_as_float(0x7f800000));
                    }
                }
            }
        }
        if (k >= ia + 1) {
            // ---- finish row r = k-1
            const int r = k - 1;
            const float gu_n = __shfl_down_sync(FULL, gu_p[0], 1);  // gamma(r, j+1)
            const float gw_n = __shfl_down_sync(FULL, gw_p[0], 1);
            const float up_n = __shfl_down_sync(FULL, up_p[0], 1);  // v'(r, j+1)
            const float wp_n = __shfl_down_sync(FULL, wp_p[0], 1);
            float oxx[VEC], ozz[VEC], oxz[VEC], ou[VEC], ow[VEC];
            float dl[VEC], dm[VEC], dxz[VEC], dbu[VEC], dbw[VEC];
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                const float gu_j = q < VEC - 1 ? gu_p[q + 1] : gu_n;
                const float gw_j = q < VEC - 1 ? gw_p[q + 1] : gw_n;
                const float up_j = q < VEC - 1 ? up_p[q + 1] : up_n;
                const float wp_j = q < VEC - 1 ? wp_p[q + 1] : wp_n;
                // b_{n-1} = beta' + Dv^T gamma
                oxx[q] = bxx_p[q] + (gu_p[q] - gu[q]) * idx;
                oxz[q] = bxz_p[q] + (gu_p[q] - gu_j) * idz + (gw_p[q] - gw[q]) * idx;
                ozz[q] = bzz_p[q] + (gw_p[q] - gw_j) * idz;
                ou[q] = au_p[q];
                ow[q] = aw_p[q];
                // gradients from v'_n (fm:369-378) and Dv(S_{n-1})
                const float u_x = (up[q] - up_p[q]) * idx;
                const float u_z = (up_j - up_p[q]) * idz;
                const float w_x = (wp[q] - wp_p[q]) * idx;
                const float w_z = (wp_j - wp_p[q]) * idz;
                const bool in = ins_p[q] != 0.f;
                const float Bxx = in ? bxx_p[q] : 0.f, Bzz = in ? bzz_p[q] : 0.f, Bxz = in ? bxz_p[q] : 0.f;
                dl[q] = dt * ((Bxx + Bzz) * (u_x + w_z));
                dm[q] = dt * (2.0f * (Bxx * u_x + Bzz * w_z));
                dxz[q] = dt * (Bxz * (u_z + w_x));
                dbu[q] = in ? au_p[q] * (dt * dvu_p[q]) : 0.f;
                dbw[q] = in ? aw_p[q] * (dt * dvw_p[q]) : 0.f;
            }
            if (owner) {
                // sources of row r: gradient of the injection scale and wavelet gradient
                const int e0 = !no_src && n < p.nt ? ldg_chk(p.src_ptr + sh.src_row0 + r) : 0;
                const int e1 = !no_src && n < p.nt ? ldg_chk(p.src_ptr + sh.src_row0 + r + 1) : 0;
                for (int e = e0; e < e1; ++e) {
                    const int2 en = ldg_chk(p.src_ent + e);
                    const int q = en.x - c0;
                    if (q < 0 || q >= VEC) continue;
                    const bool in = interior(r, en.x, nx, nz);
                    const size_t t = (size_t)en.y * p.nt + n;
                    const float f = p.src_factor;
#pragma unroll
                    for (int qq = 0; qq < VEC; ++qq) {
                        if (qq != q || !in) continue;
                        dbu[qq] += au_p[qq] * (ldg_chk(p.wav[0] + t) * f);
                        dbw[qq] += aw_p[qq] * (ldg_chk(p.wav[2] + t) * f);
                        if (p.gwav[0]) {
                            const float bu_r = ldg_chk(M(M_IRU, r) + qq), bw_r = ldg_chk(M(M_IRW, r) + qq);
                            const size_t g = (size_t)n * p.nsrc_total + en.y;
                            if (RTM_DBG_OK(p.gwav[0] + g, 4) && RTM_DBG_OK(p.gwav[2] + g, 4)) {
                                p.gwav[0][g] += au_p[qq] * f * bu_r;
                                p.gwav[2][g] += aw_p[qq] * f * bw_r;
                            }
                        }
                    }
                }
                // R^T g_{n-1}: adjoint source at the receivers (fm:445-453 transposed)
                if (!no_rec && n >= 1) {
                    const int e0r = ldg_chk(p.rec_ptr + sh.rec_row0 + r), e1r = ldg_chk(p.rec_ptr + sh.rec_row0 + r + 1);
                    for (int e = e0r; e < e1r; ++e) {
                        const int2 en = ldg_chk(p.rec_ent + e);
                        const int q = en.x - c0;
                        if (q < 0 || q >= VEC) continue;
                        const size_t t = (size_t)(n - 1) * p.nrec_total + en.y;
#pragma unroll
                        for (int qq = 0; qq < VEC; ++qq) {
                            if (qq != q) continue;
                            ou[qq] += ldg_chk(p.resid[0] + t);
                            ow[qq] += ldg_chk(p.resid[2] + t);
                        }
                    }
                }
                const long long so = soff + (long long)(r + 1) * P;
                stv<VEC>(p.aout[A_U] + so, ou);
                stv<VEC>(p.aout[A_W] + so, ow);
                stv<VEC>(p.aout[A_SXX] + so, oxx);
                stv<VEC>(p.aout[A_SZZ] + so, ozz);
                stv<VEC>(p.aout[A_SXZ] + so, oxz);
                auto acc = [&](int gi, const float (&d)[VEC]) {
                    float s[VEC];
                    if constexpr (!HOIST) ldv<VEC>(gp[gi], p.gpart[gi] + go);
#pragma unroll
                    for (int q = 0; q < VEC; ++q) s[q] = __fadd_rn(gp[gi][q], d[q]);
                    stv<VEC>(p.gpart[gi] + go, s);
                };
                acc(G_LAM, dl);
                acc(G_MU, dm);
                acc(G_MXZ, dxz);
                acc(G_BU, dbu);
                acc(G_BW, dbw);
            }
        }
        // ---- shift row k into the row k-1 registers
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            sxx_p[q] = sxx[q]; sxz_p[q] = sxz[q]; szz_p[q] = szz[q];
            uxb_p[q] = uxb[q]; wzb_p[q] = wzb[q]; xzb_p[q] = xzb[q];
            bxx_p[q] = bxx[q]; bzz_p[q] = bzz[q]; bxz_p[q] = bxz[q];
            ins_p[q] = ins[q];
            up_p[q] = up[q]; wp_p[q] = wp[q]; au_p[q] = au[q]; aw_p[q] = aw[q];
            gu_p[q] = gu[q]; gw_p[q] = gw[q]; dvu_p[q] = dvu[q]; dvw_p[q] = dvw[q];
        }
    }
}

}  // namespace rtm
