/* C/OpenMP restatement of TaichiRTM's elastic RTM hot path -- TEST
 * INFRASTRUCTURE (the oracle and the timed CPU baseline), never the product.
 *
 * It follows the reference kernels unfused and in the reference's per-step
 * order:
 *   forward  (src/forward_modeling.py:539-572):
 *     surface -> velocity -> sources -> stress -> absorb -> record
 *     -> finite check -> snapshot
 *   backward (src/backward_modeling.py:539-577):
 *     surface -> velocity -> observed-data injection -> stress -> absorb
 *     -> imaging -> finite check
 * Compiled twice: REAL=float (the reference's f32 fields, constants cast to
 * f32 like Taichi's ti.static) and REAL=double.  Built with
 * -ffp-contract=off so the double build matches the NumPy restatement.
 *
 * Layout: (nx, nz), z fastest, like the reference's fields.  Snapshots are
 * (3, nsnap, nx, nz); seismograms and observed data (3, nrec, nt).
 * modes: bit 0 = P-SV (u, w, sxx, szz, sxz), bit 1 = SH (v, syx, syz).  A
 * skipped mode keeps its fields at zero, which equals the reference whenever
 * that mode's sources are zero (the two modes never read each other's fields,
 * forward_modeling.py:330-384).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#ifndef REAL
#define REAL double
#endif
#ifndef SUFFIX
#define SUFFIX f64
#endif
#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUFFIX)

#define IDX(i, j) ((size_t)(i) * (size_t)nz + (size_t)(j))

typedef struct {
    int nx, nz;
    REAL dt, inv_dx, inv_dz, factor;
    REAL *mu, *lam, *rho;  /* borrowed */
    REAL *myx, *myz, *mxz, *rho_u, *rho_w, *inv_rho, *inv_rho_u, *inv_rho_w, *absorb;
    REAL *u, *v, *w, *sxx, *sxz, *szz, *syx, *syz;
    const REAL *surface;
} prop_t;

static REAL *zalloc(size_t n) { return (REAL *)calloc(n, sizeof(REAL)); }

/* forward_modeling.py:203-241: four loops in order, later ones overwrite. */
static void sponge(prop_t *p, int fw) {
    int nx = p->nx, nz = p->nz;
    REAL a = (REAL)0.0053, a_sq = a * a;
    for (size_t k = 0; k < (size_t)nx * nz; ++k) p->absorb[k] = (REAL)1.0;
    for (int i = 0; i < fw; ++i)
        for (int j = 0; j < nz; ++j)
            if (j < nz - i - 1 && i < nx) {
                REAL diff = (REAL)(fw - i);
                p->absorb[IDX(i, j)] = (REAL)exp((double)((-a_sq * diff) * diff));
            }
    for (int i = 0; i < fw; ++i)
        for (int j = 0; j < nz; ++j) {
            int ii = nx - i - 1;
            if (j < nz - i - 1 && ii >= 0 && ii < nx) {
                REAL diff = (REAL)(fw - i);
                p->absorb[IDX(ii, j)] = (REAL)exp((double)((-a_sq * diff) * diff));
            }
        }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < fw; ++j) {
            int jj = nz - j - 1;
            if (i >= j && i < nx - j && jj >= 0 && jj < nz) {
                REAL diff = (REAL)(fw - j);
                p->absorb[IDX(i, jj)] = (REAL)exp((double)((-a_sq * diff) * diff));
            }
        }
}

/* forward_modeling.py:243-307.  With setup_f64 the averages and inverses are
 * evaluated in double and rounded once to REAL: the reference's f32 form of
 * the 4-point harmonic mean (product of four moduli, fm:271-276) overflows
 * f32 for mu > ~4.3e9 Pa, so an f32 evaluation turns mxz into inf.  With
 * setup_f64 = 0 the f32 build reproduces that overflow. */
static void material(prop_t *p, int setup_f64) {
    int nx = p->nx, nz = p->nz;
    const REAL *mu = p->mu, *rho = p->rho;
#pragma omp parallel for
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 1; j < nz - 1; ++j) {
            if (setup_f64) {
                double a = mu[IDX(i, j)], b = mu[IDX(i + 1, j)], c = mu[IDX(i, j + 1)], d = mu[IDX(i + 1, j + 1)];
                p->myx[IDX(i, j)] = (REAL)(2.0 * a * b / (a + b));
                p->myz[IDX(i, j)] = (REAL)(2.0 * a * c / (a + c));
                double prod = a * b * c * d;
                double s = b * c * d + a * c * d + a * b * d + a * b * c;
                p->mxz[IDX(i, j)] = (REAL)(4.0 * prod / s);
                p->rho_u[IDX(i, j)] = (REAL)(0.5 * ((double)rho[IDX(i, j)] + (double)rho[IDX(i + 1, j)]));
                p->rho_w[IDX(i, j)] = (REAL)(0.5 * ((double)rho[IDX(i, j)] + (double)rho[IDX(i, j + 1)]));
            } else {
                REAL a = mu[IDX(i, j)], b = mu[IDX(i + 1, j)], c = mu[IDX(i, j + 1)], d = mu[IDX(i + 1, j + 1)];
                p->myx[IDX(i, j)] = (REAL)2.0 * a * b / (a + b);
                p->myz[IDX(i, j)] = (REAL)2.0 * a * c / (a + c);
                REAL prod = a * b * c * d;
                REAL s = b * c * d + a * c * d + a * b * d + a * b * c;
                p->mxz[IDX(i, j)] = (REAL)4.0 * prod / s;
                p->rho_u[IDX(i, j)] = (REAL)0.5 * (rho[IDX(i, j)] + rho[IDX(i + 1, j)]);
                p->rho_w[IDX(i, j)] = (REAL)0.5 * (rho[IDX(i, j)] + rho[IDX(i, j + 1)]);
            }
        }
#pragma omp parallel for
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < nz; ++j) {
            if (setup_f64) {
                /* rho_u/rho_w were rounded above; invert the exact averages */
                double ru = (i > 0 && i < nx - 1 && j > 0 && j < nz - 1)
                                ? 0.5 * ((double)rho[IDX(i, j)] + (double)rho[IDX(i + 1, j)]) : 0.0;
                double rw = (i > 0 && i < nx - 1 && j > 0 && j < nz - 1)
                                ? 0.5 * ((double)rho[IDX(i, j)] + (double)rho[IDX(i, j + 1)]) : 0.0;
                p->inv_rho[IDX(i, j)] = (REAL)(1.0 / (double)rho[IDX(i, j)]);
                p->inv_rho_u[IDX(i, j)] = (REAL)(1.0 / ru);
                p->inv_rho_w[IDX(i, j)] = (REAL)(1.0 / rw);
            } else {
                p->inv_rho[IDX(i, j)] = (REAL)1.0 / rho[IDX(i, j)];
                p->inv_rho_u[IDX(i, j)] = (REAL)1.0 / p->rho_u[IDX(i, j)];
                p->inv_rho_w[IDX(i, j)] = (REAL)1.0 / p->rho_w[IDX(i, j)];
            }
        }
}

static int prop_init(prop_t *p, int nx, int nz, double dx, double dz, double fs, int fw,
                     const REAL *mu, const REAL *lam, const REAL *rho, const REAL *surface,
                     int setup_f64) {
    memset(p, 0, sizeof(*p));
    p->nx = nx;
    p->nz = nz;
    double dt = 1.0 / fs;
    p->dt = (REAL)dt;
    p->inv_dx = (REAL)(1.0 / dx);
    p->inv_dz = (REAL)(1.0 / dz);
    p->factor = (REAL)(dt * dx * dz);
    p->mu = (REAL *)mu;
    p->lam = (REAL *)lam;
    p->rho = (REAL *)rho;
    p->surface = surface;
    size_t n = (size_t)nx * nz;
    REAL **all[] = {&p->myx, &p->myz, &p->mxz, &p->rho_u, &p->rho_w, &p->inv_rho, &p->inv_rho_u,
                    &p->inv_rho_w, &p->absorb, &p->u, &p->v, &p->w, &p->sxx, &p->sxz, &p->szz,
                    &p->syx, &p->syz};
    for (size_t k = 0; k < sizeof(all) / sizeof(all[0]); ++k) {
        *all[k] = zalloc(n);
        if (!*all[k]) return -1;
    }
    material(p, setup_f64);
    sponge(p, fw);
    return 0;
}

static void prop_free(prop_t *p) {
    REAL *all[] = {p->myx, p->myz, p->mxz, p->rho_u, p->rho_w, p->inv_rho, p->inv_rho_u,
                   p->inv_rho_w, p->absorb, p->u, p->v, p->w, p->sxx, p->sxz, p->szz, p->syx, p->syz};
    for (size_t k = 0; k < sizeof(all) / sizeof(all[0]); ++k) free(all[k]);
}

/* S0: forward_modeling.py:404-419 */
static void surface_step(prop_t *p, int modes) {
    int nx = p->nx, nz = p->nz;
    if (p->surface) {
#pragma omp parallel for
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < nz; ++j) {
                REAL sm = p->surface[IDX(i, j)];
                if (modes & 2) p->syz[IDX(i, j)] *= sm;
                if (modes & 1) { p->sxz[IDX(i, j)] *= sm; p->szz[IDX(i, j)] *= sm; }
            }
    } else {
        for (int i = 0; i < nx; ++i) {
            p->syz[IDX(i, 0)] = 0;
            p->sxz[IDX(i, 0)] = 0;
            p->szz[IDX(i, 0)] = 0;
        }
    }
}

/* S1: forward_modeling.py:309-347 (sgn=+1) / backward_modeling.py:312-345 (sgn=-1) */
static void velocity(prop_t *p, int backward, int modes) {
    int nx = p->nx, nz = p->nz;
    REAL dt = p->dt, idx = p->inv_dx, idz = p->inv_dz;
#pragma omp parallel for
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 1; j < nz - 1; ++j) {
            size_t c = IDX(i, j);
            size_t xn = backward ? IDX(i + 1, j) : IDX(i - 1, j);
            size_t zn = backward ? IDX(i, j + 1) : IDX(i, j - 1);
            if (modes & 1) {
                REAL sxx_x, szz_z, sxz_x, sxz_z;
                if (backward) {
                    sxx_x = (p->sxx[xn] - p->sxx[c]) * idx;
                    szz_z = (p->szz[zn] - p->szz[c]) * idz;
                    sxz_x = (p->sxz[xn] - p->sxz[c]) * idx;
                    sxz_z = (p->sxz[zn] - p->sxz[c]) * idz;
                    p->u[c] += -(sxx_x + sxz_z) * dt * p->inv_rho_u[c];
                    p->w[c] += -(sxz_x + szz_z) * dt * p->inv_rho_w[c];
                } else {
                    sxx_x = (p->sxx[c] - p->sxx[xn]) * idx;
                    szz_z = (p->szz[c] - p->szz[zn]) * idz;
                    sxz_x = (p->sxz[c] - p->sxz[xn]) * idx;
                    sxz_z = (p->sxz[c] - p->sxz[zn]) * idz;
                    p->u[c] += (sxx_x + sxz_z) * dt * p->inv_rho_u[c];
                    p->w[c] += (sxz_x + szz_z) * dt * p->inv_rho_w[c];
                }
            }
            if (modes & 2) {
                REAL syx_x, syz_z;
                if (backward) {
                    syx_x = (p->syx[xn] - p->syx[c]) * idx;
                    syz_z = (p->syz[zn] - p->syz[c]) * idz;
                    p->v[c] += -(syx_x + syz_z) * dt * p->inv_rho[c];
                } else {
                    syx_x = (p->syx[c] - p->syx[xn]) * idx;
                    syz_z = (p->syz[c] - p->syz[zn]) * idz;
                    p->v[c] += (syx_x + syz_z) * dt * p->inv_rho[c];
                }
            }
        }
}

/* S3: forward_modeling.py:349-384 / backward_modeling.py:347-380 */
static void stress(prop_t *p, int backward, int modes) {
    int nx = p->nx, nz = p->nz;
    REAL dt = backward ? -p->dt : p->dt, idx = p->inv_dx, idz = p->inv_dz;
#pragma omp parallel for
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 1; j < nz - 1; ++j) {
            size_t c = IDX(i, j);
            size_t xn = backward ? IDX(i - 1, j) : IDX(i + 1, j);
            size_t zn = backward ? IDX(i, j - 1) : IDX(i, j + 1);
            if (modes & 1) {
                REAL u_x, u_z, w_x, w_z;
                if (backward) {
                    u_x = (p->u[c] - p->u[xn]) * idx;
                    u_z = (p->u[c] - p->u[zn]) * idz;
                    w_x = (p->w[c] - p->w[xn]) * idx;
                    w_z = (p->w[c] - p->w[zn]) * idz;
                } else {
                    u_x = (p->u[xn] - p->u[c]) * idx;
                    u_z = (p->u[zn] - p->u[c]) * idz;
                    w_x = (p->w[xn] - p->w[c]) * idx;
                    w_z = (p->w[zn] - p->w[c]) * idz;
                }
                REAL div = u_x + w_z;
                p->sxx[c] += dt * (p->lam[c] * div + (REAL)2.0 * p->mu[c] * u_x);
                p->szz[c] += dt * (p->lam[c] * div + (REAL)2.0 * p->mu[c] * w_z);
                p->sxz[c] += dt * p->mxz[c] * (u_z + w_x);
            }
            if (modes & 2) {
                REAL v_x, v_z;
                if (backward) {
                    v_x = (p->v[c] - p->v[xn]) * idx;
                    v_z = (p->v[c] - p->v[zn]) * idz;
                } else {
                    v_x = (p->v[xn] - p->v[c]) * idx;
                    v_z = (p->v[zn] - p->v[c]) * idz;
                }
                p->syx[c] += dt * p->myx[c] * v_x;
                p->syz[c] += dt * p->myz[c] * v_z;
            }
        }
}

/* S4: forward_modeling.py:386-402 */
static void absorb(prop_t *p, int modes) {
    size_t n = (size_t)p->nx * p->nz;
#pragma omp parallel for
    for (size_t k = 0; k < n; ++k) {
        REAL c = p->absorb[k];
        if (modes & 1) { p->u[k] *= c; p->w[k] *= c; p->sxx[k] *= c; p->sxz[k] *= c; p->szz[k] *= c; }
        if (modes & 2) { p->v[k] *= c; p->syx[k] *= c; p->syz[k] *= c; }
    }
}

static int bad(REAL x) { return x != x || fabs((double)x) > (double)(REAL)1e30; }

/* forward_modeling.py:455-488 / backward_modeling.py:417-450 */
static int check_finite(prop_t *p, int base) {
    size_t n = (size_t)p->nx * p->nz;
    int code = 0;
#pragma omp parallel for reduction(max : code)
    for (size_t k = 0; k < n; ++k) {
        if (bad(p->u[k]) && code < base) code = base;
        if (bad(p->v[k]) && code < base + 1) code = base + 1;
        if (bad(p->w[k]) && code < base + 2) code = base + 2;
    }
    return code;
}

/* Snapshot storage of component c (0 u, 1 v, 2 w) in a buffer holding only
 * the components whose bit is set in `comps`, in order: its slab index, or
 * -1 when c is not stored. */
static int comp_slab(int comps, int c) {
    if (!(comps & (1 << c))) return -1;
    int k = 0;
    for (int q = 0; q < c; ++q) k += (comps >> q) & 1;
    return k;
}

int FN(rtm_oracle_forward)(int nx, int nz, double dx, double dz, int nt, double fs, int fw,
                           const REAL *mu, const REAL *lam, const REAL *rho, const REAL *surface,
                           int nsrc, const int *src, const REAL *wu, const REAL *wv, const REAL *ww,
                           int nrec, const int *rec, REAL *seis, int isnap, int save, REAL *snaps,
                           int *isnaps, int check_interval, int modes, int nthreads, int nt_run,
                           int setup_f64, int comps) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    prop_t P, *p = &P;
    if (prop_init(p, nx, nz, dx, dz, fs, fw, mu, lam, rho, surface, setup_f64)) return -1;
    size_t n = (size_t)nx * nz;
    int num_snaps = save ? nt / isnap : 0;
    int flag = 0;
    if (nt_run <= 0 || nt_run > nt) nt_run = nt;
    for (int it = 0; it < nt_run; ++it) {
        surface_step(p, modes);
        velocity(p, 0, modes);
        for (int k = 0; k < nsrc; ++k) { /* forward_modeling.py:421-443 */
            size_t c = IDX(src[2 * k], src[2 * k + 1]);
            size_t t = (size_t)k * nt + it;
            p->u[c] += wu[t] * p->factor * p->inv_rho_u[c];
            p->v[c] += wv[t] * p->factor * p->inv_rho[c];
            p->w[c] += ww[t] * p->factor * p->inv_rho_w[c];
        }
        stress(p, 0, modes);
        absorb(p, modes);
        for (int l = 0; l < nrec; ++l) { /* forward_modeling.py:445-453 */
            size_t c = IDX(rec[2 * l], rec[2 * l + 1]);
            seis[(size_t)(0 * nrec + l) * nt + it] = p->u[c];
            seis[(size_t)(1 * nrec + l) * nt + it] = p->v[c];
            seis[(size_t)(2 * nrec + l) * nt + it] = p->w[c];
        }
        if (check_interval > 0 && it % check_interval == 0) {
            flag = check_finite(p, 1);
            if (flag) break;
        }
        if (save && it % isnap == 0 && it != 0) { /* forward_modeling.py:569-572 */
            int k = it / isnap - 1;
            const REAL *src3[3] = {p->u, p->v, p->w};
            for (int c = 0; c < 3; ++c) {
                const int sl = comp_slab(comps, c);
                if (sl >= 0) memcpy(snaps + ((size_t)sl * num_snaps + k) * n, src3[c], n * sizeof(REAL));
            }
            isnaps[k] = it;
        }
    }
    prop_free(p);
    return flag;
}

int FN(rtm_oracle_backward)(int nx, int nz, double dx, double dz, int nt, double fs, int fw,
                            const REAL *mu, const REAL *lam, const REAL *rho, const REAL *surface,
                            int nrec, const int *rec, const REAL *obs, const REAL *snaps,
                            const int *isnaps, int num_snaps, int isnap, REAL *img,
                            int check_interval, int modes, int nthreads, int nt_run,
                            int setup_f64, int comps) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    prop_t P, *p = &P;
    if (prop_init(p, nx, nz, dx, dz, fs, fw, mu, lam, rho, surface, setup_f64)) return -1;
    size_t n = (size_t)nx * nz;
    int flag = 0;
    if (nt_run <= 0 || nt_run > nt) nt_run = nt;
    for (int it = 0; it < nt_run; ++it) {
        surface_step(p, modes);
        velocity(p, 1, modes);
        int t = (nt - 1) - it;
        for (int l = 0; l < nrec; ++l) { /* backward_modeling.py:452-460 */
            size_t c = IDX(rec[2 * l], rec[2 * l + 1]);
            p->u[c] += obs[(size_t)(0 * nrec + l) * nt + t];
            p->v[c] += obs[(size_t)(1 * nrec + l) * nt + t];
            p->w[c] += obs[(size_t)(2 * nrec + l) * nt + t];
        }
        stress(p, 1, modes);
        absorb(p, modes);
        if (t > 0 && t % isnap == 0) { /* backward_modeling.py:556-564 */
            int k = t / isnap - 1;
            if (k >= 0 && k < num_snaps && isnaps[k] == t) {
                const REAL *bw3[3] = {p->u, p->v, p->w};
                for (int c = 0; c < 3; ++c) {  /* components not stored image as zero */
                    const int sl = comp_slab(comps, c);
                    if (sl < 0) continue;
                    const REAL *sn = snaps + ((size_t)sl * num_snaps + k) * n;
                    const REAL *b = bw3[c];
                    REAL *im = img + (size_t)c * n;
#pragma omp parallel for
                    for (size_t q = 0; q < n; ++q) im[q] += sn[q] * b[q];
                }
            }
        }
        if (check_interval > 0 && it % check_interval == 0) {
            flag = check_finite(p, 4);
            if (flag) break;
        }
    }
    prop_free(p);
    return flag;
}

int FN(rtm_oracle_max_threads)(void) { return omp_get_max_threads(); }
