// One-time and per-call helper kernels: material set-up, layout transposes,
// image finalisation and the FP64 cross-shot stack.
#pragma once
#include <cuda_runtime.h>
#include "step_kernels.cuh"

namespace rtm {

// ForwardModeling._compute_shear_avg / _compute_rho_avg / _compute_inv_rho
// (forward_modeling.py:243-307) into the padded layout, evaluated in double
// and rounded once to float.  The reference's f32 form multiplies four
// moduli (fm:271) and overflows f32 for mu > ~4.3e9 Pa; in double the same
// formula is exact to rounding.  Averages are interior-only (0 on edges), so
// inv_rho_u / inv_rho_w are +inf on the edge cells exactly as in the
// reference.  mu, lam, rho: (nx, nz) contiguous.  Null outputs are skipped
// (fields of a mode the plan does not propagate).
static __global__ void setup_material_kernel(const float *__restrict__ mu, const float *__restrict__ lam,
                                      const float *__restrict__ rho, const float *__restrict__ surface,
                                      int nx, int nz, int pitch, float *iru, float *irw, float *olam,
                                      float *omu, float *mxz, float *ir, float *myx, float *myz,
                                      float *osurf) {
    const long long n = (long long)nx * nz;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / nz), j = (int)(idx % nz);
        const long long o = (long long)(i + 1) * pitch + j + COL_OFF;
        const bool in = i >= 1 && i <= nx - 2 && j >= 1 && j <= nz - 2;
        const double r0 = rho[idx];
        double ru = 0.0, rw = 0.0, hyx = 0.0, hyz = 0.0, hxz = 0.0;
        if (in) {
            const double a = mu[idx], b = mu[idx + nz], c = mu[idx + 1], d = mu[idx + nz + 1];
            hyx = 2.0 * a * b / (a + b);                                   // fm:265
            hyz = 2.0 * a * c / (a + c);                                   // fm:266
            const double prod = a * b * c * d;                             // fm:271
            const double s = b * c * d + a * c * d + a * b * d + a * b * c;  // fm:272-275
            hxz = 4.0 * prod / s;                                          // fm:276
            ru = 0.5 * (r0 + (double)rho[idx + nz]);                       // fm:288
            rw = 0.5 * (r0 + (double)rho[idx + 1]);                        // fm:289
        }
        if (myx) myx[o] = (float)hyx;
        if (myz) myz[o] = (float)hyz;
        if (mxz) mxz[o] = (float)hxz;
        if (ir) ir[o] = (float)(1.0 / r0);     // fm:305
        if (iru) iru[o] = (float)(1.0 / ru);   // fm:306 (+inf on edges)
        if (irw) irw[o] = (float)(1.0 / rw);   // fm:307
        if (olam) olam[o] = lam[idx];
        if (omu) omu[o] = mu[idx];
        if (osurf) osurf[o] = surface[idx];
    }
}

// (rows, cols) -> (cols, rows) for `planes` stacked matrices.
static __global__ void transpose_kernel(const float *__restrict__ in, float *__restrict__ out, int rows,
                                 int cols) {
    __shared__ float tile[32][33];
    const size_t plane = (size_t)rows * cols;
    in += blockIdx.z * plane;
    out += blockIdx.z * plane;
    const int c = blockIdx.x * 32 + threadIdx.x;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = blockIdx.y * 32 + k;
        if (r < rows && c < cols) tile[k][threadIdx.x] = in[(size_t)r * cols + c];
    }
    __syncthreads();
    const int r2 = blockIdx.y * 32 + threadIdx.x;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c2 = blockIdx.x * 32 + k;
        if (r2 < rows && c2 < cols) out[(size_t)c2 * rows + r2] = tile[threadIdx.x][k];
    }
}

// Optional source-illumination normalisation of the images: per shot cell
// I (FP64, indexed like the image), per shot the bits of max I (a
// non-negative double, so its bits order like its value), and eps.
struct IllumNorm {
    const double *illum = nullptr;             // nullptr: plain cross-correlation
    const unsigned long long *imax = nullptr;  // per shot
    double eps = 0.0;
};

__device__ __forceinline__ double normalise(double xc, const IllumNorm &nm, long long o, int shot) {
    if (!nm.illum) return xc;
    const double d = nm.illum[o] + nm.eps * __longlong_as_double((long long)nm.imax[shot]);
    return d > 0.0 ? xc / d : 0.0;
}

// Per-shot Kahan image (sum, comp) -> compact (nx, nz) float image of one shot.
static __global__ void image_out_kernel(const float *__restrict__ sum, const float *__restrict__ comp,
                                 float *__restrict__ out, long long row_off, int nx, int nz,
                                 int pitch, IllumNorm nm = IllumNorm()) {
    const long long n = (long long)nx * nz;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / nz), j = (int)(idx % nz);
        const long long o = (row_off + i) * pitch + j + COL_OFF;
        out[idx] = (float)normalise((double)sum[o] - (double)comp[o], nm, o, 0);
    }
}

// Cross-shot sum in FP64 on the global grid (imaging.py:81-93 generalised to
// windows): stack[x, j] += sum over shots covering row x of their image, in
// shot order (deterministic).
static __global__ void stack_kernel(const float *__restrict__ sum, const float *__restrict__ comp,
                             double *__restrict__ stack, const ShotDev *__restrict__ shots,
                             int nshots, int nx_g, int nz, int pitch, IllumNorm nm = IllumNorm()) {
    const long long n = (long long)nx_g * nz;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(idx / nz), j = (int)(idx % nz);
        double acc = stack[idx];
        for (int s = 0; s < nshots; ++s) {
            const int i = x - shots[s].x0;
            if (i < 0 || i >= shots[s].nx) continue;
            const long long o = (shots[s].row_off + i) * pitch + j + COL_OFF;
            acc += normalise((double)sum[o] - (double)comp[o], nm, o, s);
        }
        stack[idx] = acc;
    }
}

// Source illumination of one snapshot component: for every cell of shot
// blockIdx.y, I = sum over the imaging slots of snapshot^2 in FP64 (slot
// order), written at the image index; the shot's maximum goes to imax[shot]
// (atomicMax on the bits of a non-negative double).  Snapshot layout of the
// forward: per shot [nsnap][nx][pitch] at nsnap * row_off * pitch.
static __global__ void illum_kernel(const float *__restrict__ snap, const int *__restrict__ slots, int nslots,
                                    int nsnap, const ShotDev *__restrict__ shots, int nz, int pitch,
                                    double *__restrict__ illum, unsigned long long *__restrict__ imax) {
    const ShotDev sh = shots[blockIdx.y];
    const long long n = (long long)sh.nx * nz;
    const float *base = snap + (long long)nsnap * sh.row_off * pitch;
    double m = 0.0;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / nz), j = (int)(idx % nz);
        double acc = 0.0;
        for (int k = 0; k < nslots; ++k) {
            const double v = base[((long long)slots[k] * sh.nx + i) * pitch + j + COL_OFF];
            acc += v * v;
        }
        illum[(sh.row_off + i) * pitch + j + COL_OFF] = acc;
        m = fmax(m, acc);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(imax + blockIdx.y, (unsigned long long)__double_as_longlong(m));
}

}  // namespace rtm
