// Restore of block-scaled 16-bit wavefield checkpoints (format and store:
// ckpt_pack.cuh; the store is fused into the step launch that produces the
// checkpointed state).
//
// unpack: x = stored * 2^-S_block for the columns the warp strips
// cover (j in [0, nstrips * 30 * vec)) of every interior row of every shot;
// pad rows and the left pad columns are not written, and stay zero in the
// destination.
#pragma once
#include "ckpt_pack.cuh"
#include "step_kernels.cuh"

namespace rtm {

struct CkptIn {
    const void *data;          // NADJ fields x field_elems 16-bit values
    const int *shift;          // NADJ fields x shift_per_field block exponents
    float *dst[5];             // FP32 state fields (u, w, sxx, szz, sxz)
    long long field_elems, shift_per_field;
    const ShotDev *shots;
    int pitch, ncols, nblk, block_w, dtype;  // columns covered, blocks per padded row, block width
};

// grid: (chunks, nshots, 5 fields)
static __global__ void ckpt_unpack_kernel(CkptIn ci) {
    const int s = blockIdx.y, f = blockIdx.z;
    const ShotDev sh = ci.shots[s];
    const int ncols = ci.ncols;
    const long long n = (long long)sh.nx * ncols;
    const long long row0 = sh.state_off / ci.pitch;  // padded row 0 of the shot
    const unsigned short *h = static_cast<const unsigned short *>(ci.data) + (long long)f * ci.field_elems;
    const int *sh_blk = ci.shift + (long long)f * ci.shift_per_field;
    float *x = ci.dst[f];
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / ncols), c = (int)(idx % ncols);
        const long long e = sh.state_off + (long long)(i + 1) * ci.pitch + COL_OFF + c;
        const int S = ldg_chk(sh_blk + (row0 + i + 1) * ci.nblk + c / ci.block_w);
        const float v = ldexpf(ckpt_decode(ldg_chk(h + e), ci.dtype), -S);
        st_chk(x + e, v);
    }
}

}  // namespace rtm
