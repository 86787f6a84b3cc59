// Block-scaled 16-bit wavefield checkpoints, written by the step kernel that
// produces the stored state (no separate pass over the wavefield).
//
// Format of one compressed checkpoint slot:
//   data:   5 fields (u, w, sxx, szz, sxz) x field_elems 16-bit values, at the
//           padded state layout's element index (state_off + (i+1)*pitch + j + 4);
//   shifts: 5 fields x (padded state rows x blocks per row) int32 exponents.
// A block is one row of one shot's field over 60 columns, [60 b, 60 b + 60)
// (30 columns for plans with vec 1), so the stored values do not depend on
// the launch shape among vec 2 and 4.  Its shared exponent S is chosen from
// amax = max |x| over the block so that amax * 2^S lies in [2^14, 2^15)
// (S = 14 - floor(log2 amax); 0 for an all-zero block), found by the warp
// that owns the columns (a warp reduction at vec 2, a half-warp one at vec 4,
// whose 120-column strip holds two blocks).  Each value is stored as
//   F16 / BF16:  half(x * 2^S)            (|x * 2^S| < 2^15, inside FP16's range)
//   I16:         round(x * 2^S) as int16  (block floating point)
// and restored as stored * 2^-S.  Scaling by a power of two is exact and
// cannot overflow, however small the block (a block the wave has not reached
// holds values of 1e-40 and less).  Pad rows and pad columns are never
// stored and stay zero in the restored state.
//
// Precision: F16 keeps 11 significant bits per value wherever the value
// sits (relative error up to 2^-11), BF16 8 bits; I16 keeps its block's
// values to within 2^-15 of the block maximum, which is about 16x less
// rounding error than F16 where a block's values are within a factor of a
// few of its maximum, as in a smooth wavefield.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "debug_bounds.cuh"

namespace rtm {

enum CkptDtype { CK_F32 = 0, CK_F16 = 1, CK_BF16 = 2, CK_I16 = 3 };

// Columns per scale block for a plan with `vec` columns per lane.
__host__ __device__ constexpr int ckpt_block_cols(int vec) { return vec == 1 ? 30 : 60; }

// The compressed slot a checkpoint-storing launch writes (data == nullptr: none).
struct CkptOut {
    void *data;               // NADJ fields x field_elems 16-bit values
    int *shift;               // NADJ fields x shift_per_field block exponents S
    long long field_elems;    // padded state elements per field (all shots)
    long long shift_per_field;  // padded state rows (all shots) x nblk
    int dtype;                // CK_F16, CK_BF16 or CK_I16
    int nblk;                 // blocks per padded row (strips x 30 vec / block columns)
};

__device__ __forceinline__ unsigned short ckpt_encode(float y, int dtype) {
    if (dtype == CK_F16) return __half_as_ushort(__float2half_rn(y));
    if (dtype == CK_BF16) return __bfloat16_as_ushort(__float2bfloat16_rn(y));
    const int t = min(max(__float2int_rn(y), -32767), 32767);
    return (unsigned short)(short)t;
}

// The block's exponent: amax * 2^S in [2^14, 2^15); 0 for an all-zero (or
// non-finite, i.e. failed) block.
__device__ __forceinline__ int ckpt_shift(float amax) {
    return (amax > 0.f && amax <= 3.402823466e38f) ? 14 - ilogbf(amax) : 0;
}

__device__ __forceinline__ float ckpt_decode(unsigned short h, int dtype) {
    if (dtype == CK_F16) return __half2float(__ushort_as_half(h));
    if (dtype == CK_BF16) return __bfloat162float(__ushort_as_bfloat16(h));
    return (float)(short)h;
}

// One field of one row of a warp task: every lane of the warp calls it
// (the block maximum is a warp reduction); lanes 1..30 own the strip's
// columns and store them.  elem = the lane's first element index in the
// field, blk = the index of the strip's first block.  At vec 4 lanes 1..15
// hold block blk and lanes 16..30 block blk + 1 (lanes 0 and 31 are halo
// lanes and contribute 0).
template <int VEC>
__device__ __forceinline__ void ckpt_pack_field(const CkptOut &ck, int f, long long elem, long long blk, int lane,
                                                bool owner, const float (&v)[VEC]) {
    float m = 0.f;
    if (owner) {
#pragma unroll
        for (int q = 0; q < VEC; ++q) m = fmaxf(m, fabsf(v[q]));
    }
    float amax;
    if constexpr (VEC == 4) {
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));  // within 16-lane halves
        amax = m;
    } else {
        // max of non-negative floats = max of their bit patterns
        amax = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m)));
    }
    const int S = ckpt_shift(amax);
    if (lane == 1 || (VEC == 4 && lane == 16))
        st_chk(ck.shift + (long long)f * ck.shift_per_field + blk + (VEC == 4 ? (lane >> 4) : 0), S);
    if (!owner) return;
    unsigned short h[VEC];
#pragma unroll
    for (int q = 0; q < VEC; ++q) h[q] = ckpt_encode(ldexpf(v[q], S), ck.dtype);
    unsigned short *dst = static_cast<unsigned short *>(ck.data) + (long long)f * ck.field_elems + elem;
    if constexpr (VEC == 4) {
        st_chk(reinterpret_cast<uint2 *>(dst), make_uint2((unsigned)h[0] | ((unsigned)h[1] << 16),
                                                          (unsigned)h[2] | ((unsigned)h[3] << 16)));
    } else if constexpr (VEC == 2) {
        st_chk(reinterpret_cast<unsigned *>(dst), (unsigned)h[0] | ((unsigned)h[1] << 16));
    } else {
        st_chk(dst, h[0]);
    }
}

// The five P-SV state fields of one row, in slot order u, w, sxx, szz, sxz.
template <int VEC>
__device__ __forceinline__ void ckpt_pack_row(const CkptOut &ck, long long elem, long long blk, int lane, bool owner,
                                              const float (&u)[VEC], const float (&w)[VEC], const float (&xx)[VEC],
                                              const float (&zz)[VEC], const float (&xz)[VEC]) {
    ckpt_pack_field<VEC>(ck, 0, elem, blk, lane, owner, u);
    ckpt_pack_field<VEC>(ck, 1, elem, blk, lane, owner, w);
    ckpt_pack_field<VEC>(ck, 2, elem, blk, lane, owner, xx);
    ckpt_pack_field<VEC>(ck, 3, elem, blk, lane, owner, zz);
    ckpt_pack_field<VEC>(ck, 4, elem, blk, lane, owner, xz);
}

}  // namespace rtm
