// bank_dev.cuh -- the arithmetic of one MAS bank-solve row, z_a = sum_c P_ac r_c
// (_schwarzLocalXSym6, StiffGIPC/MASPreconditioner.cu:957-1027), shared by every kernel that
// applies the bank inverses (the PCG loop's phase D in all three loop modes, and the
// standalone stg_mas_apply), so that all of them give the same bits.
//
// The order is written out with __fmaf_rn / __fmul_rn / __fadd_rn, so it is the source's and
// not the compiler's choice of contractions.  The CPU oracle restates it (ORC_ORDER_FIXED):
//   16-vertex banks: lane (a, h) sums block row a over the column blocks 8h + ((j + a) & 7),
//                    j = 0..7, each block added with three FMAs per element (columns 0, 1, 2);
//                    the two halves are then added;
//   32-vertex banks: lane c forms the block product fma(P2, x2, fma(P1, x1, P0 x0)), and an
//                    xor butterfly over the 32 lanes (16, 8, 4, 2, 1) sums the row.
// P is the bank's packed upper inverse: 3x3 FP32 blocks, column-major; a lower block (c < a)
// is the transpose of the stored (c, a).
#pragma once

namespace stg
{

// z += H x (trans: H^T x), one FMA per element in column order
__device__ __forceinline__ void blk_fma3(const float* H, bool trans, float x0, float x1, float x2, float& z0, float& z1,
                                         float& z2)
{
    if(trans)
    {
        z0 = __fmaf_rn(H[2], x2, __fmaf_rn(H[1], x1, __fmaf_rn(H[0], x0, z0)));
        z1 = __fmaf_rn(H[5], x2, __fmaf_rn(H[4], x1, __fmaf_rn(H[3], x0, z1)));
        z2 = __fmaf_rn(H[8], x2, __fmaf_rn(H[7], x1, __fmaf_rn(H[6], x0, z2)));
    }
    else
    {
        z0 = __fmaf_rn(H[6], x2, __fmaf_rn(H[3], x1, __fmaf_rn(H[0], x0, z0)));
        z1 = __fmaf_rn(H[7], x2, __fmaf_rn(H[4], x1, __fmaf_rn(H[1], x0, z1)));
        z2 = __fmaf_rn(H[8], x2, __fmaf_rn(H[5], x1, __fmaf_rn(H[2], x0, z2)));
    }
}

// z = H x (trans: H^T x) as fma(P2, x2, fma(P1, x1, P0 x0)) per element; element (i, k) is
// H[i * si + k * sk] with (si, sk) = (1, 3), or (3, 1) transposed (strided loads instead of a
// branch: the two-branch form makes ptxas 12.9 for sm_100a abort in phase_d<32>)
__device__ __forceinline__ void blk_mul3(const float* H, bool trans, float x0, float x1, float x2, float& z0, float& z1,
                                         float& z2)
{
    const int si = trans ? 3 : 1, sk = trans ? 1 : 3;
    z0 = __fmaf_rn(H[2 * sk], x2, __fmaf_rn(H[sk], x1, __fmul_rn(H[0], x0)));
    z1 = __fmaf_rn(H[si + 2 * sk], x2, __fmaf_rn(H[si + sk], x1, __fmul_rn(H[si], x0)));
    z2 = __fmaf_rn(H[2 * si + 2 * sk], x2, __fmaf_rn(H[2 * si + sk], x1, __fmul_rn(H[2 * si], x0)));
}

// word offset of block (lo, hi), lo <= hi, in a packed upper 16-bank
__device__ __forceinline__ int bank16_off(int lo, int hi) { return 9 * (lo * 16 - lo * (lo - 1) / 2 + (hi - lo)); }

// half h of block row a of a 16-bank: the column blocks 8h + ((j + a) & 7), j = 0..7, in that
// order; rs holds the 16 residual slots (x, y, z, -)
__device__ __forceinline__ void bank16_half(const float* P, const float4* rs, int a, int h, float& z0, float& z1,
                                            float& z2)
{
    z0 = z1 = z2 = 0.f;
#pragma unroll
    for(int j = 0; j < 8; j++)
    {
        const int cc = 8 * h + ((j + a) & 7);
        const float4 r = rs[cc];
        blk_fma3(P + bank16_off(min(a, cc), max(a, cc)), cc < a, r.x, r.y, r.z, z0, z1, z2);
    }
}

// the sum of the two halves (lanes l and l ^ 16 of a warp): every lane gets z_h0 + z_h1
__device__ __forceinline__ void bank16_join(float& z0, float& z1, float& z2)
{
    z0 = __fadd_rn(z0, __shfl_xor_sync(0xffffffffu, z0, 16));
    z1 = __fadd_rn(z1, __shfl_xor_sync(0xffffffffu, z1, 16));
    z2 = __fadd_rn(z2, __shfl_xor_sync(0xffffffffu, z2, 16));
}

// xor butterfly over the 32 lanes of a warp (lane 0 holds the row sum afterwards)
__device__ __forceinline__ void warp_butterfly3(float& z0, float& z1, float& z2)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
    {
        z0 = __fadd_rn(z0, __shfl_xor_sync(0xffffffffu, z0, o));
        z1 = __fadd_rn(z1, __shfl_xor_sync(0xffffffffu, z1, o));
        z2 = __fadd_rn(z2, __shfl_xor_sync(0xffffffffu, z2, o));
    }
}

}  // namespace stg
