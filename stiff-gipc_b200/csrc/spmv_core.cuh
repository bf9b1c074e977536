// spmv_core.cuh -- per-row symmetric block SpMV shared by the standalone SpMV and the PCG.
#pragma once
#include "common.cuh"

namespace stg
{

// acc += H * x (trans == false) or H^T * x; H is a column-major 3x3 block.
template <typename T>
__device__ __forceinline__ void block_mv(const T* __restrict__ H, bool trans, T x0, T x1, T x2, T& a0, T& a1, T& a2)
{
    T h[9];
#pragma unroll
    for(int e = 0; e < 9; e++) h[e] = __ldg(H + e);
    const T h01 = trans ? h[1] : h[3], h10 = trans ? h[3] : h[1];
    const T h02 = trans ? h[2] : h[6], h20 = trans ? h[6] : h[2];
    const T h12 = trans ? h[5] : h[7], h21 = trans ? h[7] : h[5];
    a0 += h[0] * x0 + h01 * x1 + h02 * x2;
    a1 += h10 * x0 + h[4] * x1 + h12 * x2;
    a2 += h20 * x0 + h21 * x1 + h[8] * x2;
}

// Row i of y = A x, computed by the LPR lanes of one group (sub = lane within the group).
// Every lane of the warp must call this (shuffles span the warp); lanes of an invalid row
// pass valid = false.  On return all lanes of the group hold the three sums.
template <typename T, int LPR>
__device__ __forceinline__ void row_spmv(int i, bool valid, int sub, const int* __restrict__ row_ptr,
                                         const int* __restrict__ cols, const T* __restrict__ blocks,
                                         const int* __restrict__ t_ptr, const int2* __restrict__ t_ent,
                                         const T* __restrict__ x, T& a0, T& a1, T& a2)
{
    a0 = a1 = a2 = T(0);
    int u0 = 0, nu = 0, t0 = 0, nt = 0;
    if(valid)
    {
        u0 = row_ptr[i];
        nu = row_ptr[i + 1] - u0;
        t0 = t_ptr[i];
        nt = t_ptr[i + 1] - t0;
    }
    for(int e = sub; e < nu + nt; e += LPR)
    {
        int k, j;
        const bool trans = e >= nu;
        if(!trans)
        {
            k = u0 + e;
            j = __ldg(cols + k);
        }
        else
        {
            const int2 te = __ldg(t_ent + t0 + e - nu);
            k = te.x;
            j = te.y;
        }
        block_mv<T>(blocks + 9 * (size_t)k, trans, x[3 * j], x[3 * j + 1], x[3 * j + 2], a0, a1, a2);
    }
#pragma unroll
    for(int o = LPR / 2; o > 0; o >>= 1)
    {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
}

}  // namespace stg
