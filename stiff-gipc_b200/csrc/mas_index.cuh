// mas_index.cuh -- the MAS bank layout and the level-to-level block mapping, shared by the
// MAS assembly (mas.cu) and the converter's fused level-0 pass (convert.cu).
#pragma once

namespace stg
{

// upper-packed symmetric bank of B x B 3x3 blocks: B (B + 1) / 2 blocks, row-major upper order
__host__ __device__ __forceinline__ int nsym(int B) { return B * (B + 1) / 2; }
__host__ __device__ __forceinline__ int upper_index(int B, int r, int c) { return B * r - r * (r + 1) / 2 + c; }

// Map an upper block (u <= v) with value H to coarse nodes (a, b) and orient it upper:
// a < b: H; a > b: H^T at (b, a); a == b: H (u == v) or H + H^T (u < v).
__device__ __forceinline__ void coarse_triplet(int u, int v, int a, int b, const double* __restrict__ H, int* orow,
                                               int* ocol, double* oblk)
{
    double h[9];
#pragma unroll
    for(int e = 0; e < 9; e++) h[e] = H[e];
    if(a < b || (a == b && u == v))
    {
#pragma unroll
        for(int e = 0; e < 9; e++) oblk[e] = h[e];
    }
    else if(a > b)
    {
#pragma unroll
        for(int i = 0; i < 3; i++)
#pragma unroll
            for(int j = 0; j < 3; j++) oblk[j * 3 + i] = h[i * 3 + j];
        const int t = a;
        a = b;
        b = t;
    }
    else
    {
#pragma unroll
        for(int i = 0; i < 3; i++)
#pragma unroll
            for(int j = 0; j < 3; j++) oblk[j * 3 + i] = h[j * 3 + i] + h[i * 3 + j];
    }
    *orow = a;
    *ocol = b;
}

}  // namespace stg
