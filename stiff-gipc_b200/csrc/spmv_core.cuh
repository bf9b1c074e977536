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

// ---------------------------------------------------------------------------------------
// Full symmetric row-sliced copy of the matrix for the PCG SpMV, in 16-byte planes.
// Row i holds, sorted by column, its lower blocks (transposes of the upper blocks k with
// col(k) == i) followed by its upper blocks; entry e of row i sits at f = frow[i] + e.
// Entry f of a plane copy with S entries per plane is stored as
//   FP32: plane 0 {h0 h1 h2 h3} at 16 f, plane 1 {h4 h5 h6 h7} at 16 S + 16 f,
//         tail {h8, col} at 32 S + 8 f                                     (40 B per entry)
//   FP64: planes p = 0..3 {h(2p) h(2p+1)} at 16 p S + 16 f,
//         tail {h8, col, 0} at 64 S + 16 f                                 (80 B per entry)
// (h column-major).  Lanes that read consecutive entries read consecutive 16-byte (or 8-byte)
// words of every plane: coalesced in global memory and free of shared-memory bank
// conflicts, and a row range is one contiguous range of every plane (one bulk copy each).
// ---------------------------------------------------------------------------------------
template <typename T>
struct FullPlanes
{
    static constexpr int NP = sizeof(T) == 4 ? 2 : 4;     // 16-byte value planes
    static constexpr int TAIL = sizeof(T) == 4 ? 8 : 16;  // bytes of the {h8, col} plane
    static constexpr int ES = 16 * NP + TAIL;             // bytes per entry
};

__device__ __forceinline__ void load_entry(const unsigned char* base, size_t S, int f, float h[9], int& col)
{
    const float4 a = reinterpret_cast<const float4*>(base)[f];
    const float4 b = reinterpret_cast<const float4*>(base + 16 * S)[f];
    const float2 t = reinterpret_cast<const float2*>(base + 32 * S)[f];
    h[0] = a.x; h[1] = a.y; h[2] = a.z; h[3] = a.w;
    h[4] = b.x; h[5] = b.y; h[6] = b.z; h[7] = b.w;
    h[8] = t.x;
    col = __float_as_int(t.y);
}

__device__ __forceinline__ void load_entry(const unsigned char* base, size_t S, int f, double h[9], int& col)
{
#pragma unroll
    for(int p = 0; p < 4; p++)
    {
        const double2 v = reinterpret_cast<const double2*>(base + 16 * p * S)[f];
        h[2 * p] = v.x;
        h[2 * p + 1] = v.y;
    }
    const double2 t = reinterpret_cast<const double2*>(base + 64 * S)[f];
    h[8] = t.x;
    col = (int)__double_as_longlong(t.y);
}

// the same from global memory through the read-only path
__device__ __forceinline__ void ldg_entry(const unsigned char* base, size_t S, int f, float h[9], int& col)
{
    const float4 a = __ldg(reinterpret_cast<const float4*>(base) + f);
    const float4 b = __ldg(reinterpret_cast<const float4*>(base + 16 * S) + f);
    const float2 t = __ldg(reinterpret_cast<const float2*>(base + 32 * S) + f);
    h[0] = a.x; h[1] = a.y; h[2] = a.z; h[3] = a.w;
    h[4] = b.x; h[5] = b.y; h[6] = b.z; h[7] = b.w;
    h[8] = t.x;
    col = __float_as_int(t.y);
}

__device__ __forceinline__ void ldg_entry(const unsigned char* base, size_t S, int f, double h[9], int& col)
{
#pragma unroll
    for(int p = 0; p < 4; p++)
    {
        const double2 v = __ldg(reinterpret_cast<const double2*>(base + 16 * p * S) + f);
        h[2 * p] = v.x;
        h[2 * p + 1] = v.y;
    }
    const double2 t = __ldg(reinterpret_cast<const double2*>(base + 64 * S) + f);
    h[8] = t.x;
    col = (int)__double_as_longlong(t.y);
}

// writes entry f (h column-major) into a plane copy with S entries per plane
__device__ __forceinline__ void store_entry(unsigned char* base, size_t S, size_t f, const float h[9], int col)
{
    reinterpret_cast<float4*>(base)[f] = make_float4(h[0], h[1], h[2], h[3]);
    reinterpret_cast<float4*>(base + 16 * S)[f] = make_float4(h[4], h[5], h[6], h[7]);
    reinterpret_cast<float2*>(base + 32 * S)[f] = make_float2(h[8], __int_as_float(col));
}

__device__ __forceinline__ void store_entry(unsigned char* base, size_t S, size_t f, const double h[9], int col)
{
#pragma unroll
    for(int p = 0; p < 4; p++) reinterpret_cast<double2*>(base + 16 * p * S)[f] = make_double2(h[2 * p], h[2 * p + 1]);
    reinterpret_cast<double2*>(base + 64 * S)[f] = make_double2(h[8], __longlong_as_double((long long)(unsigned)col));
}

// ---------------------------------------------------------------------------------------
// Upper copy of the matrix for the PCG SpMV: entry k is the k-th block of the sorted unique
// upper BCOO (rows ascending, columns ascending within a row), so a row range is one
// contiguous range of every plane.  With S entries per plane:
//   FP32: plane 0 {h0 h1 h2 h3} at 16 k, plane 1 {h4 h5 h6 h7} at 16 S + 16 k,
//         tail {h8, col} at 32 S + 8 k, spill slot at 40 S + 4 k              (44 B per entry)
//   FP64: planes p = 0..3 {h(2p) h(2p+1)} at 16 p S + 16 k,
//         tail {h8, col, slot} at 64 S + 16 k                                 (80 B per entry)
// The spill slot of a strictly upper block k (row i, column j > i) is its position t in the
// transpose list of row j (t_ent[t].x == k): the SpMV writes H_k^T v_i there, and the owner of
// row j adds its slots t_ptr[j] .. t_ptr[j+1] in that order.  A diagonal block has slot -1.
// ---------------------------------------------------------------------------------------
template <typename T>
struct UpperPlanes
{
    static constexpr int NP = sizeof(T) == 4 ? 2 : 4;     // 16-byte value planes
    static constexpr int TAIL = sizeof(T) == 4 ? 8 : 16;  // bytes of the tail plane
    static constexpr int SLOTP = sizeof(T) == 4 ? 4 : 0;  // bytes of the separate slot plane
    static constexpr int ES = 16 * NP + TAIL + SLOTP;     // bytes per entry
};

__device__ __forceinline__ void store_upper(unsigned char* base, size_t S, size_t k, const float h[9], int col, int slot)
{
    reinterpret_cast<float4*>(base)[k] = make_float4(h[0], h[1], h[2], h[3]);
    reinterpret_cast<float4*>(base + 16 * S)[k] = make_float4(h[4], h[5], h[6], h[7]);
    reinterpret_cast<float2*>(base + 32 * S)[k] = make_float2(h[8], __int_as_float(col));
    reinterpret_cast<int*>(base + 40 * S)[k] = slot;
}

__device__ __forceinline__ void store_upper(unsigned char* base, size_t S, size_t k, const double h[9], int col, int slot)
{
#pragma unroll
    for(int p = 0; p < 4; p++) reinterpret_cast<double2*>(base + 16 * p * S)[k] = make_double2(h[2 * p], h[2 * p + 1]);
    const long long cs = (long long)(((unsigned long long)(unsigned)slot << 32) | (unsigned)col);
    reinterpret_cast<double2*>(base + 64 * S)[k] = make_double2(h[8], __longlong_as_double(cs));
}

// address of the spill slot of entry k (the slot is an int in both layouts)
template <typename T>
__device__ __forceinline__ int* upper_slot_ptr(unsigned char* base, size_t S, size_t k)
{
    if constexpr(sizeof(T) == 4)
        return reinterpret_cast<int*>(base + 40 * S) + k;
    else
        return reinterpret_cast<int*>(base + 64 * S + 16 * k + 12);
}

// entry k from global memory through the read-only path
__device__ __forceinline__ void ldg_upper(const unsigned char* base, size_t S, int k, float h[9], int& col, int& slot)
{
    const float4 a = __ldg(reinterpret_cast<const float4*>(base) + k);
    const float4 b = __ldg(reinterpret_cast<const float4*>(base + 16 * S) + k);
    const float2 t = __ldg(reinterpret_cast<const float2*>(base + 32 * S) + k);
    h[0] = a.x; h[1] = a.y; h[2] = a.z; h[3] = a.w;
    h[4] = b.x; h[5] = b.y; h[6] = b.z; h[7] = b.w;
    h[8] = t.x;
    col = __float_as_int(t.y);
    slot = __ldg(reinterpret_cast<const int*>(base + 40 * S) + k);
}

__device__ __forceinline__ void ldg_upper(const unsigned char* base, size_t S, int k, double h[9], int& col, int& slot)
{
#pragma unroll
    for(int p = 0; p < 4; p++)
    {
        const double2 v = __ldg(reinterpret_cast<const double2*>(base + 16 * p * S) + k);
        h[2 * p] = v.x;
        h[2 * p + 1] = v.y;
    }
    const double2 t = __ldg(reinterpret_cast<const double2*>(base + 64 * S) + k);
    h[8] = t.x;
    const unsigned long long cs = (unsigned long long)__double_as_longlong(t.y);
    col = (int)(unsigned)cs;
    slot = (int)(unsigned)(cs >> 32);
}

}  // namespace stg
