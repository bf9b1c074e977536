// morton.cu -- Morton keys of the vertex positions on sm_100a.
//
// Replaces _calcVertMChash (StiffGIPC/GIPC.cu:453-502) with hash_code type -1 and expand_bits
// (GIPC.cu:183-208): every position is normalised per axis to the scene's bounding box,
// scaled to 1024 cells per axis, clamped to [0, 1023] with std::max / std::min semantics and
// truncated; the three 10-bit cell coordinates are interleaved (x << 2 | y << 1 | z) and the
// key is (code << 32) | vertex index.  The keys order the vertices for the Morton-ordered MAS
// banks (stgipc.scenes.morton_renumber sorts them).
//
// One CTA finds the bounding box (min / max are exact, so the result does not depend on the
// reduction order) and then writes every key: a set-up step, run once per mesh.
#include "solver.hpp"

namespace stg
{

// expand_bits (GIPC.cu:183-190): the low 10 bits of v spread three apart
__device__ __forceinline__ uint32_t spread3(uint32_t v)
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// one axis of hash_code: std::min(std::max(t * 1024, 0), 1023), truncated
__device__ __forceinline__ uint32_t cell(double t)
{
    double v = t * 1024.0;
    v = (v < 0.0) ? 0.0 : v;
    v = (1023.0 < v) ? 1023.0 : v;
    return __double2uint_rz(v);
}

__global__ void __launch_bounds__(1024) k_morton_keys(int n, const double* __restrict__ pos,
                                                      unsigned long long* __restrict__ keys)
{
    __shared__ double red[6][32];
    __shared__ double box[6];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for(int i = threadIdx.x; i < n; i += 1024)
#pragma unroll
        for(int d = 0; d < 3; d++)
        {
            const double p = pos[3 * (size_t)i + d];
            lo[d] = fmin(lo[d], p);
            hi[d] = fmax(hi[d], p);
        }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for(int d = 0; d < 3; d++)
    {
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
        {
            lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
            hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
        if(lane == 0)
        {
            red[d][w] = lo[d];
            red[3 + d][w] = hi[d];
        }
    }
    __syncthreads();
    if(w == 0)
    {
#pragma unroll
        for(int d = 0; d < 3; d++)
        {
            double a = red[d][lane], b = red[3 + d][lane];
#pragma unroll
            for(int o = 16; o > 0; o >>= 1)
            {
                a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
                b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
            }
            if(lane == 0)
            {
                box[d] = a;
                box[3 + d] = b;
            }
        }
    }
    __syncthreads();
    const double l0 = box[0], l1 = box[1], l2 = box[2];
    const double s0 = box[3] - l0, s1 = box[4] - l1, s2 = box[5] - l2;
    for(int i = threadIdx.x; i < n; i += 1024)
    {
        const double* p = pos + 3 * (size_t)i;
        const uint32_t code = (spread3(cell((p[0] - l0) / s0)) << 2) + (spread3(cell((p[1] - l1) / s1)) << 1) +
                              spread3(cell((p[2] - l2) / s2));
        keys[i] = ((unsigned long long)code << 32) | (unsigned)i;
    }
}

}  // namespace stg

extern "C" int stg_morton_keys(int n, const double* pos, uint64_t* keys, void* stream)
{
    if(n < 0 || (n > 0 && (!pos || !keys)))
    {
        stg::set_error("stg_morton_keys: invalid arguments");
        return STG_ERR_INVALID;
    }
    if(n == 0) return STG_OK;
    stg::k_morton_keys<<<1, 1024, 0, static_cast<cudaStream_t>(stream)>>>(
        n, pos, reinterpret_cast<unsigned long long*>(keys));
    STG_CUDA_TRY(cudaGetLastError());
    return STG_OK;
}
