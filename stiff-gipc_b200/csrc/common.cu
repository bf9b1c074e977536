// common.cu -- error state and the single-CTA exclusive scan used by the build stages.
#include "common.cuh"

namespace stg
{

static thread_local std::string g_error = "no error";

void set_error(const std::string& msg) { g_error = msg; }
const char* last_error() { return g_error.c_str(); }

// Exclusive scan of n ints by one CTA of 1024 threads, 4 consecutive items per thread per
// tile (16-byte loads are not assumed: `in` may be any offset).  n = n_host, or, when n_dev
// is given, *n_dev (n_host >= 0) or ceil(*n_dev / -n_host) (n_host < 0: a bank count).
__global__ void __launch_bounds__(1024) k_scan_exclusive(const int* in, int* out, const int* n_dev, int n_host, int* total)
{
    // 16 values per thread per round (16,384 per round of the 1,024 threads), read and
    // written as int4 when both arrays are 16-byte aligned
    constexpr int PT = 16;
    __shared__ int warp_incl[32];
    __shared__ int carry;
    int n = n_host;
    if(n_dev)
    {
        const int v = *n_dev;
        n = n_host < 0 ? (v + (-n_host) - 1) / (-n_host) : v;
    }
    const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if(threadIdx.x == 0) carry = 0;
    __syncthreads();
    for(int base = 0; base < n; base += PT * 1024)
    {
        const int idx = base + threadIdx.x * PT;
        int v[PT];
        if(vec && idx + PT <= n)
        {
#pragma unroll
            for(int q = 0; q < PT / 4; q++)
            {
                const int4 t = reinterpret_cast<const int4*>(in + idx)[q];
                v[4 * q] = t.x;
                v[4 * q + 1] = t.y;
                v[4 * q + 2] = t.z;
                v[4 * q + 3] = t.w;
            }
        }
        else
        {
#pragma unroll
            for(int q = 0; q < PT; q++) v[q] = idx + q < n ? in[idx + q] : 0;
        }
        int local = 0;
#pragma unroll
        for(int q = 0; q < PT; q++) local += v[q];
        int x = local;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if(lane >= o) x += y;
        }
        if(lane == 31) warp_incl[warp] = x;
        __syncthreads();
        if(warp == 0)
        {
            int w = warp_incl[lane];
#pragma unroll
            for(int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if(lane >= o) w += y;
            }
            warp_incl[lane] = w;
        }
        __syncthreads();
        int e = carry + (warp > 0 ? warp_incl[warp - 1] : 0) + x - local;
#pragma unroll
        for(int q = 0; q < PT; q++)
        {
            const int t = v[q];
            v[q] = e;
            e += t;
        }
        if(vec && idx + PT <= n)
        {
#pragma unroll
            for(int q = 0; q < PT / 4; q++)
                reinterpret_cast<int4*>(out + idx)[q] = make_int4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
        else
        {
#pragma unroll
            for(int q = 0; q < PT; q++)
                if(idx + q < n) out[idx + q] = v[q];
        }
        __syncthreads();
        if(threadIdx.x == 0) carry += warp_incl[31];
        __syncthreads();
    }
    if(threadIdx.x == 0 && total) *total = carry;
}

}  // namespace stg
