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
    __shared__ int warp_incl[32];
    __shared__ int carry;
    int n = n_host;
    if(n_dev)
    {
        const int v = *n_dev;
        n = n_host < 0 ? (v + (-n_host) - 1) / (-n_host) : v;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if(threadIdx.x == 0) carry = 0;
    __syncthreads();
    for(int base = 0; base < n; base += 4096)
    {
        const int idx = base + threadIdx.x * 4;
        int v0 = idx < n ? in[idx] : 0;
        int v1 = idx + 1 < n ? in[idx + 1] : 0;
        int v2 = idx + 2 < n ? in[idx + 2] : 0;
        int v3 = idx + 3 < n ? in[idx + 3] : 0;
        const int local = v0 + v1 + v2 + v3;
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
        if(idx < n) out[idx] = e;
        e += v0;
        if(idx + 1 < n) out[idx + 1] = e;
        e += v1;
        if(idx + 2 < n) out[idx + 2] = e;
        e += v2;
        if(idx + 3 < n) out[idx + 3] = e;
        __syncthreads();
        if(threadIdx.x == 0) carry += warp_incl[31];
        __syncthreads();
    }
    if(threadIdx.x == 0 && total) *total = carry;
}

}  // namespace stg
