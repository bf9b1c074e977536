// common.cuh -- shared device/host helpers of libstgipc (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace stg
{
// ------------------------------------------------------------------------------------
// errors: every failure becomes a status code plus a thread-local message
// ------------------------------------------------------------------------------------
void set_error(const std::string& msg);
const char* last_error();

struct Status
{
    int code = 0;
    explicit operator bool() const { return code == 0; }
};

#define STG_CUDA_TRY(expr)                                                                        \
    do                                                                                            \
    {                                                                                             \
        cudaError_t _e = (expr);                                                                  \
        if(_e != cudaSuccess)                                                                     \
        {                                                                                         \
            ::stg::set_error(std::string(#expr) + " failed: " + cudaGetErrorString(_e) + " at " + \
                             __FILE__ + ":" + std::to_string(__LINE__));                          \
            return 2; /* STG_ERR_CUDA */                                                          \
        }                                                                                         \
    } while(0)

#define STG_LAUNCH_CHECK() STG_CUDA_TRY(cudaGetLastError())

#define STG_TRY(expr)              \
    do                             \
    {                              \
        int _s = (expr);           \
        if(_s != 0) return _s;     \
    } while(0)

// ------------------------------------------------------------------------------------
// grow-only device buffer (the reference's loose_resize, i_preconditioner.h:71-77)
// ------------------------------------------------------------------------------------
template <typename T>
struct DBuf
{
    T* ptr = nullptr;
    size_t cap = 0;
    size_t size = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release()
    {
        if(ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = size = 0;
    }
    int resize(size_t n)
    {
        if(n > cap)
        {
            size_t nc = n + n / 2 + 16;
            T* p = nullptr;
            cudaError_t e = cudaMalloc((void**)&p, nc * sizeof(T));
            if(e != cudaSuccess)
            {
                set_error(std::string("cudaMalloc of ") + std::to_string(nc * sizeof(T)) + " bytes failed: " +
                          cudaGetErrorString(e));
                return 2;
            }
            if(ptr) cudaFree(ptr);
            ptr = p;
            cap = nc;
        }
        size = n;
        return 0;
    }
    T* data() const { return ptr; }
};

inline int div_up(long a, long b) { return (int)((a + b - 1) / b); }

// Kernel attributes are per device: true the first time a call site reaches it on the
// current device (mask: one bit per device, owned by the call site, per host thread).
inline bool first_on_device(unsigned long long& mask)
{
    int d = 0;
    if(cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) return true;
    const unsigned long long bit = 1ull << d;
    if(mask & bit) return false;
    mask |= bit;
    return true;
}

// ------------------------------------------------------------------------------------
// device helpers
// ------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned lanemask_lt(int lane)
{
    return lane >= 32 ? 0xffffffffu : ((1u << lane) - 1u);
}

// Value of lane `bb` of this lane's group of B lanes, as a full-width shuffle with an explicit
// source lane.  With CUDA 12.9 for sm_100a, a fully unrolled loop of width-B shuffles inside a
// grid-stride loop made ptxas abort with a register-allocation error in some kernels; this
// form (plus partial unrolling where the abort persisted) compiles.
template <int B>
__device__ __forceinline__ float group_shfl(float v, int bb)
{
    return __shfl_sync(0xffffffffu, v, ((threadIdx.x & 31) & ~(B - 1)) + bb);
}

// 4-wide per-node vector slots {v0 v1 v2 0}: one 16-byte access (FP32) or two (FP64)
__device__ __forceinline__ void ld4(const float* p, float& a, float& b, float& c)
{
    const float4 v = *reinterpret_cast<const float4*>(p);
    a = v.x;
    b = v.y;
    c = v.z;
}
__device__ __forceinline__ void ld4(const double* p, double& a, double& b, double& c)
{
    const double2 v0 = *reinterpret_cast<const double2*>(p);
    const double2 v1 = *reinterpret_cast<const double2*>(p + 2);
    a = v0.x;
    b = v0.y;
    c = v1.x;
}
__device__ __forceinline__ void st4(float* p, float a, float b, float c)
{
    *reinterpret_cast<float4*>(p) = make_float4(a, b, c, 0.f);
}
__device__ __forceinline__ void st4(double* p, double a, double b, double c)
{
    *reinterpret_cast<double2*>(p) = make_double2(a, b);
    *reinterpret_cast<double2*>(p + 2) = make_double2(c, 0.0);
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warp_sumf(float v)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block reduction of one double; result valid in thread 0.
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v, double* smem /* BLOCK/32 */)
{
    v = warp_sum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if(lane == 0) smem[warp] = v;
    __syncthreads();
    double r = 0;
    if(warp == 0)
    {
        r = lane < BLOCK / 32 ? smem[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

// Single-CTA exclusive scan of n ints (n read from n_dev if non-null, else n_host).
// out[i] = sum in[0..i); *total = sum of all.  Launch with 1024 threads.
__global__ void k_scan_exclusive(const int* in, int* out, const int* n_dev, int n_host, int* total);

}  // namespace stg
