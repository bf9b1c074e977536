// spmv.cu -- symmetric 3x3-block BCOO SpMV on sm_100a.
//
// Replaces Spmv::srbk_spmv (StiffGIPC/linear_system/utils/spmv.cu:188-313).  The reference
// runs one thread per stored upper block, reduces row segments with cub's warp
// HeadSegmentedReduce and scatters both the row result and the transposed contribution
// H^T x_i with FP64 atomicAdd (two atomics per off-diagonal block; summation order depends
// on scheduling).
//
// Here each block row i is owned by a group of LPR lanes ("owner computes"):
//   y_i = sum_{k in row i} H_k x_{col k}  +  sum_{k: col k == i, row k < i} H_k^T x_{row k}
// The first list is the contiguous upper segment of the sorted BCOO; the second is a
// transpose reference list built once per assembly (prepare_spmv).  No atomics, fixed
// summation order, bitwise deterministic.  A transposed block is read a second time by a
// nearby row (Morton-ordered vertices keep it in the 126 MB L2), so DRAM sees each block
// about once.
#include "solver.hpp"
#include "spmv_core.cuh"

#include <mutex>

namespace stg
{

// ---------------------------------------------------------------------------------------
// structure preparation
// ---------------------------------------------------------------------------------------
// Caller-provided BCOO must be sorted by (row, col), unique, upper (row <= col) and inside
// [0, nrows) when nrows > 0 (the converter's output contract); counts violations.
__global__ void k_bcoo_validate(const int* rows, const int* cols, int nnzb, int nrows, int* bad)
{
    int cnt = 0;
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnzb; k += gridDim.x * blockDim.x)
    {
        const int r = rows[k], c = cols[k];
        bool ok = r >= 0 && c >= r && (nrows <= 0 || c < nrows);
        if(k > 0)
        {
            const int rp = rows[k - 1], cp = cols[k - 1];
            ok = ok && (rp < r || (rp == r && cp < c));
        }
        cnt += !ok;
    }
    if(cnt) atomicAdd(bad, cnt);
}

int validate_bcoo(Solver& S)
{
    const int nnzb = S.bcoo.nnzb;
    if(nnzb < 1) return 0;
    STG_TRY(S.cv.scratch.resize(4));
    int* bad = S.cv.scratch.data() + 3;
    STG_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), S.stream));
    k_bcoo_validate<<<std::max(1, std::min(div_up(nnzb, 256), kSMs * 8)), 256, 0, S.stream>>>(S.bcoo.R(), S.bcoo.C(), nnzb,
                                                                                            S.bcoo.nrows, bad);
    STG_LAUNCH_CHECK();
    S.launches++;
    int h = 0;
    STG_CUDA_TRY(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, S.stream));
    STG_CUDA_TRY(cudaStreamSynchronize(S.stream));
    if(h)
    {
        set_error("BCOO input: " + std::to_string(h) +
                  " entries are out of range, lower-triangular, unsorted or duplicated (run stg_convert first)");
        return STG_ERR_INVALID;
    }
    return 0;
}

__global__ void k_row_ptr(const int* rows, int nnzb, int nrows, int* row_ptr)
{
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k <= nnzb; k += gridDim.x * blockDim.x)
    {
        int rp = k > 0 ? rows[k - 1] : -1;
        int rc = k < nnzb ? rows[k] : nrows;
        for(int r = rp + 1; r <= rc; r++) row_ptr[r] = k;
    }
}

__global__ void k_t_count(const int* rows, const int* cols, int nnzb, int* t_cnt)
{
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnzb; k += gridDim.x * blockDim.x)
    {
        int i = rows[k], j = cols[k];
        if(i != j) atomicAdd(t_cnt + j, 1);
    }
}

__global__ void k_t_fill(const int* rows, const int* cols, int nnzb, const int* t_ptr, int* cursor, int2* t_ent)
{
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnzb; k += gridDim.x * blockDim.x)
    {
        int i = rows[k], j = cols[k];
        if(i != j)
        {
            int pos = t_ptr[j] + atomicAdd(cursor + j, 1);
            t_ent[pos] = make_int2(k, i);
        }
    }
}

// sort each transpose list by block index (insertion sort; lists are short) so that the
// summation order does not depend on atomic arrival order
__global__ void k_t_sort(const int* t_ptr, int2* t_ent, int nrows)
{
    for(int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x)
    {
        int s = t_ptr[r], e = t_ptr[r + 1];
        for(int a = s + 1; a < e; a++)
        {
            int2 v = t_ent[a];
            int b = a - 1;
            while(b >= s && t_ent[b].x > v.x)
            {
                t_ent[b + 1] = t_ent[b];
                b--;
            }
            t_ent[b + 1] = v;
        }
    }
}

__global__ void k_to_f32(const double* in, float* out, size_t count)
{
    for(size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// 3x3 inverse of every diagonal block (DiagPreconditioner::assemble,
// diag_preconditioner.cu:12-33), cofactor / determinant, column-major in and out
__global__ void k_diag_inv(const int* rows, const int* cols, const double* blocks, int nnzb, double* diag_inv)
{
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnzb; k += gridDim.x * blockDim.x)
    {
        if(rows[k] != cols[k]) continue;
        const double* H = blocks + 9 * (size_t)k;
        double a = H[0], b = H[3], c = H[6], d = H[1], e = H[4], f = H[7], g = H[2], h = H[5], i = H[8];
        double A = e * i - f * h, Bc = -(d * i - f * g), Cc = d * h - e * g;
        double inv_det = 1.0 / (a * A + b * Bc + c * Cc);
        double R[9] = {A, -(b * i - c * h), b * f - c * e, Bc, a * i - c * g, -(a * f - c * d), Cc, -(a * h - b * g), a * e - b * d};
        double* D = diag_inv + 9 * (size_t)rows[k];
#pragma unroll
        for(int r = 0; r < 3; r++)
#pragma unroll
            for(int cc = 0; cc < 3; cc++) D[cc * 3 + r] = R[r * 3 + cc] * inv_det;
    }
}

int Solver::bind_bcoo(const double* blocks, const int* rows, const int* cols, int nnzb, int nrows)
{
    bcoo.external = true;
    bcoo.ext_blocks = blocks;
    bcoo.ext_rows = rows;
    bcoo.ext_cols = cols;
    bcoo.nnzb = nnzb;
    bcoo.nrows = nrows;
    bcoo.row_ptr_valid = false;
    return validate_bcoo(*this);
}

int Solver::prepare_spmv()
{
    cudaStream_t s = stream;
    const int nnzb = bcoo.nnzb, nrows = bcoo.nrows;
    if(nrows < 1) return 0;
    STG_TRY(bcoo.row_ptr.resize(nrows + 1));
    STG_TRY(bcoo.t_ptr.resize(nrows + 1));
    STG_TRY(bcoo.t_cnt.resize(nrows + 1));
    STG_TRY(bcoo.t_ent.resize(std::max(nnzb, 1)));
    STG_TRY(cv.scratch.resize(4));
    const int g = std::max(1, std::min(div_up(nnzb + 1, 256), kSMs * 16));
    if(!bcoo.row_ptr_valid)
    {
        k_row_ptr<<<g, 256, 0, s>>>(bcoo.R(), nnzb, nrows, bcoo.row_ptr.data());
        STG_LAUNCH_CHECK();
        launches++;
        bcoo.row_ptr_valid = true;
    }
    STG_CUDA_TRY(cudaMemsetAsync(bcoo.t_cnt.data(), 0, sizeof(int) * (nrows + 1), s));
    k_t_count<<<g, 256, 0, s>>>(bcoo.R(), bcoo.C(), nnzb, bcoo.t_cnt.data());
    STG_LAUNCH_CHECK();
    k_scan_exclusive<<<1, 1024, 0, s>>>(bcoo.t_cnt.data(), bcoo.t_ptr.data(), nullptr, nrows + 1, cv.scratch.data() + 2);
    STG_LAUNCH_CHECK();
    STG_CUDA_TRY(cudaMemsetAsync(bcoo.t_cnt.data(), 0, sizeof(int) * (nrows + 1), s));
    k_t_fill<<<g, 256, 0, s>>>(bcoo.R(), bcoo.C(), nnzb, bcoo.t_ptr.data(), bcoo.t_cnt.data(), bcoo.t_ent.data());
    STG_LAUNCH_CHECK();
    k_t_sort<<<std::max(1, std::min(div_up(nrows, 256), kSMs * 16)), 256, 0, s>>>(bcoo.t_ptr.data(), bcoo.t_ent.data(), nrows);
    STG_LAUNCH_CHECK();
    launches += 4;
    if(cfg.preconditioner == STG_PRECOND_DIAG)
    {
        STG_TRY(bcoo.diag_inv.resize((size_t)nrows * 9));
        STG_CUDA_TRY(cudaMemsetAsync(bcoo.diag_inv.data(), 0, sizeof(double) * 9 * nrows, s));
        k_diag_inv<<<g, 256, 0, s>>>(bcoo.R(), bcoo.C(), bcoo.B(), nnzb, bcoo.diag_inv.data());
        STG_LAUNCH_CHECK();
        launches++;
    }
    bcoo.offdiag = -1;  // not needed on the host
    return 0;
}

// ---------------------------------------------------------------------------------------
// the standalone SpMV kernel (stg_spmv): y = a A x + b y
// ---------------------------------------------------------------------------------------
template <typename T, int LPR>
__global__ void __launch_bounds__(256) k_spmv_sym(const int* __restrict__ row_ptr, const int* __restrict__ cols,
                                                  const T* __restrict__ blocks, const int* __restrict__ t_ptr,
                                                  const int2* __restrict__ t_ent, const T* __restrict__ x, T* y, double a,
                                                  double b, int nrows)
{
    constexpr int RPW = 32 / LPR;  // rows per warp
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31, sub = lane & (LPR - 1);
    for(int base = warp * RPW; base < nrows; base += nwarps * RPW)
    {
        const int i = base + lane / LPR;
        const bool valid = i < nrows;
        T a0, a1, a2;
        row_spmv<T, LPR>(i, valid, sub, row_ptr, cols, blocks, t_ptr, t_ent, x, a0, a1, a2);
        if(valid && sub < 3)
        {
            T v = sub == 0 ? a0 : (sub == 1 ? a1 : a2);
            double out = a * (double)v;
            if(b != 0.0) out += b * (double)y[3 * i + sub];
            y[3 * i + sub] = (T)out;
        }
    }
}

int Solver::spmv(double a, const double* x, double b, double* y)
{
    const int nrows = bcoo.nrows;
    if(nrows < 1) return 0;
    const int grid = std::max(1, std::min(div_up(nrows, 256 / 16), kSMs * 8));
    k_spmv_sym<double, 16><<<grid, 256, 0, stream>>>(bcoo.row_ptr.data(), bcoo.C(), bcoo.B(), bcoo.t_ptr.data(),
                                                     bcoo.t_ent.data(), x, y, a, b, nrows);
    STG_LAUNCH_CHECK();
    launches++;
    return 0;
}

}  // namespace stg

// ---------------------------------------------------------------------------------------
// stg_spmv_noalloc: the same SpMV without a handle and without any device allocation.
//
// For callers that cannot allocate device memory: a host simulator that has reserved the
// GPU's memory for its own pool and forbids allocations outside it, or a step loop that
// cannot take cudaMalloc's implicit device-wide synchronisation.  The row pointers and
// transpose lists that stg_spmv keeps in a handle's buffers live here in one file-scope
// device array of fixed size instead (STG_NOALLOC_SCRATCH_BYTES, about 9.5 MiB), which
// every GPU that loads this library holds until the process exits.
//
// The array is shared by every call: each call rewrites all of it that it reads and clears
// what must start at zero (the counters and the per-row transpose counts), so nothing
// carries over from the previous call's contents.  Two calls that overlap on the GPU (two
// host threads, or two streams) race on the array and give wrong results.
//
// Set-up: the first call on each device resolves the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it.  Under lazy module
// loading (the CUDA 12 default) the array is only reserved when this file's module loads,
// which can be that first call; a call with n == 0 does the set-up and nothing else, so a
// caller that must have every reservation made before its own pool takes the GPU's memory
// makes such a call first (or runs with CUDA_MODULE_LOADING=EAGER).
//
// Every call validates its input on the device and reads the verdict back, then waits for
// the product: it is synchronous, and cannot be made inside a stream capture.
// ---------------------------------------------------------------------------------------
namespace
{
constexpr size_t kNaCounters = 0;                                                 // 64 ints: [0] bad, [1] scan total
constexpr size_t kNaRowInts = ((size_t)STG_NOALLOC_MAX_ROWS + 1 + 63) / 64 * 64;  // per-row array, 256 B multiple
constexpr size_t kNaRowPtr = 64 * sizeof(int);
constexpr size_t kNaTPtr = kNaRowPtr + kNaRowInts * sizeof(int);
constexpr size_t kNaTCnt = kNaTPtr + kNaRowInts * sizeof(int);
constexpr size_t kNaTEnt = kNaTCnt + kNaRowInts * sizeof(int);
constexpr size_t kNaBytes = kNaTEnt + (size_t)STG_NOALLOC_MAX_BLOCKS * sizeof(int2);
static_assert(kNaBytes == STG_NOALLOC_SCRATCH_BYTES, "header and library disagree on the scratch size");
static_assert(kNaTEnt % 256 == 0, "transpose list must stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

constexpr int kNaMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_addr[kNaMaxDevices] = {};

// device address of g_noalloc_scratch on the current device (resolved once per device)
int noalloc_scratch(unsigned char** out)
{
    int dev = -1;
    STG_CUDA_TRY(cudaGetDevice(&dev));
    if(dev < 0 || dev >= kNaMaxDevices)
    {
        stg::set_error("stg_spmv_noalloc: device ordinal " + std::to_string(dev) + " beyond the supported " +
                       std::to_string(kNaMaxDevices));
        return STG_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if(!g_noalloc_addr[dev])
    {
        void* p = nullptr;
        STG_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_addr[dev];
    return 0;
}

int spmv_noalloc(double a, const double* blocks, const int* rows, const int* cols, int nnzb, const double* x, double b,
                 double* y, int n, cudaStream_t s)
{
    using namespace stg;
    if(nnzb < 0 || n < 0 || n % 3 != 0 || (nnzb > 0 && (!blocks || !rows || !cols)) || (n > 0 && (!x || !y)))
    {
        set_error("stg_spmv_noalloc: invalid arguments");
        return STG_ERR_INVALID;
    }
    const int nrows = n / 3;
    if(nrows > STG_NOALLOC_MAX_ROWS || nnzb > STG_NOALLOC_MAX_BLOCKS)
    {
        set_error("stg_spmv_noalloc: " + std::to_string(nrows) + " block rows / " + std::to_string(nnzb) +
                  " blocks exceed the fixed scratch maximum of " + std::to_string(STG_NOALLOC_MAX_ROWS) + " / " +
                  std::to_string(STG_NOALLOC_MAX_BLOCKS) + "; use stg_spmv");
        return STG_ERR_INVALID;
    }
    unsigned char* base = nullptr;
    STG_TRY(noalloc_scratch(&base));
    if(nrows == 0) return STG_OK;
    // every array must live on the current device (or be reachable from it as managed
    // memory): a kernel given another GPU's pointers would fault or read the wrong memory
    int dev = -1;
    STG_CUDA_TRY(cudaGetDevice(&dev));
    const void* ptrs[5] = {x, y, nnzb > 0 ? blocks : nullptr, nnzb > 0 ? (const void*)rows : nullptr,
                           nnzb > 0 ? (const void*)cols : nullptr};
    for(const void* p : ptrs)
    {
        if(!p) continue;
        cudaPointerAttributes at{};
        STG_CUDA_TRY(cudaPointerGetAttributes(&at, p));
        if(!(at.type == cudaMemoryTypeManaged || (at.type == cudaMemoryTypeDevice && at.device == dev)))
        {
            set_error("stg_spmv_noalloc: an input or output is not device memory of the current device " +
                      std::to_string(dev));
            return STG_ERR_INVALID;
        }
    }
    int* counters = reinterpret_cast<int*>(base + kNaCounters);
    int* row_ptr = reinterpret_cast<int*>(base + kNaRowPtr);
    int* t_ptr = reinterpret_cast<int*>(base + kNaTPtr);
    int* t_cnt = reinterpret_cast<int*>(base + kNaTCnt);
    int2* t_ent = reinterpret_cast<int2*>(base + kNaTEnt);

    STG_CUDA_TRY(cudaMemsetAsync(counters, 0, 64 * sizeof(int), s));
    if(nnzb > 0)
    {
        k_bcoo_validate<<<std::max(1, std::min(div_up(nnzb, 256), kSMs * 8)), 256, 0, s>>>(rows, cols, nnzb, nrows,
                                                                                          counters);
        STG_LAUNCH_CHECK();
        int bad = 0;
        STG_CUDA_TRY(cudaMemcpyAsync(&bad, counters, sizeof(int), cudaMemcpyDeviceToHost, s));
        STG_CUDA_TRY(cudaStreamSynchronize(s));
        if(bad)
        {
            set_error("stg_spmv_noalloc: BCOO input: " + std::to_string(bad) +
                      " entries are out of range, lower-triangular, unsorted or duplicated (run stg_convert first)");
            return STG_ERR_INVALID;
        }
    }
    const int g = std::max(1, std::min(div_up(nnzb + 1, 256), kSMs * 16));
    k_row_ptr<<<g, 256, 0, s>>>(rows, nnzb, nrows, row_ptr);
    STG_LAUNCH_CHECK();
    STG_CUDA_TRY(cudaMemsetAsync(t_cnt, 0, sizeof(int) * (nrows + 1), s));
    k_t_count<<<g, 256, 0, s>>>(rows, cols, nnzb, t_cnt);
    STG_LAUNCH_CHECK();
    k_scan_exclusive<<<1, 1024, 0, s>>>(t_cnt, t_ptr, nullptr, nrows + 1, counters + 1);
    STG_LAUNCH_CHECK();
    STG_CUDA_TRY(cudaMemsetAsync(t_cnt, 0, sizeof(int) * (nrows + 1), s));
    k_t_fill<<<g, 256, 0, s>>>(rows, cols, nnzb, t_ptr, t_cnt, t_ent);
    STG_LAUNCH_CHECK();
    k_t_sort<<<std::max(1, std::min(div_up(nrows, 256), kSMs * 16)), 256, 0, s>>>(t_ptr, t_ent, nrows);
    STG_LAUNCH_CHECK();
    const int grid = std::max(1, std::min(div_up(nrows, 256 / 16), kSMs * 8));
    k_spmv_sym<double, 16><<<grid, 256, 0, s>>>(row_ptr, cols, blocks, t_ptr, t_ent, x, y, a, b, nrows);
    STG_LAUNCH_CHECK();
    STG_CUDA_TRY(cudaStreamSynchronize(s));
    return STG_OK;
}
}  // namespace

extern "C" int stg_spmv_noalloc(double a, const double* blocks, const int32_t* rows, const int32_t* cols, int nnzb,
                                const double* x, double b, double* y, int n, void* stream)
{
    try
    {
        return spmv_noalloc(a, blocks, rows, cols, nnzb, x, b, y, n, static_cast<cudaStream_t>(stream));
    }
    catch(const std::exception& e)
    {
        stg::set_error(std::string("stg_spmv_noalloc: ") + e.what());
        return STG_ERR_INVALID;
    }
}
