// learned.cu -- the learned coarse correction (network definition in learned.cuh): the
// coarse level's graph, the forward pass on the tensor cores (mma.sync m16n8k16 BF16 with
// FP32 accumulation), the energy loss, the backward pass, Adam, and the in-loop apply.
//
// The reference has no learned part; the network's only contract with the reference's MAS
// is the level structure it reads (restricted residuals and bank solves of one level,
// MASPreconditioner.cu:729-1027) and the Galerkin operator of that level.
#include "learned.cuh"
#include "reduce.cuh"
#include "solver.hpp"

#include <cooperative_groups.h>
#include <cuda_bf16.h>

namespace stg
{
namespace
{
constexpr int NT = 256;        // threads of the row-parallel kernels
constexpr int TILE_WARPS = 8;  // warps (16-row tiles) per CTA of the layer kernels
constexpr int XS_LD = 2 * NET_H + 8;  // bf16 row stride of a staged 16 x 128 tile (bank-conflict padding)
constexpr int WG_ROWS = 64;    // rows per CTA of the weight-gradient kernels

__device__ __forceinline__ unsigned pack_bf16(float a, float b)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const unsigned*>(&v);
}
__device__ __forceinline__ float2 unpack_bf16(unsigned u)
{
    __nv_bfloat162 v;
    *reinterpret_cast<unsigned*>(&v) = u;
    return __bfloat1622float2(v);
}
__device__ __forceinline__ float bf(const __nv_bfloat16* p, size_t i) { return __bfloat162float(p[i]); }

// D += A B for one 16x8x16 tile: A 16x16 row-major, B 16x8 column-major, BF16 in, FP32 out
__device__ __forceinline__ void mma16816(float (&d)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0,
                                         unsigned b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// One warp: acc[nt] += Xs (16 x K, bf16, row stride ldx) * W^T, W stored [N][K] bf16 with row
// stride ldw (both in shared memory), N = 8 * NTILES.
template <int K, int NTILES>
__device__ __forceinline__ void warp_gemm(const __nv_bfloat16* Xs, int ldx, const __nv_bfloat16* Ws, int ldw,
                                          float (&acc)[NTILES][4])
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for(int kk = 0; kk < K; kk += 16)
    {
        const unsigned a0 = *reinterpret_cast<const unsigned*>(Xs + g * ldx + kk + 2 * t);
        const unsigned a1 = *reinterpret_cast<const unsigned*>(Xs + (g + 8) * ldx + kk + 2 * t);
        const unsigned a2 = *reinterpret_cast<const unsigned*>(Xs + g * ldx + kk + 8 + 2 * t);
        const unsigned a3 = *reinterpret_cast<const unsigned*>(Xs + (g + 8) * ldx + kk + 8 + 2 * t);
#pragma unroll
        for(int nt = 0; nt < NTILES; nt++)
        {
            const unsigned b0 = *reinterpret_cast<const unsigned*>(Ws + (nt * 8 + g) * ldw + kk + 2 * t);
            const unsigned b1 = *reinterpret_cast<const unsigned*>(Ws + (nt * 8 + g) * ldw + kk + 8 + 2 * t);
            mma16816(acc[nt], a0, a1, a2, a3, b0, b1);
        }
    }
}

// copy an [N][K] bf16 weight matrix into shared memory with row stride ld
template <int N, int K>
__device__ __forceinline__ void stage_weights(const __nv_bfloat16* W, __nv_bfloat16* Ws, int ld)
{
    for(int i = threadIdx.x; i < N * K / 2; i += blockDim.x)
    {
        const int o = (2 * i) / K, k = (2 * i) % K;
        *reinterpret_cast<unsigned*>(Ws + o * ld + k) = *reinterpret_cast<const unsigned*>(W + 2 * (size_t)i);
    }
}

__device__ __forceinline__ bool net_gated(const int* flags)
{
    return flags && (__ldcg(flags + F_DONE) != 0 || __ldcg(flags + 3) == 0);
}

// ---------------------------------------------------------------------------------------
// the coarse level's graph
// ---------------------------------------------------------------------------------------
__global__ void k_ng_count(const int* __restrict__ urow, const int* __restrict__ ucol, const double* __restrict__ ublk,
                           int nnzu, int* cnt, float* dblk)
{
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnzu; k += gridDim.x * blockDim.x)
    {
        const int r = urow[k], c = ucol[k];
        if(r != c)
        {
            atomicAdd(cnt + r, 1);
            atomicAdd(cnt + c, 1);
        }
        else
        {
            const double* H = ublk + 9 * (size_t)k;  // column-major
#pragma unroll
            for(int a = 0; a < 3; a++)
#pragma unroll
                for(int b = 0; b < 3; b++) dblk[9 * (size_t)r + 3 * a + b] = (float)H[3 * b + a];
        }
    }
}

__global__ void k_ng_fill(const int* __restrict__ urow, const int* __restrict__ ucol, int nnzu,
                          const int* __restrict__ row, int* cur, long long* key)
{
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnzu; k += gridDim.x * blockDim.x)
    {
        const int r = urow[k], c = ucol[k];
        if(r == c) continue;
        key[row[r] + atomicAdd(cur + r, 1)] = ((long long)c << 32) | (long long)(2 * k);
        key[row[c] + atomicAdd(cur + c, 1)] = ((long long)r << 32) | (long long)(2 * k + 1);
    }
}

__device__ __forceinline__ float frob9(const float* A)
{
    float s = 0.f;
#pragma unroll
    for(int e = 0; e < 9; e++) s += A[e] * A[e];
    return sqrtf(s);
}

// per row: sort the neighbour keys by column (insertion sort; rows are short), then the
// entries' blocks (A_rc = H, A_cr = H^T with H column-major) and coupling weights
__global__ void k_ng_finish(const double* __restrict__ ublk, int n, const int* __restrict__ row, long long* key,
                            int* col, float* oblk, float* w, const float* __restrict__ dblk)
{
    for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const int b = row[i], e = row[i + 1];
        for(int p = b + 1; p < e; p++)
        {
            const long long v = key[p];
            int q = p - 1;
            while(q >= b && key[q] > v)
            {
                key[q + 1] = key[q];
                q--;
            }
            key[q + 1] = v;
        }
        const float di = frob9(dblk + 9 * (size_t)i);
        for(int p = b; p < e; p++)
        {
            const int c = (int)(key[p] >> 32);
            const int src = (int)(key[p] & 0xffffffffLL);
            const double* H = ublk + 9 * (size_t)(src >> 1);
            float* O = oblk + 9 * (size_t)p;
#pragma unroll
            for(int a = 0; a < 3; a++)
#pragma unroll
                for(int bb = 0; bb < 3; bb++) O[3 * a + bb] = (float)((src & 1) ? H[3 * a + bb] : H[3 * bb + a]);
            col[p] = c;
            // |A_rc|_F summed in H's storage order: the same float for both directions
            float h2 = 0.f;
#pragma unroll
            for(int q = 0; q < 9; q++) h2 += (float)H[q] * (float)H[q];
            const float dc = frob9(dblk + 9 * (size_t)c);
            const float den = sqrtf(di * dc);
            w[p] = den > 0.f ? sqrtf(h2) / den : 0.f;
        }
    }
}

// neighbour entries packed for the fused kernel: (owner rank << 16 | row in the owner, w)
__global__ void k_ng_pack(const int* __restrict__ col, const float* __restrict__ w, int nnz, int rpc, int2* out)
{
    for(int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x)
    {
        const int j = col[e], o = j / rpc;
        out[e] = make_int2((o << 16) | (j - o * rpc), __float_as_int(w[e]));
    }
}

// f_i = log(trace A_ii) minus its mean over the level (one CTA of 1024 threads)
__global__ void __launch_bounds__(1024) k_ng_feat(const float* __restrict__ dblk, int n, float* feat)
{
    __shared__ double red[32];
    __shared__ double mean;
    double s = 0;
    for(int i = threadIdx.x; i < n; i += 1024)
    {
        const float* D = dblk + 9 * (size_t)i;
        s += log(fmax((double)D[0] + D[4] + D[8], 1e-30));
    }
    s = block_sum<1024>(s, red);
    if(threadIdx.x == 0) mean = n > 0 ? s / n : 0.0;
    __syncthreads();
    for(int i = threadIdx.x; i < n; i += 1024)
    {
        const float* D = dblk + 9 * (size_t)i;
        feat[i] = (float)(log(fmax((double)D[0] + D[4] + D[8], 1e-30)) - mean);
    }
}
}  // namespace

int net_build_graph(cudaStream_t s, NetGraphStore& G, int n, int nnzu, const int* urow, const int* ucol,
                    const double* ublk, int* launches)
{
    G.n = n;
    STG_TRY(G.row.resize(n + 1));
    STG_TRY(G.cnt.resize(n + 1));
    STG_TRY(G.cur.resize(n + 1));
    STG_TRY(G.dblk.resize(9 * (size_t)std::max(n, 1)));
    STG_TRY(G.feat.resize(std::max(n, 1)));
    STG_CUDA_TRY(cudaMemsetAsync(G.cnt.data(), 0, sizeof(int) * (n + 1), s));
    STG_CUDA_TRY(cudaMemsetAsync(G.cur.data(), 0, sizeof(int) * (n + 1), s));
    STG_CUDA_TRY(cudaMemsetAsync(G.dblk.data(), 0, sizeof(float) * 9 * (size_t)std::max(n, 1), s));
    const int g = std::max(1, std::min(div_up(nnzu, NT), kSMs * 8));
    if(nnzu > 0)
    {
        k_ng_count<<<g, NT, 0, s>>>(urow, ucol, ublk, nnzu, G.cnt.data(), G.dblk.data());
        STG_LAUNCH_CHECK();
        (*launches)++;
    }
    k_scan_exclusive<<<1, 1024, 0, s>>>(G.cnt.data(), G.row.data(), nullptr, n, G.row.data() + n);
    STG_LAUNCH_CHECK();
    (*launches)++;
    int nnz = 0;
    STG_CUDA_TRY(cudaMemcpyAsync(&nnz, G.row.data() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    STG_CUDA_TRY(cudaStreamSynchronize(s));
    G.nnz = nnz;
    STG_TRY(G.key.resize(std::max(nnz, 1)));
    STG_TRY(G.col.resize(std::max(nnz, 1)));
    STG_TRY(G.w.resize(std::max(nnz, 1)));
    STG_TRY(G.oblk.resize(9 * (size_t)std::max(nnz, 1)));
    if(nnzu > 0)
    {
        k_ng_fill<<<g, NT, 0, s>>>(urow, ucol, nnzu, G.row.data(), G.cur.data(), G.key.data());
        STG_LAUNCH_CHECK();
        (*launches)++;
    }
    k_ng_finish<<<std::max(1, div_up(n, NT)), NT, 0, s>>>(ublk, n, G.row.data(), G.key.data(), G.col.data(),
                                                         G.oblk.data(), G.w.data(), G.dblk.data());
    STG_LAUNCH_CHECK();
    k_ng_feat<<<1, 1024, 0, s>>>(G.dblk.data(), n, G.feat.data());
    STG_LAUNCH_CHECK();
    (*launches) += 2;
    std::vector<int> hrow(n + 1);
    STG_CUDA_TRY(cudaMemcpyAsync(hrow.data(), G.row.data(), sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
    STG_CUDA_TRY(cudaStreamSynchronize(s));
    STG_TRY(net_fused_plan(hrow.data(), n, &G.fu_cl, &G.fu_rpc));
    if(G.fu_cl > 0 && nnz > 0)
    {
        STG_TRY(G.fu_nb.resize(nnz));
        k_ng_pack<<<std::max(1, std::min(div_up(nnz, NT), kSMs * 4)), NT, 0, s>>>(G.col.data(), G.w.data(), nnz, G.fu_rpc,
                                                                                  G.fu_nb.data());
        STG_LAUNCH_CHECK();
        (*launches)++;
    }
    return 0;
}

// ---------------------------------------------------------------------------------------
// forward
// ---------------------------------------------------------------------------------------
namespace
{
// per sample (one CTA each): the RMS scales and the 16-wide BF16 input rows
__global__ void __launch_bounds__(NT) k_net_input(NetGraph g, const float* __restrict__ rc, const float* __restrict__ zc,
                                                  int S, int rows_pad, __nv_bfloat16* x0, float* scale, const int* flags)
{
    if(net_gated(flags)) return;
    __shared__ double red[NT / 32];
    __shared__ float sc[2];
    const int s = blockIdx.x, n = g.n;
    const float* r = rc + 4 * (size_t)n * s;
    const float* z = zc + 4 * (size_t)n * s;
    double rr = 0, zz = 0;
    for(int i = threadIdx.x; i < n; i += NT)
    {
        const float4 a = *reinterpret_cast<const float4*>(r + 4 * (size_t)i);
        const float4 b = *reinterpret_cast<const float4*>(z + 4 * (size_t)i);
        rr += (double)a.x * a.x + (double)a.y * a.y + (double)a.z * a.z;
        zz += (double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z;
    }
    rr = block_sum<NT>(rr, red);
    zz = block_sum<NT>(zz, red);
    if(threadIdx.x == 0)
    {
        const float sr = n > 0 ? (float)sqrt(rr / n) : 0.f, sz = n > 0 ? (float)sqrt(zz / n) : 0.f;
        sc[0] = sr > 0.f ? sr : 1.f;
        sc[1] = sz > 0.f ? sz : 1.f;
        scale[2 * s] = sc[0];
        scale[2 * s + 1] = sc[1];
    }
    __syncthreads();
    const float ir = 1.f / sc[0], iz = 1.f / sc[1];
    for(int i = threadIdx.x; i < n; i += NT)
    {
        const float4 a = *reinterpret_cast<const float4*>(r + 4 * (size_t)i);
        const float4 b = *reinterpret_cast<const float4*>(z + 4 * (size_t)i);
        uint4 lo;
        lo.x = pack_bf16(a.x * ir, a.y * ir);
        lo.y = pack_bf16(a.z * ir, b.x * iz);
        lo.z = pack_bf16(b.y * iz, b.z * iz);
        lo.w = pack_bf16(g.feat[i], 1.f);
        uint4* dst = reinterpret_cast<uint4*>(x0 + NET_IN * ((size_t)s * n + i));
        dst[0] = lo;
        dst[1] = make_uint4(0u, 0u, 0u, 0u);
    }
    if(s == S - 1)  // zero the padding rows
        for(int i = S * n + threadIdx.x; i < rows_pad; i += NT)
        {
            uint4* dst = reinterpret_cast<uint4*>(x0 + NET_IN * (size_t)i);
            dst[0] = make_uint4(0u, 0u, 0u, 0u);
            dst[1] = make_uint4(0u, 0u, 0u, 0u);
        }
}

// bias + relu of one warp's 16 x 64 accumulators into BF16 rows r0 .. r0+15 (row stride 64)
__device__ __forceinline__ void store_relu(const float (&acc)[8][4], const float* __restrict__ bias, __nv_bfloat16* H,
                                           int r0)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for(int nt = 0; nt < 8; nt++)
    {
        const int c = nt * 8 + 2 * t;
        const float b0 = bias[c], b1 = bias[c + 1];
        *reinterpret_cast<unsigned*>(H + (size_t)(r0 + g) * NET_H + c) =
            pack_bf16(fmaxf(acc[nt][0] + b0, 0.f), fmaxf(acc[nt][1] + b1, 0.f));
        *reinterpret_cast<unsigned*>(H + (size_t)(r0 + g + 8) * NET_H + c) =
            pack_bf16(fmaxf(acc[nt][2] + b0, 0.f), fmaxf(acc[nt][3] + b1, 0.f));
    }
}

// h0 = relu(W0 x + b0): one warp per 16-row tile, A and B fragments straight from global
__global__ void __launch_bounds__(NT) k_net_embed(const __nv_bfloat16* __restrict__ x0, const __nv_bfloat16* __restrict__ W,
                                                  const float* __restrict__ bias, __nv_bfloat16* h0, int tiles,
                                                  const int* flags)
{
    if(net_gated(flags)) return;
    const int tile = blockIdx.x * TILE_WARPS + (threadIdx.x >> 5);
    if(tile >= tiles) return;
    float acc[8][4] = {};
    warp_gemm<NET_IN, 8>(x0 + (size_t)tile * 16 * NET_IN, NET_IN, W, NET_IN, acc);
    store_relu(acc, bias, h0, tile * 16);
}

// one message-passing layer: m = sum_j w_ij h_j (FP32, neighbours in column order, rounded
// once to BF16), then h' = relu(W [h, m] + b) on the tensor cores
__global__ void __launch_bounds__(NT) k_net_mp(NetGraph g, int rows, const __nv_bfloat16* __restrict__ hin,
                                               const __nv_bfloat16* __restrict__ W, const float* __restrict__ bias,
                                               __nv_bfloat16* mout, __nv_bfloat16* hout, int tiles, const int* flags)
{
    if(net_gated(flags)) return;
    extern __shared__ __align__(16) unsigned char net_smem[];
    __nv_bfloat16* Ws = reinterpret_cast<__nv_bfloat16*>(net_smem);
    __nv_bfloat16* Xs = Ws + NET_H * XS_LD + (threadIdx.x >> 5) * 16 * XS_LD;
    stage_weights<NET_H, 2 * NET_H>(W, Ws, XS_LD);
    __syncthreads();
    const int tile = blockIdx.x * TILE_WARPS + (threadIdx.x >> 5);
    if(tile >= tiles) return;
    const int lane = threadIdx.x & 31, n = g.n;
    for(int rr = 0; rr < 16; rr++)
    {
        const int row = tile * 16 + rr;
        unsigned self = 0u, msg = 0u;
        if(row < rows)
        {
            const int s = row / n, node = row - s * n;
            const size_t base = (size_t)s * n;
            self = *reinterpret_cast<const unsigned*>(hin + (size_t)row * NET_H + 2 * lane);
            float a0 = 0.f, a1 = 0.f;
            int e = g.row[node];
            const int ee = g.row[node + 1];
            for(; e + 4 <= ee; e += 4)
            {
                int j[4];
                float w[4];
                unsigned v[4];
#pragma unroll
                for(int u = 0; u < 4; u++)
                {
                    j[u] = g.col[e + u];
                    w[u] = g.w[e + u];
                }
#pragma unroll
                for(int u = 0; u < 4; u++) v[u] = *reinterpret_cast<const unsigned*>(hin + (base + j[u]) * NET_H + 2 * lane);
#pragma unroll
                for(int u = 0; u < 4; u++)
                {
                    const float2 f = unpack_bf16(v[u]);
                    a0 = fmaf(w[u], f.x, a0);
                    a1 = fmaf(w[u], f.y, a1);
                }
            }
            for(; e < ee; e++)
            {
                const float2 f = unpack_bf16(*reinterpret_cast<const unsigned*>(hin + (base + g.col[e]) * NET_H + 2 * lane));
                a0 = fmaf(g.w[e], f.x, a0);
                a1 = fmaf(g.w[e], f.y, a1);
            }
            msg = pack_bf16(a0, a1);
            *reinterpret_cast<unsigned*>(mout + (size_t)row * NET_H + 2 * lane) = msg;
        }
        *reinterpret_cast<unsigned*>(Xs + rr * XS_LD + 2 * lane) = self;
        *reinterpret_cast<unsigned*>(Xs + rr * XS_LD + NET_H + 2 * lane) = msg;
    }
    __syncwarp();
    float acc[8][4] = {};
    warp_gemm<2 * NET_H, 8>(Xs, XS_LD, Ws, XS_LD, acc);
    store_relu(acc, bias, hout, tile * 16);
}

// d = Wo h3 + bo (outputs 0..2 of 8): FP32 [rows_pad][4]
__global__ void __launch_bounds__(NT) k_net_head(const __nv_bfloat16* __restrict__ h3, const __nv_bfloat16* __restrict__ W,
                                                 const float* __restrict__ bias, float* delta, int tiles, const int* flags)
{
    if(net_gated(flags)) return;
    const int tile = blockIdx.x * TILE_WARPS + (threadIdx.x >> 5);
    if(tile >= tiles) return;
    float acc[1][4] = {};
    warp_gemm<NET_H, 1>(h3 + (size_t)tile * 16 * NET_H, NET_H, W, NET_H, acc);
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    if(t < 2)
    {
        const int r0 = tile * 16 + g;
        const float2 lo = t == 0 ? make_float2(acc[0][0] + bias[0], acc[0][1] + bias[1]) : make_float2(acc[0][0] + bias[2], 0.f);
        const float2 hi = t == 0 ? make_float2(acc[0][2] + bias[0], acc[0][3] + bias[1]) : make_float2(acc[0][2] + bias[2], 0.f);
        *reinterpret_cast<float2*>(delta + 4 * (size_t)r0 + 2 * t) = lo;
        *reinterpret_cast<float2*>(delta + 4 * (size_t)(r0 + 8) + 2 * t) = hi;
    }
}

// in the PCG loop (one sample): Z_level += theta s_z d, theta = 1 unless the correction
// would take r_c.g below half of r_c.z (then the largest theta that keeps it there)
__global__ void __launch_bounds__(1024) k_net_apply(int n, const float* __restrict__ rc, const float* __restrict__ delta,
                                                    const float* __restrict__ scale, float* Z, const int* flags)
{
    if(net_gated(flags)) return;
    __shared__ double red[32];
    __shared__ float th;
    const float sz = scale[1];
    double a = 0, b = 0;
    for(int i = threadIdx.x; i < n; i += 1024)
    {
        const float4 r = *reinterpret_cast<const float4*>(rc + 4 * (size_t)i);
        const float4 z = *reinterpret_cast<const float4*>(Z + 4 * (size_t)i);
        const float4 d = *reinterpret_cast<const float4*>(delta + 4 * (size_t)i);
        a += (double)r.x * z.x + (double)r.y * z.y + (double)r.z * z.z;
        b += (double)r.x * d.x + (double)r.y * d.y + (double)r.z * d.z;
    }
    a = block_sum<1024>(a, red);
    b = block_sum<1024>(b, red);
    if(threadIdx.x == 0)
    {
        b *= sz;
        th = (b < -0.5 * a && b < 0.0) ? (float)(-0.5 * a / b) : 1.f;
        if(!(th >= 0.f)) th = 0.f;
    }
    __syncthreads();
    const float f = th * sz;
    for(int i = threadIdx.x; i < n; i += 1024)
    {
        float4 z = *reinterpret_cast<const float4*>(Z + 4 * (size_t)i);
        const float4 d = *reinterpret_cast<const float4*>(delta + 4 * (size_t)i);
        z.x = fmaf(f, d.x, z.x);
        z.y = fmaf(f, d.y, z.y);
        z.z = fmaf(f, d.z, z.z);
        *reinterpret_cast<float4*>(Z + 4 * (size_t)i) = z;
    }
}
}  // namespace

// ---------------------------------------------------------------------------------------
// loss and backward
// ---------------------------------------------------------------------------------------
namespace
{
// y = A v at node i of the level (v given per node as z + f d, FP64 arithmetic)
__device__ __forceinline__ void level_row(const NetGraph& g, int i, const float* __restrict__ z,
                                          const float* __restrict__ d, double f, double (&y)[3])
{
    auto val = [&](int j, int a) -> double {
        return (double)z[4 * (size_t)j + a] + (d ? f * (double)d[4 * (size_t)j + a] : 0.0);
    };
    const float* D = g.dblk + 9 * (size_t)i;
    const double v0 = val(i, 0), v1 = val(i, 1), v2 = val(i, 2);
    y[0] = (double)D[0] * v0 + (double)D[1] * v1 + (double)D[2] * v2;
    y[1] = (double)D[3] * v0 + (double)D[4] * v1 + (double)D[5] * v2;
    y[2] = (double)D[6] * v0 + (double)D[7] * v1 + (double)D[8] * v2;
    for(int e = g.row[i]; e < g.row[i + 1]; e++)
    {
        const int j = g.col[e];
        const float* O = g.oblk + 9 * (size_t)e;
        const double u0 = val(j, 0), u1 = val(j, 1), u2 = val(j, 2);
        y[0] += (double)O[0] * u0 + (double)O[1] * u1 + (double)O[2] * u2;
        y[1] += (double)O[3] * u0 + (double)O[4] * u1 + (double)O[5] * u2;
        y[2] += (double)O[6] * u0 + (double)O[7] * u1 + (double)O[8] * u2;
    }
}

// per sample (one CTA): g = z + s_z d; loss = J(g) / |J(z)|, J(v) = 1/2 v.A v - v.r;
// ddelta = (s_z / |J(z)| / S) (A g - r)
__global__ void __launch_bounds__(NT) k_net_loss(NetGraph g, const float* __restrict__ rc, const float* __restrict__ zc,
                                                 const float* __restrict__ delta, const float* __restrict__ scale, int S,
                                                 float* ddelta, float* loss)
{
    __shared__ double red[NT / 32];
    __shared__ double coef;
    const int s = blockIdx.x, n = g.n;
    const float* r = rc + 4 * (size_t)n * s;
    const float* z = zc + 4 * (size_t)n * s;
    const float* d = delta + 4 * (size_t)n * s;
    const double sz = scale[2 * s + 1];
    double J = 0, J0 = 0;
    for(int i = threadIdx.x; i < n; i += NT)
    {
        double y[3], y0[3];
        level_row(g, i, z, d, sz, y);
        level_row(g, i, z, nullptr, 0.0, y0);
#pragma unroll
        for(int a = 0; a < 3; a++)
        {
            const double zi = z[4 * (size_t)i + a], gi = zi + sz * (double)d[4 * (size_t)i + a];
            const double ri = r[4 * (size_t)i + a];
            J += 0.5 * gi * y[a] - gi * ri;
            J0 += 0.5 * zi * y0[a] - zi * ri;
        }
    }
    J = block_sum<NT>(J, red);
    J0 = block_sum<NT>(J0, red);
    if(threadIdx.x == 0)
    {
        const double inv = J0 != 0.0 ? 1.0 / fabs(J0) : 0.0;
        loss[s] = (float)(J * inv);
        coef = sz * inv / S;
    }
    __syncthreads();
    const double cf = coef;
    for(int i = threadIdx.x; i < n; i += NT)
    {
        double y[3];
        level_row(g, i, z, d, sz, y);
        const float4 ri = *reinterpret_cast<const float4*>(r + 4 * (size_t)i);
        *reinterpret_cast<float4*>(ddelta + 4 * ((size_t)n * s + i)) =
            make_float4((float)(cf * (y[0] - ri.x)), (float)(cf * (y[1] - ri.y)), (float)(cf * (y[2] - ri.z)), 0.f);
    }
}

// dU3 = (ddelta Wo) * [h3 > 0]
__global__ void __launch_bounds__(NT) k_net_head_bwd(const float* __restrict__ ddelta, const __nv_bfloat16* __restrict__ W,
                                                     const __nv_bfloat16* __restrict__ h3, float* du, int rows)
{
    const int idx = blockIdx.x * NT + threadIdx.x;
    const int row = idx / NET_H, c = idx % NET_H;
    if(row >= rows) return;
    float v = 0.f;
#pragma unroll
    for(int o = 0; o < 3; o++) v = fmaf(ddelta[4 * (size_t)row + o], bf(W, (size_t)o * NET_H + c), v);
    du[idx] = bf(h3, idx) > 0.f ? v : 0.f;
}

// per-CTA partial weight gradients of one layer: part[o][k] = sum_rows du[r][o] x[r][k],
// part[N*K + o] = sum_rows du[r][o], over WG_ROWS rows; x = [xa (ka columns), xb].  Only
// outputs o < nvalid have a gradient.
template <int K, int N>
__global__ void __launch_bounds__(NT) k_net_wgrad(const __nv_bfloat16* __restrict__ xa, int lda, int ka,
                                                  const __nv_bfloat16* __restrict__ xb, int ldb,
                                                  const float* __restrict__ du, int ldu, int nvalid, int rows, float* part)
{
    constexpr int TPO = NT / N, KPT = K / TPO;
    __shared__ float Xs[32][K];
    __shared__ float Us[32][N];
    const int o = threadIdx.x / TPO, kq = threadIdx.x % TPO;
    float acc[KPT] = {};
    float db = 0.f;
    const int r0 = blockIdx.x * WG_ROWS;
    for(int rb = r0; rb < min(r0 + WG_ROWS, rows); rb += 32)
    {
        const int cnt = min(32, rows - rb);
        __syncthreads();
        for(int i = threadIdx.x; i < 32 * K; i += NT)
        {
            const int rr = i / K, k = i % K;
            float v = 0.f;
            if(rr < cnt) v = k < ka ? bf(xa, (size_t)(rb + rr) * lda + k) : bf(xb, (size_t)(rb + rr) * ldb + (k - ka));
            Xs[rr][k] = v;
        }
        for(int i = threadIdx.x; i < 32 * N; i += NT)
        {
            const int rr = i / N, oo = i % N;
            Us[rr][oo] = (rr < cnt && oo < nvalid) ? du[(size_t)(rb + rr) * ldu + oo] : 0.f;
        }
        __syncthreads();
        for(int rr = 0; rr < cnt; rr++)
        {
            const float u = Us[rr][o];
#pragma unroll
            for(int q = 0; q < KPT; q++) acc[q] = fmaf(u, Xs[rr][kq + TPO * q], acc[q]);
            db += u;
        }
    }
    float* P = part + (size_t)blockIdx.x * (N * K + N);
#pragma unroll
    for(int q = 0; q < KPT; q++) P[o * K + kq + TPO * q] = acc[q];
    if(kq == 0) P[N * K + o] = db;
}

// grad_w[i] = sum over CTAs of part[b][i] (fixed order), grad_b likewise
__global__ void k_net_reduce(const float* __restrict__ part, int nblk, int nw, int nb, float* gw, float* gb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= nw + nb) return;
    float s = 0.f;
    for(int b = 0; b < nblk; b++) s += part[(size_t)b * (nw + nb) + i];
    if(i < nw)
        gw[i] = s;
    else
        gb[i - nw] = s;
}

// dX = dU W (W [64][128]): first 64 columns to dha (the layer input h), last 64 to dm
__global__ void __launch_bounds__(NT) k_net_dx(const float* __restrict__ du, const __nv_bfloat16* __restrict__ W,
                                               float* dha, float* dm, int rows)
{
    __shared__ float Wf[NET_H][2 * NET_H];
    __shared__ float Us[32][NET_H];
    for(int i = threadIdx.x; i < NET_H * 2 * NET_H; i += NT) Wf[i / (2 * NET_H)][i % (2 * NET_H)] = bf(W, i);
    const int r0 = blockIdx.x * 32;
    for(int i = threadIdx.x; i < 32 * NET_H; i += NT)
    {
        const int rr = i / NET_H;
        Us[rr][i % NET_H] = r0 + rr < rows ? du[(size_t)r0 * NET_H + i] : 0.f;
    }
    __syncthreads();
    const int k = threadIdx.x % (2 * NET_H), rg = threadIdx.x / (2 * NET_H);
    for(int rr = rg * 16; rr < rg * 16 + 16; rr++)
    {
        const int row = r0 + rr;
        if(row >= rows) break;
        float v = 0.f;
#pragma unroll 16
        for(int o = 0; o < NET_H; o++) v = fmaf(Us[rr][o], Wf[o][k], v);
        if(k < NET_H)
            dha[(size_t)row * NET_H + k] = v;
        else
            dm[(size_t)row * NET_H + k - NET_H] = v;
    }
}

// dU_prev = (dha + sum_j w_ij dm_j) * [h_prev > 0]: one warp per row, 2 channels per lane
__global__ void __launch_bounds__(NT) k_net_agg_mask(NetGraph g, int rows, const float* __restrict__ dha,
                                                     const float* __restrict__ dm, const __nv_bfloat16* __restrict__ hprev,
                                                     float* du)
{
    const int row = blockIdx.x * (NT / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if(row >= rows) return;
    const int n = g.n, s = row / n, node = row - s * n;
    const size_t base = (size_t)s * n;
    float2 a = *reinterpret_cast<const float2*>(dha + (size_t)row * NET_H + 2 * lane);
    for(int e = g.row[node]; e < g.row[node + 1]; e++)
    {
        const float w = g.w[e];
        const float2 m = *reinterpret_cast<const float2*>(dm + (base + g.col[e]) * NET_H + 2 * lane);
        a.x = fmaf(w, m.x, a.x);
        a.y = fmaf(w, m.y, a.y);
    }
    const float2 h = unpack_bf16(*reinterpret_cast<const unsigned*>(hprev + (size_t)row * NET_H + 2 * lane));
    *reinterpret_cast<float2*>(du + (size_t)row * NET_H + 2 * lane) = make_float2(h.x > 0.f ? a.x : 0.f, h.y > 0.f ? a.y : 0.f);
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8); c1 / c2 the bias corrections of this step
__global__ void k_net_adam(float* p, const float* __restrict__ gr, float* m, float* v, int count, float lr, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= count) return;
    const float gi = gr[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
}

__global__ void k_net_bf16(const float* __restrict__ p, __nv_bfloat16* w, int count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < count) w[i] = __float2bfloat16_rn(p[i]);
}
// sample recorder inside the PCG loop: at iterations k = 0, every, 2 every, ... the level's
// restricted residual and bank solve (before any learned correction) go to slot k / every
__global__ void __launch_bounds__(NT) k_net_record(const float* __restrict__ R, const float* __restrict__ Z, int n,
                                                   const double* __restrict__ scal, const int* __restrict__ flags,
                                                   float* rc, float* zc, int* count, int cap, int every)
{
    if(__ldcg(flags + F_DONE)) return;
    const long k = (long)__ldcg(scal + SS_ITER);
    if(k % every != 0 || k / every >= cap) return;
    const int slot = (int)(k / every);
    for(int i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT)
    {
        reinterpret_cast<float4*>(rc)[(size_t)slot * n + i] = reinterpret_cast<const float4*>(R)[i];
        reinterpret_cast<float4*>(zc)[(size_t)slot * n + i] = reinterpret_cast<const float4*>(Z)[i];
    }
    if(blockIdx.x == 0 && threadIdx.x == 0) atomicMax(count, slot + 1);
}
}  // namespace

int net_record(cudaStream_t s, const float* R, const float* Z, int n, const double* scal, const int* flags, float* rc,
               float* zc, int* count, int cap, int every)
{
    k_net_record<<<std::max(1, std::min(div_up(n, NT), kSMs)), NT, 0, s>>>(R, Z, n, scal, flags, rc, zc, count, cap,
                                                                          every);
    STG_LAUNCH_CHECK();
    return 0;
}

// ---------------------------------------------------------------------------------------
// fused in-loop forward: the whole network in one launch of one thread-block cluster
// ---------------------------------------------------------------------------------------
namespace cg = cooperative_groups;

constexpr int FU_THREADS = 512;   // 16 warps
constexpr int FU_RPC = 128;       // max rows (level nodes) per CTA
constexpr int FU_EPC = 4096;      // max neighbour entries per CTA
constexpr int FU_HS = 2 * FU_RPC * NET_H * 2;          // own rows' h, double-buffered, bf16
constexpr int FU_XS = FU_RPC * XS_LD * 2;              // [h, m] tiles, bf16
constexpr int FU_WS = NET_H * XS_LD * 2;               // staged W_k, bf16
constexpr int FU_NB = FU_EPC * 8;                      // (owner rank << 16 | local row, w) per entry
constexpr int FU_DL = FU_RPC * 16;                     // d, float4 per row
constexpr int FU_RP = (FU_RPC + 4) * 4;                // own rows' entry offsets
constexpr int FU_RZ = 2 * FU_RPC * 16;                  // own rows' r and z
constexpr int FU_RED = 512;                             // block sums [32], cluster partials, scales
constexpr int FU_SMEM = FU_HS + FU_XS + FU_WS + FU_NB + FU_DL + FU_RED + FU_RP + FU_RZ;

namespace
{
// two deterministic block sums at once (result valid in thread 0)
__device__ __forceinline__ void block_sum2_fu(double& x, double& y, double* red)
{
    x = warp_sum(x);
    y = warp_sum(y);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if(lane == 0)
    {
        red[warp] = x;
        red[16 + warp] = y;
    }
    __syncthreads();
    if(threadIdx.x < 32)
    {
        x = warp_sum(lane < FU_THREADS / 32 ? red[lane] : 0.0);
        y = warp_sum(lane < FU_THREADS / 32 ? red[16 + lane] : 0.0);
    }
}

// lane q of warp 0 fetches CTA q's pair at red[slot], lane 0 sums them in rank order
__device__ __forceinline__ void cluster_sum2(cg::cluster_group& cluster, double* red, int slot, int nranks,
                                             double& a, double& b)
{
    const int lane = threadIdx.x & 31;
    double va = 0, vb = 0;
    if(lane < nranks)
    {
        const double* rq = cluster.map_shared_rank(red, lane);
        va = rq[slot];
        vb = rq[slot + 1];
    }
    a = 0;
    b = 0;
    for(int q = 0; q < nranks; q++)
    {
        a += __shfl_sync(0xffffffffu, va, q);
        b += __shfl_sync(0xffffffffu, vb, q);
    }
}

__device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// 16-byte load from the shared memory of CTA `rank` of the cluster at this CTA's offset `a`
__device__ __forceinline__ uint4 ld_dsmem16(unsigned a, int rank)
{
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    uint4 v;
    asm volatile("ld.shared::cluster.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(r)
                 : "memory");
    return v;
}

// W_k ([64][128] bf16) into shared memory rows of XS_LD with 16-byte asynchronous copies
__device__ __forceinline__ void stage_weights_async(const __nv_bfloat16* W, __nv_bfloat16* Ws)
{
    for(int i = threadIdx.x; i < NET_H * 2 * NET_H / 8; i += FU_THREADS)
    {
        const int o = (8 * i) / (2 * NET_H), k = (8 * i) % (2 * NET_H);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(Ws + o * XS_LD + k)),
                     "l"(W + 8 * (size_t)i)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void fma8(float (&a)[8], float w, uint4 v)
{
    const float2 f0 = unpack_bf16(v.x), f1 = unpack_bf16(v.y), f2 = unpack_bf16(v.z), f3 = unpack_bf16(v.w);
    a[0] = fmaf(w, f0.x, a[0]);
    a[1] = fmaf(w, f0.y, a[1]);
    a[2] = fmaf(w, f1.x, a[2]);
    a[3] = fmaf(w, f1.y, a[3]);
    a[4] = fmaf(w, f2.x, a[4]);
    a[5] = fmaf(w, f2.y, a[5]);
    a[6] = fmaf(w, f3.x, a[6]);
    a[7] = fmaf(w, f3.y, a[7]);
}

// The network of learned.cuh for one sample, rows split over the cluster's CTAs in
// contiguous ranges of rpc rows; a CTA keeps its rows' activations in shared memory and
// reads its neighbours' from the owning CTA (distributed shared memory).  The order of every
// sum matches the layered kernels except the RMS scales (CTA partials summed in rank order).
// nbp: the neighbour entries packed as (owner rank << 16 | row in the owner, w) (graph
// build), or null (packed here from col / w).
__global__ void __launch_bounds__(FU_THREADS) k_net_fused(NetGraph g, const int2* __restrict__ nbp,
                                                         const float* __restrict__ rc, float* Z,
                                                         const __nv_bfloat16* __restrict__ wbf,
                                                         const float* __restrict__ params, const int* flags, int rpc)
{
    if(net_gated(flags)) return;  // uniform over the cluster: nothing changes the flags meanwhile
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank(), nranks = (int)cluster.num_blocks();
    extern __shared__ __align__(16) unsigned char fu_smem[];
    __nv_bfloat16* Hs = reinterpret_cast<__nv_bfloat16*>(fu_smem);
    __nv_bfloat16* Xs = reinterpret_cast<__nv_bfloat16*>(fu_smem + FU_HS);
    __nv_bfloat16* Ws = reinterpret_cast<__nv_bfloat16*>(fu_smem + FU_HS + FU_XS);
    int2* nb = reinterpret_cast<int2*>(fu_smem + FU_HS + FU_XS + FU_WS);
    float4* dl = reinterpret_cast<float4*>(fu_smem + FU_HS + FU_XS + FU_WS + FU_NB);
    double* red = reinterpret_cast<double*>(fu_smem + FU_HS + FU_XS + FU_WS + FU_NB + FU_DL);  // [32] block sums
    int* rp = reinterpret_cast<int*>(fu_smem + FU_HS + FU_XS + FU_WS + FU_NB + FU_DL + FU_RED);
    float4* rz = reinterpret_cast<float4*>(fu_smem + FU_HS + FU_XS + FU_WS + FU_NB + FU_DL + FU_RED + FU_RP);  // [2][rpc]
    double* part = red + 32;                         // [4]: cluster partials read by the other CTAs
    float* sc = reinterpret_cast<float*>(red + 36);  // s_r, s_z, theta
    const int n = g.n, r0 = min(rank * rpc, n), own = max(0, min(rpc, n - r0));
    const int tiles = (own + 15) / 16;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = FU_THREADS / 32;

    // ---- P0: layer-0 weights (async), neighbour lists, own r / z, the RMS scales ----
    stage_weights_async(wbf + P_W1, Ws);
    const int e_base = g.row[r0], e_end = g.row[r0 + own];
    for(int i = threadIdx.x; i <= own; i += FU_THREADS) rp[i] = g.row[r0 + i] - e_base;
    if(nbp)
    {
#pragma unroll 4
        for(int e = e_base + threadIdx.x; e < e_end; e += FU_THREADS) nb[e - e_base] = nbp[e];
    }
    else
        for(int e = e_base + threadIdx.x; e < e_end; e += FU_THREADS)
        {
            const int j = g.col[e], o = j / rpc;
            nb[e - e_base] = make_int2((o << 16) | (j - o * rpc), __float_as_int(g.w[e]));
        }
    double rr = 0, zz = 0;
    for(int i = threadIdx.x; i < own; i += FU_THREADS)
    {
        const float4 a = *reinterpret_cast<const float4*>(rc + 4 * (size_t)(r0 + i));
        const float4 b = *reinterpret_cast<const float4*>(Z + 4 * (size_t)(r0 + i));
        rz[i] = a;
        rz[FU_RPC + i] = b;
        rr += (double)a.x * a.x + (double)a.y * a.y + (double)a.z * a.z;
        zz += (double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z;
    }
    block_sum2_fu(rr, zz, red);
    if(threadIdx.x == 0)
    {
        part[0] = rr;
        part[1] = zz;
    }
    cluster.sync();
    if(warp == 0)
    {
        double sr, sz;
        cluster_sum2(cluster, part, 0, nranks, sr, sz);
        if(lane == 0)
        {
            const float fr = n > 0 ? (float)sqrt(sr / n) : 0.f, fz = n > 0 ? (float)sqrt(sz / n) : 0.f;
            sc[0] = fr > 0.f ? fr : 1.f;
            sc[1] = fz > 0.f ? fz : 1.f;
        }
    }
    __syncthreads();
    const float s_r = sc[0], s_z = sc[1];

    // ---- P1: input rows (bf16, in the X tiles' first 16 columns) and the embedding ----
    {
        const float ir = 1.f / s_r, iz = 1.f / s_z;
        for(int i = threadIdx.x; i < tiles * 16; i += FU_THREADS)
        {
            uint4 lo = make_uint4(0u, 0u, 0u, 0u);
            if(i < own)
            {
                const float4 a = rz[i], b = rz[FU_RPC + i];
                lo.x = pack_bf16(a.x * ir, a.y * ir);
                lo.y = pack_bf16(a.z * ir, b.x * iz);
                lo.z = pack_bf16(b.y * iz, b.z * iz);
                lo.w = pack_bf16(g.feat[r0 + i], 1.f);
            }
            *reinterpret_cast<uint4*>(Xs + i * XS_LD) = lo;
            *reinterpret_cast<uint4*>(Xs + i * XS_LD + 8) = make_uint4(0u, 0u, 0u, 0u);
        }
        __syncthreads();
        if(warp < tiles)
        {
            float acc[8][4] = {};
            warp_gemm<NET_IN, 8>(Xs + warp * 16 * XS_LD, XS_LD, wbf + P_W0, NET_IN, acc);
            store_relu(acc, params + P_B0, Hs, warp * 16);  // buffer 0, row stride 64
        }
    }
    cluster.sync();

    // ---- P2: three message-passing layers ----
    int cur = 0;
    for(int k = 0; k < NET_LAYERS; k++)
    {
        const __nv_bfloat16* Hc = Hs + cur * FU_RPC * NET_H;
        const unsigned hbase = smem_addr(Hc);
        // gather: 4 rows per warp at a time, 8 lanes per row, 8 channels (16 bytes) per lane;
        // the neighbour rows are fetched 8 at a time, summed in entry order
        const int sub = lane >> 3, q = lane & 7;
        for(int base = warp * 4; base < tiles * 16; base += nwarps * 4)
        {
            const int i = base + sub;
            uint4 self = make_uint4(0u, 0u, 0u, 0u), msg = make_uint4(0u, 0u, 0u, 0u);
            if(i < own)
            {
                float a[8] = {};
                const int eb = rp[i], ee = rp[i + 1];
                for(int e = eb; e < ee; e += 8)
                {
                    uint4 v[8];
                    float w[8];
#pragma unroll
                    for(int u = 0; u < 8; u++)
                    {
                        const int2 t = nb[min(e + u, ee - 1)];
                        w[u] = e + u < ee ? __int_as_float(t.y) : 0.f;
                        v[u] = ld_dsmem16(hbase + ((t.x & 0xffff) * NET_H + 8 * q) * 2, t.x >> 16);
                    }
#pragma unroll
                    for(int u = 0; u < 8; u++)
                        if(e + u < ee) fma8(a, w[u], v[u]);
                }
                self = *reinterpret_cast<const uint4*>(Hc + i * NET_H + 8 * q);
                msg = make_uint4(pack_bf16(a[0], a[1]), pack_bf16(a[2], a[3]), pack_bf16(a[4], a[5]), pack_bf16(a[6], a[7]));
            }
            *reinterpret_cast<uint4*>(Xs + i * XS_LD + 8 * q) = self;
            *reinterpret_cast<uint4*>(Xs + i * XS_LD + NET_H + 8 * q) = msg;
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();
        if(warp < tiles)
        {
            float acc[8][4] = {};
            warp_gemm<2 * NET_H, 8>(Xs + warp * 16 * XS_LD, XS_LD, Ws, XS_LD, acc);
            store_relu(acc, params + P_B1 + k * NET_H, Hs + (cur ^ 1) * FU_RPC * NET_H, warp * 16);
        }
        cur ^= 1;
        __syncthreads();  // Ws is free again
        if(k + 1 < NET_LAYERS) stage_weights_async(wbf + P_W1 + (k + 1) * NET_H * 2 * NET_H, Ws);
        // the new rows are visible to the cluster, and nobody reads the old buffer any more
        cluster.sync();
    }

    // ---- P3: head, the step limit theta over the cluster, apply ----
    const float* bo = params + P_BO;
    if(warp < tiles)
    {
        float acc[1][4] = {};
        warp_gemm<NET_H, 1>(Hs + cur * FU_RPC * NET_H + warp * 16 * NET_H, NET_H, wbf + P_WO, NET_H, acc);
        const int gq = lane >> 2, t = lane & 3;
        if(t < 2)
        {
            float* d0 = reinterpret_cast<float*>(dl + warp * 16 + gq);
            float* d1 = reinterpret_cast<float*>(dl + warp * 16 + gq + 8);
            if(t == 0)
            {
                d0[0] = acc[0][0] + bo[0];
                d0[1] = acc[0][1] + bo[1];
                d1[0] = acc[0][2] + bo[0];
                d1[1] = acc[0][3] + bo[1];
            }
            else
            {
                d0[2] = acc[0][0] + bo[2];
                d0[3] = 0.f;
                d1[2] = acc[0][2] + bo[2];
                d1[3] = 0.f;
            }
        }
    }
    __syncthreads();
    double pa = 0, pb = 0;
    for(int i = threadIdx.x; i < own; i += FU_THREADS)
    {
        const float4 r = rz[i], z = rz[FU_RPC + i], d = dl[i];
        pa += (double)r.x * z.x + (double)r.y * z.y + (double)r.z * z.z;
        pb += (double)r.x * d.x + (double)r.y * d.y + (double)r.z * d.z;
    }
    block_sum2_fu(pa, pb, red);
    if(threadIdx.x == 0)
    {
        part[2] = pa;
        part[3] = pb;
    }
    cluster.sync();
    if(warp == 0)
    {
        double a, b;
        cluster_sum2(cluster, part, 2, nranks, a, b);
        if(lane == 0)
        {
            b *= s_z;
            float th = (b < -0.5 * a && b < 0.0) ? (float)(-0.5 * a / b) : 1.f;
            if(!(th >= 0.f)) th = 0.f;
            sc[2] = th;
        }
    }
    // nobody reads another CTA's shared memory after this point
    cluster.sync();
    const float f = sc[2] * s_z;
    for(int i = threadIdx.x; i < own; i += FU_THREADS)
    {
        float4 z = rz[FU_RPC + i];
        const float4 d = dl[i];
        z.x = fmaf(f, d.x, z.x);
        z.y = fmaf(f, d.y, z.y);
        z.z = fmaf(f, d.z, z.z);
        *reinterpret_cast<float4*>(Z + 4 * (size_t)(r0 + i)) = z;
    }
}

}  // namespace

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
namespace
{
constexpr int MP_SMEM = (NET_H + TILE_WARPS * 16) * XS_LD * 2;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct Layout
{
    size_t x0, h, m, delta, scale, ddelta, du, dha, dm, part, loss, wbf, total;
};

Layout layout(int n, int S)
{
    const size_t rows = (size_t)n * S, rp = (rows + 15) / 16 * 16;
    const size_t wgb = std::max<size_t>(1, (rows + WG_ROWS - 1) / WG_ROWS);
    Layout L{};
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t at = o;
        o += align256(bytes);
        return at;
    };
    L.x0 = take(rp * NET_IN * 2);
    L.h = take(4 * rp * NET_H * 2);
    L.m = take(3 * rp * NET_H * 2);
    L.delta = take(rp * 4 * 4);
    L.scale = take((size_t)S * 2 * 4);
    L.ddelta = take(rp * 4 * 4);
    L.du = take(rp * NET_H * 4);
    L.dha = take(rp * NET_H * 4);
    L.dm = take(rp * NET_H * 4);
    L.part = take(wgb * (NET_H * 2 * NET_H + NET_H) * 4);
    L.loss = take((size_t)S * 4);
    L.wbf = take((size_t)P_COUNT * 2);
    L.total = o;
    return L;
}

}  // namespace

int net_prepare()
{
    static thread_local unsigned long long done = 0;
    if(first_on_device(done))
        STG_CUDA_TRY(cudaFuncSetAttribute(k_net_mp, cudaFuncAttributeMaxDynamicSharedMemorySize, MP_SMEM));
    return 0;
}

namespace
{

const __nv_bfloat16* wb(const void* wbf, int off) { return reinterpret_cast<const __nv_bfloat16*>(wbf) + off; }
}  // namespace

size_t net_scratch_bytes(int n, int S) { return layout(n, S).total; }

int net_carve(void* scratch, size_t bytes, int n, int S, NetBuffers& b)
{
    const Layout L = layout(n, S);
    if(!scratch || bytes < L.total || n < 1 || S < 1)
    {
        set_error("learned: scratch block too small or empty graph (need " + std::to_string(L.total) + " bytes)");
        return STG_ERR_INVALID;
    }
    unsigned char* p = static_cast<unsigned char*>(scratch);
    if(reinterpret_cast<uintptr_t>(p) % 256)
    {
        set_error("learned: scratch block must be 256-byte aligned");
        return STG_ERR_INVALID;
    }
    b.S = S;
    b.rows = n * S;
    b.rows_pad = (b.rows + 15) / 16 * 16;
    b.wg_blocks = std::max(1, div_up(b.rows, WG_ROWS));
    const size_t hs = (size_t)b.rows_pad * NET_H * 2;
    b.x0 = p + L.x0;
    for(int i = 0; i < 4; i++) b.h[i] = p + L.h + i * hs;
    for(int i = 0; i < 3; i++) b.m[i] = p + L.m + i * hs;
    b.delta = reinterpret_cast<float*>(p + L.delta);
    b.scale = reinterpret_cast<float*>(p + L.scale);
    b.ddelta = reinterpret_cast<float*>(p + L.ddelta);
    b.du = reinterpret_cast<float*>(p + L.du);
    b.dha = reinterpret_cast<float*>(p + L.dha);
    b.dm = reinterpret_cast<float*>(p + L.dm);
    b.part = reinterpret_cast<float*>(p + L.part);
    b.loss = reinterpret_cast<float*>(p + L.loss);
    b.wbf = p + L.wbf;
    return 0;
}

int net_to_bf16(cudaStream_t s, const float* params, void* wbf)
{
    k_net_bf16<<<div_up(P_COUNT, NT), NT, 0, s>>>(params, reinterpret_cast<__nv_bfloat16*>(wbf), P_COUNT);
    STG_LAUNCH_CHECK();
    return 0;
}

// Cluster size and rows per CTA for the fused forward on a graph with row pointers `row`
// (host copy): the largest cluster (16, else 8) that can be resident, with at most FU_RPC
// rows and FU_EPC neighbour entries per CTA.  cl = 0: use the layered kernels.
int net_fused_plan(const int* row, int n, int* cl, int* rpc)
{
    *cl = 0;
    *rpc = 0;
    STG_CUDA_TRY(cudaFuncSetAttribute(k_net_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, FU_SMEM));
    STG_CUDA_TRY(cudaFuncSetAttribute(k_net_fused, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    for(int c : {16, 8})
    {
        const int r = (div_up(n, c) + 15) / 16 * 16;
        if(r > FU_RPC) continue;
        bool fits = true;
        for(int q = 0; q < c && fits; q++)
        {
            const int a = std::min(q * r, n), b = std::min(a + r, n);
            fits = row[b] - row[a] <= FU_EPC;
        }
        if(!fits) continue;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = c;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(c);
        cfg.blockDim = dim3(FU_THREADS);
        cfg.dynamicSmemBytes = FU_SMEM;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int clusters = 0;
        if(cudaOccupancyMaxActiveClusters(&clusters, k_net_fused, &cfg) != cudaSuccess)
        {
            cudaGetLastError();
            continue;
        }
        if(clusters < 1) continue;
        *cl = c;
        *rpc = r;
        return 0;
    }
    return 0;
}

int net_forward_fused(cudaStream_t s, const NetGraph& g, const int2* nbp, const float* rc, float* Z, const void* wbf,
                      const float* params, const int* flags, int cl, int rpc)
{
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cl);
    cfg.blockDim = dim3(FU_THREADS);
    cfg.dynamicSmemBytes = FU_SMEM;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    STG_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_net_fused, g, nbp, rc, Z, reinterpret_cast<const __nv_bfloat16*>(wbf),
                                    params, flags, rpc));
    return 0;
}

int net_forward(cudaStream_t s, const NetGraph& g, const float* rc, const float* zc, int S, const NetBuffers& b,
                const void* wbf, const float* params, float* apply, const int* flags, int* launches)
{
    STG_TRY(net_prepare());
    const int tiles = b.rows_pad / 16, grid = div_up(tiles, TILE_WARPS);
    auto H = [&](int i) { return reinterpret_cast<__nv_bfloat16*>(b.h[i]); };
    k_net_input<<<S, NT, 0, s>>>(g, rc, zc, S, b.rows_pad, reinterpret_cast<__nv_bfloat16*>(b.x0), b.scale, flags);
    STG_LAUNCH_CHECK();
    k_net_embed<<<grid, NT, 0, s>>>(reinterpret_cast<const __nv_bfloat16*>(b.x0), wb(wbf, P_W0), params + P_B0, H(0),
                                    tiles, flags);
    STG_LAUNCH_CHECK();
    for(int k = 0; k < NET_LAYERS; k++)
    {
        k_net_mp<<<grid, NT, MP_SMEM, s>>>(g, b.rows, H(k), wb(wbf, P_W1 + k * NET_H * 2 * NET_H), params + P_B1 + k * NET_H,
                                           reinterpret_cast<__nv_bfloat16*>(b.m[k]), H(k + 1), tiles, flags);
        STG_LAUNCH_CHECK();
    }
    k_net_head<<<grid, NT, 0, s>>>(H(3), wb(wbf, P_WO), params + P_BO, b.delta, tiles, flags);
    STG_LAUNCH_CHECK();
    *launches += 3 + NET_LAYERS;
    if(apply)
    {
        k_net_apply<<<1, 1024, 0, s>>>(g.n, rc, b.delta, b.scale, apply, flags);
        STG_LAUNCH_CHECK();
        (*launches)++;
    }
    return 0;
}

int net_train_step(cudaStream_t s, const NetGraph& g, const float* rc, const float* zc, int S, const NetBuffers& b,
                   float* params, float* grad, float* adam_m, float* adam_v, int step, float lr, int* launches)
{
    STG_TRY(net_to_bf16(s, params, b.wbf));
    STG_TRY(net_forward(s, g, rc, zc, S, b, b.wbf, params, nullptr, nullptr, launches));
    auto H = [&](int i) { return reinterpret_cast<const __nv_bfloat16*>(b.h[i]); };
    k_net_loss<<<S, NT, 0, s>>>(g, rc, zc, b.delta, b.scale, S, b.ddelta, b.loss);
    STG_LAUNCH_CHECK();
    const int rows = b.rows, wgb = b.wg_blocks;
    // head
    k_net_wgrad<NET_H, NET_OUT><<<wgb, NT, 0, s>>>(H(3), NET_H, NET_H, nullptr, 0, b.ddelta, 4, 3, rows, b.part);
    STG_LAUNCH_CHECK();
    k_net_reduce<<<div_up(NET_OUT * NET_H + NET_OUT, NT), NT, 0, s>>>(b.part, wgb, NET_OUT * NET_H, NET_OUT, grad + P_WO,
                                                                      grad + P_BO);
    STG_LAUNCH_CHECK();
    k_net_head_bwd<<<div_up((long)rows * NET_H, NT), NT, 0, s>>>(b.ddelta, wb(b.wbf, P_WO), H(3), b.du, rows);
    STG_LAUNCH_CHECK();
    *launches += 4;
    for(int k = NET_LAYERS - 1; k >= 0; k--)
    {
        const __nv_bfloat16* Mk = reinterpret_cast<const __nv_bfloat16*>(b.m[k]);
        k_net_wgrad<2 * NET_H, NET_H><<<wgb, NT, 0, s>>>(H(k), NET_H, NET_H, Mk, NET_H, b.du, NET_H, NET_H, rows, b.part);
        STG_LAUNCH_CHECK();
        k_net_reduce<<<div_up(NET_H * 2 * NET_H + NET_H, NT), NT, 0, s>>>(
            b.part, wgb, NET_H * 2 * NET_H, NET_H, grad + P_W1 + k * NET_H * 2 * NET_H, grad + P_B1 + k * NET_H);
        STG_LAUNCH_CHECK();
        k_net_dx<<<div_up(rows, 32), NT, 0, s>>>(b.du, wb(b.wbf, P_W1 + k * NET_H * 2 * NET_H), b.dha, b.dm, rows);
        STG_LAUNCH_CHECK();
        k_net_agg_mask<<<div_up(rows, NT / 32), NT, 0, s>>>(g, rows, b.dha, b.dm, H(k), b.du);
        STG_LAUNCH_CHECK();
        *launches += 4;
    }
    k_net_wgrad<NET_IN, NET_H><<<wgb, NT, 0, s>>>(reinterpret_cast<const __nv_bfloat16*>(b.x0), NET_IN, NET_IN, nullptr, 0,
                                                   b.du, NET_H, NET_H, rows, b.part);
    STG_LAUNCH_CHECK();
    k_net_reduce<<<div_up(NET_H * NET_IN + NET_H, NT), NT, 0, s>>>(b.part, wgb, NET_H * NET_IN, NET_H, grad + P_W0,
                                                                   grad + P_B0);
    STG_LAUNCH_CHECK();
    *launches += 3;
    if(lr > 0.f)
    {
        const float c1 = 1.f - powf(0.9f, (float)step), c2 = 1.f - powf(0.999f, (float)step);
        k_net_adam<<<div_up(P_COUNT, NT), NT, 0, s>>>(params, grad, adam_m, adam_v, P_COUNT, lr, c1, c2);
        STG_LAUNCH_CHECK();
        (*launches)++;
    }
    return 0;
}

}  // namespace stg
