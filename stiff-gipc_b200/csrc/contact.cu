// contact.cu -- barrier gradient and Hessian of the contact pairs on sm_100a.
//
// Replaces _calBarrierGradientAndHessian (StiffGIPC/GIPC.cu:3149-4988) as the reference
// builds it (NEWF and RANK 2, GIPC.cu:29-30) for the four unmollified pair types of the
// sign-encoded int4 (GIPC.cuh:49-66):
//   edge-edge       x >= 0, w >= 0            edges (x, y) and (z, w)
//   point-point     x < 0, z < 0, y >= 0      point -x-1 and y
//   point-edge      x < 0, z >= 0, w < 0, y >= 0   point -x-1, edge (y, z)
//   point-triangle  x < 0, z >= 0, w >= 0     point -x-1, triangle (y, z, w)
// With d the pair's distance (the squared-distance formulas of _d_PP / _d_PE / _d_PT / _d_EE,
// mlbvh.cu:229-257), dHat the squared activation distance and s = d / sqrt(dHat), the
// barrier energy is kappa dHat^2 (s^2 - 1)^2 ln^2(s^2) for s < 1.  The gradient is E'(s) ds/dx
// and the Hessian the rank-one E''(s) ds/dx ds/dx^T (GIPC.cu:3187-3403: PFPx's last column is
// ds/dx), with E''(s) evaluated at s^2 = 1e-6 below that (the reference's gassThreshold,
// GIPC.cu:3171); E'' >= 0 on s < 1, so the Hessian is positive semi-definite as it stands.
// ds/dx is the forward-mode derivative of the distance formula.  The mollified near-parallel
// edge-edge encodings (x >= 0 with w < 0; x < 0 with y < 0 and z < 0 or w < 0) are not
// produced here: such a pair gets zero blocks and counts in *skipped.
//
// Output per pair, in fixed slots (no atomics): 10 upper 3x3 blocks (column-major) for the
// local vertex pairs (i <= j) of up to four vertices (unused slots: a zero block on the first
// vertex's diagonal) and 12 gradient entries (3 per local vertex).
#include "solver.hpp"

namespace stg
{

// a value with its derivatives with respect to the 12 coordinates of the pair
struct Dual12
{
    double v;
    double g[12];
};

__device__ __forceinline__ Dual12 dconst(double v)
{
    Dual12 r;
    r.v = v;
#pragma unroll
    for(int k = 0; k < 12; k++) r.g[k] = 0.0;
    return r;
}
__device__ __forceinline__ Dual12 dvar(double v, int k)
{
    Dual12 r = dconst(v);
    r.g[k] = 1.0;
    return r;
}
__device__ __forceinline__ Dual12 operator+(const Dual12& a, const Dual12& b)
{
    Dual12 r;
    r.v = a.v + b.v;
#pragma unroll
    for(int k = 0; k < 12; k++) r.g[k] = a.g[k] + b.g[k];
    return r;
}
__device__ __forceinline__ Dual12 operator-(const Dual12& a, const Dual12& b)
{
    Dual12 r;
    r.v = a.v - b.v;
#pragma unroll
    for(int k = 0; k < 12; k++) r.g[k] = a.g[k] - b.g[k];
    return r;
}
__device__ __forceinline__ Dual12 operator*(const Dual12& a, const Dual12& b)
{
    Dual12 r;
    r.v = a.v * b.v;
#pragma unroll
    for(int k = 0; k < 12; k++) r.g[k] = a.g[k] * b.v + a.v * b.g[k];
    return r;
}
__device__ __forceinline__ Dual12 operator/(const Dual12& a, const Dual12& b)
{
    Dual12 r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for(int k = 0; k < 12; k++) r.g[k] = (a.g[k] - r.v * b.g[k]) * ib;
    return r;
}
__device__ __forceinline__ Dual12 dsqrt(const Dual12& a)
{
    Dual12 r;
    r.v = sqrt(a.v);
    const double h = r.v > 0.0 ? 0.5 / r.v : 0.0;
#pragma unroll
    for(int k = 0; k < 12; k++) r.g[k] = a.g[k] * h;
    return r;
}

struct DVec
{
    Dual12 x, y, z;
};
__device__ __forceinline__ DVec dsub(const DVec& a, const DVec& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ Dual12 ddot(const DVec& a, const DVec& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ DVec dcross(const DVec& a, const DVec& b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// squared distance of the pair's type (_d_PP / _d_PE / _d_PT / _d_EE, mlbvh.cu:229-257)
__device__ Dual12 squared_distance(int type, const DVec* v)
{
    if(type == 0) return ddot(dsub(v[0], v[1]), dsub(v[0], v[1]));
    if(type == 1)
    {
        const DVec c = dcross(dsub(v[1], v[0]), dsub(v[2], v[0]));
        const DVec e = dsub(v[2], v[1]);
        return ddot(c, c) / ddot(e, e);
    }
    if(type == 2)
    {
        const DVec b = dcross(dsub(v[2], v[1]), dsub(v[3], v[1]));
        const Dual12 a = ddot(dsub(v[0], v[1]), b);
        return a * a / ddot(b, b);
    }
    const DVec b = dcross(dsub(v[1], v[0]), dsub(v[3], v[2]));
    const Dual12 a = ddot(dsub(v[2], v[0]), b);
    return a * a / ddot(b, b);
}

// E'(s) and E''(s) of kappa dHat^2 (s^2 - 1)^2 ln^2(s^2) (RANK 2, GIPC.cu:3226-3230, 3285-3303)
__device__ __forceinline__ void barrier_derivs(double s, double dhat, double kappa, double& e1, double& e2)
{
    const double I = s * s, lI = log(I);
    e1 = s * 2.0 * (2.0 * kappa * dhat * dhat * lI * (I - 1.0) * (I + I * lI - 1.0)) / I;
    const double Ic = I < 1e-6 ? 1e-6 : I, l = log(Ic);
    e2 = -(4.0 * kappa * dhat * dhat *
           (4.0 * Ic + l - 3.0 * Ic * Ic * l * l + 6.0 * Ic * l - 2.0 * Ic * Ic + Ic * l * l - 7.0 * Ic * Ic * l - 2.0)) /
         Ic;
}

__global__ void k_contact_barrier(int ncp, const int4* __restrict__ pairs, const double* __restrict__ x, int nv,
                                  int block_offset, double dhat, double kappa, int* rows, int* cols, double* blocks,
                                  double* grad, int* skipped)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= ncp) return;
    const int4 q = pairs[p];
    int vid[4] = {0, 0, 0, 0}, cnt = 0, type = -1;
    if(q.x >= 0)
    {
        if(q.w >= 0)
        {
            type = 3;
            vid[0] = q.x, vid[1] = q.y, vid[2] = q.z, vid[3] = q.w, cnt = 4;
        }
    }
    else if(q.y >= 0)
    {
        const int v0 = -q.x - 1;
        if(q.z < 0)
            type = 0, vid[0] = v0, vid[1] = q.y, cnt = 2;
        else if(q.w < 0)
            type = 1, vid[0] = v0, vid[1] = q.y, vid[2] = q.z, cnt = 3;
        else
            type = 2, vid[0] = v0, vid[1] = q.y, vid[2] = q.z, vid[3] = q.w, cnt = 4;
    }
    bool ok = type >= 0;
    for(int i = 0; i < cnt; i++) ok = ok && vid[i] >= 0 && vid[i] < nv;
    for(int i = 0; i < cnt; i++)
        for(int j = i + 1; j < cnt; j++) ok = ok && vid[i] != vid[j];
    double h[12] = {0.0}, lam = 0.0, e1 = 0.0;
    if(ok)
    {
        DVec v[4];
        for(int i = 0; i < 4; i++)
        {
            const int g = vid[i < cnt ? i : 0];
            v[i] = {dvar(x[3 * (size_t)g], 3 * i), dvar(x[3 * (size_t)g + 1], 3 * i + 1), dvar(x[3 * (size_t)g + 2], 3 * i + 2)};
            if(i >= cnt) v[i] = {dconst(0.0), dconst(0.0), dconst(0.0)};
        }
        const Dual12 d = dsqrt(squared_distance(type, v));
        const double rs = 1.0 / sqrt(dhat);
        const double s = d.v * rs;
        if(s < 1.0 && s > 0.0)
        {
            barrier_derivs(s, dhat, kappa, e1, lam);
#pragma unroll
            for(int k = 0; k < 12; k++) h[k] = d.g[k] * rs;  // ds/dx
        }
    }
    else if(skipped)
        atomicAdd(skipped, 1);
    // gradient, 3 per local vertex
    for(int k = 0; k < 12; k++) grad[12 * (size_t)p + k] = e1 * h[k];
    // the 10 upper blocks (i <= j) of lam h h^T, oriented upper in the global numbering
    int slot = 0;
    for(int i = 0; i < 4; i++)
        for(int j = i; j < 4; j++, slot++)
        {
            const size_t o = 10 * (size_t)p + slot;
            double* B = blocks + 9 * o;
            if(!ok || i >= cnt || j >= cnt)
            {
                rows[o] = block_offset + (ok ? vid[0] : 0);
                cols[o] = rows[o];
                for(int e = 0; e < 9; e++) B[e] = 0.0;
                continue;
            }
            const int gi = vid[i], gj = vid[j];
            const bool sw = gi > gj;
            rows[o] = block_offset + (sw ? gj : gi);
            cols[o] = block_offset + (sw ? gi : gj);
            // block (i, j) of lam h h^T: element (a, b) = lam h[3i + a] h[3j + b]; the transposed
            // block when the global order swaps (the matrix is symmetric)
            for(int a = 0; a < 3; a++)
                for(int b = 0; b < 3; b++)
                {
                    const double val = lam * h[3 * i + a] * h[3 * j + b];
                    if(sw)
                        B[a * 3 + b] = val;  // element (b, a) of the stored block, column-major
                    else
                        B[b * 3 + a] = val;  // element (a, b), column-major
                }
        }
}

// per-pair barrier energy kappa dHat^2 (s^2 - 1)^2 ln^2(s^2) for s < 1 (the reference's
// barrier at RANK 2, GIPC.cu:3226-3230 integrated); unsupported or invalid pairs give 0
__global__ void k_contact_energy(int ncp, const int4* __restrict__ pairs, const double* __restrict__ x, int nv,
                                 double dhat, double kappa, double* energy)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= ncp) return;
    const int4 q = pairs[p];
    int vid[4] = {0, 0, 0, 0}, cnt = 0, type = -1;
    if(q.x >= 0)
    {
        if(q.w >= 0) type = 3, vid[0] = q.x, vid[1] = q.y, vid[2] = q.z, vid[3] = q.w, cnt = 4;
    }
    else if(q.y >= 0)
    {
        vid[0] = -q.x - 1, vid[1] = q.y;
        if(q.z < 0)
            type = 0, cnt = 2;
        else if(q.w < 0)
            type = 1, vid[2] = q.z, cnt = 3;
        else
            type = 2, vid[2] = q.z, vid[3] = q.w, cnt = 4;
    }
    bool ok = type >= 0;
    for(int i = 0; i < cnt; i++) ok = ok && vid[i] >= 0 && vid[i] < nv;
    for(int i = 0; i < cnt; i++)
        for(int j = i + 1; j < cnt; j++) ok = ok && vid[i] != vid[j];
    double e = 0.0;
    if(ok)
    {
        DVec v[4];
        for(int i = 0; i < 4; i++)
        {
            const int g = vid[i < cnt ? i : 0];
            v[i] = {dconst(x[3 * (size_t)g]), dconst(x[3 * (size_t)g + 1]), dconst(x[3 * (size_t)g + 2])};
        }
        const double I = squared_distance(type, v).v / dhat;
        if(I < 1.0)
        {
            const double l = log(I);
            e = kappa * dhat * dhat * (I - 1.0) * (I - 1.0) * l * l;
        }
    }
    energy[p] = e;
}

}  // namespace stg

extern "C" int stg_contact_energy(int ncp, const int32_t* pairs, const double* x, int num_verts, double dhat,
                                  double kappa, double* energy, void* stream)
{
    if(ncp < 0 || num_verts < 0 || !(dhat > 0.0) || !(kappa >= 0.0) || (ncp > 0 && (!pairs || !x || !energy)))
    {
        stg::set_error("stg_contact_energy: invalid arguments");
        return STG_ERR_INVALID;
    }
    if(ncp == 0) return STG_OK;
    stg::k_contact_energy<<<(ncp + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        ncp, reinterpret_cast<const int4*>(pairs), x, num_verts, dhat, kappa, energy);
    STG_CUDA_TRY(cudaGetLastError());
    return STG_OK;
}

extern "C" int stg_contact_barrier(int ncp, const int32_t* pairs, const double* x, int num_verts, int block_offset,
                                   double dhat, double kappa, int32_t* rows, int32_t* cols, double* blocks,
                                   double* grad, int* skipped, void* stream)
{
    if(ncp < 0 || num_verts < 0 || block_offset < 0 || !(dhat > 0.0) || !(kappa >= 0.0) ||
       (ncp > 0 && (!pairs || !x || !rows || !cols || !blocks || !grad)))
    {
        stg::set_error("stg_contact_barrier: invalid arguments");
        return STG_ERR_INVALID;
    }
    if(ncp == 0) return STG_OK;
    stg::k_contact_barrier<<<(ncp + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        ncp, reinterpret_cast<const int4*>(pairs), x, num_verts, block_offset, dhat, kappa, rows, cols, blocks, grad,
        skipped);
    STG_CUDA_TRY(cudaGetLastError());
    return STG_OK;
}
