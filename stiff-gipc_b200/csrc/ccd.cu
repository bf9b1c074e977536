// ccd.cu -- the line search's step bound from continuous collision detection on the GPU.
//
// Replaces GIPC::self_largestFeasibleStepSize + _reduct_min_selfTimeStep_to_double
// (StiffGIPC/GIPC.cu:7095-7180, 9010-9047) with the reference's additive CCD per pair
// (point_triangle_ccd / edge_edge_ccd and their distance classification, ACCD.cu:15-534):
// each pair advances conservatively along its displacement (relative to the pair's mean
// displacement) by (1 - eta) d^2 / ((d + thickness) max|dx|) until the distance has shrunk
// by the factor eta, or the step reaches 1; the bound is alpha = 1 / max over pairs of 1 / toc.
// One thread per pair, 50,000 advancement steps at most (the reference's cap).  The largest
// 1 / toc is taken with an integer atomicMax on its bit pattern (every value is >= 1, and
// positive doubles order like their bits), so the result does not depend on launch order.
// This file is compiled without FMA contraction (build.py): with the operand order of the
// reference's vector helpers kept, every toc equals the oracle's bit for bit.
#include "solver.hpp"

namespace stg
{
namespace
{
struct V3
{
    double x, y, z;
};
__device__ inline V3 v3(double x, double y, double z) { return {x, y, z}; }
__device__ inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ inline V3 vmul(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ inline double vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ inline double vsq(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
__device__ inline V3 vcross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }

// det of the matrix with columns (a, b, c), as a sum of six triple products (row-major
// m[r][k] = column k's component r: m00 m11 m22 + m10 m21 m02 + m20 m01 m12 - m20 m11 m02 -
// m00 m12 m21 - m01 m10 m22, each product evaluated left to right)
__device__ inline double det_cols(V3 a, V3 b, V3 c)
{
    return a.x * b.y * c.z + a.y * b.z * c.x + a.z * b.x * c.y - a.z * b.y * c.x - a.x * c.y * b.z - b.x * a.y * c.z;
}

// parameters of p against edge (a, b) of a triangle with normal n: (along, outward)
__device__ inline void edge_param(V3 p, V3 a, V3 b, V3 n, double& px, double& py)
{
    const V3 b0 = vsub(b, a), b1 = vcross(b0, n), b2 = vsub(p, a);
    const double D = det_cols(b0, b1, n);
    px = det_cols(b2, b1, n) / D;
    py = det_cols(b0, b2, n) / D;
}

// closest feature of triangle (t0, t1, t2) to p: 0..2 vertex, 3..5 edge, 6 interior
__device__ int pt_type(V3 p, V3 t0, V3 t1, V3 t2)
{
    const V3 n = vcross(vsub(t1, t0), vsub(t2, t0));
    double x0, y0, x1, y1, x2, y2;
    edge_param(p, t0, t1, n, x0, y0);
    if(x0 > 0 && x0 < 1 && y0 >= 0) return 3;
    edge_param(p, t1, t2, n, x1, y1);
    if(x1 > 0.0 && x1 < 1.0 && y1 >= 0.0) return 4;
    edge_param(p, t2, t0, n, x2, y2);
    if(x2 > 0.0 && x2 < 1.0 && y2 >= 0.0) return 5;
    if(x0 <= 0.0 && x2 >= 1.0) return 0;
    if(x1 <= 0.0 && x0 >= 1.0) return 1;
    if(x2 <= 0.0 && x1 >= 1.0) return 2;
    return 6;
}

// closest features of edges (v0 v1), (v2 v3): 0..8 as in the reference's _dType_edge_edge
__device__ int ee_type(V3 v0, V3 v1, V3 v2, V3 v3)
{
    const V3 u = vsub(v1, v0), v = vsub(v3, v2), w = vsub(v0, v2);
    const double a = vsq(u), b = vdot(u, v), c = vsq(v), d = vdot(u, w), e = vdot(v, w);
    const double D = a * c - b * b;
    double tD = D, tN;
    int dflt = 8;
    const double sN = (b * e - c * d);
    if(sN <= 0.0)
        tN = e, tD = c, dflt = 2;
    else if(sN >= D)
        tN = e + b, tD = c, dflt = 5;
    else
    {
        tN = (a * e - b * d);
        if(tN > 0.0 && tN < tD && (vdot(w, vcross(u, v)) == 0.0 || vsq(vcross(u, v)) < 1.0e-20 * a * c))
        {
            if(sN < D / 2)
                tN = e, tD = c, dflt = 2;
            else
                tN = e + b, tD = c, dflt = 5;
        }
    }
    if(tN <= 0.0) return -d <= 0.0 ? 0 : (-d >= a ? 3 : 6);
    if(tN >= tD) return (-d + b) <= 0.0 ? 1 : ((-d + b) >= a ? 4 : 7);
    return dflt;
}

__device__ inline double d2_pp(V3 a, V3 b) { return vsq(vsub(a, b)); }
__device__ inline double d2_pe(V3 p, V3 e0, V3 e1) { return vsq(vcross(vsub(e0, p), vsub(e1, p))) / vsq(vsub(e1, e0)); }
__device__ inline double d2_pt(V3 p, V3 t0, V3 t1, V3 t2)
{
    const V3 b = vcross(vsub(t1, t0), vsub(t2, t0));
    const double aTb = vdot(vsub(p, t0), b);
    return aTb * aTb / vsq(b);
}
__device__ inline double d2_ee(V3 a0, V3 a1, V3 b0, V3 b1)
{
    const V3 b = vcross(vsub(a1, a0), vsub(b1, b0));
    const double aTb = vdot(vsub(b0, a0), b);
    return aTb * aTb / vsq(b);
}

__device__ double ee_dist2(V3 a0, V3 a1, V3 b0, V3 b1)
{
    switch(ee_type(a0, a1, b0, b1))
    {
        case 0: return d2_pp(a0, b0);
        case 1: return d2_pp(a0, b1);
        case 2: return d2_pe(a0, b0, b1);
        case 3: return d2_pp(a1, b0);
        case 4: return d2_pp(a1, b1);
        case 5: return d2_pe(a1, b0, b1);
        case 6: return d2_pe(b0, a0, a1);
        case 7: return d2_pe(b1, a0, a1);
        default: return d2_ee(a0, a1, b0, b1);
    }
}

__device__ double pt_dist2(V3 p, V3 t0, V3 t1, V3 t2)
{
    switch(pt_type(p, t0, t1, t2))
    {
        case 0: return d2_pp(p, t0);
        case 1: return d2_pp(p, t1);
        case 2: return d2_pp(p, t2);
        case 3: return d2_pe(p, t0, t1);
        case 4: return d2_pe(p, t1, t2);
        case 5: return d2_pe(p, t2, t0);
        default: return d2_pt(p, t0, t1, t2);
    }
}

__device__ inline double ee_floor(V3 a0, V3 a1, V3 b0, V3 b1)
{
    const double s0 = vsq(vsub(a0, b0)), s1 = vsq(vsub(a0, b1)), s2 = vsq(vsub(a1, b0)), s3 = vsq(vsub(a1, b1));
    return fmin(fmin(s0, s1), fmin(s2, s3));
}

// time of impact along d: type 0 point-triangle (v = p, t0, t1, t2), 1 edge-edge
__device__ double accd(int type, V3* v, V3* d, double eta, double thickness)
{
    const double th2 = thickness * thickness;
    V3 mov;
    double mdm;
    if(type == 1)
    {
        mov = vmul(vadd(vadd(d[0], d[1]), vadd(d[2], d[3])), -0.25);
        for(int i = 0; i < 4; i++) d[i] = vadd(d[i], mov);
        mdm = sqrt(fmax(vsq(d[0]), vsq(d[1]))) + sqrt(fmax(vsq(d[2]), vsq(d[3])));
    }
    else
    {
        mov = vmul(vadd(vadd(d[1], d[2]), vadd(d[3], d[0])), -0.25);
        for(int i = 0; i < 4; i++) d[i] = vadd(d[i], mov);
        mdm = sqrt(vsq(d[0])) + sqrt(fmax(vsq(d[1]), fmax(vsq(d[2]), vsq(d[3]))));
    }
    if(mdm == 0) return 1.0;
    double dist2, dF;
    if(type == 1)
    {
        dist2 = ee_dist2(v[0], v[1], v[2], v[3]);
        dF = dist2 - th2;
        if(dF <= 0) dist2 = ee_floor(v[0], v[1], v[2], v[3]), dF = dist2 - th2;
    }
    else
        dist2 = pt_dist2(v[0], v[1], v[2], v[3]), dF = dist2 - th2;
    double dist = sqrt(dist2);
    const double gap = eta * dF / (dist + thickness);
    double toc = 0.0;
    for(int count = 1;; count++)
    {
        if(count > 50000) return toc;
        const double lb = (1 - eta) * dF / ((dist + thickness) * mdm);
        for(int i = 0; i < 4; i++) v[i] = vadd(v[i], vmul(d[i], lb));
        if(type == 1)
        {
            dist2 = ee_dist2(v[0], v[1], v[2], v[3]);
            dF = dist2 - th2;
            if(dF <= 0) dist2 = ee_floor(v[0], v[1], v[2], v[3]), dF = dist2 - th2;
        }
        else
            dist2 = pt_dist2(v[0], v[1], v[2], v[3]), dF = dist2 - th2;
        dist = sqrt(dist2);
        if(toc != 0.0 && (dF / (dist + thickness) < gap)) break;
        toc += lb;
        if(toc > 1.0) return 1.0;
    }
    return toc;
}

__global__ void k_ccd_init(unsigned long long* mx)
{
    if(threadIdx.x == 0 && blockIdx.x == 0) *mx = __double_as_longlong(1.0);
}

__global__ void k_ccd_pairs(int np, const int4* __restrict__ pairs, const double* __restrict__ x,
                            const double* __restrict__ dx, int nv, double eta, double thickness,
                            unsigned long long* mx, double* toc_out, int* bad)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= np) return;
    const int4 q = pairs[p];
    const int id[4] = {q.x < 0 ? -q.x - 1 : q.x, q.y, q.z, q.w};
    bool ok = true;
    for(int i = 0; i < 4; i++) ok = ok && id[i] >= 0 && id[i] < nv;
    double toc = 1.0;
    if(ok)
    {
        V3 v[4], d[4];
        for(int i = 0; i < 4; i++)
        {
            const size_t o = 3 * (size_t)id[i];
            v[i] = v3(x[o], x[o + 1], x[o + 2]);
            d[i] = v3(dx[o], dx[o + 1], dx[o + 2]);
        }
        toc = accd(q.x < 0 ? 0 : 1, v, d, eta, thickness);
        atomicMax(mx, (unsigned long long)__double_as_longlong(1.0 / toc));
    }
    else if(bad)
        atomicAdd(bad, 1);
    if(toc_out) toc_out[p] = toc;
}

__global__ void k_ccd_final(const unsigned long long* mx, double* alpha)
{
    if(threadIdx.x == 0 && blockIdx.x == 0) *alpha = 1.0 / __longlong_as_double((long long)*mx);
}
}  // namespace
}  // namespace stg

extern "C" int stg_ccd_step_size(int npairs, const int32_t* pairs, const double* x, const double* dx, int num_verts,
                                 double slackness, double thickness, double* alpha, double* toc, int* bad,
                                 unsigned long long* scratch, void* stream)
{
    if(npairs < 0 || num_verts < 0 || !alpha || !scratch || !(slackness > 0.0 && slackness < 1.0) ||
       !(thickness >= 0.0) || (npairs > 0 && (!pairs || !x || !dx)))
    {
        stg::set_error("stg_ccd_step_size: invalid arguments");
        return STG_ERR_INVALID;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    stg::k_ccd_init<<<1, 32, 0, s>>>(scratch);
    if(npairs > 0)
        stg::k_ccd_pairs<<<(npairs + 127) / 128, 128, 0, s>>>(npairs, reinterpret_cast<const int4*>(pairs), x, dx,
                                                             num_verts, 1.0 - slackness, thickness, scratch, toc, bad);
    stg::k_ccd_final<<<1, 32, 0, s>>>(scratch, alpha);
    STG_CUDA_TRY(cudaGetLastError());
    return STG_OK;
}
