// contact_ref.cu -- the reference's contact-distance derivatives, compiled from its sources.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref/libstg_contact_ref.so, `make -C oracle ref`; loaded by
// tests/test_contact_cpu.py).  The reference's contact Hessian (GIPC.cu:3149-4988, built with
// NEWF and RANK 2) is lambda0(I5) g g^T with g one column of the MATLAB-generated derivative
// pFpx_*2 (StiffGIPC/GIPC_PDerivative.cuh), the derivative of the scaled distance d / d_hat.
// This file includes that header where it lies and exposes those columns to the checker.  The
// header reaches Eigen only through gpu_eigen_libs.cuh for four result layouts; the layouts are
// declared here instead (row-major arrays, as the generated code indexes them).
#define _GPU_EIGEN_LIB_CUH_
#include <cuda_runtime.h>
namespace __GEIGEN__
{
struct Matrix12x9d
{
    double m[12][9];
};
struct Matrix12x4d
{
    double m[12][4];
};
struct Matrix9x4d
{
    double m[9][4];
};
struct Vector6
{
    double v[6];
};
}  // namespace __GEIGEN__
#include "GIPC_PDerivative.cuh"

// g = d(d / d_hat) / dx of one contact: type 0 point-point (2 vertices), 1 point-edge (3),
// 2 point-triangle (4), 3 edge-edge (4); x: the vertices' coordinates; g: 3 per vertex
extern "C" int orc_contact_ref_grad(int type, const double* x, double d_hat, double* g)
{
    if(type == 0)
    {
        __GEIGEN__::Vector6 r;
        pFpx_pp2(make_double3(x[0], x[1], x[2]), make_double3(x[3], x[4], x[5]), d_hat, r);
        for(int i = 0; i < 6; i++) g[i] = r.v[i];
        return 6;
    }
    if(type == 1)
    {
        __GEIGEN__::Matrix9x4d r;
        pFpx_pe2(make_double3(x[0], x[1], x[2]), make_double3(x[3], x[4], x[5]), make_double3(x[6], x[7], x[8]),
                 d_hat, r);
        for(int i = 0; i < 9; i++) g[i] = r.m[i][3];
        return 9;
    }
    __GEIGEN__::Matrix12x9d r;
    const double3 a = make_double3(x[0], x[1], x[2]), b = make_double3(x[3], x[4], x[5]);
    const double3 c = make_double3(x[6], x[7], x[8]), d = make_double3(x[9], x[10], x[11]);
    if(type == 2)
        pFpx_pt2(a, b, c, d, d_hat, r);
    else if(type == 3)
        pFpx_ee2(a, b, c, d, d_hat, r);
    else
        return -1;
    for(int i = 0; i < 12; i++) g[i] = r.m[i][8];
    return 12;
}
