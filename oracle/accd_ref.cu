// accd_ref.cu -- the reference's additive CCD, compiled from its source for the host.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref/libstg_accd_ref.so, `make -C oracle ref`; loaded by
// tests/test_ccd_cpu.py to pin orc_accd in stg_oracle.c).  StiffGIPC/ACCD.cu is included
// where it lies with its device functions made host-callable.  Its vector helpers come from
// gpu_eigen_libs.cuh, which needs Eigen (absent here); the handful ACCD.cu calls are declared
// below with the arithmetic of their definitions in gpu_eigen_libs.cu (component-wise
// operations, dot and squared norm summed x, y, z, the 3x3 determinant as six triple
// products).  Build with FMA contraction off so that the host arithmetic is the IEEE
// sequence the oracle restates.  Device qualifiers are dropped: the functions compile as host code.
#define _GPU_EIGEN_LIB_CUH_
#include <cuda_runtime.h>
#include <cmath>
#include <algorithm>
#undef __device__
#define __device__

namespace __GEIGEN__
{
struct Matrix3x3d
{
    double m[3][3];
};
inline __host__ __device__ double3 __minus(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline __host__ __device__ double3 __add(double3 a, double3 b) { return make_double3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline __host__ __device__ double3 __s_vec_multiply(const double3& a, double b) { return make_double3(a.x * b, a.y * b, a.z * b); }
inline __host__ __device__ double __squaredNorm(double3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline __host__ __device__ double __norm(const double3& n) { return sqrt(n.x * n.x + n.y * n.y + n.z * n.z); }
inline __host__ __device__ double __v_vec_dot(const double3& a, const double3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline __host__ __device__ double3 __v_vec_cross(double3 a, double3 b)
{
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline __host__ __device__ void __set_Mat_val(Matrix3x3d& M, const double& a00, const double& a01, const double& a02,
                                              const double& a10, const double& a11, const double& a12,
                                              const double& a20, const double& a21, const double& a22)
{
    M.m[0][0] = a00, M.m[0][1] = a01, M.m[0][2] = a02;
    M.m[1][0] = a10, M.m[1][1] = a11, M.m[1][2] = a12;
    M.m[2][0] = a20, M.m[2][1] = a21, M.m[2][2] = a22;
}
inline __host__ __device__ double __Determiant(const Matrix3x3d& a)
{
    return a.m[0][0] * a.m[1][1] * a.m[2][2] + a.m[1][0] * a.m[2][1] * a.m[0][2] + a.m[2][0] * a.m[0][1] * a.m[1][2] -
           a.m[2][0] * a.m[1][1] * a.m[0][2] - a.m[0][0] * a.m[1][2] * a.m[2][1] - a.m[0][1] * a.m[1][0] * a.m[2][2];
}
// the cubic root finder of ACCD.cu's vertex-face intersection test (doCCDVF / IntersectVF),
// which the step bound does not use (its call is commented out, GIPC.cu:7130-7138): no roots
inline void __NewtonSolverForCubicEquation(const double&, const double&, const double&, const double&, double*,
                                           int& num_solutions, double = 1e-6)
{
    num_solutions = 0;
}
}  // namespace __GEIGEN__

#include "ACCD.cu"

// time of impact: type 0 point-triangle (p, t0, t1, t2), 1 edge-edge (a0, a1, b0, b1)
extern "C" double orc_accd_ref(int type, const double* x, const double* dx, double eta, double thickness)
{
    double3 v[4], d[4];
    for(int i = 0; i < 4; i++)
        v[i] = make_double3(x[3 * i], x[3 * i + 1], x[3 * i + 2]), d[i] = make_double3(dx[3 * i], dx[3 * i + 1], dx[3 * i + 2]);
    if(type == 0) return point_triangle_ccd(v[0], v[1], v[2], v[3], d[0], d[1], d[2], d[3], eta, thickness);
    return edge_edge_ccd(v[0], v[1], v[2], v[3], d[0], d[1], d[2], d[3], eta, thickness);
}
