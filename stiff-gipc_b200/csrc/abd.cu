// abd.cu -- the affine-body (ABD) part of the Newton system on the GPU.
//
// An affine body carries q = (t, a1, a2, a3) (12 DOF; a_i are the rows of A, x = A xbar + t,
// abd_jacobi_matrix.inl) and owns block rows 4 b .. 4 b + 3 of the global system (4 x 4 tiles
// of 3x3 blocks).  This file builds:
//  - per body, the 12x12 Hessian and gradient of inertia + orthogonality potential
//    (ABDSystem::_cal_abd_body_gradient_and_hessian, setup_abd_system_gradient_and_hessian.cu:
//    200-262, and write_abd_body_hessian, :129-139): H = M + kappa v dt^2 PSD(d2S/da2) on the
//    a-block, g = M (q - q_tilde) + kappa v dt^2 dS/da, with M the dyadic mass
//    (ABDJacobiDyadicMass::to_mat) and S = sum (a_i.a_i - 1)^2 + sum_{i != j} (a_i.a_j)^2
//    (abd_energy.inl:9-140);
//  - the mapping of point-level 3x3 contact blocks onto body DOFs: J_i^T B J_j for two body
//    points (write_barrier_hessian / JT_H_J, setup_abd_system_gradient_and_hessian.cu:89-126,
//    abd_jacobi_matrix.inl:34-72), J_i^T B for a body point and a FEM vertex (:510-551), and
//    the FEM-FEM blocks shifted past the body rows (GIPC.cu:10328-10362);
//  - body-point positions x = J(xbar) q and the body gradient sum_i J_i^T g_i
//    (_cal_abd_system_barrier_gradient, :362-396);
//  - the block-Jacobi inverses of the bodies' diagonal tiles from the converted BCOO
//    (ABDSystem::_cal_abd_system_preconditioner, :612-655).
// All outputs go to fixed slots (no atomics, no data-dependent order).
#include "eig9.cuh"
#include "solver.hpp"

namespace stg
{
namespace
{
constexpr int AT = 128;

// the dyadic mass of one body: m, m xbar (3), m xbar xbar^T (9, row-major)
struct DyMass
{
    double m, mx[3], D[9];
};

__device__ inline void load_mass(const double* p, DyMass& M)
{
    M.m = p[0];
    for(int k = 0; k < 3; k++) M.mx[k] = p[1 + k];
    for(int k = 0; k < 9; k++) M.D[k] = p[4 + k];
}

// entry (r, c) of the 12x12 dyadic mass matrix (ABDJacobiDyadicMass::add_to)
__device__ inline double mass_entry(const DyMass& M, int r, int c)
{
    if(r < 3 && c < 3) return r == c ? M.m : 0.0;
    if(r < 3) return (c - 3) / 3 == r ? M.mx[(c - 3) % 3] : 0.0;
    if(c < 3) return (r - 3) / 3 == c ? M.mx[(r - 3) % 3] : 0.0;
    return (r - 3) / 3 == (c - 3) / 3 ? M.D[3 * ((r - 3) % 3) + (c - 3) % 3] : 0.0;
}

__global__ void k_abd_body(int N, const double* __restrict__ q, const double* __restrict__ qt,
                           const double* __restrict__ mass, const double* __restrict__ vol,
                           const int* __restrict__ fixed, double kappa, double dt, int* rows, int* cols,
                           double* blocks, double* grad)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if(b >= N) return;
    DyMass M;
    load_mass(mass + 13 * (size_t)b, M);
    double Q[12], dq[12];
    for(int k = 0; k < 12; k++) Q[k] = q[12 * (size_t)b + k], dq[k] = Q[k] - qt[12 * (size_t)b + k];
    const bool fx = fixed && fixed[b];
    double g[12];
    for(int r = 0; r < 12; r++)
    {
        double s = 0;
        for(int c = 0; c < 12; c++) s += mass_entry(M, r, c) * dq[c];
        g[r] = fx ? 0.0 : s;
    }
    double S[9][9];
    for(int i = 0; i < 9; i++)
        for(int j = 0; j < 9; j++) S[i][j] = 0.0;
    if(!fx)
    {
        const double kvt2 = kappa * vol[b] * dt * dt;
        const double* a[3] = {Q + 3, Q + 6, Q + 9};
        double dot[3][3];
        for(int i = 0; i < 3; i++)
            for(int j = 0; j < 3; j++) dot[i][j] = a[i][0] * a[j][0] + a[i][1] * a[j][1] + a[i][2] * a[j][2];
        // dS/da_i = 4 (a_i.a_i - 1) a_i + 4 sum_{j != i} (a_j.a_i) a_j
        for(int i = 0; i < 3; i++)
            for(int k = 0; k < 3; k++)
            {
                double s = 4.0 * (dot[i][i] - 1.0) * a[i][k];
                for(int j = 0; j < 3; j++)
                    if(j != i) s += 4.0 * dot[j][i] * a[j][k];
                g[3 + 3 * i + k] += kvt2 * s;
            }
        // d2S/da_i^2 = 8 a_i a_i^T + 4 (a_i.a_i - 1) I + 4 sum_{j != i} a_j a_j^T;
        // d2S/da_i da_j = 4 a_j a_i^T + 4 (a_i.a_j) I
        for(int i = 0; i < 3; i++)
            for(int j = 0; j < 3; j++)
                for(int r = 0; r < 3; r++)
                    for(int c = 0; c < 3; c++)
                    {
                        double h;
                        if(i == j)
                        {
                            h = 8.0 * a[i][r] * a[i][c] + (r == c ? 4.0 * (dot[i][i] - 1.0) : 0.0);
                            for(int k = 0; k < 3; k++)
                                if(k != i) h += 4.0 * a[k][r] * a[k][c];
                        }
                        else
                            h = 4.0 * a[j][r] * a[i][c] + (r == c ? 4.0 * dot[i][j] : 0.0);
                        S[3 * i + r][3 * j + c] = kvt2 * h;
                    }
        psd_project9(S);
    }
    for(int k = 0; k < 12; k++) grad[12 * (size_t)b + k] = g[k];
    int slot = 0;
    for(int ii = 0; ii < 4; ii++)
        for(int jj = ii; jj < 4; jj++, slot++)
        {
            const size_t o = 10 * (size_t)b + slot;
            rows[o] = 4 * b + ii;
            cols[o] = 4 * b + jj;
            for(int c = 0; c < 3; c++)
                for(int r = 0; r < 3; r++)
                {
                    const int R = 3 * ii + r, C = 3 * jj + c;
                    double v = mass_entry(M, R, C);
                    if(R >= 3 && C >= 3) v += S[R - 3][C - 3];
                    blocks[9 * o + 3 * c + r] = v;  // column-major
                }
        }
}

// X = J(x)^T B J(y) (JT_H_J, abd_jacobi_matrix.inl:34-72); B row-major 3x3
__device__ inline double jthj(const double* B, const double* x, const double* y, int R, int C)
{
    if(R < 3 && C < 3) return B[3 * R + C];
    if(R < 3) return B[3 * R + (C - 3) / 3] * y[(C - 3) % 3];
    if(C < 3) return x[(R - 3) % 3] * B[3 * ((R - 3) / 3) + C];
    return x[(R - 3) % 3] * y[(C - 3) % 3] * B[3 * ((R - 3) / 3) + (C - 3) / 3];
}

__global__ void k_abd_map(int count, const int* __restrict__ rin, const int* __restrict__ cin,
                          const double* __restrict__ bin, int P, const int* __restrict__ point_body,
                          const double* __restrict__ xbar, int N, int* rows, int* cols, double* blocks, int* bad)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= count) return;
    int i = rin[t], j = cin[t];
    double B[9];  // row-major
    const bool sw = i > j;
    for(int r = 0; r < 3; r++)
        for(int c = 0; c < 3; c++) B[3 * r + c] = sw ? bin[9 * (size_t)t + 3 * r + c] : bin[9 * (size_t)t + 3 * c + r];
    if(sw)
    {
        const int k = i;
        i = j, j = k;
    }
    const size_t base = 16 * (size_t)t;
    int slot = 0;
    auto put = [&](int r, int c, const double* V /*row-major*/) {
        const size_t o = base + slot++;
        rows[o] = r, cols[o] = c;
        for(int rr = 0; rr < 3; rr++)
            for(int cc = 0; cc < 3; cc++) blocks[9 * o + 3 * cc + rr] = V ? V[3 * rr + cc] : 0.0;
    };
    const bool ia = i < P, ja = j < P;
    int r0 = 0;
    if(i < 0 || j < 0 || (ia && (point_body[i] < 0 || point_body[i] >= N)) ||
       (ja && (point_body[j] < 0 || point_body[j] >= N)))
    {
        if(bad) atomicAdd(bad, 1);
        while(slot < 16) put(r0, r0, nullptr);
        return;
    }
    if(!ia)
    {
        // FEM-FEM: shifted past the body rows
        r0 = 4 * N + i - P;
        put(r0, 4 * N + j - P, B);
    }
    else if(!ja)
    {
        // body point - FEM vertex: J_i^T B, 4 blocks down the body's rows
        const int bi = point_body[i];
        const double* x = xbar + 3 * (size_t)i;
        r0 = 4 * bi;
        for(int k = 0; k < 4; k++)
        {
            double V[9];
            for(int r = 0; r < 3; r++)
                for(int c = 0; c < 3; c++) V[3 * r + c] = k == 0 ? B[3 * r + c] : x[r] * B[3 * (k - 1) + c];
            put(4 * bi + k, 4 * N + j - P, V);
        }
    }
    else
    {
        const int bi = point_body[i], bj = point_body[j];
        const double *x = xbar + 3 * (size_t)i, *y = xbar + 3 * (size_t)j;
        r0 = 4 * (bi < bj ? bi : bj);
        if(bi != bj)
        {
            // X at tile (bi, bj); stored upper: X itself, or X^T at (bj, bi)
            for(int ii = 0; ii < 4; ii++)
                for(int jj = 0; jj < 4; jj++)
                {
                    double V[9];
                    for(int r = 0; r < 3; r++)
                        for(int c = 0; c < 3; c++)
                            V[3 * r + c] = bi < bj ? jthj(B, x, y, 3 * ii + r, 3 * jj + c)
                                                   : jthj(B, x, y, 3 * jj + c, 3 * ii + r);
                    if(bi < bj)
                        put(4 * bi + ii, 4 * bj + jj, V);
                    else
                        put(4 * bj + jj, 4 * bi + ii, V);
                }
        }
        else
        {
            // one body: J_i^T B J_i for a diagonal point block, X + X^T for a pair of points
            for(int ii = 0; ii < 4; ii++)
                for(int jj = ii; jj < 4; jj++)
                {
                    double V[9];
                    for(int r = 0; r < 3; r++)
                        for(int c = 0; c < 3; c++)
                        {
                            const int R = 3 * ii + r, C = 3 * jj + c;
                            V[3 * r + c] = i == j ? jthj(B, x, y, R, C) : jthj(B, x, y, R, C) + jthj(B, x, y, C, R);
                        }
                    put(4 * bi + ii, 4 * bi + jj, V);
                }
        }
    }
    while(slot < 16) put(r0, r0, nullptr);
}

__global__ void k_abd_points(int P, const int* __restrict__ point_body, const double* __restrict__ xbar,
                             const double* __restrict__ q, double* x)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= P) return;
    const int b = point_body[i];
    const double* Q = q + 12 * (size_t)b;
    const double* xb = xbar + 3 * (size_t)i;
    for(int r = 0; r < 3; r++)
        x[3 * (size_t)i + r] = Q[r] + Q[3 + 3 * r] * xb[0] + Q[4 + 3 * r] * xb[1] + Q[5 + 3 * r] * xb[2];
}

__global__ void k_abd_gather_grad(int N, const int* __restrict__ start, const double* __restrict__ xbar,
                                  const double* __restrict__ pg, double* bg)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if(b >= N) return;
    double G[12];
    for(int k = 0; k < 12; k++) G[k] = 0.0;
    for(int i = start[b]; i < start[b + 1]; i++)
    {
        const double* g = pg + 3 * (size_t)i;
        const double* x = xbar + 3 * (size_t)i;
        for(int r = 0; r < 3; r++)
        {
            G[r] += g[r];
            for(int k = 0; k < 3; k++) G[3 + 3 * r + k] += x[k] * g[r];
        }
    }
    for(int k = 0; k < 12; k++) bg[12 * (size_t)b + k] += G[k];
}

// the bodies' diagonal 12x12 tiles (row-major) of a sorted unique upper BCOO
__global__ void k_abd_tiles(int nnzb, const int* __restrict__ rows, const int* __restrict__ cols,
                            const double* __restrict__ blocks, int N, double* P)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= nnzb) return;
    const int r = rows[t], c = cols[t];
    if(r >= 4 * N || r / 4 != c / 4) return;
    double* T = P + 144 * (size_t)(r / 4);
    const int R = 3 * (r % 4), C = 3 * (c % 4);
    for(int a = 0; a < 3; a++)
        for(int b = 0; b < 3; b++)
        {
            const double v = blocks[9 * (size_t)t + 3 * b + a];  // (a, b), column-major
            T[12 * (R + a) + C + b] = v;
            if(r != c) T[12 * (C + b) + R + a] = v;
        }
}

// in-place inverse of each 12x12 tile (row-major), Gauss-Jordan with partial pivoting, FP64
__global__ void k_abd_invert(int N, double* P, int* singular)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if(b >= N) return;
    double A[12][24];
    double* T = P + 144 * (size_t)b;
    for(int i = 0; i < 12; i++)
        for(int j = 0; j < 12; j++) A[i][j] = T[12 * i + j], A[i][12 + j] = i == j ? 1.0 : 0.0;
    for(int k = 0; k < 12; k++)
    {
        int p = k;
        for(int i = k + 1; i < 12; i++)
            if(fabs(A[i][k]) > fabs(A[p][k])) p = i;
        if(A[p][k] == 0.0)
        {
            if(singular) atomicAdd(singular, 1);
            for(int i = 0; i < 144; i++) T[i] = 0.0;
            return;
        }
        if(p != k)
            for(int j = 0; j < 24; j++)
            {
                const double tmp = A[k][j];
                A[k][j] = A[p][j], A[p][j] = tmp;
            }
        const double inv = 1.0 / A[k][k];
        for(int j = 0; j < 24; j++) A[k][j] *= inv;
        for(int i = 0; i < 12; i++)
            if(i != k)
            {
                const double f = A[i][k];
                if(f != 0.0)
                    for(int j = 0; j < 24; j++) A[i][j] -= f * A[k][j];
            }
    }
    for(int i = 0; i < 12; i++)
        for(int j = 0; j < 12; j++) T[12 * i + j] = A[i][12 + j];
}

}  // namespace

int abd_block_jacobi(int nnzb, const int* rows, const int* cols, const double* blocks, int N, double* P,
                     int* singular, cudaStream_t s)
{
    STG_CUDA_TRY(cudaMemsetAsync(P, 0, 144 * sizeof(double) * (size_t)N, s));
    if(nnzb > 0) k_abd_tiles<<<(nnzb + AT - 1) / AT, AT, 0, s>>>(nnzb, rows, cols, blocks, N, P);
    k_abd_invert<<<(N + 63) / 64, 64, 0, s>>>(N, P, singular);
    STG_CUDA_TRY(cudaGetLastError());
    return STG_OK;
}

}  // namespace stg

extern "C" int stg_abd_body_system(int bodies, const double* q, const double* q_tilde, const double* mass,
                                   const double* volume, const int32_t* fixed, double kappa, double dt,
                                   int32_t* rows, int32_t* cols, double* blocks, double* grad, void* stream)
{
    if(bodies < 0 || !(dt > 0.0) || !(kappa >= 0.0) ||
       (bodies > 0 && (!q || !q_tilde || !mass || !volume || !rows || !cols || !blocks || !grad)))
    {
        stg::set_error("stg_abd_body_system: invalid arguments");
        return STG_ERR_INVALID;
    }
    if(bodies == 0) return STG_OK;
    stg::k_abd_body<<<(bodies + stg::AT - 1) / stg::AT, stg::AT, 0, static_cast<cudaStream_t>(stream)>>>(
        bodies, q, q_tilde, mass, volume, fixed, kappa, dt, rows, cols, blocks, grad);
    STG_CUDA_TRY(cudaGetLastError());
    return STG_OK;
}

extern "C" int stg_abd_map_triplets(int count, const int32_t* rows, const int32_t* cols, const double* blocks,
                                    int abd_points, const int32_t* point_body, const double* xbar, int bodies,
                                    int32_t* out_rows, int32_t* out_cols, double* out_blocks, int* bad,
                                    void* stream)
{
    if(count < 0 || abd_points < 0 || bodies < 0 || (abd_points > 0 && bodies == 0) ||
       (count > 0 && (!rows || !cols || !blocks || !out_rows || !out_cols || !out_blocks)) ||
       (abd_points > 0 && (!point_body || !xbar)))
    {
        stg::set_error("stg_abd_map_triplets: invalid arguments");
        return STG_ERR_INVALID;
    }
    if(count == 0) return STG_OK;
    stg::k_abd_map<<<(count + stg::AT - 1) / stg::AT, stg::AT, 0, static_cast<cudaStream_t>(stream)>>>(
        count, rows, cols, blocks, abd_points, point_body, xbar, bodies, out_rows, out_cols, out_blocks, bad);
    STG_CUDA_TRY(cudaGetLastError());
    return STG_OK;
}

extern "C" int stg_abd_points(int abd_points, const int32_t* point_body, const double* xbar, const double* q,
                              double* x, void* stream)
{
    if(abd_points < 0 || (abd_points > 0 && (!point_body || !xbar || !q || !x)))
    {
        stg::set_error("stg_abd_points: invalid arguments");
        return STG_ERR_INVALID;
    }
    if(abd_points == 0) return STG_OK;
    stg::k_abd_points<<<(abd_points + stg::AT - 1) / stg::AT, stg::AT, 0, static_cast<cudaStream_t>(stream)>>>(
        abd_points, point_body, xbar, q, x);
    STG_CUDA_TRY(cudaGetLastError());
    return STG_OK;
}

extern "C" int stg_abd_gather_gradient(int bodies, const int32_t* body_point_start, const double* xbar,
                                       const double* point_grad, double* body_grad, void* stream)
{
    if(bodies < 0 || (bodies > 0 && (!body_point_start || !xbar || !point_grad || !body_grad)))
    {
        stg::set_error("stg_abd_gather_gradient: invalid arguments");
        return STG_ERR_INVALID;
    }
    if(bodies == 0) return STG_OK;
    stg::k_abd_gather_grad<<<(bodies + stg::AT - 1) / stg::AT, stg::AT, 0, static_cast<cudaStream_t>(stream)>>>(
        bodies, body_point_start, xbar, point_grad, body_grad);
    STG_CUDA_TRY(cudaGetLastError());
    return STG_OK;
}
