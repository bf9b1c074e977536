// cloth.cu -- cloth membrane and bending terms of the Newton system on the GPU.
//
// Membrane: replaces _calculate_triangle_fem_gradient_hessian (StiffGIPC/femEnergy.cu:2146-2216)
// with the Baraff-Witkin energy it differentiates (__computePEPF_BaraffWitkinStretch_double,
// femEnergy.cu:351-396): per triangle, F = Ds Dm^-1 (3x2, Dm in the triangle's rest plane),
// su = |F u|, sv = |F v|, I6 = (F u).(F v), and
//   E = area dt^2 [ k_st ((su - 1)^2 + (sv - 1)^2 + r ((su - 1)^3_+ + (sv - 1)^3_+)) + k_sh I6^2 ]
// with r the strain rate (the cubic only where a direction is stretched).  The Hessian in F is
// the stretch part projected per direction as the reference does analytically
// (__project_BaraffWitkinStretch_H, :535-629: the transverse term dropped where the direction
// is compressed) plus the shear part 2 (g g^T + I6 S) projected to PSD in the reference's
// closed form (__project_BaraffWitkinShear_H, :631-706), mapped to the three vertices by dF/dx.  Area is the rest area times the thickness, as the reference
// stores it.
// Bending: replaces _calculate_quad_bending_gradient_hessian (femEnergy.cu:2620-2755,
// USE_QUADRATIC_BENDING): per interior edge stencil (edge v0 v1, opposite vertices v2 v3) the
// constant 4x4 matrix Q of PrepareQuadBendingQ (:2490-2618), gradient c Q x and Hessian
// c Q (x) I3 with c = |rest edge| k_bend dt^2.
// Both write per-element gradients and the elements' upper 3x3 blocks (column-major, row <=
// col) to fixed slots: no atomics.
#include "solver.hpp"

namespace stg
{
namespace
{
constexpr int CT = 128;

// one upper block (i, j) of a per-element Hessian, oriented by the global indices
__device__ inline void put_block(int* rows, int* cols, double* blocks, size_t o, int gi, int gj, const double* Hij)
{
    // Hij: row-major 3x3 block (local i, j); stored column-major, transposed when gi > gj
    const bool sw = gi > gj;
    rows[o] = sw ? gj : gi;
    cols[o] = sw ? gi : gj;
    for(int a = 0; a < 3; a++)
        for(int b = 0; b < 3; b++)
            blocks[9 * o + (sw ? 3 * a + b : 3 * b + a)] = Hij[3 * a + b];  // element (a, b), or (b, a) if swapped
}

__global__ void k_cloth_membrane(int T, const int* __restrict__ tri, const double* __restrict__ dminv,
                                 const double* __restrict__ area, const double* __restrict__ x, int nv, double kst,
                                 double ksh, double sr, double dt2, int off, int* rows, int* cols, double* blocks,
                                 double* grad, int* bad)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= T) return;
    int v[3];
    bool ok = true;
    for(int a = 0; a < 3; a++) v[a] = tri[3 * (size_t)t + a], ok = ok && v[a] >= 0 && v[a] < nv;
    ok = ok && v[0] != v[1] && v[1] != v[2] && v[0] != v[2];
    if(!ok)
    {
        if(bad) atomicAdd(bad, 1);
        for(int k = 0; k < 6; k++)
        {
            const size_t o = 6 * (size_t)t + k;
            rows[o] = cols[o] = off;
            for(int e = 0; e < 9; e++) blocks[9 * o + e] = 0.0;
        }
        for(int k = 0; k < 9; k++) grad[9 * (size_t)t + k] = 0.0;
        return;
    }
    const double* Di = dminv + 4 * (size_t)t;  // row-major 2x2
    double X[3][3];
    for(int a = 0; a < 3; a++)
        for(int d = 0; d < 3; d++) X[a][d] = x[3 * (size_t)v[a] + d];
    double F[3][2];
    for(int d = 0; d < 3; d++)
    {
        const double e1 = X[1][d] - X[0][d], e2 = X[2][d] - X[0][d];
        for(int c = 0; c < 2; c++) F[d][c] = e1 * Di[c] + e2 * Di[2 + c];
    }
    // dF[:, c] / dx_a = w[a][c] I3
    double w[3][2];
    for(int c = 0; c < 2; c++) w[1][c] = Di[c], w[2][c] = Di[2 + c], w[0][c] = -(Di[c] + Di[2 + c]);
    const double fu[3] = {F[0][0], F[1][0], F[2][0]}, fv[3] = {F[0][1], F[1][1], F[2][1]};
    const double I5u = fu[0] * fu[0] + fu[1] * fu[1] + fu[2] * fu[2];
    const double I5v = fv[0] * fv[0] + fv[1] * fv[1] + fv[2] * fv[2];
    const double I6 = fu[0] * fv[0] + fu[1] * fv[1] + fu[2] * fv[2];
    const double su = sqrt(I5u), sv = sqrt(I5v);
    double cu = 1.0 - 1.0 / su, cv = 1.0 - 1.0 / sv;
    if(I5u > 1) cu += 1.5 * sr * (su + 1.0 / su - 2.0);
    if(I5v > 1) cv += 1.5 * sr * (sv + 1.0 / sv - 2.0);
    double P[2][3];  // dE/dF per column (u, v), without area dt^2
    for(int d = 0; d < 3; d++)
    {
        P[0][d] = kst * 2.0 * cu * fu[d] + ksh * 2.0 * I6 * fv[d];
        P[1][d] = kst * 2.0 * cv * fv[d] + ksh * 2.0 * I6 * fu[d];
    }
    const double k = area[t] * dt2;
    for(int a = 0; a < 3; a++)
        for(int d = 0; d < 3; d++) grad[9 * (size_t)t + 3 * a + d] = k * (w[a][0] * P[0][d] + w[a][1] * P[1][d]);
    // Hq (6x6, column u then v): projected stretch + projected shear
    double Hq[6][6];
    {
        // the shear term's projection in closed form (the reference's
        // __project_BaraffWitkinShear_H): with g = dI6/dF = (F v, F u) and S the swap of the two
        // columns, the Hessian 2 (g g^T + I6 S) has the eigenvector q0 ~ I6 S g + lambda0 g
        // (eigenvalue 2 lambda0, lambda0 = (I2 + sqrt(I2^2 + 12 I6^2)) / 2) and +-2 I6 on the
        // eigenspaces of S; the projection keeps 2 lambda0 q0 q0^T and 2 |I6| on the part of S's
        // sign(I6) eigenspace orthogonal to q0
        const double g[6] = {fv[0], fv[1], fv[2], fu[0], fu[1], fu[2]};
        const double Sg[6] = {fu[0], fu[1], fu[2], fv[0], fv[1], fv[2]};
        const double I2 = I5u + I5v;
        const double lam0 = 0.5 * (I2 + sqrt(I2 * I2 + 12.0 * I6 * I6));
        const double sgn = I6 >= 0 ? 1.0 : -1.0;
        double q0[6], nq = 0.0;
        for(int i = 0; i < 6; i++) q0[i] = I6 * Sg[i] + lam0 * g[i], nq += q0[i] * q0[i];
        nq = sqrt(nq);
        for(int i = 0; i < 6; i++) q0[i] = nq > 0.0 ? q0[i] / nq : 0.0;
        double Tq[6], ntq = 0.0;
        for(int i = 0; i < 6; i++) Tq[i] = 0.5 * (q0[i] + sgn * q0[(i + 3) % 6]), ntq += Tq[i] * Tq[i];
        for(int i = 0; i < 6; i++)
            for(int j = 0; j < 6; j++)
            {
                const double T = 0.5 * ((i == j ? 1.0 : 0.0) + ((i % 3 == j % 3 && i != j) ? sgn : 0.0));
                const double proj = ntq > 0.0 ? T - Tq[i] * Tq[j] / ntq : T;
                Hq[i][j] = ksh * 2.0 * (fabs(I6) * proj + lam0 * q0[i] * q0[j]);
            }
    }
    for(int c = 0; c < 2; c++)
    {
        const double s = c == 0 ? su : sv, I5 = c == 0 ? I5u : I5v;
        const double* f = c == 0 ? fu : fv;
        const double iso = s > 1 ? 2.0 * (((s - 1.0) * (3.0 * s * sr - 3.0 * sr + 2.0)) / (2.0 * s)) : 0.0;
        const double along = s > 1.0 ? (3.0 * I5 * sr - 3.0 * sr + 2.0) / s : 2.0;
        for(int i = 0; i < 3; i++)
            for(int j = 0; j < 3; j++)
                Hq[3 * c + i][3 * c + j] += kst * ((i == j ? iso : 0.0) + along * (f[i] / s) * (f[j] / s));
    }
    int slot = 0;
    for(int a = 0; a < 3; a++)
        for(int b = a; b < 3; b++, slot++)
        {
            double B[9];
            for(int i = 0; i < 3; i++)
                for(int j = 0; j < 3; j++)
                {
                    double sum = 0;
                    for(int c = 0; c < 2; c++)
                        for(int e = 0; e < 2; e++) sum += w[a][c] * w[b][e] * Hq[3 * c + i][3 * e + j];
                    B[3 * i + j] = k * sum;
                }
            put_block(rows, cols, blocks, 6 * (size_t)t + slot, off + v[a], off + v[b], B);
        }
}

__global__ void k_cloth_bending(int E, const int* __restrict__ st, const double* __restrict__ Q,
                                const double* __restrict__ len, const double* __restrict__ x, int nv, double kb,
                                double dt2, int off, int* rows, int* cols, double* blocks, double* grad, int* bad)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if(e >= E) return;
    int v[4];
    bool ok = true;
    for(int a = 0; a < 4; a++) v[a] = st[4 * (size_t)e + a], ok = ok && v[a] >= 0 && v[a] < nv;
    if(!ok)
    {
        // a boundary edge (no second triangle) or a bad index: no term
        if(bad && v[3] >= 0) atomicAdd(bad, 1);
        const int r0 = off + (v[0] >= 0 && v[0] < nv ? v[0] : 0);
        for(int kk = 0; kk < 10; kk++)
        {
            const size_t o = 10 * (size_t)e + kk;
            rows[o] = cols[o] = r0;
            for(int q = 0; q < 9; q++) blocks[9 * o + q] = 0.0;
        }
        for(int q = 0; q < 12; q++) grad[12 * (size_t)e + q] = 0.0;
        return;
    }
    const double* Qe = Q + 16 * (size_t)e;  // row-major 4x4
    const double c = len[e] * kb * dt2;
    for(int i = 0; i < 4; i++)
        for(int d = 0; d < 3; d++)
        {
            double s = 0;
            for(int j = 0; j < 4; j++) s += Qe[4 * i + j] * x[3 * (size_t)v[j] + d];
            grad[12 * (size_t)e + 3 * i + d] = c * s;
        }
    int slot = 0;
    for(int i = 0; i < 4; i++)
        for(int j = i; j < 4; j++, slot++)
        {
            const double q = c * Qe[4 * i + j];
            const double B[9] = {q, 0, 0, 0, q, 0, 0, 0, q};
            put_block(rows, cols, blocks, 10 * (size_t)e + slot, off + v[i], off + v[j], B);
        }
}
}  // namespace
}  // namespace stg

extern "C" int stg_cloth_membrane(int tris, const int32_t* tri_verts, const double* dminv, const double* area,
                                  const double* x, int num_verts, double stretch, double shear, double strain_rate,
                                  double dt, int block_offset, int32_t* rows, int32_t* cols, double* blocks,
                                  double* grad, int* bad, void* stream)
{
    if(tris < 0 || num_verts < 0 || block_offset < 0 || !(dt > 0.0) || !(stretch >= 0.0) || !(shear >= 0.0) ||
       !(strain_rate >= 0.0) || (tris > 0 && (!tri_verts || !dminv || !area || !x || !rows || !cols || !blocks || !grad)))
    {
        stg::set_error("stg_cloth_membrane: invalid arguments");
        return STG_ERR_INVALID;
    }
    if(tris == 0) return STG_OK;
    stg::k_cloth_membrane<<<(tris + stg::CT - 1) / stg::CT, stg::CT, 0, static_cast<cudaStream_t>(stream)>>>(
        tris, tri_verts, dminv, area, x, num_verts, stretch, shear, strain_rate, dt * dt, block_offset, rows, cols,
        blocks, grad, bad);
    STG_CUDA_TRY(cudaGetLastError());
    return STG_OK;
}

extern "C" int stg_cloth_bending(int edges, const int32_t* stencil, const double* Q, const double* rest_length,
                                 const double* x, int num_verts, double bend_stiff, double dt, int block_offset,
                                 int32_t* rows, int32_t* cols, double* blocks, double* grad, int* bad, void* stream)
{
    if(edges < 0 || num_verts < 0 || block_offset < 0 || !(dt > 0.0) || !(bend_stiff >= 0.0) ||
       (edges > 0 && (!stencil || !Q || !rest_length || !x || !rows || !cols || !blocks || !grad)))
    {
        stg::set_error("stg_cloth_bending: invalid arguments");
        return STG_ERR_INVALID;
    }
    if(edges == 0) return STG_OK;
    stg::k_cloth_bending<<<(edges + stg::CT - 1) / stg::CT, stg::CT, 0, static_cast<cudaStream_t>(stream)>>>(
        edges, stencil, Q, rest_length, x, num_verts, bend_stiff, dt * dt, block_offset, rows, cols, blocks, grad,
        bad);
    STG_CUDA_TRY(cudaGetLastError());
    return STG_OK;
}
