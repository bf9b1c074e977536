// fem.cu -- the Hessian producer of one implicit-Euler Newton iteration on the GPU: per-tet
// stable Neo-Hookean gradient and PSD-projected Hessian (12x12, written as the 10 upper 3x3
// blocks of the tet), lumped mass, the kinetic term and IPC plane barriers, as the device
// triplets and gradient that GlobalLinearSystem::solve_linear_system receives.
//
// The reference builds these in femEnergy.cu:1719-1855 (_calculate_fem_gradient_hessian, its
// SNH variants and Eigen-SVD eigensystem projection) and GIPC.cu:6524-6551 (ground barrier).
// This file follows the formulation of the synthetic scenes (stgipc/scenes.py: SNH of Smith
// et al. 2018 without the log term, psi = mu/2 (|F|^2 - 3) + lam/2 (J - alpha)^2,
// alpha = 1 + mu / lam, whose 9x9 Hessian in F is projected to PSD by clamping negative
// eigenvalues), and the reference's plane barrier on the squared distance.
#include "solver.hpp"
#include "eig9.cuh"

namespace stg
{
namespace
{
constexpr int FT = 128;  // threads per CTA

__device__ __forceinline__ double det3(const double (&M)[3][3])
{
    return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
}

// one thread per tet: the 10 upper blocks (column-major, upper orientation) into the
// triplets at t * 10 + kk, the tet's 12 gradient entries and its lumped mass share
__global__ void __launch_bounds__(FT) k_fem_tet(const double* __restrict__ rest, const double* __restrict__ pos,
                                                const int* __restrict__ tets, const double* __restrict__ E, int T,
                                                double nu, double rho, double dt, int* rows, int* cols, double* blocks,
                                                double* ft, double* mt)
{
    const int t = blockIdx.x * FT + threadIdx.x;
    if(t >= T) return;
    int v[4];
    for(int a = 0; a < 4; a++) v[a] = tets[4 * (size_t)t + a];
    double Dm[3][3], Ds[3][3];
    for(int r = 0; r < 3; r++)
        for(int a = 0; a < 3; a++)
        {
            Dm[r][a] = rest[3 * (size_t)v[a + 1] + r] - rest[3 * (size_t)v[0] + r];
            Ds[r][a] = pos[3 * (size_t)v[a + 1] + r] - pos[3 * (size_t)v[0] + r];
        }
    const double dd = det3(Dm);
    const double vol = fabs(dd) / 6.0;
    double Di[3][3];  // Dm^-1 = adj(Dm) / det
    Di[0][0] = (Dm[1][1] * Dm[2][2] - Dm[1][2] * Dm[2][1]) / dd;
    Di[0][1] = (Dm[0][2] * Dm[2][1] - Dm[0][1] * Dm[2][2]) / dd;
    Di[0][2] = (Dm[0][1] * Dm[1][2] - Dm[0][2] * Dm[1][1]) / dd;
    Di[1][0] = (Dm[1][2] * Dm[2][0] - Dm[1][0] * Dm[2][2]) / dd;
    Di[1][1] = (Dm[0][0] * Dm[2][2] - Dm[0][2] * Dm[2][0]) / dd;
    Di[1][2] = (Dm[0][2] * Dm[1][0] - Dm[0][0] * Dm[1][2]) / dd;
    Di[2][0] = (Dm[1][0] * Dm[2][1] - Dm[1][1] * Dm[2][0]) / dd;
    Di[2][1] = (Dm[0][1] * Dm[2][0] - Dm[0][0] * Dm[2][1]) / dd;
    Di[2][2] = (Dm[0][0] * Dm[1][1] - Dm[0][1] * Dm[1][0]) / dd;
    double F[3][3];
    for(int i = 0; i < 3; i++)
        for(int j = 0; j < 3; j++) F[i][j] = Ds[i][0] * Di[0][j] + Ds[i][1] * Di[1][j] + Ds[i][2] * Di[2][j];
    const double mu = E[t] / (2.0 * (1.0 + nu)), lam = E[t] * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double J = det3(F), alpha = 1.0 + mu / lam;
    // cofactor g = dJ/dF (row-major vec) and the Hessian of J (HJ[ij][kl] = eps_ikm eps_jln F_mn)
    double g[9];
    g[0] = F[1][1] * F[2][2] - F[1][2] * F[2][1];
    g[1] = F[1][2] * F[2][0] - F[1][0] * F[2][2];
    g[2] = F[1][0] * F[2][1] - F[1][1] * F[2][0];
    g[3] = F[0][2] * F[2][1] - F[0][1] * F[2][2];
    g[4] = F[0][0] * F[2][2] - F[0][2] * F[2][0];
    g[5] = F[0][1] * F[2][0] - F[0][0] * F[2][1];
    g[6] = F[0][1] * F[1][2] - F[0][2] * F[1][1];
    g[7] = F[0][2] * F[1][0] - F[0][0] * F[1][2];
    g[8] = F[0][0] * F[1][1] - F[0][1] * F[1][0];
    double H[9][9];
    const double k = lam * (J - alpha);
    for(int i = 0; i < 3; i++)
        for(int j = 0; j < 3; j++)
            for(int kk = 0; kk < 3; kk++)
                for(int l = 0; l < 3; l++)
                {
                    // eps_ikm eps_jln F_mn: nonzero only for i != k, j != l; m, n the third indices
                    double hj = 0;
                    if(i != kk && j != l)
                    {
                        const int m = 3 - i - kk, n = 3 - j - l;
                        const double sik = ((kk - i + 3) % 3 == 1) ? 1.0 : -1.0;  // eps_ikm
                        const double sjl = ((l - j + 3) % 3 == 1) ? 1.0 : -1.0;  // eps_jln
                        hj = sik * sjl * F[m][n];
                    }
                    H[3 * i + j][3 * kk + l] = (3 * i + j == 3 * kk + l ? mu : 0.0) + lam * g[3 * i + j] * g[3 * kk + l] + k * hj;
                }
    for(int i = 0; i < 9; i++)
        for(int j = i + 1; j < 9; j++)
        {
            const double a = 0.5 * (H[i][j] + H[j][i]);
            H[i][j] = a;
            H[j][i] = a;
        }
    double P[9];
    for(int i = 0; i < 3; i++)
        for(int j = 0; j < 3; j++) P[3 * i + j] = mu * F[i][j] + k * g[3 * i + j];
    // PSD projection: clamp negative eigenvalues (only when there is one)
    psd_project9(H);
    // d[a][j]: dF_ij / dx_a,i
    double d[4][3];
    for(int j = 0; j < 3; j++)
    {
        d[1][j] = Di[0][j];
        d[2][j] = Di[1][j];
        d[3][j] = Di[2][j];
        d[0][j] = -(Di[0][j] + Di[1][j] + Di[2][j]);
    }
    const double w = vol * dt * dt;
    for(int a = 0; a < 4; a++)
        for(int i = 0; i < 3; i++)
            ft[12 * (size_t)t + 3 * a + i] = w * (d[a][0] * P[3 * i] + d[a][1] * P[3 * i + 1] + d[a][2] * P[3 * i + 2]);
    mt[t] = rho * vol / 4.0;
    int kk = 0;
    for(int a = 0; a < 4; a++)
        for(int b = a; b < 4; b++, kk++)
        {
            double B[3][3];  // H12[3a+i][3b+k] = w sum_jl d[a][j] d[b][l] H9[3i+j][3k+l]
            for(int i = 0; i < 3; i++)
                for(int q = 0; q < 3; q++)
                {
                    double s = 0;
                    for(int j = 0; j < 3; j++)
                        for(int l = 0; l < 3; l++) s += d[a][j] * d[b][l] * H[3 * i + j][3 * q + l];
                    B[i][q] = w * s;
                }
            const bool swap = v[a] > v[b];
            const size_t o = 10 * (size_t)t + kk;
            rows[o] = swap ? v[b] : v[a];
            cols[o] = swap ? v[a] : v[b];
            // column-major storage of the upper-oriented block (B^T when swapped)
            for(int r = 0; r < 3; r++)
                for(int c = 0; c < 3; c++) blocks[9 * o + 3 * c + r] = swap ? B[c][r] : B[r][c];
        }
}

__global__ void k_fem_count(const int* __restrict__ tets, int T, int* cnt)
{
    for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < 4 * T; i += gridDim.x * blockDim.x) atomicAdd(cnt + tets[i], 1);
}

__global__ void k_fem_fill(const int* __restrict__ tets, int T, const int* __restrict__ start, int* cur, int* inc)
{
    for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < 4 * T; i += gridDim.x * blockDim.x)
    {
        const int v = tets[i];
        inc[start[v] + atomicAdd(cur + v, 1)] = i;  // i = 4 t + a
    }
}

// per vertex: incident (tet, slot) entries in increasing order, then the gradient and mass
// gathered in that order, the kinetic term, plane barriers, and the vertex's diagonal triplet
__global__ void k_fem_vertex(const int* __restrict__ start, int* inc, const double* __restrict__ ft,
                             const double* __restrict__ mt, const double* __restrict__ pos,
                             const double* __restrict__ vel, const double* __restrict__ xtilde, int V, int T,
                             double dt, double gy,
                             const double* __restrict__ planes, int nplanes, int* rows, int* cols, double* blocks,
                             double* b)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if(v >= V) return;
    const int s0 = start[v], s1 = start[v + 1];
    for(int p = s0 + 1; p < s1; p++)
    {
        const int x = inc[p];
        int q = p - 1;
        while(q >= s0 && inc[q] > x)
        {
            inc[q + 1] = inc[q];
            q--;
        }
        inc[q + 1] = x;
    }
    double g0 = 0, g1 = 0, g2 = 0, m = 0;
    for(int p = s0; p < s1; p++)
    {
        const int e = inc[p], t = e >> 2, a = e & 3;
        g0 += ft[12 * (size_t)t + 3 * a];
        g1 += ft[12 * (size_t)t + 3 * a + 1];
        g2 += ft[12 * (size_t)t + 3 * a + 2];
        m += mt[t];
    }
    // kinetic: M (x - x_tilde), x_tilde given, or x_tilde = x + dt v + dt^2 (0, gy, 0) at x = x_n
    if(xtilde)
    {
        g0 += m * (pos[3 * (size_t)v] - xtilde[3 * (size_t)v]);
        g1 += m * (pos[3 * (size_t)v + 1] - xtilde[3 * (size_t)v + 1]);
        g2 += m * (pos[3 * (size_t)v + 2] - xtilde[3 * (size_t)v + 2]);
    }
    else
    {
        g0 += m * (-dt * vel[3 * (size_t)v]);
        g1 += m * (-dt * vel[3 * (size_t)v + 1] - dt * dt * gy);
        g2 += m * (-dt * vel[3 * (size_t)v + 2]);
    }
    double Hb[9] = {m, 0, 0, 0, m, 0, 0, 0, m};
    const double px = pos[3 * (size_t)v], py = pos[3 * (size_t)v + 1], pz = pos[3 * (size_t)v + 2];
    for(int k = 0; k < nplanes; k++)
    {
        const double* pl = planes + 6 * k;  // normal xyz, offset, dhat, kappa
        const double dist = px * pl[0] + py * pl[1] + pz * pl[2] - pl[3];
        const double dhat = pl[4], kappa = pl[5];
        if(!(dist < dhat)) continue;
        // IPC plane barrier on the squared distance (GIPC.cu:6524-6551)
        const double d2 = dist * dist, dh2 = dhat * dhat, tt = d2 - dh2, lg = log(d2 / dh2);
        const double gb = tt * lg * -2.0 - (tt * tt) / d2;
        const double hb = (lg * -2.0 - tt * 4.0 / d2) + 1.0 / (d2 * d2) * (tt * tt);
        const double gr = kappa * gb * 2.0 * dist, sc = kappa * (4.0 * hb * d2 + 2.0 * gb);
        g0 += gr * pl[0];
        g1 += gr * pl[1];
        g2 += gr * pl[2];
        for(int r = 0; r < 3; r++)
            for(int c = 0; c < 3; c++) Hb[3 * c + r] += sc * pl[r] * pl[c];
    }
    b[3 * (size_t)v] = g0;
    b[3 * (size_t)v + 1] = g1;
    b[3 * (size_t)v + 2] = g2;
    const size_t o = 10 * (size_t)T + v;
    rows[o] = v;
    cols[o] = v;
    for(int e = 0; e < 9; e++) blocks[9 * o + e] = Hb[e];
}

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

// incremental potential of the Newton iteration's objective, per CTA: dt^2 vol psi(F) per
// tet; 1/2 m |x - x_tilde|^2 and kappa b(d^2) per vertex (m from the tets' lumped mass);
// CTA partials in part[blockIdx.x] (tets) and part[tet_ctas + blockIdx.x] (vertices)
__global__ void __launch_bounds__(256) k_fem_energy_tet(const double* __restrict__ rest, const double* __restrict__ pos,
                                                         const int* __restrict__ tets, const double* __restrict__ E,
                                                         int T, double nu, double rho, double dt, double* mt, double* part)
{
    __shared__ double red[8];
    double e = 0;
    for(int t = blockIdx.x * 256 + threadIdx.x; t < T; t += gridDim.x * 256)
    {
        int v[4];
        for(int a = 0; a < 4; a++) v[a] = tets[4 * (size_t)t + a];
        double Dm[3][3], Ds[3][3];
        for(int r = 0; r < 3; r++)
            for(int a = 0; a < 3; a++)
            {
                Dm[r][a] = rest[3 * (size_t)v[a + 1] + r] - rest[3 * (size_t)v[0] + r];
                Ds[r][a] = pos[3 * (size_t)v[a + 1] + r] - pos[3 * (size_t)v[0] + r];
            }
        const double dd = det3(Dm), vol = fabs(dd) / 6.0;
        // F = Ds Dm^-1: |F|^2 and det F = det Ds / det Dm
        double Di[3][3];
        Di[0][0] = (Dm[1][1] * Dm[2][2] - Dm[1][2] * Dm[2][1]) / dd;
        Di[0][1] = (Dm[0][2] * Dm[2][1] - Dm[0][1] * Dm[2][2]) / dd;
        Di[0][2] = (Dm[0][1] * Dm[1][2] - Dm[0][2] * Dm[1][1]) / dd;
        Di[1][0] = (Dm[1][2] * Dm[2][0] - Dm[1][0] * Dm[2][2]) / dd;
        Di[1][1] = (Dm[0][0] * Dm[2][2] - Dm[0][2] * Dm[2][0]) / dd;
        Di[1][2] = (Dm[0][2] * Dm[1][0] - Dm[0][0] * Dm[1][2]) / dd;
        Di[2][0] = (Dm[1][0] * Dm[2][1] - Dm[1][1] * Dm[2][0]) / dd;
        Di[2][1] = (Dm[0][1] * Dm[2][0] - Dm[0][0] * Dm[2][1]) / dd;
        Di[2][2] = (Dm[0][0] * Dm[1][1] - Dm[0][1] * Dm[1][0]) / dd;
        double F[3][3], f2 = 0;
        for(int i = 0; i < 3; i++)
            for(int j = 0; j < 3; j++)
            {
                F[i][j] = Ds[i][0] * Di[0][j] + Ds[i][1] * Di[1][j] + Ds[i][2] * Di[2][j];
                f2 += F[i][j] * F[i][j];
            }
        const double mu = E[t] / (2.0 * (1.0 + nu)), lam = E[t] * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
        const double J = det3(F), alpha = 1.0 + mu / lam;
        e += vol * dt * dt * (0.5 * mu * (f2 - 3.0) + 0.5 * lam * (J - alpha) * (J - alpha));
        if(mt) mt[t] = rho * vol / 4.0;
    }
    e = block_sum<256>(e, red);
    if(threadIdx.x == 0) part[blockIdx.x] = e;
}

__global__ void __launch_bounds__(256) k_fem_energy_vertex(const int* __restrict__ start, const int* __restrict__ inc,
                                                            const double* __restrict__ mt, const double* __restrict__ pos,
                                                            const double* __restrict__ xtilde, int V,
                                                            const double* __restrict__ planes, int nplanes, double* part,
                                                            int* violations)
{
    __shared__ double red[8];
    double e = 0;
    for(int v = blockIdx.x * 256 + threadIdx.x; v < V; v += gridDim.x * 256)
    {
        double m = 0;
        for(int p = start[v]; p < start[v + 1]; p++) m += mt[inc[p] >> 2];
        const double d0 = pos[3 * (size_t)v] - xtilde[3 * (size_t)v], d1 = pos[3 * (size_t)v + 1] - xtilde[3 * (size_t)v + 1],
                     d2 = pos[3 * (size_t)v + 2] - xtilde[3 * (size_t)v + 2];
        e += 0.5 * m * (d0 * d0 + d1 * d1 + d2 * d2);
        for(int k = 0; k < nplanes; k++)
        {
            const double* pl = planes + 6 * k;
            const double dist = pos[3 * (size_t)v] * pl[0] + pos[3 * (size_t)v + 1] * pl[1] + pos[3 * (size_t)v + 2] * pl[2] - pl[3];
            if(!(dist > 0.0))
            {
                atomicAdd(violations, 1);
                continue;
            }
            if(dist < pl[4])
            {
                const double dd2 = dist * dist, dh2 = pl[4] * pl[4], tt = dd2 - dh2;
                e += pl[5] * (-(tt * tt) * log(dd2 / dh2));
            }
        }
    }
    e = block_sum<256>(e, red);
    if(threadIdx.x == 0) part[blockIdx.x] = e;
}
}  // namespace

constexpr int FEM_PARTS = 2 * kSMs * 4 + 8;  // energy: CTA partials of both passes + violation count

size_t fem_scratch_bytes(int V, int T)
{
    return a256(sizeof(double) * 12 * (size_t)T) + a256(sizeof(double) * (size_t)T) + 3 * a256(sizeof(int) * (V + 1)) +
           a256(sizeof(int) * 4 * (size_t)T) + a256(sizeof(double) * FEM_PARTS);
}

int fem_newton_system(cudaStream_t s, int V, const double* rest, const double* pos, const double* vel,
                      const double* xtilde, int T, const int* tets, const double* E, double nu, double rho, double dt,
                      double gy, int nplanes, const double* planes, int* rows, int* cols, double* blocks, double* b,
                      void* scratch, size_t bytes)
{
    if(V < 1 || T < 0 || !rest || !pos || (!vel && !xtilde) || (T > 0 && (!tets || !E)) || (nplanes > 0 && !planes) || !rows ||
       !cols || !blocks || !b || !(dt > 0) || !(nu > 0 && nu < 0.5))
    {
        set_error("stg_fem_newton_system: invalid arguments");
        return STG_ERR_INVALID;
    }
    if(!scratch || bytes < fem_scratch_bytes(V, T) || reinterpret_cast<uintptr_t>(scratch) % 256)
    {
        set_error("stg_fem_newton_system: scratch too small or not 256-byte aligned");
        return STG_ERR_INVALID;
    }
    unsigned char* p = static_cast<unsigned char*>(scratch);
    double* ft = reinterpret_cast<double*>(p);
    p += a256(sizeof(double) * 12 * (size_t)T);
    double* mt = reinterpret_cast<double*>(p);
    p += a256(sizeof(double) * (size_t)T);
    int* cnt = reinterpret_cast<int*>(p);
    p += a256(sizeof(int) * (V + 1));
    int* start = reinterpret_cast<int*>(p);
    p += a256(sizeof(int) * (V + 1));
    int* cur = reinterpret_cast<int*>(p);
    p += a256(sizeof(int) * (V + 1));
    int* inc = reinterpret_cast<int*>(p);
    STG_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int) * (V + 1), s));
    STG_CUDA_TRY(cudaMemsetAsync(cur, 0, sizeof(int) * (V + 1), s));
    if(T > 0)
    {
        k_fem_tet<<<div_up(T, FT), FT, 0, s>>>(rest, pos, tets, E, T, nu, rho, dt, rows, cols, blocks, ft, mt);
        STG_LAUNCH_CHECK();
        const int g = std::max(1, std::min(div_up(4L * T, 256), kSMs * 8));
        k_fem_count<<<g, 256, 0, s>>>(tets, T, cnt);
        STG_LAUNCH_CHECK();
        k_scan_exclusive<<<1, 1024, 0, s>>>(cnt, start, nullptr, V, start + V);
        STG_LAUNCH_CHECK();
        k_fem_fill<<<g, 256, 0, s>>>(tets, T, start, cur, inc);
        STG_LAUNCH_CHECK();
    }
    else
        STG_CUDA_TRY(cudaMemsetAsync(start, 0, sizeof(int) * (V + 1), s));
    k_fem_vertex<<<div_up(V, 256), 256, 0, s>>>(start, inc, ft, mt, pos, vel, xtilde, V, T, dt, gy, planes, nplanes,
                                                rows, cols, blocks, b);
    STG_LAUNCH_CHECK();
    return 0;
}

// the incremental potential at pos (tet CTA partials, then vertex CTA partials, summed on the
// host in CTA order); `violations` counts vertices on the wrong side of a plane (energy
// infinite: the caller must reject the step).  Uses the same scratch as fem_newton_system.
int fem_energy(cudaStream_t s, int V, const double* rest, const double* pos, const double* xtilde, int T,
               const int* tets, const double* E, double nu, double rho, double dt, int nplanes, const double* planes,
               void* scratch, size_t bytes, double* energy, int* violations)
{
    if(V < 1 || T < 0 || !rest || !pos || !xtilde || (T > 0 && (!tets || !E)) || (nplanes > 0 && !planes) || !energy)
    {
        set_error("stg_fem_energy: invalid arguments");
        return STG_ERR_INVALID;
    }
    if(!scratch || bytes < fem_scratch_bytes(V, T) || reinterpret_cast<uintptr_t>(scratch) % 256)
    {
        set_error("stg_fem_energy: scratch too small or not 256-byte aligned");
        return STG_ERR_INVALID;
    }
    unsigned char* p = static_cast<unsigned char*>(scratch);
    p += a256(sizeof(double) * 12 * (size_t)T);
    double* mt = reinterpret_cast<double*>(p);
    p += a256(sizeof(double) * (size_t)T);
    int* cnt = reinterpret_cast<int*>(p);
    p += a256(sizeof(int) * (V + 1));
    int* start = reinterpret_cast<int*>(p);
    p += a256(sizeof(int) * (V + 1));
    int* cur = reinterpret_cast<int*>(p);
    p += a256(sizeof(int) * (V + 1));
    int* inc = reinterpret_cast<int*>(p);
    p += a256(sizeof(int) * 4 * (size_t)T);
    double* part = reinterpret_cast<double*>(p);
    const int gt = std::max(1, std::min(div_up(T, 256), kSMs * 4)), gv = std::max(1, std::min(div_up(V, 256), kSMs * 4));
    int* viol = reinterpret_cast<int*>(part + gt + gv);
    STG_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int) * (V + 1), s));
    STG_CUDA_TRY(cudaMemsetAsync(cur, 0, sizeof(int) * (V + 1), s));
    STG_CUDA_TRY(cudaMemsetAsync(viol, 0, sizeof(int), s));
    if(T > 0)
    {
        k_fem_energy_tet<<<gt, 256, 0, s>>>(rest, pos, tets, E, T, nu, rho, dt, mt, part);
        STG_LAUNCH_CHECK();
        const int g = std::max(1, std::min(div_up(4L * T, 256), kSMs * 8));
        k_fem_count<<<g, 256, 0, s>>>(tets, T, cnt);
        STG_LAUNCH_CHECK();
        k_scan_exclusive<<<1, 1024, 0, s>>>(cnt, start, nullptr, V, start + V);
        STG_LAUNCH_CHECK();
        k_fem_fill<<<g, 256, 0, s>>>(tets, T, start, cur, inc);
        STG_LAUNCH_CHECK();
    }
    else
        STG_CUDA_TRY(cudaMemsetAsync(start, 0, sizeof(int) * (V + 1), s));
    k_fem_energy_vertex<<<gv, 256, 0, s>>>(start, inc, mt, pos, xtilde, V, planes, nplanes, part + gt, viol);
    STG_LAUNCH_CHECK();
    std::vector<double> h(gt + gv);
    int hv = 0;
    STG_CUDA_TRY(cudaMemcpyAsync(h.data(), part, sizeof(double) * (gt + gv), cudaMemcpyDeviceToHost, s));
    STG_CUDA_TRY(cudaMemcpyAsync(&hv, viol, sizeof(int), cudaMemcpyDeviceToHost, s));
    STG_CUDA_TRY(cudaStreamSynchronize(s));
    double e = 0;
    for(int i = 0; i < gt + gv; i++) e += h[i];
    *energy = e;
    if(violations) *violations = hv;
    return 0;
}

}  // namespace stg
