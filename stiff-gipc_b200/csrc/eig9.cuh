// eig9.cuh -- eigen-decomposition of a symmetric 9x9 matrix on the device (FP64), shared by
// the PSD projections of the tet Hessian (fem.cu) and the affine-body shape Hessian (abd.cu).
#pragma once

namespace stg
{

// eigen-decomposition of a symmetric 9x9 matrix by cyclic Jacobi rotations (FP64);
// A is overwritten (its diagonal holds the eigenvalues), V receives the eigenvectors
__device__ inline void jacobi9(double (&A)[9][9], double (&V)[9][9])
{
    for(int i = 0; i < 9; i++)
        for(int j = 0; j < 9; j++) V[i][j] = i == j ? 1.0 : 0.0;
    double norm = 0;
    for(int i = 0; i < 9; i++)
        for(int j = 0; j < 9; j++) norm += A[i][j] * A[i][j];
    for(int sweep = 0; sweep < 30; sweep++)
    {
        double off = 0;
        for(int p = 0; p < 9; p++)
            for(int q = p + 1; q < 9; q++) off += A[p][q] * A[p][q];
        if(off <= 1e-30 * norm) break;
        for(int p = 0; p < 8; p++)
            for(int q = p + 1; q < 9; q++)
            {
                const double apq = A[p][q];
                if(fabs(apq) <= 1e-300) continue;
                const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for(int k = 0; k < 9; k++)
                {
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
                for(int k = 0; k < 9; k++)
                {
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
                for(int k = 0; k < 9; k++)
                {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
}

// project a symmetric 9x9 matrix to PSD in place: negative eigenvalues clamped to zero (the
// matrix is rebuilt only when it has one)
__device__ inline void psd_project9(double (&H)[9][9])
{
    double A[9][9], V[9][9];
    for(int i = 0; i < 9; i++)
        for(int j = 0; j < 9; j++) A[i][j] = H[i][j];
    jacobi9(A, V);
    bool neg = false;
    for(int i = 0; i < 9; i++) neg |= A[i][i] < 0.0;
    if(!neg) return;
    for(int i = 0; i < 9; i++)
        for(int j = i; j < 9; j++)
        {
            double s = 0;
            for(int q = 0; q < 9; q++) s += V[i][q] * fmax(A[q][q], 0.0) * V[j][q];
            H[i][j] = s;
            H[j][i] = s;
        }
}

}  // namespace stg
