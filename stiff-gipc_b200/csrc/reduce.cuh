// reduce.cuh -- deterministic grid reductions finished by the last CTA, plus the PCG scalar
// updates that follow each reduction (all on the device; no host round-trip).
#pragma once
#include "common.cuh"

namespace stg
{

struct PcgParams
{
    double tol;        // stop threshold (see stop_rule)
    long max_iter;     // (long)(max_iter_ratio * n) as PCGSolver::solve computes it
    int stop_rule;     // 0: |rz| <= tol * rz0 (reference), 1: ||r|| <= tol ||b||
    int refine;        // FP32 mode residual replacement interval (0 = off)
    int judge;         // learned correction without replacements (FP64): judge the recursive
                       // FP64 residual every `judge` iterations (0 = off)
};

enum PostOp : int
{
    POST_STORE = 0,    // scal[slot] = total
    POST_INIT_RZ = 1,  // rz = rz0 = total; beta = 0
    POST_ALPHA = 2,    // pq = total; alpha = rz / pq (breakdown check)
    POST_CHECK = 3,    // rr = total; iteration k completed; stop tests
    POST_BETA = 4,     // beta = total / rz; rz = total
    POST_RECHECK = 5,  // rr = total after residual replacement; stop test only
    POST_CHECK_PQ = 6  // as POST_CHECK, with p.q (aux) and r.z (aux2) finished by the
                       // consumer: rz recorded, the breakdown test of POST_ALPHA first,
                       // alpha and pq recorded
};

enum : int
{
    F_DONE = 0,        // nonzero: loop finished
    F_STATUS = 1,      // STG_OK / STG_MAX_ITER / STG_BREAKDOWN
    F_REPL = 2,        // residual replacements performed
    F_LEARN = 3,       // nonzero: the learned coarse correction is applied
    F_LACC = 4,        // replacement checkpoints the learned correction passed
    F_LREJ = 5         // checkpoints it failed (the correction is then switched off)
};

// scalar slots (mirror solver.hpp)
enum : int
{
    SS_RZ = 0, SS_RZ0 = 1, SS_PQ = 2, SS_ALPHA = 3, SS_BETA = 4, SS_RZNEW = 5, SS_RR = 6, SS_BB = 7, SS_ITER = 9,
    SS_LRR = 10
};

__device__ __forceinline__ void post_op(int op, int slot, double total, double* scal, int* flags, const PcgParams& p,
                                        double aux = 0.0, double aux2 = 0.0)
{
    if(op == POST_CHECK_PQ)
    {
        scal[SS_RZ] = aux2;
        scal[SS_PQ] = aux;
        if(!(aux > 0.0) || !isfinite(aux))
        {
            flags[F_DONE] = 1;
            flags[F_STATUS] = 5;  // STG_BREAKDOWN: no update was applied
            return;
        }
        scal[SS_ALPHA] = scal[SS_RZ] / aux;
        op = POST_CHECK;
    }
    switch(op)
    {
        case POST_STORE: scal[slot] = total; break;
        case POST_INIT_RZ:
            scal[SS_RZ] = total;
            scal[SS_RZ0] = total;
            scal[SS_BETA] = 0.0;
            scal[SS_ITER] = 0.0;
            scal[SS_LRR] = scal[SS_BB];
            break;
        case POST_ALPHA:
        {
            scal[SS_PQ] = total;
            if(!(total > 0.0) || !isfinite(total))
            {
                flags[F_DONE] = 1;
                flags[F_STATUS] = 5;  // STG_BREAKDOWN
            }
            else
                scal[SS_ALPHA] = scal[SS_RZ] / total;
            break;
        }
        case POST_CHECK:
        case POST_RECHECK:
        {
            scal[SS_RR] = total;
            if(op == POST_RECHECK && flags[F_LEARN])
            {
                // the FP64 residual judges the learned correction: it must have fallen since
                // the previous replacement (or since r0 = b); else plain MAS from here on
                if(total < scal[SS_LRR])
                    flags[F_LACC] += 1;
                else
                {
                    flags[F_LREJ] += 1;
                    flags[F_LEARN] = 0;
                }
            }
            if(op == POST_RECHECK) scal[SS_LRR] = total;
            long k = (long)scal[SS_ITER];
            if(op == POST_CHECK)
            {
                k += 1;
                scal[SS_ITER] = (double)k;
                if(p.judge > 0 && flags[F_LEARN] && k % p.judge == 0)
                {
                    // FP64 recurrence: its residual judges the learned correction directly
                    if(total < scal[SS_LRR])
                        flags[F_LACC] += 1;
                    else
                    {
                        flags[F_LREJ] += 1;
                        flags[F_LEARN] = 0;
                    }
                    scal[SS_LRR] = total;
                }
            }
            bool conv;
            if(p.stop_rule == 0)
                conv = fabs(scal[SS_RZ]) <= p.tol * scal[SS_RZ0];
            else
                conv = total <= p.tol * p.tol * scal[SS_BB];
            if(!isfinite(total))
            {
                flags[F_DONE] = 1;
                flags[F_STATUS] = 5;
            }
            else if(conv)
            {
                flags[F_DONE] = 1;
                flags[F_STATUS] = 0;
            }
            else if(k + 1 >= p.max_iter)
            {
                // the reference loop runs k = 1 .. max_iter-1 and returns max_iter
                scal[SS_ITER] = (double)p.max_iter;
                flags[F_DONE] = 1;
                flags[F_STATUS] = 4;  // STG_MAX_ITER
            }
            break;
        }
        case POST_BETA:
        {
            const double rz = scal[SS_RZ];
            scal[SS_RZNEW] = total;
            scal[SS_BETA] = total / rz;
            scal[SS_RZ] = total;
            break;
        }
        default: break;
    }
}

// This thread's sum of p[t] for t = threadIdx.x, threadIdx.x + BLOCK, ... < count, added in
// that order from zero.  The loads are issued four at a time before their adds: a loop that
// adds each load as it comes waits one memory round trip per term.  Adding the zeros of the
// idle slots changes no bit (a sum that starts from +0 is never -0).
template <int BLOCK>
__device__ __forceinline__ double strided_sum(const double* p, int count)
{
    double a = 0.0;
    for(int t0 = threadIdx.x; t0 < count; t0 += 4 * BLOCK)
    {
        double v[4];
#pragma unroll
        for(int u = 0; u < 4; u++)
        {
            const int t = t0 + u * BLOCK;
            v[u] = t < count ? __ldcg(p + t) : 0.0;
        }
#pragma unroll
        for(int u = 0; u < 4; u++) a += v[u];
    }
    return a;
}

// Every CTA contributes `v` (valid in all threads; summed over the block).  The last CTA to
// arrive sums the per-CTA partials in index order and applies the post-op.  Deterministic
// for a fixed grid size.  Must be called by all threads of every CTA of the grid.
template <int BLOCK>
__device__ __forceinline__ void grid_reduce_finish(double v, double* partials, unsigned* counter, int op, int slot,
                                                   double* scal, int* flags, const PcgParams& p)
{
    __shared__ double red[BLOCK / 32];
    __shared__ bool last;
    const double bs = block_sum<BLOCK>(v, red);
    if(threadIdx.x == 0)
    {
        partials[blockIdx.x] = bs;
        __threadfence();
        const unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if(!last) return;
    __threadfence();
    const double acc = strided_sum<BLOCK>(partials, (int)gridDim.x);
    const double tot = block_sum<BLOCK>(acc, red);
    if(threadIdx.x == 0)
    {
        post_op(op, slot, tot, scal, flags, p);
        *counter = 0u;
        __threadfence();
    }
}

}  // namespace stg
