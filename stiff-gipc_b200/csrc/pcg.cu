// pcg.cu -- preconditioned conjugate gradient on sm_100a.
//
// Replaces PCGSolver::solve / pcg (StiffGIPC/linear_system/solver/pcg_solver.cu:158-332) and
// GlobalLinearSystem::apply_preconditioner (global_linear_system.cu:167-180).  Same
// recurrence and stopping rule as the reference:
//   x0 = 0, r = b, z = M^-1 r, rz = r.z, p = z, rz0 = rz
//   for k = 1 .. max_iter-1:
//       q = A p; alpha = rz / p.q; x += alpha p; r -= alpha q
//       if |rz| <= tol * rz0: break          (rz from before the update)
//       z = M^-1 r; rz_new = r.z; beta = rz_new / rz; p = z + beta p; rz = rz_new
//
// The reference runs ~8 kernels per iteration, copies each dot product to the host
// (pcg_solver.cu:148) and synchronises six times per iteration.  Here one iteration is five
// fused phases with every scalar on the device:
//   A  q = A p_new with p_new = z + beta p_old formed on the fly from the gathered z / p_old
//      (p is double-buffered, so the p update costs no pass), p.q -> alpha
//   B  x += alpha p; r -= alpha q per MAS level-0 bank, restricting r to level 0 and summing
//      each level-0 component into level 1 in the same pass; r.r -> stop test
//   C  restriction of levels >= 2 from level 1 (one CTA, level by level)
//   D  bank solves z_b = P_b r_b for every bank of every level
//   E  prolongation z = sum_l P_l z_l (+ ABD 12x12 block-Jacobi), r.z -> beta
// (non-MAS preconditioners: B is a plain axpy, C/D vanish, E applies block-Jacobi/identity).
// Every reduction is finished by the last CTA in a fixed order (deterministic).  In FP32 mode
// every `refine` iterations r is recomputed as b - A x with the FP64 blocks and restricted
// again (residual replacement).
//
// Three drivers share these phases:
//   LOOP_HOST   one launch per phase, a flag read after every iteration;
//   LOOP_GRAPH  the iteration is captured once as the body of a device-side WHILE node of a
//               CUDA graph (the replacement as an IF node); one graph launch runs the whole
//               solve, the loop condition is set by the stop test on the device;
//   LOOP_PERSISTENT  one cooperative kernel runs all iterations; phases are separated by a
//               bounded grid barrier that also finishes the reductions.
#include "solver.hpp"
#include "reduce.cuh"
#include "spmv_core.cuh"
#include "bank_dev.cuh"

#include <map>
#include <mutex>

namespace stg
{

constexpr int PB = 256;  // threads per CTA in every PCG kernel

enum Site : int
{
    SITE_A = 0,
    SITE_B = 1,
    SITE_R = 2,
    SITE_E = 3,
    SITE_INIT = 4,
    SITE_INIT_RZ = 5,
    SITE_F = 6  // r_(k+1).z_k of phase E (flexible PCG)
};
// last-CTA counters (PcgDev::counters): one per reduction site finished by its producer,
// plus the scenes' stop test (k_seg<SEG_B>)
constexpr int CNT_SEG = 6;

// ---------------------------------------------------------------------------------------
// reductions: last CTA finishes, optionally drives the graph's conditional nodes
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void set_conditionals(const PcgDev& c, int op)
{
    if(!c.use_cond) return;
    const bool done = c.flags[F_DONE] != 0;
    if(op == POST_CHECK || op == POST_RECHECK || op == POST_ALPHA) cudaGraphSetConditional(c.h_while, done ? 0u : 1u);
    if(op == POST_CHECK && c.use_cond == 2)
    {
        const long k = (long)c.scal[SS_ITER];
        const bool repl = !done && c.prm.refine > 0 && k % c.prm.refine == 0;
        cudaGraphSetConditional(c.h_if, repl ? 1u : 0u);
    }
}

template <int BLOCK = PB>
__device__ __forceinline__ void finish_reduction(const PcgDev& c, double v, int site, int op, int slot = 0,
                                                 double aux = 0.0, double aux2 = 0.0)
{
    __shared__ double red[BLOCK / 32];
    __shared__ bool last;
    double* partials = c.partials + (size_t)site * c.slots;
    unsigned* counter = c.counters + site;
    const double bs = block_sum<BLOCK>(v, red);
    if(threadIdx.x == 0)
    {
        partials[blockIdx.x] = bs;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if(!last) return;
    __threadfence();
    // The post-op reads the scalars and flags (one 128-byte line each) one after another;
    // fetched into L1 now, while the partials are summed, those reads do not wait on L2.
    // Only this CTA writes them while the kernel runs, so the L1 copies stay current.
    if(threadIdx.x == 0)
    {
        asm volatile("prefetch.global.L1 [%0];" ::"l"(c.scal));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(c.flags));
    }
    const double acc = strided_sum<BLOCK>(partials, (int)gridDim.x);
    const double tot = block_sum<BLOCK>(acc, red);
    if(threadIdx.x == 0)
    {
        post_op(op, slot, tot, c.scal, c.flags, c.prm, aux, aux2);
        set_conditionals(c, op == POST_CHECK_PQ ? (int)POST_CHECK : op);
        *counter = 0u;
        __threadfence();
    }
}

// A reduction finished by each CTA of its consumer from the producer's per-CTA partials,
// in the same fixed order in every CTA (so every CTA gets the same value): p.q of the SpMV
// phase (consumed by phase B) and r.z of phase E (consumed by the next SpMV phase for beta
// and by phase B for alpha).  The producers need no last-CTA step of their own.
template <int BLOCK>
__device__ __forceinline__ double consume_sum(const PcgDev& c, int site, int count)
{
    __shared__ double red[BLOCK / 32];
    __shared__ double tot;
    const double* part = c.partials + (size_t)site * c.slots;
    const double a = strided_sum<BLOCK>(part, count);
    const double s = block_sum<BLOCK>(a, red);
    if(threadIdx.x == 0) tot = s;
    __syncthreads();
    return tot;
}

// Two such reductions in one pass (both partial arrays loaded together, one set of
// barriers); each result is bitwise the one consume_sum gives.
template <int BLOCK>
__device__ __forceinline__ void consume_sum2(const PcgDev& c, int site_a, int count_a, int site_b, int count_b,
                                             double& ra, double& rb)
{
    __shared__ double red[2][BLOCK / 32];
    __shared__ double tot[2];
    const double* pa = c.partials + (size_t)site_a * c.slots;
    const double* pb = c.partials + (size_t)site_b * c.slots;
    double a = strided_sum<BLOCK>(pa, count_a), b = strided_sum<BLOCK>(pb, count_b);
    a = warp_sum(a);
    b = warp_sum(b);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if(lane == 0)
    {
        red[0][warp] = a;
        red[1][warp] = b;
    }
    __syncthreads();
    if(warp == 0)
    {
        double x = lane < BLOCK / 32 ? red[0][lane] : 0.0, y = lane < BLOCK / 32 ? red[1][lane] : 0.0;
        x = warp_sum(x);
        y = warp_sum(y);
        if(lane == 0)
        {
            tot[0] = x;
            tot[1] = y;
        }
    }
    __syncthreads();
    ra = tot[0];
    rb = tot[1];
}

// consume_sum2 in two steps, so that the partials' loads can be issued early and other
// work done while they are in flight: consume2_load fetches this thread's partials (at most
// K per site; the caller checks K * BLOCK against the counts), consume2_finish sums them in
// consume_sum2's order (bitwise its result).
template <int BLOCK, int K>
__device__ __forceinline__ void consume2_load(const PcgDev& c, int site_a, int count_a, int site_b, int count_b,
                                              double (&a)[K], double (&b)[K])
{
    const double* pa = c.partials + (size_t)site_a * c.slots;
    const double* pb = c.partials + (size_t)site_b * c.slots;
#pragma unroll
    for(int k = 0; k < K; k++)
    {
        const int t = threadIdx.x + k * BLOCK;
        a[k] = t < count_a ? __ldcg(pa + t) : 0.0;
        b[k] = t < count_b ? __ldcg(pb + t) : 0.0;
    }
}

template <int BLOCK, int K>
__device__ __forceinline__ void consume2_finish(const double (&a)[K], const double (&b)[K], double& ra, double& rb)
{
    __shared__ double red[2][BLOCK / 32];
    __shared__ double tot[2];
    double x = 0, y = 0;
#pragma unroll
    for(int k = 0; k < K; k++)
    {
        x += a[k];
        y += b[k];
    }
    x = warp_sum(x);
    y = warp_sum(y);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if(lane == 0)
    {
        red[0][warp] = x;
        red[1][warp] = y;
    }
    __syncthreads();
    if(warp == 0)
    {
        double u = lane < BLOCK / 32 ? red[0][lane] : 0.0, v = lane < BLOCK / 32 ? red[1][lane] : 0.0;
        u = warp_sum(u);
        v = warp_sum(v);
        if(lane == 0)
        {
            tot[0] = u;
            tot[1] = v;
        }
    }
    __syncthreads();
    ra = tot[0];
    rb = tot[1];
}

// ---------------------------------------------------------------------------------------
// block loads (16-byte vector loads of the padded layouts)
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void load_block(const float* base, size_t k, float h[9])
{
    const float4* p = reinterpret_cast<const float4*>(base) + 3 * k;
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    h[0] = a.x; h[1] = a.y; h[2] = a.z; h[3] = a.w;
    h[4] = b.x; h[5] = b.y; h[6] = b.z; h[7] = b.w;
    h[8] = c.x;
}

__device__ __forceinline__ void load_block(const double* base, size_t k, double h[9])
{
    const double2* p = reinterpret_cast<const double2*>(base) + 5 * k;
    const double2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3), e = __ldg(p + 4);
    h[0] = a.x; h[1] = a.y; h[2] = b.x; h[3] = b.y; h[4] = c.x; h[5] = c.y; h[6] = d.x; h[7] = d.y;
    h[8] = e.x;
}

// acc += H x (trans: H^T x); h column-major
template <typename T>
__device__ __forceinline__ void mv3(const T h[9], bool trans, T x0, T x1, T x2, T& a0, T& a1, T& a2)
{
    const T h01 = trans ? h[1] : h[3], h10 = trans ? h[3] : h[1];
    const T h02 = trans ? h[2] : h[6], h20 = trans ? h[6] : h[2];
    const T h12 = trans ? h[5] : h[7], h21 = trans ? h[7] : h[5];
    a0 += h[0] * x0 + h01 * x1 + h02 * x2;
    a1 += h10 * x0 + h[4] * x1 + h12 * x2;
    a2 += h20 * x0 + h21 * x1 + h[8] * x2;
}

// Row i of A * v with v_j = z_j + beta p_j gathered from the interleaved zp slots (x_plain:
// a plain [3n] FP64 vector instead, for the residual replacement).  LPR lanes per row,
// warp-wide shuffles: every lane of the warp must call it.
template <typename T, int LPR>
__device__ __forceinline__ void row_spmv_zp(const PcgDev& c, const T* blk, int i, bool valid, int sub, const T* zp,
                                            T beta, const double* x_plain, T& a0, T& a1, T& a2)
{
    a0 = a1 = a2 = T(0);
    int u0 = 0, nu = 0, t0 = 0, nt = 0;
    if(valid)
    {
        u0 = __ldg(c.row_ptr + i);
        nu = __ldg(c.row_ptr + i + 1) - u0;
        t0 = __ldg(c.t_ptr + i);
        nt = __ldg(c.t_ptr + i + 1) - t0;
    }
    for(int e = sub; e < nu + nt; e += LPR)
    {
        int k, j;
        const bool trans = e >= nu;
        if(!trans)
        {
            k = u0 + e;
            j = __ldg(c.cols + k);
        }
        else
        {
            const int2 te = __ldg(c.t_ent + t0 + e - nu);
            k = te.x;
            j = te.y;
        }
        T h[9];
        load_block(blk, (size_t)k, h);
        T x0, x1, x2;
        if(x_plain)
        {
            x0 = (T)x_plain[3 * j];
            x1 = (T)x_plain[3 * j + 1];
            x2 = (T)x_plain[3 * j + 2];
        }
        else
        {
            T p0, p1, p2;
            ld4(zp + 8 * (size_t)j, x0, x1, x2);
            ld4(zp + 8 * (size_t)j + 4, p0, p1, p2);
            x0 += beta * p0;
            x1 += beta * p1;
            x2 += beta * p2;
        }
        mv3<T>(h, trans, x0, x1, x2, a0, a1, a2);
    }
#pragma unroll
    for(int o = LPR / 2; o > 0; o >>= 1)
    {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
}

// Row i of A * (z + beta p) on the full symmetric plane copy (untiled phase A).  LPR lanes
// per row, warp-wide shuffles: every lane of the warp must call it.
template <typename T, int LPR>
__device__ __forceinline__ void row_spmv_full(const PcgDev& c, int i, bool valid, int sub, const T* zp, T beta, T& a0,
                                              T& a1, T& a2)
{
    a0 = a1 = a2 = T(0);
    int f0 = 0, deg = 0;
    if(valid)
    {
        f0 = __ldg(c.frow + i);
        deg = __ldg(c.frow + i + 1) - f0;
    }
    for(int e = sub; e < deg; e += LPR)
    {
        int j;
        T h[9];
        ldg_entry(c.fent, c.fstride, f0 + e, h, j);
        T x0, x1, x2, p0, p1, p2;
        ld4(zp + 8 * (size_t)j, x0, x1, x2);
        ld4(zp + 8 * (size_t)j + 4, p0, p1, p2);
        x0 += beta * p0;
        x1 += beta * p1;
        x2 += beta * p2;
        mv3<T>(h, false, x0, x1, x2, a0, a1, a2);
    }
#pragma unroll
    for(int o = LPR / 2; o > 0; o >>= 1)
    {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
}

// ---------------------------------------------------------------------------------------
// phases (gt / gn: this thread's index and the thread count of the grid)
// ---------------------------------------------------------------------------------------
// zp buffer parity: phase A of iteration k runs with ITER = k-1 and reads zp[(k-1)&1]
// (z_{k-1}, p_{k-1}), writing p_k into zp[k&1]; B reads p_k there; E (ITER = k) writes z_k
// into zp[k&1] too, which phase A of iteration k+1 reads.
template <typename T>
__device__ __forceinline__ T* zpbuf(const PcgDev& c, int parity)
{
    return reinterpret_cast<T*>(parity ? c.zp1 : c.zp0);
}
// scalars are read with ld.global.cg: in the persistent kernel they change between phases
__device__ __forceinline__ int iter_parity(const PcgDev& c) { return ((long)__ldcg(c.scal + SS_ITER)) & 1; }

// A: q = A p_new, p_new = z + beta p_old; returns this thread's share of p_new . q
template <typename T>
__device__ __forceinline__ double phase_a(const PcgDev& c, int gt, int gn)
{
    constexpr int LPR = 16, RPW = 32 / LPR;
    const int par = iter_parity(c);
    const T* zp = zpbuf<T>(c, par);
    T* zpn = zpbuf<T>(c, par ^ 1);
    T* q = reinterpret_cast<T*>(c.q);
    const T beta = (T)__ldcg(c.scal + SS_BETA);
    const int warp = gt >> 5, nwarps = gn >> 5, lane = gt & 31, sub = lane & (LPR - 1);
    double acc = 0;
    for(int base = warp * RPW; base < c.nrows; base += nwarps * RPW)
    {
        const int i = base + lane / LPR;
        const bool valid = i < c.nrows;
        T a0, a1, a2;
        row_spmv_full<T, LPR>(c, i, valid, sub, zp, beta, a0, a1, a2);
        if(valid && sub == 0)
        {
            T z0, z1, z2, p0, p1, p2;
            ld4(zp + 8 * (size_t)i, z0, z1, z2);
            ld4(zp + 8 * (size_t)i + 4, p0, p1, p2);
            p0 = z0 + beta * p0;
            p1 = z1 + beta * p1;
            p2 = z2 + beta * p2;
            st4(zpn + 8 * (size_t)i + 4, p0, p1, p2);
            st4(q + 4 * (size_t)i, a0, a1, a2);
            acc += (double)p0 * (double)a0 + (double)p1 * (double)a1 + (double)p2 * (double)a2;
        }
    }
    return acc;
}

// The transposed products H_k^T p_row(k) that the upper SpMV phase spilled for row i (slots
// t0 .. t1 of its transpose list), added to q_i in list order: a fixed order, so the sum is
// deterministic.  SPB slots are loaded at a time, all loads of a batch before the first add.
constexpr int SPB = 8;
template <typename T>
__device__ __forceinline__ void spill_add(const PcgDev& c, int t0, int t1, T& q0, T& q1, T& q2)
{
    const T* sp = reinterpret_cast<const T*>(c.spill);
    for(int tb = t0; tb < t1; tb += SPB)
    {
        T a[SPB][3];
#pragma unroll
        for(int u = 0; u < SPB; u++)
        {
            a[u][0] = a[u][1] = a[u][2] = T(0);
            if(tb + u < t1) ld4(sp + 4 * (size_t)(tb + u), a[u][0], a[u][1], a[u][2]);
        }
#pragma unroll
        for(int u = 0; u < SPB; u++)
            if(tb + u < t1)
            {
                q0 += a[u][0];
                q1 += a[u][1];
                q2 += a[u][2];
            }
    }
}

// q_i of the SpMV phase: after the upper kernel (c.spill set) q holds the upper part of the
// row, and its spilled products are added here
template <typename T>
__device__ __forceinline__ void load_q(const PcgDev& c, const T* q, size_t i, T& q0, T& q1, T& q2)
{
    ld4(q + 4 * i, q0, q1, q2);
    if(c.spill) spill_add<T>(c, __ldg(c.t_ptr + i), __ldg(c.t_ptr + i + 1), q0, q1, q2);
}

// B (MAS): axpy over the FEM range in level-0 slot order + level-0/1 restriction; plain axpy
// over the ABD range.  Returns this thread's share of r.r.
// x_i += alpha p_i; r_i -= alpha q_i for block row i (3 dofs); returns the new r_i and adds
// its squared norm to acc
template <typename T>
__device__ __forceinline__ void axpy_row(const PcgDev& c, const T* pn, const T* q, double alpha, int i, double& r0,
                                         double& r1, double& r2, double& acc)
{
    T p0, p1, p2, q0, q1, q2;
    ld4(pn + 8 * (size_t)i + 4, p0, p1, p2);
    load_q<T>(c, q, (size_t)i, q0, q1, q2);
    double* x = c.x + 3 * (size_t)i;
    double* r = c.r + 3 * (size_t)i;
    x[0] += alpha * (double)p0;
    x[1] += alpha * (double)p1;
    x[2] += alpha * (double)p2;
    r0 = r[0] - alpha * (double)q0;
    r1 = r[1] - alpha * (double)q1;
    r2 = r[2] - alpha * (double)q2;
    r[0] = r0;
    r[1] = r1;
    r[2] = r2;
    acc += r0 * r0 + r1 * r1 + r2 * r2;
}

// One level-0 slot of phase B (MAS): its row's p, q, x, r, closed mask and level-1 parent,
// loaded before alpha is known (the loads do not depend on it), and after the upper SpMV the
// bounds of its row's spilled products (loaded and added to q when the slot is updated)
template <typename T>
struct BSlot
{
    int v = -1;
    T p[3], q[3];
    double x[3], r[3];
    unsigned msk = 0u;
    int gnext = 0;
    int t0 = 0, t1 = 0;
};

// SPILL: q may need the upper SpMV's spilled products (the persistent kernel never runs that
// SpMV and compiles without the loop: with it, ptxas 12.9 for sm_100a aborts on that kernel)
template <typename T, bool SPILL = true>
__device__ __forceinline__ void b_load(const PcgDev& c, const T* pn, const T* q, int s, BSlot<T>& L)
{
    L.v = c.identity ? (s < c.V ? s : -1) : (s < c.M ? c.part_map[s] : -1);
    if(L.v < 0) return;
    const size_t row = (size_t)(c.fem_dof / 3) + L.v;
    ld4(pn + 8 * row + 4, L.p[0], L.p[1], L.p[2]);
    ld4(q + 4 * row, L.q[0], L.q[1], L.q[2]);
    if constexpr(SPILL)
    {
        if(c.spill)
        {
            L.t0 = __ldg(c.t_ptr + row);
            L.t1 = __ldg(c.t_ptr + row + 1);
        }
    }
#pragma unroll
    for(int d = 0; d < 3; d++)
    {
        L.x[d] = c.x[3 * row + d];
        L.r[d] = c.r[3 * row + d];
    }
    L.msk = c.fine_mask[L.v];
    L.gnext = c.going_next[L.v];
}

// x_i += alpha p_i, r_i -= alpha q_i of the slot, the level-0 residual slot and the level-0 ->
// 1 restriction (each component of a level-0 bank sums its members in lane order); every lane
// of the warp calls it (group shuffles).  Returns the slot's |r_i|^2.
// st / [slo, shi): the calling warp's staged spill slots (shared memory), or null
template <typename T, int B>
__device__ __forceinline__ double b_update(const PcgDev& c, BSlot<T>& L, int s, double alpha, const T* st = nullptr,
                                           int slo = 0, int shi = 0)
{
    float r0 = 0.f, r1 = 0.f, r2 = 0.f;
    double rr = 0.0;
    if(L.v >= 0)
    {
        const size_t row = (size_t)(c.fem_dof / 3) + L.v;
        if(L.t1 > L.t0)
        {
            if(st && L.t0 >= slo && L.t1 <= shi)
            {
                for(int t = L.t0; t < L.t1; t++)
                {
                    const T* a = st + 4 * (t - slo);
                    L.q[0] += a[0];
                    L.q[1] += a[1];
                    L.q[2] += a[2];
                }
            }
            else
                spill_add<T>(c, L.t0, L.t1, L.q[0], L.q[1], L.q[2]);
        }
        const double a = c.seg_of_row ? __ldcg(c.seg + SEG_N * c.seg_of_row[row] + SG_ALPHA) : alpha;
#pragma unroll
        for(int d = 0; d < 3; d++)
        {
            L.x[d] = fma(a, (double)L.p[d], L.x[d]);
            L.r[d] = fma(-a, (double)L.q[d], L.r[d]);
            c.x[3 * row + d] = L.x[d];
            c.r[3 * row + d] = L.r[d];
        }
        rr = fma(L.r[2], L.r[2], fma(L.r[1], L.r[1], L.r[0] * L.r[0]));
        if(c.seg_of_row) c.seg_row[(size_t)c.nrows + row] = rr;
        r0 = (float)L.r[0];
        r1 = (float)L.r[1];
        r2 = (float)L.r[2];
    }
    if(s < c.M) st4(c.R + 4 * (size_t)s, r0, r1, r2);
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
    for(int bb = 0; bb < B; bb++)
    {
        const float x0 = group_shfl<B>(r0, bb);
        const float x1 = group_shfl<B>(r1, bb);
        const float x2 = group_shfl<B>(r2, bb);
        if(L.msk & (1u << bb))
        {
            a0 += x0;
            a1 += x1;
            a2 += x2;
        }
    }
    if(L.v >= 0 && __popc(L.msk & lanemask_lt(s % B)) == 0) st4(c.R + 4 * (size_t)L.gnext, a0, a1, a2);
    return rr;
}

// B (MAS): x / r update over the FEM range in level-0 slot order + level-0/1 restriction;
// plain axpy over the ABD range.  `first` (with have_first): slot gt's loads, issued by the
// caller before alpha was known.  Returns this thread's share of r.r.
template <typename T, int B, bool SPILL = true>
__device__ __forceinline__ double phase_b_mas(const PcgDev& c, int gt, int gn, double alpha, BSlot<T>& first,
                                              bool have_first, const T* st = nullptr, int slo = 0, int shi = 0)
{
    const T* pn = zpbuf<T>(c, iter_parity(c) ^ 1);
    const T* q = reinterpret_cast<const T*>(c.q);
    double acc = 0;
    const int span = (c.M + 31) / 32 * 32;
    int s = gt;
    if(have_first && s < span)
    {
        acc += b_update<T, B>(c, first, s, alpha, st, slo, shi);
        s += gn;
    }
    for(; s < span; s += gn)
    {
        BSlot<T> L;
        b_load<T, SPILL>(c, pn, q, s, L);
        acc += b_update<T, B>(c, L, s, alpha);
    }
    for(int i = gt; i < c.abd_bodies * 4; i += gn)
    {
        double d0, d1, d2;
        axpy_row<T>(c, pn, q, alpha, i, d0, d1, d2, acc);
    }
    return acc;
}

// B (block-Jacobi / identity): plain axpy over all block rows
template <typename T>
__device__ __forceinline__ double phase_b_plain(const PcgDev& c, int gt, int gn, double alpha)
{
    const T* pn = zpbuf<T>(c, iter_parity(c) ^ 1);
    const T* q = reinterpret_cast<const T*>(c.q);
    double acc = 0;
    for(int i = gt; i < c.nrows; i += gn)
    {
        double d0, d1, d2;
        const double a = c.seg_of_row ? __ldcg(c.seg + SEG_N * c.seg_of_row[i] + SG_ALPHA) : alpha;
        axpy_row<T>(c, pn, q, a, i, d0, d1, d2, acc);
        if(c.seg_of_row) c.seg_row[(size_t)c.nrows + i] = d0 * d0 + d1 * d1 + d2 * d2;
    }
    return acc;
}

// residual replacement: r = b - A x with the FP64 blocks; returns the share of r.r
__device__ __forceinline__ double phase_replace(const PcgDev& c, int gt, int gn)
{
    constexpr int LPR = 16, RPW = 32 / LPR;
    const int warp = gt >> 5, nwarps = gn >> 5, lane = gt & 31, sub = lane & (LPR - 1);
    const double* blk = reinterpret_cast<const double*>(c.blk64);
    double acc = 0;
    for(int base = warp * RPW; base < c.nrows; base += nwarps * RPW)
    {
        const int i = base + lane / LPR;
        const bool valid = i < c.nrows;
        double a0, a1, a2;
        row_spmv_zp<double, LPR>(c, blk, i, valid, sub, nullptr, 0.0, c.x, a0, a1, a2);
        if(valid && sub < 3)
        {
            const int d = 3 * i + sub;
            const double ri = c.b[d] - (sub == 0 ? a0 : (sub == 1 ? a1 : a2));
            c.r[d] = ri;
            acc += ri * ri;
        }
    }
    return acc;
}

// level 0/1 restriction alone (after a residual replacement)
template <int B>
__device__ __forceinline__ void phase_restrict01(const PcgDev& c, int gt, int gn)
{
    const int span = (c.M + 31) / 32 * 32;
    for(int s = gt; s < span; s += gn)
    {
        const int v = s < c.M ? c.part_map[s] : -1;
        float r0 = 0.f, r1 = 0.f, r2 = 0.f;
        unsigned msk = 0;
        if(v >= 0)
        {
            const int d = c.fem_dof + 3 * v;
            r0 = (float)c.r[d];
            r1 = (float)c.r[d + 1];
            r2 = (float)c.r[d + 2];
            msk = c.fine_mask[v];
        }
        // the bank's values through shared memory (same lane-order sums as the shuffle form in
        // phase_b_mas); this kernel runs at set-up and after residual replacements only
        __shared__ float sv[PB * 3];
        const int w0 = (threadIdx.x & ~(B - 1)) * 3;
        sv[3 * threadIdx.x] = r0;
        sv[3 * threadIdx.x + 1] = r1;
        sv[3 * threadIdx.x + 2] = r2;
        __syncwarp();
        if(s < c.M)
        {
            st4(c.R + 4 * (size_t)s, r0, r1, r2);
        }
        const int lane = s % B;
        if(v >= 0 && __popc(msk & lanemask_lt(lane)) == 0)
        {
            float a0 = 0.f, a1 = 0.f, a2 = 0.f;
            for(int bb = 0; bb < B; bb++)
                if(msk & (1u << bb))
                {
                    a0 += sv[w0 + 3 * bb];
                    a1 += sv[w0 + 3 * bb + 1];
                    a2 += sv[w0 + 3 * bb + 2];
                }
            const int g = c.going_next[v];
            st4(c.R + 4 * (size_t)g, a0, a1, a2);
        }
        __syncwarp();
    }
}

// C: restriction level l -> l+1 for l in [l0, l1): each component of a level-l bank sums its
// nodes in lane order.  Threads gt, gt+gn, ... of the caller; the caller separates levels
// (C1: level 1 -> 2 over the whole grid; C2: levels >= 2 inside one CTA, which passes
// block_sync = true).
template <int B>
__device__ __forceinline__ void restrict_level(const PcgDev& c, int number, int begin, int gt, int gn,
                                               bool skip_stores = false)
{
    const int span = (number + 31) / 32 * 32;
    for(int i = gt; i < span; i += gn)
    {
        const bool valid = i < number;
        float r0 = 0.f, r1 = 0.f, r2 = 0.f;
        unsigned msk = 0;
        if(valid)
        {
            ld4(c.R + 4 * (size_t)(begin + i), r0, r1, r2);
            msk = c.closed[begin + i];
        }
        float a0 = 0.f, a1 = 0.f, a2 = 0.f;
        // partial unroll: full unrolling of this loop makes ptxas 12.9 (sm_100a) abort
#pragma unroll 4
        for(int bb = 0; bb < B; bb++)
        {
            const float x0 = group_shfl<B>(r0, bb);
            const float x1 = group_shfl<B>(r1, bb);
            const float x2 = group_shfl<B>(r2, bb);
            if(msk & (1u << bb))
            {
                a0 += x0;
                a1 += x1;
                a2 += x2;
            }
        }
        if(valid && !skip_stores && __popc(msk & lanemask_lt(i % B)) == 0)
        {
            const int g = c.going_next[begin + i];
            st4(c.R + 4 * (size_t)g, a0, a1, a2);
        }
    }
}

template <int B>
__device__ __forceinline__ void phase_c(const PcgDev& c, int l0, int l1, int gt, int gn, bool block_sync)
{
    for(int level = l0; level < l1 && level < c.L - 1; level++)
    {
        restrict_level<B>(c, __ldg(c.ls_dev + 2 * level), __ldg(c.ls_dev + 2 * level + 1), gt, gn);
        if(block_sync) __syncthreads();
    }
}

// D: bank solves for banks b0, b0 + bstep, ... < b1, with the arithmetic of bank_dev.cuh.
// B = 16: the CTA's eight warps take one bank each per pass (warp w the w-th bank of the
// pass), the packed inverse (4,896 B) and residual slots staged per warp with 16-byte loads.
// B = 32: one bank per pass of the CTA (PB = 256 threads, 4 (row, col) pairs each).
template <int B>
__device__ __forceinline__ void phase_d(const PcgDev& c, int b0, int b1, int bstep)
{
    if constexpr(B == 16)
    {
        constexpr int W = PB / 32;
        __shared__ __align__(16) float P16[W][136 * 9];
        __shared__ float4 r16[W][16];
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for(int bk = b0 + w * bstep; bk < b1; bk += W * bstep)
        {
            const float4* src = reinterpret_cast<const float4*>(c.inv + (size_t)bk * 136 * 9);
            float4* dst = reinterpret_cast<float4*>(P16[w]);
            for(int t = lane; t < 136 * 9 / 4; t += 32) dst[t] = __ldg(src + t);
            if(lane < 16) r16[w][lane] = *reinterpret_cast<const float4*>(c.R + 4 * ((size_t)bk * 16 + lane));
            __syncwarp();
            const int a = lane & 15, h = lane >> 4;
            float z0, z1, z2;
            bank16_half(P16[w], r16[w], a, h, z0, z1, z2);
            bank16_join(z0, z1, z2);
            if(h == 0) st4(c.Z + ((size_t)bk * 16 + a) * 4, z0, z1, z2);
            __syncwarp();
        }
    }
    else
    {
        constexpr int NS = B * (B + 1) / 2;
        __shared__ __align__(16) float P[NS * 9];
        __shared__ float rr[3 * B];
        for(int bk = b0; bk < b1; bk += bstep)
        {
            const float4* src = reinterpret_cast<const float4*>(c.inv + (size_t)bk * NS * 9);
            float4* dst = reinterpret_cast<float4*>(P);
            for(int t = threadIdx.x; t < NS * 9 / 4; t += PB) dst[t] = __ldg(src + t);
            if(threadIdx.x < B) ld4(c.R + 4 * ((size_t)bk * B + threadIdx.x), rr[3 * threadIdx.x], rr[3 * threadIdx.x + 1],
                                    rr[3 * threadIdx.x + 2]);
            __syncthreads();
            constexpr int REP = (B * B + PB - 1) / PB;
#pragma unroll
            for(int rep = 0; rep < REP; rep++)
            {
                const int pair = threadIdx.x + rep * PB;
                const int a = pair / B, cc = pair % B;
                const float x0 = rr[3 * cc], x1 = rr[3 * cc + 1], x2 = rr[3 * cc + 2];
                const int lo = min(a, cc), hi = max(a, cc);
                float z0, z1, z2;
                blk_mul3(P + (B * lo - lo * (lo + 1) / 2 + hi) * 9, cc < a, x0, x1, x2, z0, z1, z2);
                warp_butterfly3(z0, z1, z2);
                if(cc == 0)
                {
                    st4(c.Z + ((size_t)bk * B + a) * 4, z0, z1, z2);
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------
// D (16-vertex banks): one warp per bank, the bank's packed inverse (136 3x3 FP32 blocks,
// 4,896 B) and its 16 residual slots (256 B) staged in shared memory by the Tensor Memory
// Accelerator (cp.async.bulk, completion on an mbarrier), double-buffered so that the copy
// of the warp's next bank overlaps the solve of the current one.  Lane (a, h) = (l & 15,
// l >> 4) forms block row a of z = P r over the column blocks cc = 8h + ((j + a) & 7),
// j < 8 (upper block (a, cc) as stored, lower ones as the transpose of (cc, a)); the two
// halves meet in one shuffle.  The rotation by a spreads a warp's block reads over the
// shared-memory banks (1.9 wavefronts per load on average, at most 2).
// ---------------------------------------------------------------------------------------
constexpr int D_WARPS = 4;                        // warps per CTA
constexpr int D_PBYTES = 136 * 9 * 4;             // packed inverse of one bank
constexpr int D_RBYTES = 16 * 16;                 // 16 float4 residual slots
constexpr int D_BUF = D_PBYTES + D_RBYTES;        // one stage (16-byte multiple)
constexpr int D_WARP_BYTES = 2 * D_BUF + 16;      // two stages + two mbarriers
constexpr unsigned long long WAIT_NS = 1000000000ull;  // every bounded wait gives up after 1 s

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

// L2 eviction priorities for the bulk copies: the SpMV phase streams about 75 MB of block
// planes per iteration, more than half of L2, which would push out the MAS bank inverses
// (38.5 MB on the 352,947-DOF cube) and the vectors that the other phases reread every
// iteration.  Its planes are copied evict-first and the inverses evict-last.
__device__ __forceinline__ unsigned long long l2_evict_first()
{
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ unsigned long long l2_evict_last()
{
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ void tma_load_1d_hint(void* dst, const void* src, unsigned bytes, unsigned bar,
                                                 unsigned long long policy)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;"
        :
        : "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(bar), "l"(policy)
        : "memory");
}

__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, unsigned bytes, unsigned bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :
                 : "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// waits for phase `parity` of the mbarrier; false when the bounded wait gave up (WAIT_NS of
// the global timer, read every 256 polls)
__device__ __noinline__ bool mbar_wait_slow(unsigned bar, unsigned parity);

__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return ok != 0;
}

// fast path inline (one poll); the timed loop out of line (inlining it into the pipelined
// kernels makes ptxas 12.9 for sm_100a abort in register allocation)
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity)
{
    return mbar_try(bar, parity) || mbar_wait_slow(bar, parity);
}

__device__ __noinline__ bool mbar_wait_slow(unsigned bar, unsigned parity)
{
    unsigned long long t0 = 0;
    for(unsigned it = 1; it != 0u; it++)  // the timer ends it; the count only bounds the loop
    {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if(ok) return true;
        if((it & 255u) == 0u)
        {
            const unsigned long long t = global_ns();
            if(t0 == 0)
                t0 = t;
            else if(t - t0 > WAIT_NS)
                return false;
        }
    }
    return false;
}

__device__ __forceinline__ void d16_issue(const PcgDev& c, char* stage, unsigned bar, int bk)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"((unsigned)D_BUF) : "memory");
    const unsigned long long keep = l2_evict_last();
    tma_load_1d_hint(stage, c.inv + (size_t)bk * 136 * 9, D_PBYTES, bar, keep);
    tma_load_1d_hint(stage + D_PBYTES, c.R + (size_t)bk * 16 * 4, D_RBYTES, bar, keep);
}

// Banks [b0, b1).  guarded: only on residual-replacement iterations (host loop).
__global__ void __launch_bounds__(D_WARPS * 32) k_phase_d16(PcgDev c, int b0, int b1, int guarded)
{
    // the stop flag (and the replacement test) are loaded with the first bank's copy in
    // flight, not before it: their latency overlaps the copy's
    const int done = __ldcg(c.flags + F_DONE);
    const long k_it = guarded ? (long)__ldcg(c.scal + SS_ITER) : 0;
    extern __shared__ __align__(128) char dsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    char* base = dsm + (size_t)warp * D_WARP_BYTES;
    char* const stage0 = base;
    char* const stage1 = base + D_BUF;
    const unsigned bar0 = smem_u32(base + 2 * D_BUF), bar1 = bar0 + 8;
    const int gw = b0 + blockIdx.x * D_WARPS + warp, nw = gridDim.x * D_WARPS;
    if(gw >= b1) return;
    // this lane's eight blocks: word offset of block k in the packed upper order and
    // whether it is used transposed (the stored block is (cc, a) with cc < a)
    const int a = lane & 15, h = lane >> 4;
    int koff[8], rcol[8];
    unsigned tmask = 0u;
#pragma unroll
    for(int j = 0; j < 8; j++)
    {
        const int cc = 8 * h + ((j + a) & 7);
        const int lo = min(a, cc), hi = max(a, cc);
        koff[j] = 9 * (lo * 16 - lo * (lo - 1) / 2 + (hi - lo));
        rcol[j] = 4 * cc;
        if(cc < a) tmask |= 1u << j;
    }
    if(lane == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        d16_issue(c, stage0, bar0, gw);
    }
    __syncwarp();
    if(done || (guarded && (c.prm.refine <= 0 || k_it % c.prm.refine != 0)))
    {
        // nothing to solve: let the first copy land before the warp's shared memory goes
        if(lane == 0) mbar_wait(bar0, 0u);
        return;
    }
    unsigned ph0 = 0u, ph1 = 0u;
    int buf = 0;
    for(int bk = gw; bk < b1; bk += nw, buf ^= 1)
    {
        char* const cur = buf ? stage1 : stage0;
        const unsigned bcur = buf ? bar1 : bar0, bnext = buf ? bar0 : bar1;
        // prefetch the next bank into the other stage (its previous contents are consumed)
        const int nxt = bk + nw;
        if(lane == 0 && nxt < b1)
        {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            d16_issue(c, buf ? stage0 : stage1, bnext, nxt);
        }
        if(!__all_sync(0xffffffffu, mbar_wait(bcur, buf ? ph1 : ph0)))
        {
            if(lane == 0)
            {
                atomicExch(c.flags + F_STATUS, 6);  // STG_ERR_TIMEOUT
                atomicExch(c.flags + F_DONE, 1);
            }
            // let any copy still in flight land before the CTA's shared memory is released
            if(nxt < b1) mbar_wait(bnext, buf ? ph0 : ph1);
            return;
        }
        if(buf)
            ph1 ^= 1u;
        else
            ph0 ^= 1u;
        const float* P = reinterpret_cast<const float*>(cur);
        const float* rs = reinterpret_cast<const float*>(cur + D_PBYTES);
        // bank16_half's order with the block offsets precomputed (bank_dev.cuh)
        float z0 = 0.f, z1 = 0.f, z2 = 0.f;
#pragma unroll
        for(int j = 0; j < 8; j++)
        {
            const float4 r = *reinterpret_cast<const float4*>(rs + rcol[j]);
            blk_fma3(P + koff[j], (tmask >> j) & 1u, r.x, r.y, r.z, z0, z1, z2);
        }
        bank16_join(z0, z1, z2);
        if(h == 0) st4(c.Z + ((size_t)bk * 16 + a) * 4, z0, z1, z2);
        __syncwarp();
    }
}

// 16-byte asynchronous copy global -> shared (L2 only)
__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// ---------------------------------------------------------------------------------------
// A, tiled: the SpMV phase with its matrix stream staged in shared memory by the Tensor
// Memory Accelerator.  Each CTA owns a contiguous, balanced range of rows, cut into tiles of
// RT rows (64 FP32, 32 FP64).  A tile's entries are one contiguous range [frow[r0], frow[r1])
// of every plane of the full copy (FullPlanes), so one producer lane moves a whole tile with
// one bulk copy per plane, plus one for the tile's row bounds, into a ring of stages that
// complete on per-stage mbarriers.  Eight consumer warps compute the tile from shared memory
// (16-byte loads) with LPR lanes per row (4 FP32, 8 FP64): lane `sub`
// sums the entries sub, sub + LPR, ... of its row in order, four at a time with their
// neighbour gathers of z / p issued before the block values are read, and an xor tree over
// the LPR lanes finishes the row.  A tile with more entries than a stage holds is computed
// from global memory (only its row bounds are copied).  Every wait is bounded; a wait that
// gives up sets STG_ERR_TIMEOUT and the kernel drains its copies in flight before returning.
// ---------------------------------------------------------------------------------------
constexpr int A_CW = 8;            // consumer warps
constexpr int A_THREADS = (A_CW + 1) * 32;

// Tile shapes of the SpMV phase: rows per tile x lanes per row = 8 warps x 32.  The
// default for each precision is the first of its candidates; the autotuner may pick the
// other (Solver::spmv_rt).
template <typename T> constexpr int a_rt_default() { return sizeof(T) == 4 ? 64 : 32; }
constexpr int SPMV_HALO = -2;   // stg_spmv_tiles value selecting the halo kernel
constexpr int SPMV_UPPER = -3;  // stg_spmv_tiles value selecting the upper kernel

// The autotuner's choices, one per shape class (precision, block rows, unique blocks) for
// the whole process: the first handle that meets a class times the candidates, every later
// solve of that class reuses the choice, so results stay reproducible within the process.
struct TuneKey
{
    int prec, nrows, nnzb;
    bool operator<(const TuneKey& o) const
    {
        return prec != o.prec ? prec < o.prec : (nrows != o.nrows ? nrows < o.nrows : nnzb < o.nnzb);
    }
};
struct TuneVal
{
    int pick;
    float us[4];
};
static std::mutex g_tune_mu;
static std::map<TuneKey, TuneVal> g_tune;

static bool tuned_choice(int prec, int nrows, int nnzb, int* pick, float* us)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    const auto it = g_tune.find(TuneKey{prec, nrows, nnzb});
    if(it == g_tune.end()) return false;
    *pick = it->second.pick;
    for(int i = 0; i < 4; i++) us[i] = it->second.us[i];
    return true;
}

static void record_choice(int prec, int nrows, int nnzb, int pick, const float* us)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    TuneVal v{pick, {us[0], us[1], us[2], us[3]}};
    g_tune[TuneKey{prec, nrows, nnzb}] = v;
}
template <typename T> constexpr int a_rt_alt() { return sizeof(T) == 4 ? 32 : 16; }

template <typename T, int RT_ = a_rt_default<T>()>
struct ATile
{
    using FP = FullPlanes<T>;
    static constexpr int RT = RT_;                               // rows per tile
    static constexpr int LPR = 32 * A_CW / RT;                   // consumer lanes per row
    static constexpr int CAP = 20 * RT;                          // entries per stage (even)
    static constexpr int STAGES = 2;
    static constexpr int FROW = 4 * (RT + 4);                    // frow[r0 .. r0 + RT + 4)
    static constexpr int STAGE = CAP * FP::ES + FROW;            // planes + row bounds
    static constexpr int META = 16 * STAGES;                     // per stage: {F0a, overflow}
    static constexpr int BARS = 16 * STAGES;                     // full[s], empty[s]
    static constexpr int SMEM = STAGES * STAGE + META + BARS;
    static constexpr int MIN_CTAS = 2;                           // resident CTAs per SM
};

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// shared-memory loads by 32-bit shared address
__device__ __forceinline__ int lds_s32(unsigned a)
{
    int v;
    asm volatile("ld.shared.b32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}

// entry f of a stage's planes (CAP entries per plane) at shared address sb: the tail
// {h8, col} and the eight other values, loaded separately so that the neighbour gather can
// be issued before the bulk of the block is read
template <int CAP>
__device__ __forceinline__ void lds_tail(unsigned sb, int f, float& h8, int& col)
{
    unsigned tc;
    asm volatile("ld.shared.v2.b32 {%0, %1}, [%2];" : "=f"(h8), "=r"(tc) : "r"(sb + 32u * CAP + 8u * f));
    col = (int)tc;
}
template <int CAP>
__device__ __forceinline__ void lds_tail(unsigned sb, int f, double& h8, int& col)
{
    unsigned long long tc;
    asm volatile("ld.shared.v2.b64 {%0, %1}, [%2];" : "=d"(h8), "=l"(tc) : "r"(sb + 64u * CAP + 16u * f));
    col = (int)tc;
}
template <int CAP>
__device__ __forceinline__ void lds_main(unsigned sb, int f, float h[9])
{
    const unsigned a0 = sb + 16u * f, a1 = sb + 16u * CAP + 16u * f;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(h[0]), "=f"(h[1]), "=f"(h[2]), "=f"(h[3]) : "r"(a0));
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(h[4]), "=f"(h[5]), "=f"(h[6]), "=f"(h[7]) : "r"(a1));
}
template <int CAP>
__device__ __forceinline__ void lds_main(unsigned sb, int f, double h[9])
{
#pragma unroll
    for(int p = 0; p < 4; p++)
        asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];"
                     : "=d"(h[2 * p]), "=d"(h[2 * p + 1])
                     : "r"(sb + 16u * p * CAP + 16u * f));
}

// a row's whole zp slot {z0 z1 z2 -, p0 p1 p2 -} in one 32-byte load (FP32) or two (FP64)
// (sm_100 256-bit vector loads; the slots are 32- / 64-byte aligned): a neighbour gather is
// one L1 wavefront per lane instead of two (FP32) or four (FP64)
__device__ __forceinline__ void ld_zp(const float* a, float& z0, float& z1, float& z2, float& p0, float& p1, float& p2)
{
    float w0, w1;
    asm("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(z0), "=f"(z1), "=f"(z2), "=f"(w0), "=f"(p0), "=f"(p1), "=f"(p2), "=f"(w1)
        : "l"(a));
    (void)w0;
    (void)w1;
}
__device__ __forceinline__ void ld_zp(const double* a, double& z0, double& z1, double& z2, double& p0, double& p1,
                                      double& p2)
{
    double w0, w1;
    asm("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(z0), "=d"(z1), "=d"(z2), "=d"(w0) : "l"(a));
    asm("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(p0), "=d"(p1), "=d"(p2), "=d"(w1) : "l"(a + 4));
    (void)w0;
    (void)w1;
}

// v_j = z_j + beta p_j gathered from the zp slots
template <typename T>
__device__ __forceinline__ void a_gather(int j, const T* zp, T beta, T& x0, T& x1, T& x2)
{
    T p0, p1, p2;
    ld_zp(zp + 8 * (size_t)j, x0, x1, x2, p0, p1, p2);
    x0 += beta * p0;
    x1 += beta * p1;
    x2 += beta * p2;
}

template <typename T, int RTT>
__global__ void __launch_bounds__(A_THREADS, ATile<T, RTT>::MIN_CTAS) k_phase_a_tiled(PcgDev c)
{
    using G = ATile<T, RTT>;
    using FP = FullPlanes<T>;
    constexpr int RT = G::RT, LPR = G::LPR, CAP = G::CAP;
    extern __shared__ __align__(128) unsigned char asm_[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // this CTA's rows: a contiguous range [rb, re) of about nrows / gridDim.x rows (starts
    // are multiples of 4, so that every tile's row-bound copy is 16-byte aligned), cut into
    // tiles of RT rows: tile k is [rb + k RT, min(rb + (k + 1) RT, re))
    auto range_start = [&](long long b) -> int {
        return b == 0 ? 0 : (b >= gridDim.x ? c.nrows : (int)((b * c.nrows / gridDim.x) & ~3LL));
    };
    const int rb = range_start(blockIdx.x), re = range_start(blockIdx.x + 1LL);
    const int mine = re > rb ? (re - rb + RT - 1) / RT : 0;
    // the loads the start depends on are independent: issue them together
    const int done = __ldcg(c.flags + F_DONE);
    const double s_iter = __ldcg(c.scal + SS_ITER), rz_old = __ldcg(c.scal + SS_RZ);
    int lo = 0, hi = 0;  // producer: entry bounds of the next 32 tiles, one per lane
    if(warp == A_CW && lane < mine)
    {
        const int r0 = rb + lane * RT;
        lo = __ldg(c.frow + r0);
        hi = __ldg(c.frow + min(r0 + RT, re));
    }
    int* meta = reinterpret_cast<int*>(asm_ + G::STAGES * G::STAGE);
    const unsigned sbase = smem_u32(asm_);
    const unsigned bar_full = smem_u32(asm_ + G::STAGES * G::STAGE + G::META);
    const unsigned bar_empty = bar_full + 8 * G::STAGES;
    if(threadIdx.x == 0)
    {
        for(int s = 0; s < G::STAGES; s++)
        {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, A_CW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // tile k into stage k % STAGES (producer lane 0): the row bounds and every plane's range
    auto issue_tile = [&](int k, int F0, int F1) {
        const int s = k % G::STAGES;
        const int F0a = F0 & ~1, n2 = ((F1 + 1) & ~1) - F0a;
        const bool ovf = n2 > CAP;
        const int nc = ovf ? 0 : n2;
        meta[4 * s] = F0a;
        meta[4 * s + 1] = ovf ? 1 : 0;
        unsigned char* st = asm_ + (size_t)s * G::STAGE;
        const unsigned bf = bar_full + 8 * s;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(bf, (unsigned)(G::FROW + nc * FP::ES));
        tma_load_1d(st + CAP * FP::ES, c.frow + rb + (size_t)k * RT, G::FROW, bf);
        if(nc)
        {
            const unsigned long long stream = l2_evict_first();
#pragma unroll 1
            for(int pl = 0; pl < FP::NP; pl++)
                tma_load_1d_hint(st + (size_t)16 * pl * CAP, c.fent + 16 * (pl * c.fstride + F0a), (unsigned)(16 * nc),
                                 bf, stream);
            tma_load_1d_hint(st + (size_t)16 * FP::NP * CAP, c.fent + 16 * FP::NP * c.fstride + (size_t)FP::TAIL * F0a,
                             (unsigned)(FP::TAIL * nc), bf, stream);
        }
    };
    // The first STAGES tiles depend neither on beta nor on the stop flag: their copies start
    // now and run while the r.z partials are summed.  A stopped solve drains them and returns.
    const int pre = min(G::STAGES, mine);
    if(warp == A_CW)
        for(int u = 0; u < pre; u++)
        {
            const int F0 = __shfl_sync(0xffffffffu, lo, u), F1 = __shfl_sync(0xffffffffu, hi, u);
            if(lane == 0) issue_tile(u, F0, F1);
        }
    // beta = rz_k / rz_(k-1): rz_k from phase E's partials, rz_(k-1) as phase B recorded it
    // (the first iteration has p_0 = 0: beta = 0)
    // flexible PCG (learned correction): beta = r_k.(z_k - z_(k-1)) / r_(k-1).z_(k-1)
    double rz_new, rz_mix = 0.0;
    if(c.flex && (long)s_iter > 0)
        consume_sum2<A_THREADS>(c, SITE_E, c.grid_e, SITE_F, c.grid_e, rz_new, rz_mix);
    else
        rz_new = consume_sum<A_THREADS>(c, SITE_E, c.grid_e);
    if(done)
    {
        if(warp == A_CW && lane == 0)
            for(int k = 0; k < pre; k++) mbar_wait(bar_full + 8 * k, 0u);
        return;
    }
    const double s_beta = (long)s_iter == 0 ? 0.0 : (rz_new - rz_mix) / rz_old;

    const int par = ((long)s_iter) & 1;
    const T* zp = zpbuf<T>(c, par);
    T* zpn = zpbuf<T>(c, par ^ 1);
    T* q = reinterpret_cast<T*>(c.q);
    const T beta = (T)s_beta;
    double acc = 0;
    bool failed = false;

    if(warp == A_CW)
    {
        // ---- producer warp: lane 0 issues, all lanes fetch the tile bounds ----
        int issued = pre;
        for(int k0 = 0; k0 < mine && !failed; k0 += 32)
        {
            if(k0 > 0)
            {
                lo = hi = 0;
                if(k0 + lane < mine)
                {
                    const int r0 = rb + (k0 + lane) * RT;
                    lo = __ldg(c.frow + r0);
                    hi = __ldg(c.frow + min(r0 + RT, re));
                }
            }
            const int cnt = min(32, mine - k0);
            for(int u = 0; u < cnt; u++)
            {
                const int F0 = __shfl_sync(0xffffffffu, lo, u), F1 = __shfl_sync(0xffffffffu, hi, u);
                const int k = k0 + u, s = k % G::STAGES;
                if(k < pre) continue;
                if(lane == 0)
                {
                    if(!mbar_wait(bar_empty + 8 * s, ((k / G::STAGES) - 1) & 1)) failed = true;
                    if(!failed)
                    {
                        issue_tile(k, F0, F1);
                        issued = k + 1;
                    }
                }
                failed = __shfl_sync(0xffffffffu, failed ? 1 : 0, 0) != 0;
                if(failed) break;
            }
        }
        if(lane == 0)
        {
            if(failed)
            {
                atomicExch(c.flags + F_STATUS, 6);  // STG_ERR_TIMEOUT
                atomicExch(c.flags + F_DONE, 1);
            }
            // drain: every issued stage's copies must have landed before the CTA exits
            for(int k = max(0, issued - G::STAGES); k < issued; k++)
                mbar_wait(bar_full + 8 * (k % G::STAGES), (k / G::STAGES) & 1);
        }
    }
    else
    {
        // ---- consumer warps: LPR lanes per row; lane `sub` of row r (tile-local) sums the
        //      entries e = sub, sub + LPR, ... of that row in order, up to four at a time ----
        // The lane whose entry is the row's diagonal block gathers v_i = z_i + beta p_i, which
        // is p_new of the row; it is shuffled to the row's first lane (a row without a
        // diagonal block gathers it there).
        const int sub = lane & (LPR - 1);
        const int rloc = warp * (32 / LPR) + lane / LPR;
        const unsigned grp = (LPR == 32 ? 0xffffffffu : ((1u << LPR) - 1u)) << (lane & ~(LPR - 1));
        for(int k = 0; k < mine; k++)
        {
            const int s = k % G::STAGES;
            const int r0 = rb + k * RT, r1 = min(r0 + RT, re);
            const int i = r0 + rloc;
            if(!__all_sync(0xffffffffu, mbar_wait(bar_full + 8 * s, (k / G::STAGES) & 1)))
            {
                failed = true;
                break;
            }
            const unsigned sb = sbase + (unsigned)(s * G::STAGE);
            const unsigned sfrow = sb + CAP * FP::ES;
            const int F0a = meta[4 * s];
            const bool ovf = meta[4 * s + 1] != 0;
            int f = 0, d = 0;
            if(i < r1)
            {
                const int x0 = lds_s32(sfrow + 4 * rloc), x1 = lds_s32(sfrow + 4 * rloc + 4);
                f = x0 - F0a;
                d = x1 - x0;
            }
            T y0 = T(0), y1 = T(0), y2 = T(0), pn0 = T(0), pn1 = T(0), pn2 = T(0);
            bool hit = false;
            // scenes: the row's own beta (its neighbours are in the same scene)
            const T bta = (c.seg_of_row && i < r1) ? (T)__ldcg(c.seg + SEG_N * c.seg_of_row[i] + SG_BETA) : beta;
            for(int e0 = sub; e0 < d; e0 += 4 * LPR)
            {
                T h8[4], x[4][3];
                int j[4];
#pragma unroll
                for(int u = 0; u < 4; u++)
                {
                    const int e = e0 + u * LPR;
                    h8[u] = T(0);
                    j[u] = 0;
                    if(e < d)
                    {
                        if(!ovf)
                            lds_tail<CAP>(sb, f + e, h8[u], j[u]);
                        else
                        {
                            T hh[9];
                            ldg_entry(c.fent, c.fstride, F0a + f + e, hh, j[u]);
                            h8[u] = hh[8];
                        }
                    }
                }
#pragma unroll
                for(int u = 0; u < 4; u++)
                    if(e0 + u * LPR < d) a_gather<T>(j[u], zp, bta, x[u][0], x[u][1], x[u][2]);
#pragma unroll
                for(int u = 0; u < 4; u++)
                {
                    const int e = e0 + u * LPR;
                    if(e < d)
                    {
                        T h[9];
                        int jj;
                        if(!ovf)
                            lds_main<CAP>(sb, f + e, h);
                        else
                            ldg_entry(c.fent, c.fstride, F0a + f + e, h, jj);
                        h[8] = h8[u];
                        mv3<T>(h, false, x[u][0], x[u][1], x[u][2], y0, y1, y2);
                        if(j[u] == i)
                        {
                            pn0 = x[u][0];
                            pn1 = x[u][1];
                            pn2 = x[u][2];
                            hit = true;
                        }
                    }
                }
            }
            __syncwarp();
            if(lane == 0) mbar_arrive(bar_empty + 8 * s);
#pragma unroll
            for(int o = LPR / 2; o > 0; o >>= 1)
            {
                y0 += __shfl_xor_sync(0xffffffffu, y0, o);
                y1 += __shfl_xor_sync(0xffffffffu, y1, o);
                y2 += __shfl_xor_sync(0xffffffffu, y2, o);
            }
            const unsigned hm = __ballot_sync(0xffffffffu, hit) & grp;
            const int src = hm ? __ffs(hm) - 1 : lane;
            T p0 = __shfl_sync(0xffffffffu, pn0, src);
            T p1 = __shfl_sync(0xffffffffu, pn1, src);
            T p2 = __shfl_sync(0xffffffffu, pn2, src);
            if(sub == 0 && i < r1)
            {
                if(!hm) a_gather<T>(i, zp, bta, p0, p1, p2);
                st4(zpn + 8 * (size_t)i + 4, p0, p1, p2);
                st4(q + 4 * (size_t)i, y0, y1, y2);
                const double pq = (double)p0 * (double)y0 + (double)p1 * (double)y1 + (double)p2 * (double)y2;
                acc += pq;
                if(c.seg_of_row) c.seg_row[i] = pq;
            }
        }
        if(failed && lane == 0)
        {
            atomicExch(c.flags + F_STATUS, 6);  // STG_ERR_TIMEOUT
            atomicExch(c.flags + F_DONE, 1);
        }
    }
    // p.q: this CTA's partial only; phase B finishes the sum (consume_sum)
    __shared__ double red[A_THREADS / 32];
    const double bs = block_sum<A_THREADS>(acc, red);
    if(threadIdx.x == 0) c.partials[(size_t)SITE_A * c.slots + blockIdx.x] = bs;
}

// ---------------------------------------------------------------------------------------
// A, upper: the SpMV phase streaming each upper block once (UpperPlanes).  The tiling, the
// bulk-copy ring and the bounded waits are those of k_phase_a_tiled, over the upper copy's
// entry ranges [row_ptr[r0], row_ptr[r1]) (rounded out to multiples of 4 entries, so that
// every plane's copy is a 16-byte multiple).  For block k of row i (column j):
//   - the row's lanes add H_k v_j to q_i in entry order (v = z + beta p gathered; v_i, which
//     every lane of the row gathers once, is p_new of the row), exactly as the full-copy
//     kernel adds its upper entries;
//   - j > i: the lane writes H_k^T v_i into the spill slot of k (its place in row j's
//     transpose list); phase B adds row j's slots to q_j in list order, so every row's sum
//     has a fixed order and the phase stays deterministic.
// q therefore holds the upper part of A p only.  p.q = p^T A p is formed from it without the
// spilled part: p^T A p = sum_i (2 v_i . (upper row i of A) v - v_i . H_ii v_i).
// ---------------------------------------------------------------------------------------
// First row of CTA b of the upper SpMV phase's G CTAs (multiples of 4, so that every tile's
// row-bound copy is 16-byte aligned); CTA b owns [a_range_start(b), a_range_start(b + 1)).
__host__ __device__ __forceinline__ int a_range_start(long long b, int G, int nrows)
{
    return b == 0 ? 0 : (b >= G ? nrows : (int)((b * nrows / G) & ~3LL));
}

template <typename T>
struct AUpper
{
    using UP = UpperPlanes<T>;
    // a row holds about half the entries of its full-copy row: two entries per lane and
    // batch, and a stage about half the size of the full-copy kernel's, so that three CTAs
    // fit per SM (72 registers per thread): the phase is latency-bound, and the third CTA
    // hides more of the gathers' latency than deeper batches or a deeper ring did
    static constexpr int RT = sizeof(T) == 4 ? 64 : 32;            // rows per tile
    static constexpr int LPR = 32 * A_CW / RT;                     // consumer lanes per row
    static constexpr int CAP = 9 * RT;                             // entries per stage (mult. of 4)
    static constexpr int UB = 2;                                   // entries per lane per batch
    static constexpr int STAGES = 2;
    static constexpr int FROW = 4 * (RT + 4);                      // row_ptr[r0 .. r0 + RT + 4)
    static constexpr int SLOT_OFF = (16 * UP::NP + UP::TAIL) * CAP;  // FP32 slot plane in a stage
    static constexpr int STAGE = CAP * UP::ES + FROW;
    static constexpr int META = 16 * STAGES;
    static constexpr int BARS = 16 * STAGES;
    static constexpr int SMEM = STAGES * STAGE + META + BARS;
    static constexpr int MIN_CTAS = 3;
    static_assert(STAGE % 16 == 0 && SLOT_OFF % 16 == 0, "stage planes must stay 16-byte aligned");
    static_assert(RT + 4 <= 136, "row-bound copies must stay inside the padded row pointers");
};

// tail {h8, col} and spill slot of stage entry f
template <int CAP, int SLOT_OFF>
__device__ __forceinline__ void lds_utail(unsigned sb, int f, float& h8, int& col, int& slot)
{
    unsigned tc;
    asm volatile("ld.shared.v2.b32 {%0, %1}, [%2];" : "=f"(h8), "=r"(tc) : "r"(sb + 32u * CAP + 8u * f));
    col = (int)tc;
    slot = lds_s32(sb + SLOT_OFF + 4u * f);
}
template <int CAP, int SLOT_OFF>
__device__ __forceinline__ void lds_utail(unsigned sb, int f, double& h8, int& col, int& slot)
{
    unsigned long long tc;
    asm volatile("ld.shared.v2.b64 {%0, %1}, [%2];" : "=d"(h8), "=l"(tc) : "r"(sb + 64u * CAP + 16u * f));
    col = (int)(unsigned)tc;
    slot = (int)(unsigned)(tc >> 32);
}

template <typename T>
__global__ void __launch_bounds__(A_THREADS, AUpper<T>::MIN_CTAS) k_phase_a_upper(PcgDev c)
{
    using G = AUpper<T>;
    using UP = UpperPlanes<T>;
    constexpr int RT = G::RT, LPR = G::LPR, CAP = G::CAP;
    extern __shared__ __align__(128) unsigned char asm_[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int rb = a_range_start(blockIdx.x, gridDim.x, c.nrows), re = a_range_start(blockIdx.x + 1LL, gridDim.x, c.nrows);
    const int mine = re > rb ? (re - rb + RT - 1) / RT : 0;
    const int done = __ldcg(c.flags + F_DONE);
    const double s_iter = __ldcg(c.scal + SS_ITER), rz_old = __ldcg(c.scal + SS_RZ);
    int lo = 0, hi = 0;  // producer: entry bounds of the next 32 tiles, one per lane
    if(warp == A_CW && lane < mine)
    {
        const int r0 = rb + lane * RT;
        lo = __ldg(c.urow + r0);
        hi = __ldg(c.urow + min(r0 + RT, re));
    }
    int* meta = reinterpret_cast<int*>(asm_ + G::STAGES * G::STAGE);
    const unsigned sbase = smem_u32(asm_);
    const unsigned bar_full = smem_u32(asm_ + G::STAGES * G::STAGE + G::META);
    const unsigned bar_empty = bar_full + 8 * G::STAGES;
    if(threadIdx.x == 0)
    {
        for(int s = 0; s < G::STAGES; s++)
        {
            mbar_init(bar_full + 8 * s, 1);
            mbar_init(bar_empty + 8 * s, A_CW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // tile k into stage k % STAGES (producer lane 0): the row bounds and every plane's range
    auto issue_tile = [&](int k, int F0, int F1) {
        const int s = k % G::STAGES;
        // 4-entry aligned range: F0a + n4 <= round_up(nnzb, 4) <= the plane stride
        const int F0a = F0 & ~3, n4 = ((F1 + 3) & ~3) - F0a;
        const bool ovf = n4 > CAP;
        const int nc = ovf ? 0 : n4;
        meta[4 * s] = F0a;
        meta[4 * s + 1] = ovf ? 1 : 0;
        unsigned char* st = asm_ + (size_t)s * G::STAGE;
        const unsigned bf = bar_full + 8 * s;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(bf, (unsigned)(G::FROW + nc * UP::ES));
        tma_load_1d(st + CAP * UP::ES, c.urow + rb + (size_t)k * RT, G::FROW, bf);
        if(nc)
        {
            const unsigned long long stream = l2_evict_first();
            const size_t S = c.ustride;
#pragma unroll 1
            for(int pl = 0; pl < UP::NP; pl++)
                tma_load_1d_hint(st + (size_t)16 * pl * CAP, c.uent + 16 * (pl * S + F0a), (unsigned)(16 * nc), bf,
                                 stream);
            tma_load_1d_hint(st + (size_t)16 * UP::NP * CAP, c.uent + 16 * UP::NP * S + (size_t)UP::TAIL * F0a,
                             (unsigned)(UP::TAIL * nc), bf, stream);
            if constexpr(UP::SLOTP > 0)
                tma_load_1d_hint(st + G::SLOT_OFF, c.uent + (16 * UP::NP + UP::TAIL) * S + (size_t)UP::SLOTP * F0a,
                                 (unsigned)(UP::SLOTP * nc), bf, stream);
        }
    };
    // The first STAGES tiles depend neither on beta nor on the stop flag: their copies start
    // now and run while the r.z partials are summed.  A stopped solve drains them and returns.
    const int pre = min(G::STAGES, mine);
    if(warp == A_CW)
        for(int u = 0; u < pre; u++)
        {
            const int F0 = __shfl_sync(0xffffffffu, lo, u), F1 = __shfl_sync(0xffffffffu, hi, u);
            if(lane == 0) issue_tile(u, F0, F1);
        }
    double rz_new, rz_mix = 0.0;
    if(c.flex && (long)s_iter > 0)
        consume_sum2<A_THREADS>(c, SITE_E, c.grid_e, SITE_F, c.grid_e, rz_new, rz_mix);
    else
        rz_new = consume_sum<A_THREADS>(c, SITE_E, c.grid_e);
    if(done)
    {
        if(warp == A_CW && lane == 0)
            for(int k = 0; k < pre; k++) mbar_wait(bar_full + 8 * k, 0u);
        return;
    }
    const double s_beta = (long)s_iter == 0 ? 0.0 : (rz_new - rz_mix) / rz_old;

    const int par = ((long)s_iter) & 1;
    const T* zp = zpbuf<T>(c, par);
    T* zpn = zpbuf<T>(c, par ^ 1);
    T* q = reinterpret_cast<T*>(c.q);
    T* spill = reinterpret_cast<T*>(c.spill);
    const T beta = (T)s_beta;
    double acc = 0;
    bool failed = false;

    if(warp == A_CW)
    {
        // ---- producer warp: lane 0 issues, all lanes fetch the tile bounds ----
        int issued = pre;
        for(int k0 = 0; k0 < mine && !failed; k0 += 32)
        {
            if(k0 > 0)
            {
                lo = hi = 0;
                if(k0 + lane < mine)
                {
                    const int r0 = rb + (k0 + lane) * RT;
                    lo = __ldg(c.urow + r0);
                    hi = __ldg(c.urow + min(r0 + RT, re));
                }
            }
            const int cnt = min(32, mine - k0);
            for(int u = 0; u < cnt; u++)
            {
                const int F0 = __shfl_sync(0xffffffffu, lo, u), F1 = __shfl_sync(0xffffffffu, hi, u);
                const int k = k0 + u, s = k % G::STAGES;
                if(k < pre) continue;
                if(lane == 0)
                {
                    if(!mbar_wait(bar_empty + 8 * s, ((k / G::STAGES) - 1) & 1)) failed = true;
                    if(!failed)
                    {
                        issue_tile(k, F0, F1);
                        issued = k + 1;
                    }
                }
                failed = __shfl_sync(0xffffffffu, failed ? 1 : 0, 0) != 0;
                if(failed) break;
            }
        }
        if(lane == 0)
        {
            if(failed)
            {
                atomicExch(c.flags + F_STATUS, 6);  // STG_ERR_TIMEOUT
                atomicExch(c.flags + F_DONE, 1);
            }
            for(int k = max(0, issued - G::STAGES); k < issued; k++)
                mbar_wait(bar_full + 8 * (k % G::STAGES), (k / G::STAGES) & 1);
        }
    }
    else
    {
        // ---- consumer warps: LPR lanes per row; lane `sub` of row r sums the entries
        //      sub, sub + LPR, ... of the row in order, UB at a time ----
        const int sub = lane & (LPR - 1);
        const int rloc = warp * (32 / LPR) + lane / LPR;
        for(int k = 0; k < mine; k++)
        {
            const int s = k % G::STAGES;
            const int r0 = rb + k * RT, r1 = min(r0 + RT, re);
            const int i = r0 + rloc;
            // v_i (p_new of the row) does not depend on the stage: gather it before the wait
            const T bta = (c.seg_of_row && i < r1) ? (T)__ldcg(c.seg + SEG_N * c.seg_of_row[i] + SG_BETA) : beta;
            T v0 = T(0), v1 = T(0), v2 = T(0);
            if(i < r1) a_gather<T>(i, zp, bta, v0, v1, v2);
            if(!__all_sync(0xffffffffu, mbar_wait(bar_full + 8 * s, (k / G::STAGES) & 1)))
            {
                failed = true;
                break;
            }
            const unsigned sb = sbase + (unsigned)(s * G::STAGE);
            const unsigned sfrow = sb + CAP * UP::ES;
            const int F0a = meta[4 * s];
            const bool ovf = meta[4 * s + 1] != 0;
            int f = 0, d = 0;
            if(i < r1)
            {
                const int x0 = lds_s32(sfrow + 4 * rloc), x1 = lds_s32(sfrow + 4 * rloc + 4);
                f = x0 - F0a;
                d = x1 - x0;
            }
            T y0 = T(0), y1 = T(0), y2 = T(0);
            double dd = 0.0;  // v_i . H_ii v_i
            for(int e0 = sub; e0 < d; e0 += G::UB * LPR)
            {
                T h8[G::UB], x[G::UB][3];
                int j[G::UB], sl[G::UB];
#pragma unroll
                for(int u = 0; u < G::UB; u++)
                {
                    const int e = e0 + u * LPR;
                    h8[u] = T(0);
                    j[u] = i;
                    sl[u] = -1;
                    if(e < d)
                    {
                        if(!ovf)
                            lds_utail<CAP, G::SLOT_OFF>(sb, f + e, h8[u], j[u], sl[u]);
                        else
                        {
                            T hh[9];
                            ldg_upper(c.uent, c.ustride, F0a + f + e, hh, j[u], sl[u]);
                            h8[u] = hh[8];
                        }
                    }
                }
#pragma unroll
                for(int u = 0; u < G::UB; u++)
                {
                    x[u][0] = v0;
                    x[u][1] = v1;
                    x[u][2] = v2;
                    if(e0 + u * LPR < d && j[u] != i) a_gather<T>(j[u], zp, bta, x[u][0], x[u][1], x[u][2]);
                }
#pragma unroll
                for(int u = 0; u < G::UB; u++)
                {
                    const int e = e0 + u * LPR;
                    if(e < d)
                    {
                        T h[9];
                        int jj, ss;
                        if(!ovf)
                            lds_main<CAP>(sb, f + e, h);
                        else
                            ldg_upper(c.uent, c.ustride, F0a + f + e, h, jj, ss);
                        h[8] = h8[u];
                        mv3<T>(h, false, x[u][0], x[u][1], x[u][2], y0, y1, y2);
                        T t0 = T(0), t1 = T(0), t2 = T(0);
                        mv3<T>(h, j[u] != i, v0, v1, v2, t0, t1, t2);
                        if(j[u] == i)
                            dd += (double)v0 * (double)t0 + (double)v1 * (double)t1 + (double)v2 * (double)t2;
                        else if(sl[u] >= 0)
                            st4(spill + 4 * (size_t)sl[u], t0, t1, t2);
                    }
                }
            }
            __syncwarp();
            if(lane == 0) mbar_arrive(bar_empty + 8 * s);
#pragma unroll
            for(int o = LPR / 2; o > 0; o >>= 1)
            {
                y0 += __shfl_xor_sync(0xffffffffu, y0, o);
                y1 += __shfl_xor_sync(0xffffffffu, y1, o);
                y2 += __shfl_xor_sync(0xffffffffu, y2, o);
                dd += __shfl_xor_sync(0xffffffffu, dd, o);
            }
            if(sub == 0 && i < r1)
            {
                st4(zpn + 8 * (size_t)i + 4, v0, v1, v2);
                st4(q + 4 * (size_t)i, y0, y1, y2);
                const double vy = (double)v0 * (double)y0 + (double)v1 * (double)y1 + (double)v2 * (double)y2;
                const double pq = 2.0 * vy - dd;
                acc += pq;
                if(c.seg_of_row) c.seg_row[i] = pq;
            }
        }
        if(failed && lane == 0)
        {
            atomicExch(c.flags + F_STATUS, 6);  // STG_ERR_TIMEOUT
            atomicExch(c.flags + F_DONE, 1);
        }
    }
    __shared__ double red[A_THREADS / 32];
    const double bs = block_sum<A_THREADS>(acc, red);
    if(threadIdx.x == 0) c.partials[(size_t)SITE_A * c.slots + blockIdx.x] = bs;
}

// ---------------------------------------------------------------------------------------
// A with a staged halo: the SpMV phase with every operand in shared memory.  Rows are cut
// into fixed tiles of RT rows (tile t: [RT t, RT t + RT)), and CTA b takes the contiguous
// tiles [b T / G, (b + 1) T / G).  Preparation (k_tile_halo) lists, per tile, the distinct
// columns its entries read outside the tile (the halo: about a quarter of the entries on a
// Morton-ordered mesh) and rewrites each entry's column as a slot of the tile's operand
// window: col - r0 for a column inside the tile, RT + its rank in the halo list otherwise.
// The producer warp fills a stage per tile: its lanes copy the halo's {z, p} slots with
// cp.async (16-byte pieces; each lane ties its copies to the stage's mbarrier), then lane 0
// starts the bulk copies of the tile's matrix planes, row bounds and own rows' {z, p}.  The
// consumers read blocks and operands from shared memory only: no gather waits on L2.
// ---------------------------------------------------------------------------------------
template <typename T>
struct AHalo
{
    using FP = FullPlanes<T>;
    static constexpr int RT = sizeof(T) == 4 ? 64 : 32;           // rows per tile
    static constexpr int LPR = 32 * A_CW / RT;                     // consumer lanes per row
    static constexpr int CAP = sizeof(T) == 4 ? 1024 : 512;        // entries per stage (even)
    static constexpr int HCAP = sizeof(T) == 4 ? 320 : 192;        // halo slots per tile
    static constexpr int SLOT = 8 * (int)sizeof(T);                // {z0 z1 z2 -, p0 p1 p2 -}
    static constexpr int TAIL = FP::TAIL;
    static constexpr int FROW = 4 * (RT + 4);                      // frow[r0 .. r0 + RT + 4)
    static constexpr int HALO = (RT + HCAP) * SLOT;                // own rows, then the halo
    static constexpr int PLANES = CAP * FP::ES;
    static constexpr int STAGE = PLANES + FROW + HALO;             // 16-byte multiple
    static constexpr int STAGES = 2;
    static constexpr int META = 16 * STAGES;
    static constexpr int SMEM = STAGES * STAGE + META + 16 * STAGES;
    static constexpr int MAXE = 2048;                              // entries per tile the preparation sorts
};

// Preparation, one CTA per tile: the tile's sorted halo (hcnt[t], hlist[t * HCAP ..]) and
// the slot-tail plane {h8, slot} that replaces {h8, col} for the halo kernel.  A tile with
// more than CAP entries or HCAP halo columns counts in *bad (the solve keeps the plain tiled
// kernel then).
template <typename T>
__global__ void __launch_bounds__(256) k_tile_halo(const int* __restrict__ frow, const unsigned char* __restrict__ fent,
                                                   size_t S, int nrows, int* hcnt, int* hlist, unsigned char* htail,
                                                   int* bad)
{
    using G = AHalo<T>;
    constexpr int RT = G::RT, MAXE = G::MAXE, PER = MAXE / 256;
    __shared__ int key[MAXE];
    __shared__ int uniq[MAXE];
    __shared__ int wsum[8];
    __shared__ int total;
    const int t = blockIdx.x, tid = threadIdx.x;
    const int r0 = t * RT, r1 = min(r0 + RT, nrows);
    const int F0 = frow[r0], n = frow[r1] - F0;
    if(n + 2 > G::CAP || n > MAXE)  // a stage's copy starts at an even entry: up to n + 2
    {
        if(tid == 0)
        {
            atomicAdd(bad, 1);
            hcnt[t] = 0;
        }
        return;
    }
    const unsigned char* tail = fent + (size_t)16 * FullPlanes<T>::NP * S;  // {h8, col} plane
    auto col_of = [&](int f) -> int {
        return sizeof(T) == 4 ? reinterpret_cast<const int*>(tail)[2 * (size_t)f + 1]
                              : (int)reinterpret_cast<const long long*>(tail)[2 * (size_t)f + 1];
    };
    int P = 1;
    while(P < n) P <<= 1;
    for(int i = tid; i < MAXE; i += 256)
    {
        int k = 0x7fffffff;
        if(i < n)
        {
            const int cc = col_of(F0 + i);
            if(cc < r0 || cc >= r1) k = cc;
        }
        key[i] = k;
    }
    __syncthreads();
    // bitonic sort of key[0, P)
    for(int k = 2; k <= P; k <<= 1)
        for(int j = k >> 1; j > 0; j >>= 1)
        {
            for(int i = tid; i < P; i += 256)
            {
                const int ixj = i ^ j;
                if(ixj > i)
                {
                    const int a = key[i], b = key[ixj];
                    if(((i & k) == 0) == (a > b))
                    {
                        key[i] = b;
                        key[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    // distinct keys, in order: thread tid owns key[PER tid, PER tid + PER)
    int cnt = 0;
#pragma unroll
    for(int u = 0; u < PER; u++)
    {
        const int i = PER * tid + u;
        cnt += (i < P && key[i] != 0x7fffffff && (i == 0 || key[i] != key[i - 1])) ? 1 : 0;
    }
    const int lane = tid & 31, w = tid >> 5;
    int incl = cnt;
#pragma unroll
    for(int o = 1; o < 32; o <<= 1)
    {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if(lane >= o) incl += y;
    }
    if(lane == 31) wsum[w] = incl;
    __syncthreads();
    int before = 0;
    for(int u = 0; u < w; u++) before += wsum[u];
    if(tid == 255) total = before + incl;
    int pos = before + incl - cnt;
#pragma unroll
    for(int u = 0; u < PER; u++)
    {
        const int i = PER * tid + u;
        if(i < P && key[i] != 0x7fffffff && (i == 0 || key[i] != key[i - 1])) uniq[pos++] = key[i];
    }
    __syncthreads();
    const int H = total;
    if(H > G::HCAP)
    {
        if(tid == 0)
        {
            atomicAdd(bad, 1);
            hcnt[t] = 0;
        }
        return;
    }
    if(tid == 0) hcnt[t] = H;
    for(int i = tid; i < H; i += 256) hlist[(size_t)t * G::HCAP + i] = uniq[i];
    for(int e = tid; e < n; e += 256)
    {
        const size_t f = (size_t)F0 + e;
        const int cc = col_of((int)f);
        int slot;
        if(cc >= r0 && cc < r1)
            slot = cc - r0;
        else
        {
            int lo = 0, hi = H;  // first uniq >= cc
            while(lo < hi)
            {
                const int mid = (lo + hi) >> 1;
                if(uniq[mid] < cc)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            slot = RT + lo;
        }
        if(sizeof(T) == 4)
        {
            const float2 v = reinterpret_cast<const float2*>(tail)[f];
            reinterpret_cast<float2*>(htail)[f] = make_float2(v.x, __int_as_float(slot));
        }
        else
        {
            const double2 v = reinterpret_cast<const double2*>(tail)[f];
            reinterpret_cast<double2*>(htail)[f] = make_double2(v.x, __longlong_as_double((long long)slot));
        }
    }
}

// Producer of the halo kernel: fills stage k % STAGES with tile tb + k.  Lane 0 starts the
// tile's bulk copies (planes, row bounds, own rows' {z, p}); every lane copies its share of
// the halo with cp.async and arrives (.noinc) on the stage's barrier, which expects lane 0
// plus the 32 lanes.  hc: the halo sizes of the 32 tiles from k & ~31 on, one per lane.
template <typename T>
__device__ __forceinline__ void halo_issue(const PcgDev& c, unsigned char* hsm_, int* meta, unsigned bar_full,
                                           const T* zp, int tb, int k, int hc, int lane)
{
    using G = AHalo<T>;
    using FP = FullPlanes<T>;
    constexpr int RT = G::RT, CAP = G::CAP;
    const int s = k % G::STAGES, t = tb + k;
    const int r0 = t * RT, r1 = min(r0 + RT, c.nrows);
    unsigned char* st = hsm_ + (size_t)s * G::STAGE;
    const unsigned bf = bar_full + 8 * s;
    if(lane == 0)
    {
        const int F0 = __ldg(c.frow + r0), F1 = __ldg(c.frow + r1);
        const int F0a = F0 & ~1, n2 = ((F1 + 1) & ~1) - F0a;
        meta[4 * s] = F0a;
        const unsigned own = (unsigned)((r1 - r0) * G::SLOT);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(bf, (unsigned)(n2 * FP::ES + G::FROW) + own);
        const unsigned long long stream = l2_evict_first();
#pragma unroll 1
        for(int pl = 0; pl < FP::NP; pl++)
            tma_load_1d_hint(st + (size_t)16 * pl * CAP, c.fent + 16 * (pl * c.fstride + F0a), (unsigned)(16 * n2), bf,
                             stream);
        tma_load_1d_hint(st + (size_t)16 * FP::NP * CAP, c.htail + (size_t)FP::TAIL * F0a, (unsigned)(FP::TAIL * n2),
                         bf, stream);
        tma_load_1d(st + G::PLANES, c.frow + r0, G::FROW, bf);
        tma_load_1d(st + G::PLANES + G::FROW, zp + 8 * (size_t)r0, own, bf);
    }
    // the halo: {z, p} slots of the tile's outside columns; a lane's column ids are loaded
    // together before its copies are issued
    const int H = __shfl_sync(0xffffffffu, hc, k % 32);
    const int* hl = c.hlist + (size_t)t * G::HCAP;
    unsigned char* hs = st + G::PLANES + G::FROW + (size_t)RT * G::SLOT;
    constexpr int PER = (G::HCAP + 31) / 32;
    int cols[PER];
#pragma unroll
    for(int u = 0; u < PER; u++) cols[u] = lane + 32 * u < H ? __ldg(hl + lane + 32 * u) : -1;
#pragma unroll
    for(int u = 0; u < PER; u++)
        if(cols[u] >= 0)
        {
            const unsigned char* src = reinterpret_cast<const unsigned char*>(zp + 8 * (size_t)cols[u]);
            unsigned char* dst = hs + (size_t)(lane + 32 * u) * G::SLOT;
#pragma unroll
            for(int pc = 0; pc < G::SLOT / 16; pc++) cp_async16(dst + 16 * pc, src + 16 * pc);
        }
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bf) : "memory");
}

template <typename T>
__global__ void __launch_bounds__(A_THREADS, 2) k_phase_a_halo(PcgDev c)
{
    using G = AHalo<T>;
    constexpr int RT = G::RT, LPR = G::LPR, CAP = G::CAP;
    extern __shared__ __align__(128) unsigned char hsm_[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = (c.nrows + RT - 1) / RT;
    const int tb = (int)((long long)blockIdx.x * ntiles / gridDim.x);
    const int te = (int)((long long)(blockIdx.x + 1) * ntiles / gridDim.x);
    const int mine = te - tb;
    const int done = __ldcg(c.flags + F_DONE);
    const double s_iter = __ldcg(c.scal + SS_ITER), rz_old = __ldcg(c.scal + SS_RZ);
    if(done) return;
    int* meta = reinterpret_cast<int*>(hsm_ + G::STAGES * G::STAGE);
    const unsigned sbase = smem_u32(hsm_);
    const unsigned bar_full = smem_u32(hsm_ + G::STAGES * G::STAGE + G::META);
    const unsigned bar_empty = bar_full + 8 * G::STAGES;
    if(threadIdx.x == 0)
    {
        for(int s = 0; s < G::STAGES; s++)
        {
            mbar_init(bar_full + 8 * s, 33);  // lane 0's expect_tx arrival + one per producer lane
            mbar_init(bar_empty + 8 * s, A_CW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int par = ((long)s_iter) & 1;
    const T* zp = zpbuf<T>(c, par);
    T* zpn = zpbuf<T>(c, par ^ 1);
    T* q = reinterpret_cast<T*>(c.q);
    // the first stages need nothing of beta: the producer starts them before the reduction
    int hc = 0;
    if(warp == A_CW)
    {
        hc = lane < mine ? __ldg(c.hcnt + tb + lane) : 0;
        for(int k = 0; k < min(G::STAGES, mine); k++) halo_issue<T>(c, hsm_, meta, bar_full, zp, tb, k, hc, lane);
    }
    // beta = rz_k / rz_(k-1) (flexible PCG: r_k.(z_k - z_(k-1)) / r_(k-1).z_(k-1)); 0 at first
    double rz_new, rz_mix = 0.0;
    if(c.flex && (long)s_iter > 0)
        consume_sum2<A_THREADS>(c, SITE_E, c.grid_e, SITE_F, c.grid_e, rz_new, rz_mix);
    else
        rz_new = consume_sum<A_THREADS>(c, SITE_E, c.grid_e);
    const double s_beta = (long)s_iter == 0 ? 0.0 : (rz_new - rz_mix) / rz_old;
    const T beta = (T)s_beta;
    double acc = 0;
    bool failed = false;

    if(warp == A_CW)
    {
        // ---- producer warp: the remaining tiles, each once its stage is released ----
        int issued = min(G::STAGES, mine);
        for(int k = G::STAGES; k < mine && !failed; k++)
        {
            if(k % 32 == 0) hc = k + lane < mine ? __ldg(c.hcnt + tb + k + lane) : 0;
            const int s = k % G::STAGES;
            bool ok = true;
            if(lane == 0) ok = mbar_wait(bar_empty + 8 * s, ((k / G::STAGES) - 1) & 1);
            failed = __shfl_sync(0xffffffffu, ok ? 0 : 1, 0) != 0;
            if(failed) break;
            halo_issue<T>(c, hsm_, meta, bar_full, zp, tb, k, hc, lane);
            issued = k + 1;
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        if(lane == 0)
        {
            if(failed)
            {
                atomicExch(c.flags + F_STATUS, 6);  // STG_ERR_TIMEOUT
                atomicExch(c.flags + F_DONE, 1);
            }
            // drain: every issued stage's copies must have landed before the CTA exits
            for(int k = max(0, issued - G::STAGES); k < issued; k++)
                mbar_wait(bar_full + 8 * (k % G::STAGES), (k / G::STAGES) & 1);
        }
    }
    else
    {
        // ---- consumer warps: LPR lanes per row, lane `sub` sums the row's entries sub,
        //      sub + LPR, ... in order, four at a time; operands from the stage's window ----
        const int sub = lane & (LPR - 1);
        const int rloc = warp * (32 / LPR) + lane / LPR;
        for(int k = 0; k < mine; k++)
        {
            const int s = k % G::STAGES, t = tb + k;
            const int r0 = t * RT, r1 = min(r0 + RT, c.nrows);
            const int i = r0 + rloc;
            if(!__all_sync(0xffffffffu, mbar_wait(bar_full + 8 * s, (k / G::STAGES) & 1)))
            {
                failed = true;
                break;
            }
            const unsigned sb = sbase + (unsigned)(s * G::STAGE);
            const unsigned sfrow = sb + G::PLANES;
            const T* win = reinterpret_cast<const T*>(hsm_ + (size_t)s * G::STAGE + G::PLANES + G::FROW);
            const int F0a = meta[4 * s];
            int f = 0, d = 0;
            if(i < r1)
            {
                const int x0 = lds_s32(sfrow + 4 * rloc), x1 = lds_s32(sfrow + 4 * rloc + 4);
                f = x0 - F0a;
                d = x1 - x0;
            }
            const T bta = (c.seg_of_row && i < r1) ? (T)__ldcg(c.seg + SEG_N * c.seg_of_row[i] + SG_BETA) : beta;
            T y0 = T(0), y1 = T(0), y2 = T(0);
            for(int e0 = sub; e0 < d; e0 += 4 * LPR)
            {
                T h8[4];
                int sl[4];
#pragma unroll
                for(int u = 0; u < 4; u++)
                {
                    h8[u] = T(0);
                    sl[u] = 0;
                    if(e0 + u * LPR < d) lds_tail<CAP>(sb, f + e0 + u * LPR, h8[u], sl[u]);
                }
#pragma unroll
                for(int u = 0; u < 4; u++)
                {
                    const int e = e0 + u * LPR;
                    if(e < d)
                    {
                        const T* w = win + 8 * sl[u];
                        T x0, x1, x2, p0, p1, p2;
                        ld4(w, x0, x1, x2);
                        ld4(w + 4, p0, p1, p2);
                        x0 += bta * p0;
                        x1 += bta * p1;
                        x2 += bta * p2;
                        T h[9];
                        lds_main<CAP>(sb, f + e, h);
                        h[8] = h8[u];
                        mv3<T>(h, false, x0, x1, x2, y0, y1, y2);
                    }
                }
            }
            T p0 = T(0), p1 = T(0), p2 = T(0);
            if(sub == 0 && i < r1)
            {
                const T* w = win + 8 * rloc;
                T z0, z1, z2, o0, o1, o2;
                ld4(w, z0, z1, z2);
                ld4(w + 4, o0, o1, o2);
                p0 = z0 + bta * o0;
                p1 = z1 + bta * o1;
                p2 = z2 + bta * o2;
            }
            __syncwarp();
            if(lane == 0) mbar_arrive(bar_empty + 8 * s);
#pragma unroll
            for(int o = LPR / 2; o > 0; o >>= 1)
            {
                y0 += __shfl_xor_sync(0xffffffffu, y0, o);
                y1 += __shfl_xor_sync(0xffffffffu, y1, o);
                y2 += __shfl_xor_sync(0xffffffffu, y2, o);
            }
            if(sub == 0 && i < r1)
            {
                st4(zpn + 8 * (size_t)i + 4, p0, p1, p2);
                st4(q + 4 * (size_t)i, y0, y1, y2);
                const double pq = (double)p0 * (double)y0 + (double)p1 * (double)y1 + (double)p2 * (double)y2;
                acc += pq;
                if(c.seg_of_row) c.seg_row[i] = pq;
            }
        }
        if(failed && lane == 0)
        {
            atomicExch(c.flags + F_STATUS, 6);  // STG_ERR_TIMEOUT
            atomicExch(c.flags + F_DONE, 1);
        }
    }
    // p.q: this CTA's partial only; phase B finishes the sum (consume_sum)
    __shared__ double red[A_THREADS / 32];
    const double bs = block_sum<A_THREADS>(acc, red);
    if(threadIdx.x == 0) c.partials[(size_t)SITE_A * c.slots + blockIdx.x] = bs;
}

// E (MAS): z = sum over levels (FP32) on the FEM range + ABD block-Jacobi; share of r.z
// ABD 12x12 block-Jacobi (abd_preconditioner.cu:20-38): one thread per dof of the first
// 12 * bodies dofs, z written into the zp slots; returns the share of r.z
// skip: the solve has stopped (stop flag read with the loads): nothing is stored
template <typename T>
__device__ __forceinline__ double abd_apply(const PcgDev& c, T* zp, int gt, int gn, bool skip = false)
{
    double acc = 0;
    for(int t = gt; t < c.abd_bodies * 12; t += gn)
    {
        const int body = t / 12, row = t % 12;
        const double* J = c.abd_inv + (size_t)body * 144 + row * 12;
        double s = 0;
#pragma unroll
        for(int cc = 0; cc < 12; cc++) s += J[cc] * c.r[body * 12 + cc];
        if(skip) continue;
        zp[8 * (size_t)(t / 3) + t % 3] = (T)s;
        acc += c.r[t] * (double)(T)s;
    }
    return acc;
}

template <typename T>
__device__ __forceinline__ double phase_e_mas(const PcgDev& c, int gt, int gn, bool skip = false)
{
    T* zp = zpbuf<T>(c, iter_parity(c));
    double acc = 0;
    const int fem_row = c.fem_dof / 3;
    for(int v = gt; v < c.V; v += gn)
    {
        const int s = c.real_map[v];
        float c0, c1, c2;
        ld4(c.Z + 4 * (size_t)s, c0, c1, c2);
        for(int l = 1; l < c.L; l++)
        {
            const int now = c.coarse_table[(size_t)v * (c.L - 1) + l - 1];
            float t0, t1, t2;
            ld4(c.Z + 4 * (size_t)now, t0, t1, t2);
            c0 += t0;
            c1 += t1;
            c2 += t2;
        }
        const int row = fem_row + v;
        const double* r = c.r + 3 * (size_t)row;
        const double rz = r[0] * (double)(T)c0 + r[1] * (double)(T)c1 + r[2] * (double)(T)c2;
        acc += rz;
        if(skip) continue;
        st4(zp + 8 * (size_t)row, (T)c0, (T)c1, (T)c2);
        if(c.seg_of_row) c.seg_row[2 * (size_t)c.nrows + row] = rz;
    }
    return acc + abd_apply<T>(c, zp, gt, gn, skip);
}

// E (global block-Jacobi / identity, then the ABD local preconditioner); share of r.z
template <typename T>
__device__ __forceinline__ double phase_e_plain(const PcgDev& c, int gt, int gn, bool skip = false)
{
    T* zp = zpbuf<T>(c, iter_parity(c));
    double acc = 0;
    for(int bi = c.abd_bodies * 4 + gt; bi < c.nrows; bi += gn)
    {
        const double r0 = c.r[3 * bi], r1 = c.r[3 * bi + 1], r2 = c.r[3 * bi + 2];
        double z0 = r0, z1 = r1, z2 = r2;
        if(c.diag_inv)
        {
            const double* D = c.diag_inv + 9 * (size_t)bi;
            z0 = D[0] * r0 + D[3] * r1 + D[6] * r2;
            z1 = D[1] * r0 + D[4] * r1 + D[7] * r2;
            z2 = D[2] * r0 + D[5] * r1 + D[8] * r2;
        }
        const double rz = r0 * (double)(T)z0 + r1 * (double)(T)z1 + r2 * (double)(T)z2;
        acc += rz;
        if(skip) continue;
        st4(zp + 8 * (size_t)bi, (T)z0, (T)z1, (T)z2);
        if(c.seg_of_row) c.seg_row[2 * (size_t)c.nrows + bi] = rz;
    }
    return acc + abd_apply<T>(c, zp, gt, gn, skip);
}

// ---------------------------------------------------------------------------------------
// one kernel per phase (LOOP_HOST / LOOP_GRAPH)
// ---------------------------------------------------------------------------------------
#define GT (blockIdx.x * PB + threadIdx.x)
#define GN (gridDim.x * PB)

// r = b, x = 0, both zp slots = 0 (p_0 = 0 so that p_1 = z_0 + 0 p_0); b.b
template <typename T>
__global__ void __launch_bounds__(PB) k_init(PcgDev c)
{
    double acc = 0;
    T* zp0 = reinterpret_cast<T*>(c.zp0);
    T* zp1 = reinterpret_cast<T*>(c.zp1);
    for(int i = GT; i < c.n; i += GN)
    {
        const double bi = c.b[i];
        c.r[i] = bi;
        c.x[i] = 0.0;
        acc += bi * bi;
    }
    for(int i = GT; i < 8 * c.nrows; i += GN)
    {
        zp0[i] = T(0);
        zp1[i] = T(0);
    }
    finish_reduction(c, acc, SITE_INIT, POST_STORE, SS_BB);
}

template <typename T>
__global__ void __launch_bounds__(PB) k_phase_a(PcgDev c)
{
    if(c.flags[F_DONE]) return;
    finish_reduction(c, phase_a<T>(c, GT, GN), SITE_A, POST_ALPHA);
}

template <typename T, int B>
__global__ void __launch_bounds__(PB, 4) k_phase_b(PcgDev c)
{
    // the first slot's loads depend neither on alpha nor on the stop flag: issue them with
    // the flag's load, before the reductions
    const int done = __ldcg(c.flags + F_DONE);
    BSlot<T> first;
    if(B > 0)
        b_load<T>(c, zpbuf<T>(c, iter_parity(c) ^ 1), reinterpret_cast<const T*>(c.q), GT, first);
    // the p.q and r.z partials, in flight with the slot's loads (a grid too large for the
    // registers sums them in consume_sum2 below)
    constexpr int PK = 3;
    const bool early = c.grid_a <= PK * PB && c.grid_e <= PK * PB;
    double pa[PK], pe[PK];
    if(early) consume2_load<PB, PK>(c, SITE_A, c.grid_a, SITE_E, c.grid_e, pa, pe);
    if(done) return;
    // After the upper SpMV, the spilled products of a warp's 32 consecutive rows (Morton
    // order: consecutive slots are consecutive rows) are one contiguous run of slots: the warp
    // copies up to SPW of them into shared memory with coalesced asynchronous copies, issued
    // before the reductions, instead of each lane reading its own run (32 lines per load).
    constexpr int SPW = 4096 / (4 * (int)sizeof(T));  // staged slots per warp (4 KB)
    __shared__ __align__(16) T stage[B > 0 ? PB / 32 : 1][B > 0 ? 4 * SPW : 4];
    const int lane = threadIdx.x & 31;
    int slo = 0, shi = 0;
    if(B > 0 && c.spill && c.identity)
    {
        const bool valid = first.v >= 0;
        const unsigned vm = __ballot_sync(0xffffffffu, valid);
        if(vm & 1u)
        {
            slo = __shfl_sync(0xffffffffu, first.t0, 0);
            const int hi = __reduce_max_sync(0xffffffffu, valid ? first.t1 : 0);
            shi = slo + min(hi - slo, SPW);
            T* sw = stage[threadIdx.x >> 5];
            const unsigned char* src = reinterpret_cast<const unsigned char*>(c.spill) + (size_t)slo * 4 * sizeof(T);
            for(int e = lane; e < shi - slo; e += 32)
#pragma unroll
                for(int h = 0; h < (int)sizeof(T) / 4; h++)
                    cp_async16(reinterpret_cast<unsigned char*>(sw) + (size_t)e * 4 * sizeof(T) + 16 * h,
                               src + (size_t)e * 4 * sizeof(T) + 16 * h);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    double pq, rz;
    if(early)
        consume2_finish<PB, PK>(pa, pe, pq, rz);
    else
        consume_sum2<PB>(c, SITE_A, c.grid_a, SITE_E, c.grid_e, pq, rz);
    if(B > 0 && c.spill && c.identity)
    {
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncwarp();
    }
    double v = 0;
    if(pq > 0.0 && isfinite(pq))  // else breakdown: no update; the last CTA reports it
    {
        const double alpha = rz / pq;
        v = B > 0 ? phase_b_mas<T, (B > 0 ? B : 16)>(c, GT, GN, alpha, first, true, shi > slo ? stage[threadIdx.x >> 5] : nullptr,
                                                     slo, shi)
                  : phase_b_plain<T>(c, GT, GN, alpha);
    }
    finish_reduction(c, v, SITE_B, POST_CHECK_PQ, 0, pq, rz);
}

// guarded: runs only when this iteration is a replacement iteration (host / plain graph),
// or unconditionally inside the graph's IF node
__global__ void __launch_bounds__(PB) k_replace(PcgDev c, int guarded)
{
    if(c.flags[F_DONE]) return;
    if(guarded)
    {
        const long k = (long)c.scal[SS_ITER];
        if(c.prm.refine <= 0 || k % c.prm.refine != 0) return;
    }
    if(blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(c.flags + F_REPL, 1);
    finish_reduction(c, phase_replace(c, GT, GN), SITE_R, POST_RECHECK);
}

template <int B>
__global__ void __launch_bounds__(PB) k_restrict01(PcgDev c, int guarded)
{
    if(c.flags[F_DONE]) return;
    if(guarded)
    {
        const long k = (long)c.scal[SS_ITER];
        if(c.prm.refine <= 0 || k % c.prm.refine != 0) return;
    }
    phase_restrict01<B>(c, GT, GN);
}

// C1: level 1 -> 2 over the whole grid
template <int B>
__global__ void __launch_bounds__(PB) k_phase_c1(PcgDev c)
{
    // the stop flag only gates the stores: its load overlaps the level's loads
    const int done = __ldcg(c.flags + F_DONE);
    if(c.L > 2) restrict_level<B>(c, c.ls[2], c.ls[3], GT, GN, done != 0);  // level 1's (count, begin)
}

// C2: levels 2 -> 3 -> ... (small) by one CTA.  All nodes of the levels >= 2 (contiguous
// from the first level-2 node) fit in shared memory: their residuals, closed masks and
// parents are loaded in one round, each level is restricted inside shared memory (the
// component leader sums its members in lane order, as restrict_level does), and the levels
// >= 3 are stored once at the end.  More nodes than C2_SMEM_NODES: level by level through
// global memory.
constexpr int C2_SMEM_NODES = 4096;
constexpr int C2_SMEM_BYTES = C2_SMEM_NODES * (16 + 4 + 4);

template <int B>
__global__ void __launch_bounds__(1024) k_phase_c2(PcgDev c)
{
    // the stop flag only gates the stores: its load overlaps the nodes' loads
    const int done = __ldcg(c.flags + F_DONE);
    // level sizes from the parameter block (unrolled constant indices: no dependent loads)
    int last_n = 0, last_b = 0;
#pragma unroll
    for(int l = 0; l <= kMaxLevelsDev; l++)
        if(l == c.L - 1)
        {
            last_n = c.ls[2 * l];
            last_b = c.ls[2 * l + 1];
        }
    const int b2 = c.ls[5];  // first level-2 node
    const int total = last_b + last_n - b2;
    if(total > C2_SMEM_NODES)
    {
        if(!done) phase_c<B>(c, 2, c.L - 1, threadIdx.x, blockDim.x, true);
        return;
    }
    extern __shared__ float4 c2_smem[];
    float4* rv = c2_smem;
    unsigned* cm = reinterpret_cast<unsigned*>(rv + C2_SMEM_NODES);
    int* par = reinterpret_cast<int*>(cm + C2_SMEM_NODES);
    const int n2 = c.ls[4];
    for(int i = threadIdx.x; i < total; i += 1024)
    {
        rv[i] = i < n2 ? *reinterpret_cast<const float4*>(c.R + 4 * (size_t)(b2 + i)) : make_float4(0.f, 0.f, 0.f, 0.f);
        cm[i] = c.closed[b2 + i];
        par[i] = c.going_next[b2 + i] - b2;
    }
    __syncthreads();
    for(int level = 2; level < c.L - 1; level++)
    {
        int number = 0, begin = 0;
#pragma unroll
        for(int l = 0; l < kMaxLevelsDev; l++)
            if(l == level)
            {
                number = c.ls[2 * l];
                begin = c.ls[2 * l + 1] - b2;
            }
        const int span = (number + 31) / 32 * 32;
        for(int i = threadIdx.x; i < span; i += 1024)
        {
            const bool valid = i < number;
            float r0 = 0.f, r1 = 0.f, r2 = 0.f;
            unsigned msk = 0;
            if(valid)
            {
                const float4 v = rv[begin + i];
                r0 = v.x;
                r1 = v.y;
                r2 = v.z;
                msk = cm[begin + i];
            }
            float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll 4
            for(int bb = 0; bb < B; bb++)
            {
                const float x0 = group_shfl<B>(r0, bb);
                const float x1 = group_shfl<B>(r1, bb);
                const float x2 = group_shfl<B>(r2, bb);
                if(msk & (1u << bb))
                {
                    a0 += x0;
                    a1 += x1;
                    a2 += x2;
                }
            }
            if(valid && __popc(msk & lanemask_lt(i % B)) == 0) rv[par[begin + i]] = make_float4(a0, a1, a2, 0.f);
        }
        __syncthreads();
    }
    if(done) return;
    for(int i = n2 + threadIdx.x; i < total; i += 1024)
        *reinterpret_cast<float4*>(c.R + 4 * (size_t)(b2 + i)) = rv[i];
}

template <int B>
__global__ void __launch_bounds__(PB) k_phase_d(PcgDev c)
{
    if(c.flags[F_DONE]) return;
    phase_d<B>(c, blockIdx.x, c.nbanks, gridDim.x);
}

template <typename T, int B>
__global__ void __launch_bounds__(PB, 8) k_phase_e(PcgDev c, int op)
{
    // the stop flag only gates the stores: its load overlaps the prolongation's loads
    const int done = __ldcg(c.flags + F_DONE);
    const double v = B > 0 ? phase_e_mas<T>(c, GT, GN, done != 0) : phase_e_plain<T>(c, GT, GN, done != 0);
    if(done) return;
    if(op == POST_INIT_RZ)
    {
        finish_reduction(c, v, SITE_E, POST_INIT_RZ);
        return;
    }
    // r.z: this CTA's partial only; the next SpMV phase and phase B finish the sum
    __shared__ double red[PB / 32];
    const double bs = block_sum<PB>(v, red);
    if(threadIdx.x == 0) c.partials[(size_t)SITE_E * c.slots + blockIdx.x] = bs;
    if(c.flex && (long)__ldcg(c.scal + SS_ITER) > 0)
    {
        // flexible PCG: r_(k+1).z_k with z_k still in the other zp buffer
        const T* zo = zpbuf<T>(c, iter_parity(c) ^ 1);
        double vo = 0;
        for(int bi = GT; bi < c.nrows; bi += GN)
        {
            T z0, z1, z2;
            ld4(zo + 8 * (size_t)bi, z0, z1, z2);
            vo += c.r[3 * bi] * (double)z0 + c.r[3 * bi + 1] * (double)z1 + c.r[3 * bi + 2] * (double)z2;
        }
        const double bo = block_sum<PB>(vo, red);
        if(threadIdx.x == 0) c.partials[(size_t)SITE_F * c.slots + blockIdx.x] = bo;
    }
}

// ---------------------------------------------------------------------------------------
// independent scenes (PcgDev::seg_of_row): one CTA per scene sums the scene's per-row
// contributions in row order and updates its scalars
//   SEG_INIT after the first preconditioner application: r.z, b.b, beta = 0
//   SEG_A    after the SpMV phase: p.q, alpha = r.z / p.q (0 once the scene is done)
//   SEG_B    after the x / r update: r.r and the scene's stop test; the last CTA ends the
//            loop when every scene is done
//   SEG_E    after the preconditioner: beta = r.z_new / r.z, r.z = r.z_new
// ---------------------------------------------------------------------------------------
enum SegMode : int
{
    SEG_INIT = 0,
    SEG_A = 1,
    SEG_B = 2,
    SEG_E = 3
};

template <int MODE>
__global__ void __launch_bounds__(PB) k_seg(PcgDev c)
{
    __shared__ double red[PB / 32];
    __shared__ bool last;
    if(MODE != SEG_INIT && __ldcg(c.flags + F_DONE)) return;
    const int sc = blockIdx.x;
    const int r0 = c.seg_row_off[sc], r1 = c.seg_row_off[sc + 1];
    double* S = c.seg + SEG_N * (size_t)sc;
    const double* src = c.seg_row + (size_t)(MODE == SEG_A ? 0 : (MODE == SEG_B ? 1 : 2)) * c.nrows;
    double v = 0, bb = 0;
    for(int i = r0 + threadIdx.x; i < r1; i += PB) v += __ldcg(src + i);
    if(MODE == SEG_INIT)
        for(int i = 3 * r0 + threadIdx.x; i < 3 * r1; i += PB) bb += c.b[i] * c.b[i];
    v = block_sum<PB>(v, red);
    if(MODE == SEG_INIT) bb = block_sum<PB>(bb, red);
    if(threadIdx.x == 0)
    {
        if(MODE == SEG_INIT)
        {
            S[SG_RZ] = v;
            S[SG_BB] = bb;
            S[SG_BETA] = 0.0;
            S[SG_ALPHA] = 0.0;
            S[SG_RR] = bb;
            S[SG_DONE] = bb > 0.0 ? 0.0 : 1.0;
            S[SG_ITER] = 0.0;
        }
        else if(MODE == SEG_A)
        {
            S[SG_PQ] = v;
            // a scene whose p.q is not positive stops (no update), the others go on
            const bool go = S[SG_DONE] == 0.0 && v > 0.0 && isfinite(v);
            S[SG_ALPHA] = go ? S[SG_RZ] / v : 0.0;
            if(!go && S[SG_DONE] == 0.0)
            {
                S[SG_DONE] = 1.0;
                S[SG_ITER] = __ldcg(c.scal + SS_ITER);
            }
        }
        else if(MODE == SEG_E)
        {
            if(S[SG_DONE] == 0.0) S[SG_BETA] = S[SG_RZ] != 0.0 ? v / S[SG_RZ] : 0.0;
            S[SG_RZ] = v;
        }
        else
        {
            S[SG_RR] = v;
            if(S[SG_DONE] == 0.0 && v <= c.seg_tol2 * S[SG_BB])
            {
                S[SG_DONE] = 1.0;
                S[SG_ITER] = __ldcg(c.scal + SS_ITER);
            }
            __threadfence();
            last = atomicAdd(c.counters + CNT_SEG, 1u) == (unsigned)(gridDim.x - 1);
        }
    }
    if(MODE != SEG_B) return;
    __syncthreads();
    if(!last) return;
    __threadfence();
    double open = 0;
    for(int q = threadIdx.x; q < c.nseg; q += PB) open += __ldcg(c.seg + SEG_N * (size_t)q + SG_DONE) == 0.0 ? 1.0 : 0.0;
    open = block_sum<PB>(open, red);
    if(threadIdx.x == 0)
    {
        if(open == 0.0)
        {
            c.flags[F_DONE] = 1;
            c.flags[F_STATUS] = 0;
            if(c.use_cond) cudaGraphSetConditional(c.h_while, 0u);
        }
        c.counters[CNT_SEG] = 0u;
        __threadfence();
    }
}

// ---------------------------------------------------------------------------------------
// persistent kernel (LOOP_PERSISTENT): all iterations in one cooperative launch
// ---------------------------------------------------------------------------------------
// Grid barrier that also finishes a reduction: every CTA deposits its partial, the last CTA
// to arrive sums them in index order, applies the post-op and releases the others.  Waits
// are bounded (~2^22 polls with backoff, a few seconds): a CTA that gives up marks the solve
// STG_ERR_TIMEOUT and every CTA leaves at the next check instead of spinning forever.
__device__ __forceinline__ void grid_barrier(const PcgDev& c, double v, int site, int op, unsigned& gen)
{
    __shared__ double red[PB / 32];
    __shared__ bool last;
    const double bs = (op >= 0) ? block_sum<PB>(v, red) : 0.0;
    if(threadIdx.x == 0)
    {
        if(op >= 0) c.partials[(size_t)site * c.slots + blockIdx.x] = bs;
        __threadfence();
        last = atomicAdd(c.bar, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if(last)
    {
        __threadfence();
        if(op >= 0)
        {
            const double* partials = c.partials + (size_t)site * c.slots;
            double acc = 0;
            for(int i = threadIdx.x; i < (int)gridDim.x; i += PB) acc += __ldcg(partials + i);
            const double tot = block_sum<PB>(acc, red);
            if(threadIdx.x == 0) post_op(op, 0, tot, c.scal, c.flags, c.prm);
        }
        if(threadIdx.x == 0)
        {
            c.bar[0] = 0u;
            __threadfence();
            atomicExch(c.bar + 1, gen + 1u);
        }
    }
    else if(threadIdx.x == 0)
    {
        unsigned polls = 0, ns = 32;
        while(true)
        {
            unsigned g;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(g) : "l"(c.bar + 1) : "memory");
            if(g != gen) break;
            if(++polls > (1u << 22))
            {
                atomicExch(c.flags + F_DONE, 1);
                atomicExch(c.flags + F_STATUS, 6);  // STG_ERR_TIMEOUT
                break;
            }
            __nanosleep(ns);
            if(ns < 256) ns <<= 1;
        }
    }
    gen += 1u;
    __syncthreads();
    __threadfence();
}

__device__ __forceinline__ bool is_done(const PcgDev& c)
{
    return *((volatile int*)c.flags + F_DONE) != 0;
}

template <typename T, int B>
__global__ void __launch_bounds__(PB) k_pcg_persistent(PcgDev c)
{
    unsigned gen = 0;
    const int gt = GT, gn = GN;
    constexpr int BB = B > 0 ? B : 16;
    // banks of levels 0..2 need only R_0..R_2 (ready after C1); the coarser ones wait for C2,
    // which CTA 0 runs before solving them while the other CTAs solve the finer banks
    const int split = c.L > 3 ? c.ls[2 * 3 + 1] / BB : c.nbanks;
    for(long guard = 0; guard < c.prm.max_iter + 2; guard++)
    {
        if(is_done(c)) break;
        grid_barrier(c, phase_a<T>(c, gt, gn), SITE_A, POST_ALPHA, gen);
        if(is_done(c)) break;
        const double alpha = __ldcg(c.scal + SS_ALPHA);
        BSlot<T> none;
        const double vb =
            B > 0 ? phase_b_mas<T, BB, false>(c, gt, gn, alpha, none, false) : phase_b_plain<T>(c, gt, gn, alpha);
        grid_barrier(c, vb, SITE_B, POST_CHECK, gen);
        if(is_done(c)) break;
        const long k = (long)__ldcg(c.scal + SS_ITER);
        if(c.prm.refine > 0 && k % c.prm.refine == 0)
        {
            if(blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(c.flags + F_REPL, 1);
            grid_barrier(c, phase_replace(c, gt, gn), SITE_R, POST_RECHECK, gen);
            if(is_done(c)) break;
            if(B > 0)
            {
                phase_restrict01<BB>(c, gt, gn);
                grid_barrier(c, 0.0, 0, -1, gen);
            }
        }
        if(B > 0)
        {
            phase_c<BB>(c, 1, 2, gt, gn, false);
            grid_barrier(c, 0.0, 0, -1, gen);
            if(gridDim.x == 1)
            {
                phase_c<BB>(c, 2, c.L - 1, threadIdx.x, blockDim.x, true);
                phase_d<BB>(c, 0, c.nbanks, 1);
            }
            else if(blockIdx.x == 0)
            {
                phase_c<BB>(c, 2, c.L - 1, threadIdx.x, blockDim.x, true);
                phase_d<BB>(c, split, c.nbanks, 1);
            }
            else
                phase_d<BB>(c, blockIdx.x - 1, split, gridDim.x - 1);
            grid_barrier(c, 0.0, 0, -1, gen);
        }
        const double ve = B > 0 ? phase_e_mas<T>(c, gt, gn) : phase_e_plain<T>(c, gt, gn);
        grid_barrier(c, ve, SITE_E, POST_BETA, gen);
    }
}

// ---------------------------------------------------------------------------------------
// layout preparation
// ---------------------------------------------------------------------------------------
__global__ void k_pack_blocks(const double* __restrict__ src, int nnzb, float* dst32, double* dst64)
{
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnzb; k += gridDim.x * blockDim.x)
    {
        const double* s = src + 9 * (size_t)k;
        if(dst32)
        {
            float4* d = reinterpret_cast<float4*>(dst32) + 3 * (size_t)k;
            d[0] = make_float4((float)s[0], (float)s[1], (float)s[2], (float)s[3]);
            d[1] = make_float4((float)s[4], (float)s[5], (float)s[6], (float)s[7]);
            d[2] = make_float4((float)s[8], 0.f, 0.f, 0.f);
        }
        if(dst64)
        {
            double2* d = reinterpret_cast<double2*>(dst64) + 5 * (size_t)k;
            d[0] = make_double2(s[0], s[1]);
            d[1] = make_double2(s[2], s[3]);
            d[2] = make_double2(s[4], s[5]);
            d[3] = make_double2(s[6], s[7]);
            d[4] = make_double2(s[8], 0.0);
        }
    }
}

// Builds the full symmetric plane copy (FullPlanes) used by the PCG SpMV (phase A): row i
// holds its lower blocks (transposes of the upper blocks k with col(k) == i, in transpose-
// list order) followed by its upper blocks.  16 lanes per row, one entry per lane.
template <typename T>
__global__ void k_build_full(const int* __restrict__ row_ptr, const int* __restrict__ cols,
                             const int* __restrict__ t_ptr, const int2* __restrict__ t_ent,
                             const double* __restrict__ blocks, int nrows, size_t S, unsigned char* fent)
{
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, sub = gt & 15;
    for(int i = gt >> 4; i < nrows; i += (gridDim.x * blockDim.x) >> 4)
    {
        const int u0 = row_ptr[i], nu = row_ptr[i + 1] - u0;
        const int t0 = t_ptr[i], nt = t_ptr[i + 1] - t0;
        const size_t f0 = (size_t)u0 + t0;
        for(int e = sub; e < nt + nu; e += 16)
        {
            T h[9];
            int col;
            if(e < nt)
            {
                const int2 te = t_ent[t0 + e];
                const double* H = blocks + 9 * (size_t)te.x;
#pragma unroll
                for(int a = 0; a < 3; a++)
#pragma unroll
                    for(int b = 0; b < 3; b++) h[b * 3 + a] = (T)H[a * 3 + b];  // H^T
                col = te.y;
            }
            else
            {
                const int k = u0 + e - nt;
                const double* H = blocks + 9 * (size_t)k;
#pragma unroll
                for(int t = 0; t < 9; t++) h[t] = (T)H[t];
                col = cols[k];
            }
            store_entry(fent, S, f0 + e, h, col);
        }
    }
}

// first full-copy entry of every row: frow[i] = row_ptr[i] + t_ptr[i], i <= nrows
__global__ void k_frow(const int* __restrict__ row_ptr, const int* __restrict__ t_ptr, int nrows, int* frow)
{
    for(int i = blockIdx.x * blockDim.x + threadIdx.x; i <= nrows; i += gridDim.x * blockDim.x)
        frow[i] = row_ptr[i] + t_ptr[i];
}

// Builds the upper copy (UpperPlanes) used by the upper SpMV phase: entry k is upper block k
// in the iteration precision with its column and slot -1; k_upper_slots then gives every
// block of a transpose list its place t in that list.
template <typename T>
__global__ void k_build_upper(const int* __restrict__ cols, const double* __restrict__ blocks, int nnzb, size_t S,
                              unsigned char* uent)
{
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnzb; k += gridDim.x * blockDim.x)
    {
        T h[9];
        const double* H = blocks + 9 * (size_t)k;
#pragma unroll
        for(int t = 0; t < 9; t++) h[t] = (T)H[t];
        store_upper(uent, S, (size_t)k, h, cols[k], -1);
    }
}

template <typename T>
__global__ void k_upper_slots(const int2* __restrict__ t_ent, const int* __restrict__ t_ptr, int nrows, size_t S,
                              unsigned char* uent)
{
    const int count = t_ptr[nrows];
    for(int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x)
        *upper_slot_ptr<T>(uent, S, (size_t)t_ent[t].x) = t;
}

// Whether the SpMV phase of the next solve runs the upper kernel: when chosen
// (stg_spmv_tiles), picked by the autotuner, or by default in FP32.  Measured on the
// 352,947-DOF cube, the FP32 solve takes the same time with either kernel (the upper one
// moves 1.05x its algorithmic bytes, the full copy 1.68x, and holds half the matrix
// bytes); in FP64 the upper kernel's spill (32 B per transposed product) costs more than it
// saves and the full copy is the default.  The persistent loop's SpMV reads the full copy.
static bool upper_spmv_selected(const Solver& S)
{
    if(S.cfg.loop_mode == STG_LOOP_PERSISTENT) return false;
    if(S.spmv_rt == SPMV_UPPER) return true;
    if(S.spmv_rt != 0) return false;
    return S.spmv_tune ? S.tuned_rt == SPMV_UPPER : S.cfg.precision == STG_PREC_FP32;
}

int pack_blocks(Solver& S)
{
    Bcoo& A = S.bcoo;
    const int nnzb = A.nnzb;
    A.upper_built = false;
    if(nnzb < 1) return 0;
    STG_TRY(A.blk64p.resize((size_t)nnzb * 10));
    const bool fp32 = S.cfg.precision == STG_PREC_FP32;
    k_pack_blocks<<<std::max(1, std::min(div_up(nnzb, 256), kSMs * 16)), 256, 0, S.stream>>>(A.B(), nnzb, nullptr,
                                                                                           A.blk64p.data());
    STG_LAUNCH_CHECK();
    // the autotuner times every kernel: both copies; otherwise the copy the chosen kernel reads
    const bool tuning = S.spmv_tune && S.spmv_rt == 0 && S.cfg.loop_mode != STG_LOOP_PERSISTENT;
    const bool need_upper = tuning || upper_spmv_selected(S);
    const bool need_full = tuning || !upper_spmv_selected(S);
    if(need_upper)
    {
        // plane stride: a multiple of 4 entries covering every 4-aligned tile range
        A.ustride = ((size_t)nnzb + 7) & ~(size_t)3;
        STG_TRY(A.urow.resize((size_t)A.nrows + 1 + 136));  // tiles copy row_ptr[r0 .. r0 + RT + 4)
        STG_CUDA_TRY(cudaMemcpyAsync(A.urow.data(), A.row_ptr.data(), sizeof(int) * ((size_t)A.nrows + 1),
                                     cudaMemcpyDeviceToDevice, S.stream));
        const int gu = std::max(1, std::min(div_up(nnzb, 256), kSMs * 16));
        if(fp32)
        {
            STG_TRY(A.uent.resize(A.ustride * UpperPlanes<float>::ES));
            k_build_upper<float><<<gu, 256, 0, S.stream>>>(A.C(), A.B(), nnzb, A.ustride, A.uent.data());
            STG_LAUNCH_CHECK();
            k_upper_slots<float><<<gu, 256, 0, S.stream>>>(A.t_ent.data(), A.t_ptr.data(), A.nrows, A.ustride,
                                                          A.uent.data());
        }
        else
        {
            STG_TRY(A.uent.resize(A.ustride * UpperPlanes<double>::ES));
            k_build_upper<double><<<gu, 256, 0, S.stream>>>(A.C(), A.B(), nnzb, A.ustride, A.uent.data());
            STG_LAUNCH_CHECK();
            k_upper_slots<double><<<gu, 256, 0, S.stream>>>(A.t_ent.data(), A.t_ptr.data(), A.nrows, A.ustride,
                                                           A.uent.data());
        }
        STG_LAUNCH_CHECK();
        S.launches += 2;
        // spill slots: 4 values of the iteration precision per transpose-list entry (< nnzb)
        STG_TRY(S.pcg.spill.resize((size_t)nnzb * (fp32 ? 2 : 4)));
        A.upper_built = true;
    }
    if(!need_full)
    {
        A.halo_ok = false;
        return 0;
    }
    // full symmetric copy: at most 2 * nnzb entries per plane, rounded up to an even count
    // so that every even-aligned entry range of the 8-byte tail plane is a 16-byte multiple
    A.fstride = ((size_t)2 * nnzb + 2) & ~(size_t)1;
    STG_TRY(A.frow.resize((size_t)A.nrows + 1 + 72));  // tiles copy frow[r0 .. r0 + RT + 4)
    k_frow<<<std::max(1, std::min(div_up(A.nrows + 1, 256), kSMs * 8)), 256, 0, S.stream>>>(
        A.row_ptr.data(), A.t_ptr.data(), A.nrows, A.frow.data());
    STG_LAUNCH_CHECK();
    S.launches++;
    const int g = std::max(1, std::min(div_up(A.nrows, 16), kSMs * 16));
    if(fp32)
    {
        STG_TRY(A.fent.resize(A.fstride * FullPlanes<float>::ES));
        k_build_full<float><<<g, 256, 0, S.stream>>>(A.row_ptr.data(), A.C(), A.t_ptr.data(), A.t_ent.data(), A.B(),
                                                     A.nrows, A.fstride, A.fent.data());
    }
    else
    {
        STG_TRY(A.fent.resize(A.fstride * FullPlanes<double>::ES));
        k_build_full<double><<<g, 256, 0, S.stream>>>(A.row_ptr.data(), A.C(), A.t_ptr.data(), A.t_ent.data(), A.B(),
                                                      A.nrows, A.fstride, A.fent.data());
    }
    STG_LAUNCH_CHECK();
    S.launches += 2;
    // operand windows of the halo SpMV phase (one CTA per tile), when that kernel may run
    A.halo_ok = false;
    if(S.spmv_rt == SPMV_HALO || S.spmv_tune)
    {
        const int rt = fp32 ? AHalo<float>::RT : AHalo<double>::RT;
        const int hcap = fp32 ? AHalo<float>::HCAP : AHalo<double>::HCAP;
        const int tiles = div_up(A.nrows, rt);
        STG_TRY(A.hcnt.resize(tiles));
        STG_TRY(A.hlist.resize((size_t)tiles * hcap));
        STG_TRY(A.htail.resize(A.fstride * (size_t)FullPlanes<double>::TAIL));
        STG_TRY(S.cv.scratch.resize(4));
        int* bad = S.cv.scratch.data() + 3;
        STG_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), S.stream));
        if(fp32)
            k_tile_halo<float><<<tiles, 256, 0, S.stream>>>(A.frow.data(), A.fent.data(), A.fstride, A.nrows,
                                                            A.hcnt.data(), A.hlist.data(), A.htail.data(), bad);
        else
            k_tile_halo<double><<<tiles, 256, 0, S.stream>>>(A.frow.data(), A.fent.data(), A.fstride, A.nrows,
                                                             A.hcnt.data(), A.hlist.data(), A.htail.data(), bad);
        STG_LAUNCH_CHECK();
        S.launches++;
        int h = 0;
        STG_CUDA_TRY(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, S.stream));
        STG_CUDA_TRY(cudaStreamSynchronize(S.stream));
        A.halo_ok = h == 0;
    }
    return 0;
}

// Diagnostic for the bounded waits: one thread arms an mbarrier that no arrival or copy will
// ever complete and waits on it with the same bounded poll as the bulk-copy pipelines
// (mbar_wait).  The wait gives up, the kernel records STG_ERR_TIMEOUT and the elapsed
// nanoseconds, and returns; nothing is in flight, so the context stays usable.
__global__ void k_selftest_wait(int* status, unsigned long long* ns)
{
    __shared__ __align__(8) unsigned long long bar;
    if(threadIdx.x != 0) return;
    const unsigned b = smem_u32(&bar);
    mbar_init(b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    unsigned long long t0, t1;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    const bool ok = mbar_wait(b, 0);
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
    *status = ok ? 0 : 6;  // STG_ERR_TIMEOUT
    *ns = t1 - t0;
}

int selftest_wait(int* status, double* seconds)
{
    int* d_status = nullptr;
    unsigned long long* d_ns = nullptr;
    STG_CUDA_TRY(cudaMalloc(&d_status, sizeof(int) + sizeof(unsigned long long) * 2));
    d_ns = reinterpret_cast<unsigned long long*>(d_status + 2);
    k_selftest_wait<<<1, 32>>>(d_status, d_ns);
    cudaError_t e = cudaGetLastError();
    int h_status = -1;
    unsigned long long h_ns = 0;
    if(e == cudaSuccess) e = cudaMemcpy(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if(e == cudaSuccess) e = cudaMemcpy(&h_ns, d_ns, sizeof(h_ns), cudaMemcpyDeviceToHost);
    cudaFree(d_status);
    STG_CUDA_TRY(e);
    if(status) *status = h_status;
    if(seconds) *seconds = 1e-9 * (double)h_ns;
    return 0;
}

// ---------------------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------------------
// MAS levels >= 2 restriction (C1 parallel, C2 one CTA) and the bank solves (D)
// the 16-bank solves of banks [b0, b1): warp per bank, TMA-staged; one resident wave of CTAs
static int launch_d16(Solver& S, const PcgDev& c, int b0, int b1, int guarded)
{
    if(b1 <= b0) return 0;
    const int smem = D_WARPS * D_WARP_BYTES;
    static thread_local unsigned long long attr_done = 0;
    if(first_on_device(attr_done))
        STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_d16, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0;
    STG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_phase_d16, D_WARPS * 32, smem));
    const int grid = std::max(1, std::min(div_up(b1 - b0, D_WARPS), std::max(per_sm, 1) * kSMs));
    k_phase_d16<<<grid, D_WARPS * 32, smem, S.stream>>>(c, b0, b1, guarded);
    STG_LAUNCH_CHECK();
    S.launches++;
    return 0;
}

// Restriction of the coarse levels and the bank solves of every level.
template <int B>
static int launch_mas_cd(Solver& S, const PcgDev& c)
{
    cudaStream_t s = S.stream;
    if(c.L > 2)
    {
        const int n1 = (c.ls[2] + 31) / 32 * 32;
        k_phase_c1<B><<<std::max(1, std::min(div_up(n1, PB), kSMs * 4)), PB, 0, s>>>(c);
        STG_LAUNCH_CHECK();
        S.launches++;
    }
    if(c.L > 3)
    {
        k_phase_c2<B><<<1, 1024, C2_SMEM_BYTES, s>>>(c);
        STG_LAUNCH_CHECK();
        S.launches++;
    }
    if(B == 16) return launch_d16(S, c, 0, c.nbanks, 0);
    k_phase_d<B><<<std::max(1, std::min(c.nbanks, kSMs * 8)), PB, 0, s>>>(c);
    STG_LAUNCH_CHECK();
    S.launches++;
    return 0;
}


// tiled phase A: the shared-memory opt-in and one resident wave of CTAs, per tile shape
template <typename T, int RT>
static int phase_a_grid_rt(int nrows, int* grid)
{
    static thread_local unsigned long long seen = 0;
    static thread_local int per_sm_dev[64];
    int dev = 0;
    STG_CUDA_TRY(cudaGetDevice(&dev));
    int& per_sm = per_sm_dev[dev & 63];
    if(first_on_device(seen))
    {
        STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_a_tiled<T, RT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          ATile<T, RT>::SMEM));
        STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_a_tiled<T, RT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                          cudaSharedmemCarveoutMaxShared));
        STG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_phase_a_tiled<T, RT>, A_THREADS,
                                                                   ATile<T, RT>::SMEM));
    }
    *grid = std::max(1, std::min(div_up(nrows, RT), std::max(per_sm, 1) * kSMs));
    return 0;
}

// the halo SpMV phase: one resident wave of CTAs over the fixed tiles
template <typename T>
static int phase_a_grid_halo(int nrows, int* grid)
{
    static thread_local unsigned long long seen = 0;
    static thread_local int per_sm_dev[64];
    int dev = 0;
    STG_CUDA_TRY(cudaGetDevice(&dev));
    int& per_sm = per_sm_dev[dev & 63];
    if(first_on_device(seen))
    {
        STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_a_halo<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, AHalo<T>::SMEM));
        STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_a_halo<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                          cudaSharedmemCarveoutMaxShared));
        STG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_phase_a_halo<T>, A_THREADS, AHalo<T>::SMEM));
    }
    *grid = std::max(1, std::min(div_up(nrows, AHalo<T>::RT), std::max(per_sm, 1) * kSMs));
    return 0;
}

// the upper SpMV phase: one resident wave of CTAs
template <typename T>
static int phase_a_grid_upper(int nrows, int* grid)
{
    static thread_local unsigned long long seen = 0;
    static thread_local int per_sm_dev[64];
    int dev = 0;
    STG_CUDA_TRY(cudaGetDevice(&dev));
    int& per_sm = per_sm_dev[dev & 63];
    if(first_on_device(seen))
    {
        STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_a_upper<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          AUpper<T>::SMEM));
        STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_a_upper<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                          cudaSharedmemCarveoutMaxShared));
        STG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_phase_a_upper<T>, A_THREADS,
                                                                   AUpper<T>::SMEM));
    }
    *grid = std::max(1, std::min(div_up(nrows, AUpper<T>::RT), std::max(per_sm, 1) * kSMs));
    return 0;
}

template <typename T>
static int phase_a_grid(int nrows, int rt, int* grid, bool halo = false, bool upper = false)
{
    if(upper) return phase_a_grid_upper<T>(nrows, grid);
    if(halo) return phase_a_grid_halo<T>(nrows, grid);
    if(rt == a_rt_alt<T>()) return phase_a_grid_rt<T, a_rt_alt<T>()>(nrows, grid);
    return phase_a_grid_rt<T, a_rt_default<T>()>(nrows, grid);
}

template <typename T>
static int launch_phase_a(const PcgDev& c, cudaStream_t s)
{
    int grid = 0;
    STG_TRY(phase_a_grid<T>(c.nrows, c.a_rt, &grid, c.halo != 0, c.upper != 0));
    if(grid != c.grid_a)
    {
        set_error("SpMV phase grid differs from the one phase B sums over");
        return STG_ERR_INVALID;
    }
    if(c.upper)
        k_phase_a_upper<T><<<grid, A_THREADS, AUpper<T>::SMEM, s>>>(c);
    else if(c.halo)
        k_phase_a_halo<T><<<grid, A_THREADS, AHalo<T>::SMEM, s>>>(c);
    else if(c.a_rt == a_rt_alt<T>())
        k_phase_a_tiled<T, a_rt_alt<T>()><<<grid, A_THREADS, ATile<T, a_rt_alt<T>()>::SMEM, s>>>(c);
    else
        k_phase_a_tiled<T, a_rt_default<T>()><<<grid, A_THREADS, ATile<T>::SMEM, s>>>(c);
    STG_LAUNCH_CHECK();
    return 0;
}

// BCOO tile autotuner: every candidate of the SpMV phase launched on this system (3 untimed,
// then `reps` timed with CUDA events): the two tile shapes of the tiled kernel and, when its
// operand windows fit (halo_ok), the halo kernel.  Returns the fastest (its rows per tile, or
// SPMV_HALO) and each mean.
template <typename T>
static int tune_phase_a(Solver& S, PcgDev c, float* us, int* out)
{
    const int cand[4] = {a_rt_default<T>(), a_rt_alt<T>(), SPMV_HALO, SPMV_UPPER};
    float best = 0.f;
    int pick = cand[0];
    for(int v = 0; v < 4; v++)
    {
        us[v] = 0.f;
        if((cand[v] == SPMV_HALO && !S.bcoo.halo_ok) || (cand[v] == SPMV_UPPER && !S.bcoo.upper_built)) continue;
        c.halo = cand[v] == SPMV_HALO ? 1 : 0;
        c.upper = cand[v] == SPMV_UPPER ? 1 : 0;
        c.spill = c.upper ? S.pcg.spill.data() : nullptr;
        c.a_rt = (c.halo || c.upper) ? a_rt_default<T>() : cand[v];
        STG_TRY(phase_a_grid<T>(c.nrows, c.a_rt, &c.grid_a, c.halo != 0, c.upper != 0));
        for(int i = 0; i < 3; i++) STG_TRY(launch_phase_a<T>(c, S.stream));
        const int reps = 10;
        STG_CUDA_TRY(cudaEventRecord(S.ev[4], S.stream));
        for(int i = 0; i < reps; i++) STG_TRY(launch_phase_a<T>(c, S.stream));
        STG_CUDA_TRY(cudaEventRecord(S.ev[5], S.stream));
        STG_CUDA_TRY(cudaEventSynchronize(S.ev[5]));
        float ms = 0.f;
        STG_CUDA_TRY(cudaEventElapsedTime(&ms, S.ev[4], S.ev[5]));
        us[v] = 1e3f * ms / reps;
        S.launches += 3 + reps;
        if(v == 0 || us[v] < best)
        {
            best = us[v];
            pick = cand[v];
        }
    }
    *out = pick;
    return 0;
}

// learned coarse correction after the bank solves: the sample recorder (the level's r and
// z before any correction), then the network's forward pass and apply on the level's Z
static int launch_learned(Solver& S, const PcgDev& c)
{
    LearnedState& Ls = S.learned;
    const float* R = c.R + 4 * (size_t)Ls.begin;
    float* Z = c.Z + 4 * (size_t)Ls.begin;
    if(c.net_mode & 2)
    {
        STG_TRY(net_record(S.stream, R, Z, Ls.graph.n, c.scal, c.flags, Ls.rec_rc, Ls.rec_zc, Ls.rec_count.data(),
                           Ls.rec_cap, Ls.rec_every));
        S.launches++;
    }
    if((c.net_mode & 1) && Ls.graph.fu_cl > 0)
    {
        STG_TRY(net_forward_fused(S.stream, Ls.graph.view(), Ls.graph.nnz > 0 ? Ls.graph.fu_nb.data() : nullptr, R, Z,
                                  Ls.wbf.data(), Ls.params.data(), c.flags, Ls.graph.fu_cl, Ls.graph.fu_rpc));
        S.launches++;
    }
    else if(c.net_mode & 1)
        STG_TRY(net_forward(S.stream, Ls.graph.view(), R, Z, 1, Ls.buf, Ls.wbf.data(), Ls.params.data(), Z, c.flags,
                            &S.launches));
    return 0;
}

template <typename T, int B>
static int launch_iteration(Solver& S, const PcgDev& c, int grid_vec, int grid_rows, bool in_graph_cond)
{
    cudaStream_t s = S.stream;
    const bool fp32 = sizeof(T) == 4;
    STG_TRY(launch_phase_a<T>(c, s));
    if(c.seg_of_row)
    {
        k_seg<SEG_A><<<c.nseg, PB, 0, s>>>(c);
        STG_LAUNCH_CHECK();
        S.launches++;
    }
    k_phase_b<T, B><<<B > 0 ? std::max(1, std::min(div_up(c.M, PB), kSMs * 4)) : grid_vec, PB, 0, s>>>(c);
    STG_LAUNCH_CHECK();
    S.launches += 2;
    if(c.seg_of_row)
    {
        k_seg<SEG_B><<<c.nseg, PB, 0, s>>>(c);
        STG_LAUNCH_CHECK();
        S.launches++;
    }
    if(fp32 && c.prm.refine > 0)
    {
        if(in_graph_cond)
        {
            // IF node: replacement (+ re-restriction) only on replacement iterations
            cudaStreamCaptureStatus st;
            cudaGraph_t capg;
            const cudaGraphNode_t* deps;
            size_t ndeps = 0;
            STG_CUDA_TRY(cudaStreamGetCaptureInfo(s, &st, nullptr, &capg, &deps, &ndeps));
            cudaGraphNodeParams ip = {};
            ip.type = cudaGraphNodeTypeConditional;
            ip.conditional.handle = c.h_if;
            ip.conditional.type = cudaGraphCondTypeIf;
            ip.conditional.size = 1;
            cudaGraphNode_t ifnode;
            STG_CUDA_TRY(cudaGraphAddNode(&ifnode, capg, deps, ndeps, &ip));
            STG_CUDA_TRY(cudaStreamUpdateCaptureDependencies(s, &ifnode, 1, cudaStreamSetCaptureDependencies));
            // the IF body is recorded by the caller (see record_if_body)
            S.pending_if_body = ip.conditional.phGraph_out[0];
        }
        else
        {
            k_replace<<<grid_rows, PB, 0, s>>>(c, 1);
            STG_LAUNCH_CHECK();
            S.launches++;
            if(B > 0)
            {
                k_restrict01<(B > 0 ? B : 16)><<<std::max(1, std::min(div_up(c.M, PB), kSMs * 4)), PB, 0, s>>>(c, 1);
                STG_LAUNCH_CHECK();
                S.launches++;
            }
        }
    }
    if(B > 0) STG_TRY(launch_mas_cd<(B > 0 ? B : 16)>(S, c));
    if(c.net_mode) STG_TRY(launch_learned(S, c));
    k_phase_e<T, B><<<grid_vec, PB, 0, s>>>(c, POST_BETA);
    STG_LAUNCH_CHECK();
    S.launches++;
    if(c.seg_of_row)
    {
        k_seg<SEG_E><<<c.nseg, PB, 0, s>>>(c);
        STG_LAUNCH_CHECK();
        S.launches++;
    }
    return 0;
}

template <typename T, int B>
static int record_if_body(Solver& S, const PcgDev& c, int grid_rows, cudaGraph_t body)
{
    cudaStream_t s = S.stream;
    STG_CUDA_TRY(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    k_replace<<<grid_rows, PB, 0, s>>>(c, 0);
    cudaError_t e1 = cudaGetLastError();
    if(B > 0 && e1 == cudaSuccess)
    {
        k_restrict01<(B > 0 ? B : 16)><<<std::max(1, std::min(div_up(c.M, PB), kSMs * 4)), PB, 0, s>>>(c, 0);
        e1 = cudaGetLastError();
    }
    cudaGraph_t out = body;
    cudaError_t e2 = cudaStreamEndCapture(s, &out);
    STG_CUDA_TRY(e1);
    STG_CUDA_TRY(e2);
    return 0;
}

// Every kernel of the iteration asks for the same shared-memory carveout (the largest), so
// that consecutive phases do not make the SMs switch their L1 / shared split between
// launches.
template <typename T, int B>
static int set_carveouts()
{
    static thread_local unsigned long long done = 0;
    if(!first_on_device(done)) return 0;
    const int cv = cudaSharedmemCarveoutMaxShared;
    constexpr int BB = B > 0 ? B : 16;
    STG_CUDA_TRY(cudaFuncSetAttribute(k_init<T>, cudaFuncAttributePreferredSharedMemoryCarveout, cv));
    STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_b<T, B>, cudaFuncAttributePreferredSharedMemoryCarveout, cv));
    STG_CUDA_TRY(cudaFuncSetAttribute(k_replace, cudaFuncAttributePreferredSharedMemoryCarveout, cv));
    STG_CUDA_TRY(cudaFuncSetAttribute(k_restrict01<BB>, cudaFuncAttributePreferredSharedMemoryCarveout, cv));
    STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_c1<BB>, cudaFuncAttributePreferredSharedMemoryCarveout, cv));
    STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_c2<BB>, cudaFuncAttributePreferredSharedMemoryCarveout, cv));
    STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_c2<BB>, cudaFuncAttributeMaxDynamicSharedMemorySize, C2_SMEM_BYTES));
    STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_d<BB>, cudaFuncAttributePreferredSharedMemoryCarveout, cv));
    STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_d16, cudaFuncAttributePreferredSharedMemoryCarveout, cv));
    STG_CUDA_TRY(cudaFuncSetAttribute(k_phase_e<T, B>, cudaFuncAttributePreferredSharedMemoryCarveout, cv));
    return 0;
}

template <typename T, int B>
static int pcg_run(Solver& S, PcgDev& c, int& h_done)
{
    STG_TRY((set_carveouts<T, B>()));
    STG_TRY(phase_a_grid<T>(c.nrows, c.a_rt, &c.grid_a, c.halo != 0, c.upper != 0));
    c.grid_e = std::max(1, std::min(div_up(c.n, PB), kSMs * 4));  // grid_vec below
    if(c.grid_a > c.slots || c.grid_e > c.slots)
    {
        set_error("SpMV phase grid larger than the reduction slots");
        return STG_ERR_INVALID;
    }
    cudaStream_t s = S.stream;
    PcgState& P = S.pcg;
    const int grid_vec = std::max(1, std::min(div_up(c.n, PB), kSMs * 4));
    // the SpMV phase runs as exactly one resident wave (grid-stride over the rows)
    int per_sm_a = 0;
    STG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_a, k_phase_a<T>, PB, 0));
    const int grid_rows = std::max(1, std::min(div_up(c.nrows, PB / 16), std::max(per_sm_a, 1) * kSMs));
    const int grid_b = B > 0 ? std::max(1, std::min(div_up(c.M, PB), kSMs * 4)) : grid_vec;
    // init: r = b, x = 0, p = 0, b.b; z = M^-1 r, rz = rz0 = r.z (beta = 0 so p_new = z)
    k_init<T><<<grid_vec, PB, 0, s>>>(c);
    STG_LAUNCH_CHECK();
    S.launches++;
    if(B > 0)
    {
        constexpr int BB = B > 0 ? B : 16;
        k_restrict01<BB><<<grid_b, PB, 0, s>>>(c, 0);
        STG_LAUNCH_CHECK();
        S.launches++;
        STG_TRY(launch_mas_cd<BB>(S, c));
        if(c.net_mode) STG_TRY(launch_learned(S, c));
    }
    k_phase_e<T, B><<<grid_vec, PB, 0, s>>>(c, POST_INIT_RZ);
    STG_LAUNCH_CHECK();
    S.launches++;
    if(c.seg_of_row)
    {
        k_seg<SEG_INIT><<<c.nseg, PB, 0, s>>>(c);
        STG_LAUNCH_CHECK();
        S.launches++;
    }

    int h_flags[4] = {0, 0, 0, 0};
    const long max_iter = c.prm.max_iter;
    if(max_iter <= 1)
    {
        h_done = 1;
        return 0;
    }
    const int mode = S.cfg.loop_mode;
    if(mode == STG_LOOP_HOST)
    {
        for(long it = 1; it <= max_iter; it++)
        {
            STG_TRY((launch_iteration<T, B>(S, c, grid_vec, grid_rows, false)));
            STG_CUDA_TRY(cudaMemcpyAsync(h_flags, P.flags.data(), sizeof(int) * 4, cudaMemcpyDeviceToHost, s));
            STG_CUDA_TRY(cudaStreamSynchronize(s));
            if(h_flags[F_DONE]) break;
        }
    }
    else if(mode == STG_LOOP_GRAPH)
    {
        // graph: WHILE(cond) { iteration }, cond initialised to 1 (at every launch) and set by
        // the stop test.  The captured kernels hold the parameter block by value: when it is
        // bytewise the one of the last capture (same buffers, sizes, scalars and kernel
        // variant), the instantiated graph is launched again instead of re-captured.
        PcgDev key = c;
        key.h_while = 0;
        key.h_if = 0;
        key.use_cond = 0;
        const int variant = (int)sizeof(T) * 1000 + B;
        if(P.graph && P.graph_variant == variant && std::memcmp(&key, &P.graph_key, sizeof(key)) == 0)
        {
            c.h_while = P.graph_dev.h_while;
            c.h_if = P.graph_dev.h_if;
            c.use_cond = P.graph_dev.use_cond;
            STG_CUDA_TRY(cudaGraphLaunch(P.graph, s));
            STG_CUDA_TRY(cudaMemcpyAsync(h_flags, P.flags.data(), sizeof(int) * 4, cudaMemcpyDeviceToHost, s));
            STG_CUDA_TRY(cudaStreamSynchronize(s));
            c.use_cond = 0;
            h_done = h_flags[F_DONE];
            return 0;
        }
        if(P.graph)
        {
            cudaGraphExecDestroy(P.graph);
            P.graph = nullptr;
        }
        if(!S.capture_stream) STG_CUDA_TRY(cudaStreamCreateWithFlags(&S.capture_stream, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        STG_CUDA_TRY(cudaGraphCreate(&g, 0));
        int rc = 0;
        do
        {
            // a conditional handle must belong to exactly one conditional node: the IF handle
            // exists only when the body holds the residual-replacement node (FP32 mode)
            const bool need_if = sizeof(T) == 4 && c.prm.refine > 0;
            cudaGraphConditionalHandle hw = 0, hi = 0;
            if(cudaGraphConditionalHandleCreate(&hw, g, 1, cudaGraphCondAssignDefault) != cudaSuccess ||
               (need_if && cudaGraphConditionalHandleCreate(&hi, g, 0, cudaGraphCondAssignDefault) != cudaSuccess))
            {
                set_error(std::string("cudaGraphConditionalHandleCreate failed: ") + cudaGetErrorString(cudaGetLastError()));
                rc = STG_ERR_CUDA;
                break;
            }
            c.h_while = hw;
            c.h_if = hi;
            c.use_cond = need_if ? 2 : 1;  // 2: the stop test also drives the IF node
            cudaGraphNodeParams wp = {};
            wp.type = cudaGraphNodeTypeConditional;
            wp.conditional.handle = hw;
            wp.conditional.type = cudaGraphCondTypeWhile;
            wp.conditional.size = 1;
            cudaGraphNode_t wnode;
            if(cudaGraphAddNode(&wnode, g, nullptr, 0, &wp) != cudaSuccess)
            {
                set_error(std::string("cudaGraphAddNode(WHILE) failed: ") + cudaGetErrorString(cudaGetLastError()));
                rc = STG_ERR_CUDA;
                break;
            }
            cudaGraph_t body = wp.conditional.phGraph_out[0];
            cudaStream_t user = S.stream;
            S.stream = S.capture_stream;
            S.pending_if_body = nullptr;
            cudaError_t cb = cudaStreamBeginCaptureToGraph(S.stream, body, nullptr, nullptr, 0,
                                                           cudaStreamCaptureModeThreadLocal);
            if(cb != cudaSuccess)
            {
                S.stream = user;
                set_error(std::string("cudaStreamBeginCaptureToGraph failed: ") + cudaGetErrorString(cb));
                rc = STG_ERR_CUDA;
                break;
            }
            const int l0 = S.launches;
            rc = launch_iteration<T, B>(S, c, grid_vec, grid_rows, true);
            cudaGraph_t out = body;
            cudaError_t ce = cudaStreamEndCapture(S.stream, &out);
            if(rc == 0 && ce != cudaSuccess)
            {
                set_error(std::string("cudaStreamEndCapture failed: ") + cudaGetErrorString(ce));
                rc = STG_ERR_CUDA;
            }
            if(rc == 0 && S.pending_if_body) rc = record_if_body<T, B>(S, c, grid_rows, S.pending_if_body);
            S.stream = user;
            S.launches_per_batch = S.launches - l0;
            S.launches = l0;
            if(rc) break;
            cudaError_t ie = cudaGraphInstantiate(&P.graph, g, 0);
            if(ie != cudaSuccess)
            {
                set_error(std::string("cudaGraphInstantiate failed: ") + cudaGetErrorString(ie));
                rc = STG_ERR_CUDA;
            }
        } while(0);
        cudaGraphDestroy(g);
        if(rc) return rc;
        P.graph_key = key;
        P.graph_dev = c;
        P.graph_variant = variant;
        STG_CUDA_TRY(cudaGraphLaunch(P.graph, s));
        STG_CUDA_TRY(cudaMemcpyAsync(h_flags, P.flags.data(), sizeof(int) * 4, cudaMemcpyDeviceToHost, s));
        STG_CUDA_TRY(cudaStreamSynchronize(s));
        c.use_cond = 0;
    }
    else
    {
        // persistent cooperative kernel: every CTA must be resident
        int per_sm = 0;
        STG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_persistent<T, B>, PB, 0));
        int dev = 0, sms = kSMs;
        STG_CUDA_TRY(cudaGetDevice(&dev));
        STG_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const int grid = std::max(1, std::min(per_sm, 4) * sms);
        if(grid > c.slots)
        {
            set_error("persistent grid larger than the reduction slots");
            return STG_ERR_INVALID;
        }
        STG_CUDA_TRY(cudaMemsetAsync(c.bar, 0, sizeof(unsigned) * 2, s));
        void* args[] = {&c};
        STG_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k_pcg_persistent<T, B>, grid, PB, args, 0, s));
        S.launches++;
        STG_CUDA_TRY(cudaMemcpyAsync(h_flags, P.flags.data(), sizeof(int) * 4, cudaMemcpyDeviceToHost, s));
        STG_CUDA_TRY(cudaStreamSynchronize(s));
    }
    h_done = h_flags[F_DONE];
    return 0;
}

// reads `n` 16-byte words (evicts the L2 without leaving dirty lines to write back)
__global__ void k_l2_scrub(const uint4* __restrict__ buf, size_t n, unsigned* sink)
{
    unsigned acc = 0;
    for(size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    {
        const uint4 v = __ldcs(buf + i);
        acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
    if(acc == 0x9e3779b9u) *sink = acc;  // keeps the loads; the buffer is zero, never taken
}

// Times `reps` launches of the phase-A SpMV (the tiled kernel the iteration runs) on the
// last solved system (measurement hook).  Before every launch a 256 MiB buffer (twice the
// L2) is read, so each launch starts with the matrix out of L2 as in the PCG loop, where
// the bank inverses and vectors stream through L2 between two SpMVs; each launch is timed
// alone with CUDA events on the handle's stream and the durations are averaged.
int profile_spmv(Solver& S, int reps, float* avg_ms, double* bytes)
{
    if(!S.pcg_ready)
    {
        set_error("stg_profile_spmv: run a solve first");
        return STG_ERR_NOT_READY;
    }
    const bool fp32 = S.cfg.precision == STG_PREC_FP32;
    PcgDev c = S.pcg_dev;
    cudaStream_t s = S.stream;
    const size_t flush_bytes = (size_t)256 << 20;
    STG_CUDA_TRY(cudaFuncSetAttribute(k_l2_scrub, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      cudaSharedmemCarveoutMaxShared));
    const bool fresh = S.pcg.flush.cap < flush_bytes;
    STG_TRY(S.pcg.flush.resize(flush_bytes));
    if(fresh) STG_CUDA_TRY(cudaMemsetAsync(S.pcg.flush.data(), 0, flush_bytes, s));
    int saved[4];
    STG_CUDA_TRY(cudaMemcpyAsync(saved, c.flags, sizeof(saved), cudaMemcpyDeviceToHost, s));
    STG_CUDA_TRY(cudaStreamSynchronize(s));
    STG_CUDA_TRY(cudaMemsetAsync(c.flags, 0, sizeof(int) * 4, s));
    auto launch = [&]() -> int {
        if(fp32)
            STG_TRY(launch_phase_a<float>(c, s));
        else
            STG_TRY(launch_phase_a<double>(c, s));
        return 0;
    };
    for(int i = 0; i < 3; i++) STG_TRY(launch());
    double total = 0;
    for(int i = 0; i < reps; i++)
    {
        k_l2_scrub<<<kSMs * 8, 256, 0, s>>>(reinterpret_cast<const uint4*>(S.pcg.flush.data()), flush_bytes / 16,
                                            reinterpret_cast<unsigned*>(c.counters + 7));
        STG_LAUNCH_CHECK();
        STG_CUDA_TRY(cudaEventRecord(S.ev[4], s));
        STG_TRY(launch());
        STG_CUDA_TRY(cudaEventRecord(S.ev[5], s));
        STG_CUDA_TRY(cudaEventSynchronize(S.ev[5]));
        float ms = 0;
        STG_CUDA_TRY(cudaEventElapsedTime(&ms, S.ev[4], S.ev[5]));
        total += ms;
    }
    S.launches += 2 * reps + 3;
    STG_CUDA_TRY(cudaMemcpyAsync(c.flags, saved, sizeof(saved), cudaMemcpyHostToDevice, s));
    STG_CUDA_TRY(cudaStreamSynchronize(s));
    if(avg_ms) *avg_ms = (float)(total / std::max(reps, 1));
    const double blk = fp32 ? 36.0 : 72.0, vec = fp32 ? 4.0 : 8.0;
    if(bytes) *bytes = (double)S.bcoo.nnzb * (blk + 8.0) + 3.0 * c.n * vec;
    return 0;
}

int Solver::pcg_solve(const double* b, double* x, int n, int abd_bodies, const double* abd_inv, stg_stats* st)
{
    cudaStream_t s = stream;
    const bool fp32 = cfg.precision == STG_PREC_FP32;
    const bool use_mas = cfg.preconditioner == STG_PRECOND_MAS;
    if(n != 3 * bcoo.nrows)
    {
        set_error("stg_pcg_solve: n must be 3 * block rows of the BCOO");
        return STG_ERR_INVALID;
    }
    if(use_mas && !mas.assembled)
    {
        set_error("stg_pcg_solve: MAS preconditioner not assembled");
        return STG_ERR_NOT_READY;
    }
    if(use_mas && 3 * (mas_fem_offset + mas.V) > n)
    {
        set_error("stg_pcg_solve: MAS range exceeds the system");
        return STG_ERR_INVALID;
    }
    if(abd_bodies > 0 && 4 * abd_bodies > bcoo.nrows)
    {
        set_error("stg_pcg_solve: ABD bodies exceed the system");
        return STG_ERR_INVALID;
    }
    PcgState& P = pcg;
    if(abd_bodies > 0 && !abd_inv)
    {
        // ABDPreconditioner::assemble: inverses of the bodies' diagonal tiles of this BCOO
        STG_TRY(P.abd_inv.resize((size_t)abd_bodies * 144));
        STG_TRY(abd_block_jacobi(bcoo.nnzb, bcoo.R(), bcoo.C(), bcoo.B(), abd_bodies, P.abd_inv.data(), nullptr, s));
        launches += 3;
        abd_inv = P.abd_inv.data();
    }
    const size_t es = fp32 ? sizeof(float) : sizeof(double);
    STG_TRY(P.r.resize(n));
    const size_t nr = (size_t)bcoo.nrows;
    // zp0, zp1 (8 slots per block row), q (4 slots), each region 256-byte aligned
    const size_t zp_bytes = (8 * nr * es + 255) / 256 * 256, q_bytes = (4 * nr * es + 255) / 256 * 256;
    STG_TRY(P.vbuf.resize((2 * zp_bytes + q_bytes) / sizeof(double) + 32));
    STG_TRY(pack_blocks(*this));
    const int slots = kSMs * 8;
    STG_TRY(P.partials.resize((size_t)slots * 8));
    STG_TRY(P.scal.resize(S_COUNT));
    STG_TRY(P.counters.resize(8));
    STG_TRY(P.flags.resize(8));
    STG_TRY(P.bar.resize(2));
    STG_CUDA_TRY(cudaMemsetAsync(P.counters.data(), 0, sizeof(unsigned) * 8, s));
    STG_CUDA_TRY(cudaMemsetAsync(P.flags.data(), 0, sizeof(int) * 8, s));
    STG_CUDA_TRY(cudaMemsetAsync(P.scal.data(), 0, sizeof(double) * S_COUNT, s));

    // zeroed bytewise (padding included): the graph loop compares parameter blocks with memcmp
    PcgDev c;
    std::memset(&c, 0, sizeof(c));
    c.row_ptr = bcoo.row_ptr.data();
    c.cols = bcoo.C();
    c.t_ptr = bcoo.t_ptr.data();
    c.t_ent = bcoo.t_ent.data();
    c.blk64 = reinterpret_cast<const double2*>(bcoo.blk64p.data());
    c.fent = bcoo.fent.data();
    c.frow = bcoo.frow.data();
    c.fstride = bcoo.fstride;
    c.htail = bcoo.htail.data();
    c.hcnt = bcoo.hcnt.data();
    c.hlist = bcoo.hlist.data();
    c.halo = 0;
    c.uent = bcoo.uent.data();
    c.urow = bcoo.urow.data();
    c.ustride = bcoo.ustride;
    c.nrows = bcoo.nrows;
    c.n = n;
    char* vb = reinterpret_cast<char*>(P.vbuf.data());
    c.zp0 = vb;
    c.zp1 = vb + zp_bytes;
    c.q = vb + 2 * zp_bytes;
    c.x = x;
    c.r = P.r.data();
    c.b = b;
    if(use_mas)
    {
        c.part_map = mas.part_map.data();
        c.fine_mask = mas.fine_mask.data();
        c.going_next = mas.going_next.data();
        c.closed = mas.closed.data();
        c.R = mas.R.data();
        c.Z = mas.Z.data();
        c.inv = mas.inv.data();
        c.real_map = mas.real_map.data();
        c.coarse_table = mas.coarse_table.data();
        c.M = mas.M;
        c.V = mas.V;
        c.L = mas.L;
        c.nbanks = mas.nbanks;
        c.fem_dof = 3 * mas_fem_offset;
        c.identity = mas.identity ? 1 : 0;
        for(int i = 0; i < 2 * (kMaxLevels + 1); i++) c.ls[i] = mas.level_size[i];
        c.ls_dev = reinterpret_cast<const int*>(mas.level_size_d.data());
    }
    c.diag_inv = cfg.preconditioner == STG_PRECOND_DIAG ? bcoo.diag_inv.data() : nullptr;
    c.abd_bodies = abd_bodies;
    c.abd_inv = abd_inv;
    c.partials = P.partials.data();
    c.counters = P.counters.data();
    c.scal = P.scal.data();
    c.flags = P.flags.data();
    c.slots = slots;
    c.prm.tol = cfg.tol;
    c.prm.max_iter = (long)(cfg.max_iter_ratio * (double)n);
    c.prm.stop_rule = cfg.stop_rule;
    c.prm.refine = fp32 ? cfg.refine_interval : 0;
    c.bar = P.bar.data();
    // SpMV kernel: a fixed tile shape (or the halo kernel), the autotuner's choice for this
    // shape class (precision, block rows, unique blocks; one choice per class and process), or
    // the precision's default shape
    c.a_rt = fp32 ? a_rt_default<float>() : a_rt_default<double>();
    c.halo = 0;
    c.upper = 0;
    if(spmv_rt == SPMV_HALO)
        c.halo = bcoo.halo_ok ? 1 : 0;
    else if(spmv_rt > 0)
        c.a_rt = spmv_rt;
    else if(spmv_tune && cfg.loop_mode != STG_LOOP_PERSISTENT)
    {
        if(tuned_prec != (fp32 ? 1 : 0) || tuned_nrows != bcoo.nrows || tuned_nnzb != bcoo.nnzb)
        {
            int r = 0;
            if(!tuned_choice(fp32 ? 1 : 0, bcoo.nrows, bcoo.nnzb, &r, tune_us))
            {
                PcgDev t = c;
                t.grid_e = std::max(1, std::min(div_up(n, PB), kSMs * 4));
                STG_TRY(fp32 ? tune_phase_a<float>(*this, t, tune_us, &r) : tune_phase_a<double>(*this, t, tune_us, &r));
                record_choice(fp32 ? 1 : 0, bcoo.nrows, bcoo.nnzb, r, tune_us);
            }
            tuned_rt = r;
            tuned_prec = fp32 ? 1 : 0;
            tuned_nrows = bcoo.nrows;
            tuned_nnzb = bcoo.nnzb;
        }
        if(tuned_rt == SPMV_HALO)
            c.halo = bcoo.halo_ok ? 1 : 0;
        else if(tuned_rt == SPMV_UPPER)
            c.upper = bcoo.upper_built ? 1 : 0;
        else
            c.a_rt = tuned_rt;
    }
    else if(upper_spmv_selected(*this))
        c.upper = bcoo.upper_built ? 1 : 0;
    c.spill = c.upper ? pcg.spill.data() : nullptr;
    if(nseg > 0)
    {
        if(seg_off_host.back() != bcoo.nrows || abd_bodies > 0 || cfg.loop_mode == STG_LOOP_PERSISTENT ||
           cfg.learned || cfg.stop_rule != STG_STOP_RELATIVE_RESIDUAL)
        {
            set_error("stg_pcg_solve: scenes need their offsets to end at the block-row count, no ABD bodies, the host "
                      "or graph loop, no learned correction and the relative-residual stop rule");
            return STG_ERR_INVALID;
        }
        STG_TRY(seg_row.resize(3 * (size_t)bcoo.nrows));
        STG_TRY(seg_scal.resize((size_t)SEG_N * nseg));
        c.seg_of_row = seg_of_row.data();
        c.seg_row_off = seg_off.data();
        c.seg = seg_scal.data();
        c.seg_row = seg_row.data();
        c.nseg = nseg;
        c.seg_tol2 = cfg.tol * cfg.tol;
        c.prm.tol = 0.0;  // the scenes' own tests end the loop
    }
    const bool net_apply = cfg.learned != 0, net_rec = learned.rec_cap > 0;
    if(net_apply || net_rec)
    {
        if(!use_mas)
        {
            set_error("stg_pcg_solve: the learned coarse correction and its recorder need the MAS preconditioner");
            return STG_ERR_INVALID;
        }
        if(!learned.graph_ready)
        {
            set_error("stg_pcg_solve: no graph of the learned level: configure the level (stg_net_configure) before "
                      "the MAS assembly, with a level below the hierarchy's level count");
            return STG_ERR_NOT_READY;
        }
        if(cfg.loop_mode == STG_LOOP_PERSISTENT)
        {
            set_error("stg_pcg_solve: the learned coarse correction runs in the host and graph loops only");
            return STG_ERR_INVALID;
        }
        if(net_apply && !learned.has_params)
        {
            set_error("stg_pcg_solve: learned is on but no parameters were set (stg_net_set_params)");
            return STG_ERR_NOT_READY;
        }
        STG_TRY(net_prepare());
        c.flex = net_apply ? 1 : 0;
        c.prm.judge = (net_apply && c.prm.refine == 0) ? std::max(1, cfg.refine_interval) : 0;
        c.net_mode = (net_apply ? 1 : 0) | (net_rec ? 2 : 0);
        c.net_n = learned.graph.n;
        c.net_rec_cap = learned.rec_cap;
        c.net_rec_every = learned.rec_every;
        c.net_ptrs[0] = learned.graph.row.data();
        c.net_ptrs[1] = learned.scratch.data();
        c.net_ptrs[2] = learned.params.data();
        c.net_ptrs[3] = learned.rec_rc;
        c.net_ptrs[4] = learned.rec_zc;
        c.net_ptrs[5] = learned.rec_count.data();
        if(net_apply)
        {
            const int on = 1;
            STG_CUDA_TRY(cudaMemcpyAsync(P.flags.data() + F_LEARN, &on, sizeof(int), cudaMemcpyHostToDevice, s));
        }
        if(net_rec) STG_CUDA_TRY(cudaMemsetAsync(learned.rec_count.data(), 0, sizeof(int), s));
    }

    int done = 0;
    if(fp32)
    {
        if(!use_mas)
            STG_TRY((pcg_run<float, 0>(*this, c, done)));
        else if(cfg.bank_size == 32)
            STG_TRY((pcg_run<float, 32>(*this, c, done)));
        else
            STG_TRY((pcg_run<float, 16>(*this, c, done)));
    }
    else
    {
        if(!use_mas)
            STG_TRY((pcg_run<double, 0>(*this, c, done)));
        else if(cfg.bank_size == 32)
            STG_TRY((pcg_run<double, 32>(*this, c, done)));
        else
            STG_TRY((pcg_run<double, 16>(*this, c, done)));
    }
    pcg_dev = c;
    pcg_ready = true;

    double h_scal[S_COUNT];
    int h_flags[8];
    STG_CUDA_TRY(cudaMemcpyAsync(h_scal, P.scal.data(), sizeof(double) * S_COUNT, cudaMemcpyDeviceToHost, s));
    STG_CUDA_TRY(cudaMemcpyAsync(h_flags, P.flags.data(), sizeof(int) * 8, cudaMemcpyDeviceToHost, s));
    STG_CUDA_TRY(cudaStreamSynchronize(s));
    const long max_iter = c.prm.max_iter;
    int status = h_flags[F_DONE] ? h_flags[F_STATUS] : STG_MAX_ITER;
    if(status == STG_ERR_TIMEOUT) set_error("persistent PCG: a grid barrier wait gave up");
    const long iters = max_iter <= 1 ? 1 : (long)h_scal[S_ITER];
    if(cfg.loop_mode == STG_LOOP_GRAPH && max_iter > 1)
    {
        // the graph's body ran once per iteration; its IF node (residual replacement plus
        // the level-0/1 re-restriction) once per replacement
        launches += (int)iters * launches_per_batch + h_flags[F_REPL] * (use_mas ? 2 : 1);
    }
    if(st)
    {
        st->iterations = (int)iters;
        st->rz0 = h_scal[S_RZ0];
        st->rz_final = h_scal[S_RZ];
        st->rel_residual_recursive = h_scal[S_BB] > 0 ? std::sqrt(h_scal[S_RR] / h_scal[S_BB]) : 0.0;
        st->replacements = h_flags[F_REPL];
        st->learned_accepted = h_flags[F_LACC];
        st->learned_rejected = h_flags[F_LREJ];
    }
    if(nseg > 0)
    {
        seg_host.resize((size_t)SEG_N * nseg);
        STG_CUDA_TRY(cudaMemcpyAsync(seg_host.data(), seg_scal.data(), sizeof(double) * SEG_N * nseg, cudaMemcpyDeviceToHost, s));
        STG_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return status;
}

}  // namespace stg
