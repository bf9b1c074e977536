// mas.cu -- multilevel additive Schwarz (MAS / CEMAS) preconditioner on sm_100a.
//
// Replaces MASPreconditioner (StiffGIPC/MASPreconditioner.cu):
//   hierarchy  ReorderRealtime (1785-1826) and its kernels (29-625, 1132-1548)
//   assembly   PrepareHessian_bcoo (1829-2075) + __inverse6_P96x96 (630-726)
//   apply      preconditioning (2248-2289): __buildMultiLevelR_optimized_new (729-847),
//              _schwarzLocalXSym6 (957-1027), __collectFinalZ_new (850-879)
//
// Bank size B (BANKSIZE, eigen_data.h:17) is a template parameter: 16 (CEMAS as shipped) or
// 32 (Morton-ordered GPU MAS).  Integer results (masks, coarse ids, tables) are bit-exact
// with the reference's intended semantics; the reference's warp-synchronous shared-memory
// races are replaced by explicit barriers:
//   * in-bank closure (_preparePrefixSumL0_new / _nextLevelCluster) reads the original
//     masks from shared memory written before a __syncthreads;
//   * the union of coarse connectivity masks (_buildConnectMaskLx_new) is formed with
//     atomicOr on the node mask (OR is order independent);
//   * component leaders and counts use ballots instead of racy shared atomics.
// Restriction sums are computed per bank in lane order (deterministic) instead of float
// atomics, and the coarse-level Galerkin blocks are formed level by level with the
// deterministic sort/merge of convert.cu instead of FP64 atomics (see the assembly section).
#include "solver.hpp"
#include "bank_dev.cuh"
#include "mas_index.cuh"

namespace stg
{


// group-local ballot: the B lanes of this lane's bank
template <int B>
__device__ __forceinline__ unsigned group_ballot(bool pred)
{
    const unsigned all = __ballot_sync(0xffffffffu, pred);
    if(B == 32) return all;
    const int shift = (threadIdx.x & 31) & ~(B - 1);
    return (all >> shift) & ((1u << B) - 1u);
}

// ---------------------------------------------------------------------------------------
// hierarchy
// ---------------------------------------------------------------------------------------
// _buildCML0_new (MASPreconditioner.cu:62-98): in-bank neighbour bits; inter-bank neighbours
// are compacted to the front of the vertex's list.
template <int B>
__global__ void k_mas_l0_mask(const int* __restrict__ part_map, const int* __restrict__ real_map,
                              const unsigned* __restrict__ nstart, unsigned* nnum, unsigned* nlist, unsigned* fine_mask,
                              int M)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if(s >= M) return;
    const int v = part_map[s];
    if(v < 0) return;
    const int bank = s / B, lane = s % B;
    unsigned msk = 1u << lane;
    unsigned nk = 0;
    const unsigned st = nstart[v], num = nnum[v];
    for(unsigned i = 0; i < num; i++)
    {
        const unsigned u = nlist[st + i];
        const int su = real_map[u];
        if(su / B == bank)
            msk |= 1u << (su % B);
        else
            nlist[st + nk++] = u;
    }
    nnum[v] = nk;
    fine_mask[v] = msk;
}

// _buildCollisionConnection_new (MASPreconditioner.cu:1132-1548).  coarse == nullptr: level 0
// (ids via real_map, OR into conn[vertex]); otherwise the previous level's coarse table
// (OR into conn[coarse id]).
template <int B>
__global__ void k_mas_contacts(unsigned* conn, const int* __restrict__ coarse, const int* __restrict__ real_map,
                               const int4* __restrict__ pairs, int ncp, int node_offset, int V)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= ncp) return;
    const int4 q = pairs[p];
    int v[4] = {q.x, q.y, q.z, q.w};
    int cnt = 4;
    if(v[0] >= 0)
    {
        if(v[3] < 0) v[3] = -v[3] - 1;
    }
    else
    {
        v[0] = -v[0] - 1;
        if(v[2] < 0)
        {
            if(v[1] < 0)
            {
                v[1] = -v[1] - 1;
                v[2] = -v[2] - 1;
                v[3] = -v[3] - 1;
            }
            else
                cnt = 2;
        }
        else if(v[3] < 0)
        {
            if(v[1] < 0)
            {
                v[1] = -v[1] - 1;
                v[3] = -v[3] - 1;
            }
            else
                cnt = 3;
        }
    }
    int vid[4], cpv[4];
    unsigned msk[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for(int i = 0; i < 4; i++)
    {
        const int id = v[i] - node_offset;
        vid[i] = (i < cnt && id >= 0 && id < V) ? id : -1;
        cpv[i] = vid[i] >= 0 ? (coarse ? coarse[vid[i]] : real_map[vid[i]]) : -1;
    }
#pragma unroll
    for(int i = 0; i < 4; i++)
#pragma unroll
        for(int j = i + 1; j < 4; j++)
        {
            const int a = cpv[i], b = cpv[j];
            if(a == b || a < 0 || b < 0) continue;
            if(a / B == b / B)
            {
                msk[i] |= 1u << (b % B);
                msk[j] |= 1u << (a % B);
            }
        }
#pragma unroll
    for(int i = 0; i < 4; i++)
    {
        if(coarse)
        {
            if(cpv[i] >= 0 && msk[i]) atomicOr(conn + cpv[i], msk[i]);
        }
        else if(vid[i] >= 0 && msk[i])
            atomicOr(conn + vid[i], msk[i]);
    }
}

// Reachable set of `lane` through the bank's original masks (the visit loop of
// _preparePrefixSumL0_new / _nextLevelCluster), masks read from shared memory.
__device__ __forceinline__ unsigned bank_closure(const unsigned* orig, int lane, unsigned start)
{
    unsigned conn = start, visited = 1u << lane;
    for(;;)
    {
        const unsigned todo = visited ^ conn;
        if(!todo) break;
        const int nv = __ffs(todo) - 1;
        visited |= 1u << nv;
        conn |= orig[nv];
    }
    return conn;
}

// _preparePrefixSumL0_new (MASPreconditioner.cu:159-214): closure + component count per bank.
template <int B>
__global__ void __launch_bounds__(256) k_mas_l0_closure(const int* __restrict__ part_map, unsigned* fine_mask,
                                                        int* prefix_orig, int M)
{
    __shared__ unsigned orig[256];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = s % B;
    const int v = s < M ? part_map[s] : -1;
    orig[threadIdx.x] = v >= 0 ? fine_mask[v] : 0u;
    __syncthreads();
    bool leader = false;
    if(v >= 0)
    {
        const unsigned* bank_orig = orig + (threadIdx.x & ~(B - 1));
        const unsigned c = bank_closure(bank_orig, lane, bank_orig[lane]);
        fine_mask[v] = c;
        leader = __popc(c & lanemask_lt(lane)) == 0;
    }
    const unsigned lm = group_ballot<B>(leader);
    if(lane == 0 && s < M) prefix_orig[s / B] = __popc(lm);
}

// _buildLevel1_new (MASPreconditioner.cu:270-328): level-1 ids in leader-lane order.
template <int B>
__global__ void k_mas_l1_assign(const int* __restrict__ part_map, const unsigned* __restrict__ fine_mask,
                                const int* __restrict__ prefix_sum_orig, int* coarse_tables, int* going_next, int M)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = s % B;
    const int v = s < M ? part_map[s] : -1;
    const unsigned c = v >= 0 ? fine_mask[v] : 0u;
    const bool leader = v >= 0 && __popc(c & lanemask_lt(lane)) == 0;
    const unsigned elected = group_ballot<B>(leader);
    if(v < 0) return;
    const int lead = __ffs(c) - 1;
    const int id = __popc(elected & lanemask_lt(lead)) + prefix_sum_orig[s / B];
    coarse_tables[v] = id;
    going_next[v] = id + M;
}

// _buildConnectMaskLx_new (MASPreconditioner.cu:401-470) with union semantics.
template <int B>
__global__ void k_mas_lx_mask(const int* __restrict__ part_map, const unsigned* __restrict__ nstart, unsigned* nnum,
                              unsigned* nlist, const int* __restrict__ prev, unsigned* next_mask, int M)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if(s >= M) return;
    const int v = part_map[s];
    if(v < 0) return;
    const unsigned c = (unsigned)prev[v];
    unsigned msk = 0, nk = 0;
    const unsigned st = nstart[v], num = nnum[v];
    for(unsigned i = 0; i < num; i++)
    {
        const unsigned u = nlist[st + i];
        const unsigned cu = (unsigned)prev[u];
        if(c / B == cu / B)
            msk |= 1u << (cu % B);
        else
            nlist[st + nk++] = u;
    }
    nnum[v] = nk;
    if(msk) atomicOr(next_mask + c, msk);
}

// _nextLevelCluster (MASPreconditioner.cu:473-520): closure over level-l banks.
// ls: level sizes (count, begin) pairs; level = l.
template <int B>
__global__ void __launch_bounds__(256) k_mas_lx_closure(unsigned* next_mask, unsigned* closed, int* next_prefix,
                                                        const int* __restrict__ ls, int level)
{
    __shared__ unsigned orig[256];
    const int number = ls[2 * level], begin = ls[2 * level + 1];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = i % B;
    const bool valid = i < number;
    orig[threadIdx.x] = valid ? ((1u << lane) | next_mask[i]) : 0u;
    __syncthreads();
    bool leader = false;
    if(valid)
    {
        const unsigned* bank_orig = orig + (threadIdx.x & ~(B - 1));
        const unsigned c = bank_closure(bank_orig, lane, bank_orig[lane]);
        next_mask[i] = c;
        closed[begin + i] = c;
        leader = __popc(c & lanemask_lt(lane)) == 0;
    }
    const unsigned lm = group_ballot<B>(leader);
    if(lane == 0 && i < number) next_prefix[i / B] = __popc(lm);
}

// _prefixSumLx (MASPreconditioner.cu:522-566): next-level ids; also records the level size.
template <int B>
__global__ void k_mas_lx_assign(unsigned* next_mask, const int* __restrict__ next_prefix_sum, int* going_next, int* ls,
                                int level)
{
    const int number = ls[2 * level], begin = ls[2 * level + 1];
    const int rounded = (number + B - 1) / B * B;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = i % B;
    const bool valid = i < number;
    const unsigned c = valid ? next_mask[i] : 0u;
    const bool leader = valid && __popc(c & lanemask_lt(lane)) == 0;
    const unsigned elected = group_ballot<B>(leader);
    if(i == 0) ls[2 * (level + 1) + 1] = begin + rounded;
    if(!valid) return;
    const int lead = __ffs(c) - 1;
    const int id = __popc(elected & lanemask_lt(lead)) + next_prefix_sum[i / B];
    next_mask[i] = (unsigned)id;
    going_next[begin + i] = id + begin + rounded;
}

// _computeNextLevel (MASPreconditioner.cu:568-579)
__global__ void k_mas_compute_next(int* coarse_tables, const unsigned* __restrict__ next_mask, int level, int V)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if(v >= V) return;
    coarse_tables[(size_t)level * V + v] = (int)next_mask[coarse_tables[(size_t)(level - 1) * V + v]];
}

// _aggregationKernel (MASPreconditioner.cu:581-608)
__global__ void k_mas_aggregate(const int* __restrict__ going_next, int* coarse_table, int L, int V)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if(v >= V) return;
    int cur = v;
    for(int l = 0; l < L - 1; l++)
    {
        cur = going_next[cur];
        coarse_table[(size_t)v * (L - 1) + l] = cur;
    }
}

// scan driver: n = ceil(ls[2*level] / div) when ls != nullptr
__global__ void k_set_level1(int* ls, const int* total, int M)
{
    ls[2] = *total;
    ls[3] = M;
}

// ---------------------------------------------------------------------------------------
// assembly (PrepareHessian_bcoo) and inverse
// ---------------------------------------------------------------------------------------
// PrepareHessian_bcoo (MASPreconditioner.cu:1829-2075) accumulates, for every level l, the
// bank-diagonal blocks of the Galerkin operator P_l^T A P_l: block (a, b) of a level-l bank
// is the sum of A(u, v) over all fine pairs with coarse_l(u) = a, coarse_l(v) = b.  The
// reference walks every BCOO entry and every in-bank level-0 pair up the levels with FP64
// atomics, which serialise on the few coarse blocks every pair reaches.  Here the same sums
// are formed level by level: A_1 = aggregate(A_0), A_{l+1} = aggregate(A_l) (aggregate =
// map both indices to the coarse node and merge duplicates with the deterministic sorter of
// convert.cu), and each level's bank blocks are read off A_l.  Level-0 in-bank entries with
// slot(col) < slot(row) are not stored by the reference (lambda 1 only stores col >= row
// slots, and lambda 2 propagates the stored bank matrix); they are left out here too.

// level-0 bank blocks (lambda 1, level-0 branch): direct stores, entries are unique
template <int B>
__global__ void k_mas_store_l0(const int* __restrict__ rows, const int* __restrict__ cols,
                               const double* __restrict__ blocks, int nnzb, int offset, int V,
                               const int* __restrict__ real_map, double* mat)
{
    const int NS = nsym(B);
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnzb; k += gridDim.x * blockDim.x)
    {
        const int rr = rows[k] - offset, cc = cols[k] - offset;
        if(rr < 0 || rr >= V || cc < 0 || cc >= V) continue;
        const int sc = real_map[cc], sr = real_map[rr];
        if(sc / B != sr / B || sc < sr) continue;
        const double* H = blocks + 9 * (size_t)k;
        double* D = mat + ((size_t)(sc / B) * NS + upper_index(B, sr % B, sc % B)) * 9;
#pragma unroll
        for(int e = 0; e < 9; e++) D[e] = H[e];
    }
}

// A_0 (FEM range of the BCOO) -> level-1 triplets; masked entries get row -1
template <int B>
__global__ void k_mas_agg_l0(const int* __restrict__ rows, const int* __restrict__ cols, const double* __restrict__ blocks,
                             int nnzb, int offset, int V, const int* __restrict__ real_map, const int* __restrict__ c1,
                             int* orow, int* ocol, double* oblk)
{
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnzb; k += gridDim.x * blockDim.x)
    {
        const int rr = rows[k] - offset, cc = cols[k] - offset;
        bool use = rr >= 0 && rr < V && cc >= 0 && cc < V;
        if(use)
        {
            const int sc = real_map[cc], sr = real_map[rr];
            use = !(sc / B == sr / B && sc < sr);
        }
        if(!use)
        {
            orow[k] = -1;
            ocol[k] = 0;
            continue;
        }
        coarse_triplet(rr, cc, c1[rr], c1[cc], blocks + 9 * (size_t)k, orow + k, ocol + k, oblk + 9 * (size_t)k);
    }
}

// A_l -> level-(l+1) triplets through going_next (global ids) of level-l nodes
__global__ void k_mas_agg_lx(const int* __restrict__ rows, const int* __restrict__ cols, const double* __restrict__ blocks,
                             int nnz, const int* __restrict__ going_next, int begin, int begin_next, int* orow, int* ocol,
                             double* oblk)
{
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x)
    {
        const int u = rows[k], v = cols[k];
        coarse_triplet(u, v, going_next[begin + u] - begin_next, going_next[begin + v] - begin_next,
                       blocks + 9 * (size_t)k, orow + k, ocol + k, oblk + 9 * (size_t)k);
    }
}

// bank-diagonal blocks of A_l (level-local ids, upper) into the packed bank matrices
template <int B>
__global__ void k_mas_extract(const int* __restrict__ rows, const int* __restrict__ cols, const double* __restrict__ blocks,
                              int nnz, int begin, double* mat)
{
    const int NS = nsym(B);
    for(int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x)
    {
        const int ga = begin + rows[k], gb = begin + cols[k];
        if(ga / B != gb / B) continue;
        double* D = mat + ((size_t)(ga / B) * NS + upper_index(B, ga % B, gb % B)) * 9;
        const double* H = blocks + 9 * (size_t)k;
#pragma unroll
        for(int e = 0; e < 9; e++) D[e] = H[e];
    }
}

// __inverse6_P96x96 (MASPreconditioner.cu:630-726): in-place Gauss-Jordan without pivoting
// of each bank's dense 3B x 3B matrix in FP64 (zero diagonal -> 1 for padding), lower
// triangle of the diagonal 3x3 blocks mirrored from the upper one, upper blocks stored FP32.
// One CTA per bank, thread i owns column i.  The pivot row is scaled by the correctly rounded
// reciprocal of the pivot (the reference divides; k_mas_invert16 does the same as here, so
// both bank sizes follow one order, the CPU oracle's ORC_ORDER_FIXED).
template <int B>
__global__ void __launch_bounds__(3 * B) k_mas_invert(const double* __restrict__ mat, float* inv, int nbanks)
{
    constexpr int N = 3 * B;
    const int NS = nsym(B);
    extern __shared__ double sm[];
    double* A = sm;            // N*N row-major
    double* colm = sm + N * N; // N
    const int bk = blockIdx.x;
    const int i = threadIdx.x;
    const double* Mb = mat + (size_t)bk * NS * 9;
    for(int j = 0; j < N; j++)
    {
        const int rowId = j / 3, colId = i / 3;
        double v;
        if(colId >= rowId)
            v = Mb[upper_index(B, rowId, colId) * 9 + (i % 3) * 3 + (j % 3)];
        else
            v = Mb[upper_index(B, colId, rowId) * 9 + (j % 3) * 3 + (i % 3)];
        if(i == j && v == 0.0) v = 1.0;
        A[j * N + i] = v;
    }
    for(int j = 0; j < N; j++)
    {
        __syncthreads();
        const double rt = A[j * N + j];
        colm[i] = A[i * N + j];
        __syncthreads();
        A[i * N + j] = (i == j) ? 1.0 : 0.0;
        __syncthreads();
        A[j * N + i] = __dmul_rn(A[j * N + i], 1.0 / rt);
        __syncthreads();
        const double aji = A[j * N + i];
        for(int k = 0; k < N; k++)
        {
            if(k == j) continue;
            A[k * N + i] = fma(-colm[k], aji, A[k * N + i]);
        }
    }
    __syncthreads();
    if(i % 3 < 2)
        A[(i + 1) * N + i] = A[i * N + i + 1];
    else
        A[i * N + i - 2] = A[(i - 2) * N + i];
    __syncthreads();
    float* P = inv + (size_t)bk * NS * 9;
    for(int j = 0; j < N; j++)
    {
        const int rowId = j / 3, colId = i / 3;
        if(colId >= rowId) P[upper_index(B, rowId, colId) * 9 + (i % 3) * 3 + (j % 3)] = (float)A[j * N + i];
    }
}

// The same Gauss-Jordan for 16-banks, one CTA of 256 threads per bank, thread (bi, bj) owning
// the 3x3 tile at block row bi, block column bj in registers.  Pivot j: the tiles of block
// column j / 3 publish column j; those of block row j / 3 scale row j by the reciprocal of
// the pivot (one FP64 division per thread and pivot: divisions on the pivot's critical path
// made a per-element division three times slower) and publish it; then every tile updates
// itself with fma(-colm[k], A[j][i], A[k][i]) as k_mas_invert does.  The broadcasts are
// double-buffered (two barriers per pivot).  Scaling by the reciprocal instead of dividing
// changes the last bit of some FP64 entries against the reference's per-element division;
// k_mas_invert scales the same way, and the CPU oracle (ORC_ORDER_FIXED) restates it.
__global__ void __launch_bounds__(256) k_mas_invert16(const double* __restrict__ mat, float* inv, int nbanks)
{
    constexpr int B = 16;
    const int NS = nsym(B);
    __shared__ double rowj[2][3 * B], colj[2][3 * B];
    const int bk = blockIdx.x;
    const int bi = threadIdx.x / B, bj = threadIdx.x % B;
    const double* Mb = mat + (size_t)bk * NS * 9;
    double a[3][3];
    if(bj >= bi)
    {
        const double* H = Mb + upper_index(B, bi, bj) * 9;  // column-major
#pragma unroll
        for(int r = 0; r < 3; r++)
#pragma unroll
            for(int cc = 0; cc < 3; cc++) a[r][cc] = H[cc * 3 + r];
    }
    else
    {
        const double* H = Mb + upper_index(B, bj, bi) * 9;  // the mirror block, transposed
#pragma unroll
        for(int r = 0; r < 3; r++)
#pragma unroll
            for(int cc = 0; cc < 3; cc++) a[r][cc] = H[r * 3 + cc];
    }
    if(bi == bj)
    {
#pragma unroll
        for(int r = 0; r < 3; r++)
            if(a[r][r] == 0.0) a[r][r] = 1.0;
    }
    for(int j = 0; j < 3 * B; j++)
    {
        const int pb = j / 3, pr = j % 3, buf = j & 1;
        // 1: block column pb publishes the old column j
        if(bj == pb)
        {
#pragma unroll
            for(int r = 0; r < 3; r++) colj[buf][3 * bi + r] = pr == 0 ? a[r][0] : (pr == 1 ? a[r][1] : a[r][2]);
        }
        __syncthreads();
        // 2: block row pb forms row j after the column replacement (e_j) and the division by
        // the pivot, keeps it and publishes it
        if(bi == pb)
        {
            const double rinv = 1.0 / colj[buf][j];
#pragma unroll
            for(int cc = 0; cc < 3; cc++)
            {
                const int col = 3 * bj + cc;
                const double x = col == j ? 1.0 : (pr == 0 ? a[0][cc] : (pr == 1 ? a[1][cc] : a[2][cc]));
                const double v = __dmul_rn(x, rinv);
                rowj[buf][col] = v;
                if(pr == 0)
                    a[0][cc] = v;
                else if(pr == 1)
                    a[1][cc] = v;
                else
                    a[2][cc] = v;
            }
        }
        __syncthreads();
        // 3: every other row: A[k][i] = fma(-colm[k], A[j][i], A[k][i]) (column j replaced by e_j)
#pragma unroll
        for(int r = 0; r < 3; r++)
        {
            const int row = 3 * bi + r;
            if(row == j) continue;
            const double cm = colj[buf][row];
#pragma unroll
            for(int cc = 0; cc < 3; cc++)
            {
                const double old = (3 * bj + cc == j) ? 0.0 : a[r][cc];
                a[r][cc] = fma(-cm, rowj[buf][3 * bj + cc], old);
            }
        }
        // the next pivot writes the other buffers; this pivot's are reused two pivots later,
        // after two more barriers
    }
    if(bj < bi) return;
    if(bi == bj)
    {
        // lower triangle of the diagonal 3x3 block mirrored from the upper one
        a[1][0] = a[0][1];
        a[2][1] = a[1][2];
        a[2][0] = a[0][2];
    }
    float* P = inv + ((size_t)bk * NS + upper_index(B, bi, bj)) * 9;
#pragma unroll
    for(int r = 0; r < 3; r++)
#pragma unroll
        for(int cc = 0; cc < 3; cc++) P[cc * 3 + r] = (float)a[r][cc];
}

// ---------------------------------------------------------------------------------------
// apply
// ---------------------------------------------------------------------------------------
// Level 0 + level 1 of __buildMultiLevelR_optimized_new (MASPreconditioner.cu:729-847):
// slot values (FP32) and, for each level-0 component, the sum of its members in lane order.
template <int B>
__global__ void k_mas_restrict0(const double* __restrict__ r, const int* __restrict__ part_map,
                                const unsigned* __restrict__ fine_mask, const int* __restrict__ going_next, float* R, int M,
                                const int* done)
{
    if(done && *done) return;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = s % B;
    const int v = s < M ? part_map[s] : -1;
    float r0 = 0.f, r1 = 0.f, r2 = 0.f;
    unsigned msk = 0;
    if(v >= 0)
    {
        r0 = (float)r[3 * v];
        r1 = (float)r[3 * v + 1];
        r2 = (float)r[3 * v + 2];
        msk = fine_mask[v];
    }
    if(s < M) st4(R + 4 * (size_t)s, r0, r1, r2);
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
    for(int b = 0; b < B; b++)
    {
        const float x0 = group_shfl<B>(r0, b);
        const float x1 = group_shfl<B>(r1, b);
        const float x2 = group_shfl<B>(r2, b);
        if(msk & (1u << b))
        {
            a0 += x0;
            a1 += x1;
            a2 += x2;
        }
    }
    if(v >= 0 && __popc(msk & lanemask_lt(lane)) == 0)
    {
        const int g = going_next[v];
        st4(R + 4 * (size_t)g, a0, a1, a2);
    }
}

// Levels l -> l+1 (l >= 1): each component of a level-l bank sums its nodes in lane order.
template <int B>
__global__ void k_mas_restrict_lx(float* R, const unsigned* __restrict__ closed, const int* __restrict__ going_next,
                                  int number, int begin, const int* done)
{
    if(done && *done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = i % B;
    const bool valid = i < number;
    float r0 = 0.f, r1 = 0.f, r2 = 0.f;
    unsigned msk = 0;
    if(valid)
    {
        ld4(R + 4 * (size_t)(begin + i), r0, r1, r2);
        msk = closed[begin + i];
    }
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
    for(int b = 0; b < B; b++)
    {
        const float x0 = group_shfl<B>(r0, b);
        const float x1 = group_shfl<B>(r1, b);
        const float x2 = group_shfl<B>(r2, b);
        if(msk & (1u << b))
        {
            a0 += x0;
            a1 += x1;
            a2 += x2;
        }
    }
    if(valid && __popc(msk & lanemask_lt(lane)) == 0)
    {
        const int g = going_next[begin + i];
        st4(R + 4 * (size_t)g, a0, a1, a2);
    }
}

// _schwarzLocalXSym6 (MASPreconditioner.cu:957-1027): z_b = P_b r_b for every bank of every
// level, with the row arithmetic of bank_dev.cuh (the PCG loop's phase D gives the same bits).
// 16-banks: one warp per bank (4 per CTA), lane (a, h) forms half h of block row a; the
// packed inverse (4,896 B) and the 16 residual slots are staged per warp with 16-byte loads.
constexpr int SCHWARZ16_WARPS = 4;

__global__ void __launch_bounds__(SCHWARZ16_WARPS * 32) k_mas_schwarz16(const float* __restrict__ inv,
                                                                        const float* __restrict__ R, float* Z,
                                                                        int nbanks, const int* done)
{
    if(done && *done) return;
    __shared__ __align__(16) float P[SCHWARZ16_WARPS][136 * 9];
    __shared__ float4 rs[SCHWARZ16_WARPS][16];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bk = blockIdx.x * SCHWARZ16_WARPS + w;
    if(bk >= nbanks) return;
    const float4* src = reinterpret_cast<const float4*>(inv + (size_t)bk * 136 * 9);
    float4* dst = reinterpret_cast<float4*>(P[w]);
    for(int t = lane; t < 136 * 9 / 4; t += 32) dst[t] = __ldg(src + t);
    if(lane < 16) rs[w][lane] = *reinterpret_cast<const float4*>(R + 4 * ((size_t)bk * 16 + lane));
    __syncwarp();
    const int a = lane & 15, h = lane >> 4;
    float z0, z1, z2;
    bank16_half(P[w], rs[w], a, h, z0, z1, z2);
    bank16_join(z0, z1, z2);
    if(h == 0) st4(Z + ((size_t)bk * 16 + a) * 4, z0, z1, z2);
}

// 32-banks: one CTA of 1,024 threads per bank, thread (a, c) forms the block product of
// block (a, c) and the 32 lanes of row a sum them with the xor butterfly.
__global__ void __launch_bounds__(1024) k_mas_schwarz32(const float* __restrict__ inv, const float* __restrict__ R,
                                                        float* Z, const int* done)
{
    if(done && *done) return;
    constexpr int B = 32, NS = B * (B + 1) / 2;
    __shared__ __align__(16) float P[NS * 9];
    __shared__ float r[3 * B];
    const int bk = blockIdx.x;
    const float4* src = reinterpret_cast<const float4*>(inv + (size_t)bk * NS * 9);
    float4* dst = reinterpret_cast<float4*>(P);
    for(int t = threadIdx.x; t < NS * 9 / 4; t += B * B) dst[t] = __ldg(src + t);
    if(threadIdx.x < B) ld4(R + 4 * ((size_t)bk * B + threadIdx.x), r[3 * threadIdx.x], r[3 * threadIdx.x + 1], r[3 * threadIdx.x + 2]);
    __syncthreads();
    const int a = threadIdx.x / B, c = threadIdx.x % B;
    const int lo = min(a, c), hi = max(a, c);
    float z0, z1, z2;
    blk_mul3(P + upper_index(B, lo, hi) * 9, c < a, r[3 * c], r[3 * c + 1], r[3 * c + 2], z0, z1, z2);
    warp_butterfly3(z0, z1, z2);
    if(c == 0) st4(Z + ((size_t)bk * B + a) * 4, z0, z1, z2);
}

// __collectFinalZ_new (MASPreconditioner.cu:850-879): Z_v = sum over levels (FP32) -> FP64.
__global__ void k_mas_prolong(const float* __restrict__ Z, const int* __restrict__ real_map,
                              const int* __restrict__ coarse_table, int L, int V, double* z)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if(v >= V) return;
    const int s = real_map[v];
    float c0, c1, c2;
    ld4(Z + 4 * (size_t)s, c0, c1, c2);
    for(int l = 1; l < L; l++)
    {
        const int now = coarse_table[(size_t)v * (L - 1) + l - 1];
        float t0, t1, t2;
        ld4(Z + 4 * (size_t)now, t0, t1, t2);
        c0 += t0;
        c1 += t1;
        c2 += t2;
    }
    z[3 * v] = c0;
    z[3 * v + 1] = c1;
    z[3 * v + 2] = c2;
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
static int num_levels(int n, int B)
{
    int nLevel = 1;
    int levelSz = (n + B - 1) / B * B;
    while(levelSz > B)
    {
        levelSz /= B;
        nLevel++;
        levelSz = (levelSz + B - 1) / B * B;
    }
    nLevel = nLevel + 1;
    return nLevel > kMaxLevels ? kMaxLevels : nLevel;
}

int Solver::mas_init(int V, int node_offset, const uint32_t* ns, const uint32_t* nn, const uint32_t* nl, int nls,
                     const int* pm, int pms, const int* rm)
{
    MasState& m = mas;
    const int B = cfg.bank_size;
    if(V < 1 || pms < V || pms % B != 0 || nls < 0)
    {
        set_error("stg_mas_init: need vert_num >= 1, part_map_size >= vert_num and a multiple of bank_size");
        return STG_ERR_INVALID;
    }
    // host-side validation of the maps (an out-of-range id would be an out-of-bounds access)
    for(int s = 0; s < pms; s++)
        if(pm[s] < -1 || pm[s] >= V)
        {
            set_error("stg_mas_init: part_map entry out of range");
            return STG_ERR_INVALID;
        }
    for(int v = 0; v < V; v++)
        if(rm[v] < 0 || rm[v] >= pms || pm[rm[v]] != v)
        {
            set_error("stg_mas_init: real_map is not the inverse of part_map");
            return STG_ERR_INVALID;
        }
    for(int v = 0; v < V; v++)
        if((long)ns[v] + nn[v] > nls)
        {
            set_error("stg_mas_init: neighbour list overruns neighbor_list_size");
            return STG_ERR_INVALID;
        }
    for(int e = 0; e < nls; e++)
        if(nl[e] >= (uint32_t)V)
        {
            set_error("stg_mas_init: neighbour id out of range");
            return STG_ERR_INVALID;
        }
    m.bank = B;
    m.V = V;
    m.M = pms;
    m.identity = true;
    for(int s = 0; s < pms && m.identity; s++) m.identity = pm[s] == (s < V ? s : -1);
    m.nb0 = pms / B;
    m.node_offset = node_offset;
    m.nlist_size = nls;
    m.L = num_levels(std::max(pms, V), B);
    const int L = m.L;
    cudaStream_t s = stream;
    STG_TRY(m.nstart.resize(V));
    STG_TRY(m.nnum_init.resize(V));
    STG_TRY(m.nnum.resize(V));
    STG_TRY(m.nlist_init.resize(std::max(nls, 1)));
    STG_TRY(m.nlist.resize(std::max(nls, 1)));
    STG_TRY(m.part_map.resize(pms));
    STG_TRY(m.real_map.resize(V));
    STG_TRY(m.fine_mask.resize(V));
    STG_TRY(m.next_mask.resize(V + B));
    STG_TRY(m.prefix_orig.resize(m.nb0 + 1));
    STG_TRY(m.prefix_sum_orig.resize(m.nb0 + 1));
    STG_TRY(m.next_prefix.resize(V / B + 2));
    STG_TRY(m.next_prefix_sum.resize(V / B + 2));
    STG_TRY(m.coarse_tables.resize((size_t)L * V));
    m.gn_size = pms + L * (V + B);  // >= total clusters: level l >= 1 holds <= V nodes, rounded to B
    STG_TRY(m.going_next.resize(m.gn_size));
    STG_TRY(m.closed.resize(m.gn_size));
    STG_TRY(m.coarse_table.resize((size_t)V * std::max(L - 1, 1)));
    STG_TRY(m.level_size_d.resize(kMaxLevels + 2));
    STG_TRY(m.scratch.resize(kMaxLevels + 2));
    STG_CUDA_TRY(cudaMemcpyAsync(m.nstart.data(), ns, sizeof(unsigned) * V, cudaMemcpyHostToDevice, s));
    STG_CUDA_TRY(cudaMemcpyAsync(m.nnum_init.data(), nn, sizeof(unsigned) * V, cudaMemcpyHostToDevice, s));
    if(nls > 0) STG_CUDA_TRY(cudaMemcpyAsync(m.nlist_init.data(), nl, sizeof(unsigned) * nls, cudaMemcpyHostToDevice, s));
    STG_CUDA_TRY(cudaMemcpyAsync(m.part_map.data(), pm, sizeof(int) * pms, cudaMemcpyHostToDevice, s));
    STG_CUDA_TRY(cudaMemcpyAsync(m.real_map.data(), rm, sizeof(int) * V, cudaMemcpyHostToDevice, s));
    STG_CUDA_TRY(cudaMemsetAsync(m.going_next.data(), 0, sizeof(int) * m.gn_size, s));
    STG_CUDA_TRY(cudaMemsetAsync(m.closed.data(), 0, sizeof(unsigned) * m.gn_size, s));
    STG_CUDA_TRY(cudaStreamSynchronize(s));
    m.inited = true;
    m.built = m.assembled = false;
    return 0;
}

template <int B>
static int mas_build_t(Solver& S, const int* contacts, int ncp)
{
    MasState& m = S.mas;
    cudaStream_t s = S.stream;
    const int V = m.V, M = m.M, L = m.L;
    int* ls = reinterpret_cast<int*>(m.level_size_d.data());
    STG_CUDA_TRY(cudaMemcpyAsync(m.nlist.data(), m.nlist_init.data(), sizeof(unsigned) * std::max(m.nlist_size, 1),
                                 cudaMemcpyDeviceToDevice, s));
    STG_CUDA_TRY(cudaMemcpyAsync(m.nnum.data(), m.nnum_init.data(), sizeof(unsigned) * V, cudaMemcpyDeviceToDevice, s));
    STG_CUDA_TRY(cudaMemsetAsync(ls, 0, sizeof(int2) * (kMaxLevels + 2), s));
    const int gM = div_up(M, 256), gV = div_up(V, 256);
    const int4* pairs = reinterpret_cast<const int4*>(contacts);
    k_mas_l0_mask<B><<<gM, 256, 0, s>>>(m.part_map.data(), m.real_map.data(), m.nstart.data(), m.nnum.data(),
                                        m.nlist.data(), m.fine_mask.data(), M);
    STG_LAUNCH_CHECK();
    if(ncp > 0)
    {
        k_mas_contacts<B><<<div_up(ncp, 256), 256, 0, s>>>(m.fine_mask.data(), nullptr, m.real_map.data(), pairs, ncp,
                                                          m.node_offset, V);
        STG_LAUNCH_CHECK();
        S.launches++;
    }
    k_mas_l0_closure<B><<<gM, 256, 0, s>>>(m.part_map.data(), m.fine_mask.data(), m.prefix_orig.data(), M);
    STG_LAUNCH_CHECK();
    k_scan_exclusive<<<1, 1024, 0, s>>>(m.prefix_orig.data(), m.prefix_sum_orig.data(), nullptr, m.nb0, m.scratch.data());
    STG_LAUNCH_CHECK();
    k_set_level1<<<1, 1, 0, s>>>(ls, m.scratch.data(), M);
    STG_LAUNCH_CHECK();
    k_mas_l1_assign<B><<<gM, 256, 0, s>>>(m.part_map.data(), m.fine_mask.data(), m.prefix_sum_orig.data(),
                                          m.coarse_tables.data(), m.going_next.data(), M);
    STG_LAUNCH_CHECK();
    S.launches += 5;
    const int gN = div_up(V + B, 256);
    for(int level = 1; level < L; level++)
    {
        const int* prev = m.coarse_tables.data() + (size_t)(level - 1) * V;
        STG_CUDA_TRY(cudaMemsetAsync(m.next_mask.data(), 0, sizeof(unsigned) * (V + B), s));
        k_mas_lx_mask<B><<<gM, 256, 0, s>>>(m.part_map.data(), m.nstart.data(), m.nnum.data(), m.nlist.data(), prev,
                                            m.next_mask.data(), M);
        STG_LAUNCH_CHECK();
        if(ncp > 0)
        {
            k_mas_contacts<B><<<div_up(ncp, 256), 256, 0, s>>>(m.next_mask.data(), prev, m.real_map.data(), pairs, ncp,
                                                              m.node_offset, V);
            STG_LAUNCH_CHECK();
            S.launches++;
        }
        k_mas_lx_closure<B><<<gN, 256, 0, s>>>(m.next_mask.data(), m.closed.data(), m.next_prefix.data(), ls, level);
        STG_LAUNCH_CHECK();
        // n = ceil(ls[2*level] / B) banks
        k_scan_exclusive<<<1, 1024, 0, s>>>(m.next_prefix.data(), m.next_prefix_sum.data(), ls + 2 * level, -B,
                                            ls + 2 * (level + 1));
        STG_LAUNCH_CHECK();
        k_mas_lx_assign<B><<<gN, 256, 0, s>>>(m.next_mask.data(), m.next_prefix_sum.data(), m.going_next.data(), ls, level);
        STG_LAUNCH_CHECK();
        k_mas_compute_next<<<gV, 256, 0, s>>>(m.coarse_tables.data(), m.next_mask.data(), level, V);
        STG_LAUNCH_CHECK();
        S.launches += 5;
    }
    if(L > 1)
    {
        k_mas_aggregate<<<gV, 256, 0, s>>>(m.going_next.data(), m.coarse_table.data(), L, V);
        STG_LAUNCH_CHECK();
        S.launches++;
    }
    STG_CUDA_TRY(cudaMemcpyAsync(m.level_size, ls, sizeof(int) * 2 * (L + 1), cudaMemcpyDeviceToHost, s));
    STG_CUDA_TRY(cudaStreamSynchronize(s));
    m.total_clusters = m.level_size[2 * L + 1];
    m.nbanks = m.total_clusters / B;
    if(m.total_clusters > m.gn_size || m.total_clusters % B != 0)
    {
        set_error("MAS build produced an inconsistent cluster count");
        return STG_ERR_INVALID;
    }
    m.built = true;
    return 0;
}

int Solver::mas_build(const int* contacts, int ncp)
{
    if(!mas.inited)
    {
        set_error("MAS not initialised (stg_mas_init)");
        return STG_ERR_NOT_READY;
    }
    if(cfg.bank_size == 32) return mas_build_t<32>(*this, contacts, ncp);
    return mas_build_t<16>(*this, contacts, ncp);
}

int convert_into(Solver& S, ConvertScratch& cv, int count, const int* rows, const int* cols, const double* blocks,
                 int nrows, bool skip_negative, DBuf<int>& out_rows, DBuf<int>& out_cols, DBuf<double>& out_blocks,
                 DBuf<int>& row_ptr, int* unique, bool fuse = false);

template <int B>
static int mas_assemble_t(Solver& S, int offset)
{
    MasState& m = S.mas;
    cudaStream_t s = S.stream;
    const int NS = nsym(B);
    const size_t nvals = (size_t)m.nbanks * NS * 9;
    STG_TRY(m.mat.resize(nvals));
    STG_TRY(m.inv.resize(nvals));
    // R, Z: one {x y z 0} float4 slot per node of every level
    STG_TRY(m.R.resize((size_t)m.total_clusters * 4));
    STG_TRY(m.Z.resize((size_t)m.total_clusters * 4));
    // the fine convert of stg_solve_linear_system already stored level 0 and emitted the
    // level-1 triplets (ConvFuse) when it ran for this offset
    const bool fused = m.l0_fused && m.l0_offset == offset;
    m.l0_fused = false;
    if(!fused) STG_CUDA_TRY(cudaMemsetAsync(m.mat.data(), 0, nvals * sizeof(double), s));
    STG_CUDA_TRY(cudaMemsetAsync(m.R.data(), 0, sizeof(float) * 4 * m.total_clusters, s));
    const int nnzb = S.bcoo.nnzb;
    const int g = std::max(1, std::min(div_up(nnzb, 256), kSMs * 16));
    if(nnzb > 0 && !fused)
    {
        k_mas_store_l0<B><<<g, 256, 0, s>>>(S.bcoo.R(), S.bcoo.C(), S.bcoo.B(), nnzb, offset, m.V, m.real_map.data(),
                                            m.mat.data());
        STG_LAUNCH_CHECK();
        S.launches++;
    }
    bool learned_captured = false;
    S.learned.graph_ready = false;
    if(m.L > 1 && nnzb > 0)
    {
        // level 1 from the fine matrix
        if(!fused)
        {
            STG_TRY(m.tr_rows.resize(nnzb));
            STG_TRY(m.tr_cols.resize(nnzb));
            STG_TRY(m.tr_blocks.resize((size_t)nnzb * 9));
            k_mas_agg_l0<B><<<g, 256, 0, s>>>(S.bcoo.R(), S.bcoo.C(), S.bcoo.B(), nnzb, offset, m.V,
                                              m.real_map.data(), m.coarse_tables.data(), m.tr_rows.data(),
                                              m.tr_cols.data(), m.tr_blocks.data());
            STG_LAUNCH_CHECK();
            S.launches++;
        }
        int nnz = 0;
        STG_TRY(convert_into(S, m.gcv, nnzb, m.tr_rows.data(), m.tr_cols.data(), m.tr_blocks.data(), m.level_size[2],
                             true, m.ga_rows, m.ga_cols, m.ga_blocks, m.g_rowptr, &nnz));
        for(int level = 1;; level++)
        {
            const int begin = m.level_size[2 * level + 1];
            if(level == S.learned.level && nnz > 0)
            {
                // the learned level's Galerkin operator, kept for its graph (built below)
                LearnedState& Ls = S.learned;
                STG_TRY(Ls.urow.resize(nnz));
                STG_TRY(Ls.ucol.resize(nnz));
                STG_TRY(Ls.ublk.resize(9 * (size_t)nnz));
                STG_CUDA_TRY(cudaMemcpyAsync(Ls.urow.data(), m.ga_rows.data(), sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s));
                STG_CUDA_TRY(cudaMemcpyAsync(Ls.ucol.data(), m.ga_cols.data(), sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s));
                STG_CUDA_TRY(cudaMemcpyAsync(Ls.ublk.data(), m.ga_blocks.data(), sizeof(double) * 9 * nnz,
                                             cudaMemcpyDeviceToDevice, s));
                Ls.unnz = nnz;
                learned_captured = true;
            }
            if(nnz > 0)
            {
                k_mas_extract<B><<<std::max(1, std::min(div_up(nnz, 256), kSMs * 16)), 256, 0, s>>>(
                    m.ga_rows.data(), m.ga_cols.data(), m.ga_blocks.data(), nnz, begin, m.mat.data());
                STG_LAUNCH_CHECK();
                S.launches++;
            }
            if(level + 1 >= m.L || nnz == 0) break;
            const int begin_next = m.level_size[2 * (level + 1) + 1];
            STG_TRY(m.tr_rows.resize(nnz));
            STG_TRY(m.tr_cols.resize(nnz));
            STG_TRY(m.tr_blocks.resize((size_t)nnz * 9));
            k_mas_agg_lx<<<std::max(1, std::min(div_up(nnz, 256), kSMs * 16)), 256, 0, s>>>(
                m.ga_rows.data(), m.ga_cols.data(), m.ga_blocks.data(), nnz, m.going_next.data(), begin, begin_next,
                m.tr_rows.data(), m.tr_cols.data(), m.tr_blocks.data());
            STG_LAUNCH_CHECK();
            S.launches++;
            int nnz2 = 0;
            STG_TRY(convert_into(S, m.gcv, nnz, m.tr_rows.data(), m.tr_cols.data(), m.tr_blocks.data(),
                                 m.level_size[2 * (level + 1)], false, m.gb_rows, m.gb_cols, m.gb_blocks, m.g_rowptr,
                                 &nnz2));
            std::swap(m.ga_rows.ptr, m.gb_rows.ptr);
            std::swap(m.ga_rows.cap, m.gb_rows.cap);
            std::swap(m.ga_cols.ptr, m.gb_cols.ptr);
            std::swap(m.ga_cols.cap, m.gb_cols.cap);
            std::swap(m.ga_blocks.ptr, m.gb_blocks.ptr);
            std::swap(m.ga_blocks.cap, m.gb_blocks.cap);
            nnz = nnz2;
        }
    }
    if(B == 16)
    {
        k_mas_invert16<<<m.nbanks, 256, 0, s>>>(m.mat.data(), m.inv.data(), m.nbanks);
        STG_LAUNCH_CHECK();
    }
    else
    {
        const size_t smem = sizeof(double) * (3 * B * 3 * B + 3 * B);
        if(smem > 48 * 1024)
            STG_CUDA_TRY(cudaFuncSetAttribute(k_mas_invert<B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_mas_invert<B><<<m.nbanks, 3 * B, smem, s>>>(m.mat.data(), m.inv.data(), m.nbanks);
        STG_LAUNCH_CHECK();
    }
    S.launches++;
    if(learned_captured)
    {
        LearnedState& Ls = S.learned;
        const int n = m.level_size[2 * Ls.level];
        Ls.begin = m.level_size[2 * Ls.level + 1];
        STG_TRY(net_build_graph(s, Ls.graph, n, Ls.unnz, Ls.urow.data(), Ls.ucol.data(), Ls.ublk.data(), &S.launches));
        Ls.graph.level = Ls.level;
        const size_t bytes = net_scratch_bytes(n, 1);
        STG_TRY(Ls.scratch.resize(bytes));
        STG_TRY(net_carve(Ls.scratch.data(), bytes, n, 1, Ls.buf));
        Ls.graph_ready = true;
    }
    m.assembled = true;
    return 0;
}

int Solver::mas_assemble(int offset)
{
    if(!mas.built)
    {
        set_error("MAS hierarchy not built");
        return STG_ERR_NOT_READY;
    }
    if(cfg.bank_size == 32) return mas_assemble_t<32>(*this, offset);
    return mas_assemble_t<16>(*this, offset);
}

template <int B>
int mas_restrict_solve_t(Solver& S, const double* r, const int* done)
{
    MasState& m = S.mas;
    cudaStream_t s = S.stream;
    k_mas_restrict0<B><<<div_up(m.M, 256), 256, 0, s>>>(r, m.part_map.data(), m.fine_mask.data(), m.going_next.data(),
                                                        m.R.data(), m.M, done);
    STG_LAUNCH_CHECK();
    S.launches++;
    for(int level = 1; level < m.L - 1; level++)
    {
        const int number = m.level_size[2 * level], begin = m.level_size[2 * level + 1];
        if(number < 1) continue;
        k_mas_restrict_lx<B><<<div_up((number + B - 1) / B * B, 256), 256, 0, s>>>(m.R.data(), m.closed.data(),
                                                                                   m.going_next.data(), number, begin, done);
        STG_LAUNCH_CHECK();
        S.launches++;
    }
    if(B == 16)
        k_mas_schwarz16<<<div_up(m.nbanks, SCHWARZ16_WARPS), SCHWARZ16_WARPS * 32, 0, s>>>(m.inv.data(), m.R.data(),
                                                                                          m.Z.data(), m.nbanks, done);
    else
        k_mas_schwarz32<<<m.nbanks, 1024, 0, s>>>(m.inv.data(), m.R.data(), m.Z.data(), done);
    STG_LAUNCH_CHECK();
    S.launches++;
    return 0;
}

// restriction + bank solves; kernels return immediately when *done != 0 (done may be null)
int mas_restrict_solve_guarded(Solver& S, const double* r, const int* done)
{
    if(S.cfg.bank_size == 32) return mas_restrict_solve_t<32>(S, r, done);
    return mas_restrict_solve_t<16>(S, r, done);
}

int mas_restrict_solve(Solver& S, const double* r) { return mas_restrict_solve_guarded(S, r, nullptr); }

int Solver::mas_apply(const double* r, double* z)
{
    if(!mas.assembled)
    {
        set_error("MAS not assembled");
        return STG_ERR_NOT_READY;
    }
    STG_TRY(mas_restrict_solve(*this, r));
    k_mas_prolong<<<div_up(mas.V, 256), 256, 0, stream>>>(mas.Z.data(), mas.real_map.data(), mas.coarse_table.data(),
                                                          mas.L, mas.V, z);
    STG_LAUNCH_CHECK();
    launches++;
    return 0;
}

}  // namespace stg
