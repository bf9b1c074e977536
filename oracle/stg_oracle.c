/*
 * stg_oracle.c -- CPU oracle for the StiffGIPC Newton linear solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the GPU path is compared against; it
 * is loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and by
 * nothing else.  The product (libstgipc.so) never links or calls it.
 *
 * It restates, serially and in plain C, the reference's algorithms for the hot path:
 *   - srbk_convert  : StiffGIPC/linear_system/utils/converter.cu:32-51, 88-131, 171-238
 *   - srbk_spmv     : StiffGIPC/linear_system/utils/spmv.cu:188-313
 *   - PCG           : StiffGIPC/linear_system/solver/pcg_solver.cu:158-332
 *   - preconditioner composition: global_linear_system.cu:167-180,
 *                     abd_preconditioner.cu:20-38, diag_preconditioner.cu:9-66
 *   - MAS hierarchy : StiffGIPC/MASPreconditioner.cu:29-625 (kernels), 1132-1548 (contacts),
 *                     1551-1826 (drivers), 1731-1750 (level count)
 *   - MAS assembly  : MASPreconditioner.cu:1829-2075 (PrepareHessian_bcoo), 2207-2245
 *   - MAS inverse   : MASPreconditioner.cu:630-726 (__inverse6_P96x96)
 *   - MAS apply     : MASPreconditioner.cu:729-879, 957-1027, 2248-2289
 *   - subsystem index selection: i_preconditioner.cu:32-73
 *
 * Where the reference kernels rely on warp-synchronous shared-memory races
 * (_preparePrefixSumL0_new, _buildConnectMaskLx_new, _nextLevelCluster, _buildLevel1_new),
 * this oracle implements the intended semantics: per-bank connected components of the
 * in-bank connectivity graph, and the union of connectivity masks over all vertices that
 * share a coarse node.
 *
 * Parity status: the integer ordering inputs are pinned by the reference's
 * Assets/sorted_mesh .part fixtures (tests/golden); the floating-point results of convert /
 * SpMV / MAS / PCG are "parity unpinned" -- the reference needs Eigen 3.4, which is absent, so
 * it cannot be built and run to produce golden outputs.
 *
 * Bank size is a run-time parameter (16 = CEMAS as shipped, 32 = Morton-ordered GPU MAS).
 */
#define _POSIX_C_SOURCE 199309L
#include <math.h>
#include <stdint.h>
#include <time.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAX_LEVELS 6

/* Summation orders of the MAS.  The reference forms the coarse bank matrices with FP64
 * atomicAdd (PrepareHessian_bcoo, MASPreconditioner.cu:1849-2075) and the multilevel residual
 * with float atomicAdd (__buildMultiLevelR_optimized_new, :729-847), so its sums have no
 * defined order, and the dot products inside the bank solves (_schwarzLocalXSym6, :957-1027)
 * are a warp reduction whose contraction into FMAs the compiler chooses.
 *   ORC_ORDER_WALK  follows the reference's loops literally: every fine entry and every
 *                   fine residual is walked up the levels (lambda 1 / lambda 2, the atomics
 *                   taken in loop order), pivots divide (`/= rt`), bank rows are summed
 *                   column by column.
 *   ORC_ORDER_FIXED (default) fixes one order, the one the sm_100a kernels use, so that the
 *                   two can be compared bit for bit:
 *     - level l+1 bank matrices from the level-l Galerkin operator A_l, one level at a time:
 *       each upper entry of A_l (in sorted order) is mapped to its coarse pair and oriented
 *       upper, and duplicates are summed in that order (orc_convert);
 *     - Gauss-Jordan rows are scaled by the correctly rounded reciprocal of the pivot;
 *     - the residual of a level-(l+1) node is the FP32 sum, from 0 and in lane order, of the
 *       members of its level-l component;
 *     - 16-vertex bank rows: two partial sums of eight 3x3 blocks each, half h over the
 *       column blocks 8h + ((j + a) mod 8), j = 0..7, each block added with three FMAs
 *       (columns 0, 1, 2); then half 0 + half 1;
 *     - 32-vertex bank rows: the 32 block products (fma(P2, x2, fma(P1, x1, P0 x0))) are
 *       summed by an xor butterfly over 32 lanes (offsets 16, 8, 4, 2, 1);
 *     - prolongation: level 0 + level 1 + ... in FP32, as the reference. */
#define ORC_ORDER_WALK 0
#define ORC_ORDER_FIXED 1

/* ------------------------------------------------------------------------------------ */
/* 3x3 helpers; blocks are column-major (Eigen Matrix3d): element (i,j) at [j*3+i]       */
/* ------------------------------------------------------------------------------------ */
static inline double bget(const double* b, int i, int j) { return b[j * 3 + i]; }

/* ------------------------------------------------------------------------------------ */
/* srbk_convert: triplets -> sorted unique BCOO (converter.cu:88-238).                  */
/* Key = (row << 32) + col, stable sort (cub radix sort keeps input order on ties),     */
/* duplicates summed.  Returns the unique count.                                        */
/* ------------------------------------------------------------------------------------ */
typedef struct { uint64_t key; int idx; } orc_kv;

static int kv_cmp(const void* a, const void* b)
{
    const orc_kv* x = (const orc_kv*)a;
    const orc_kv* y = (const orc_kv*)b;
    if(x->key < y->key) return -1;
    if(x->key > y->key) return 1;
    return (x->idx < y->idx) ? -1 : (x->idx > y->idx);
}

int orc_convert(int count, const int* rows, const int* cols, const double* blocks,
                int* out_rows, int* out_cols, double* out_blocks)
{
    if(count < 1) return 0;
    orc_kv* kv = (orc_kv*)malloc(sizeof(orc_kv) * (size_t)count);
    for(int i = 0; i < count; i++)
    {
        kv[i].key = ((uint64_t)(uint32_t)rows[i] << 32) + (uint64_t)(uint32_t)cols[i];
        kv[i].idx = i;
    }
    qsort(kv, (size_t)count, sizeof(orc_kv), kv_cmp);
    int u = -1;
    uint64_t prev = 0;
    for(int i = 0; i < count; i++)
    {
        if(i == 0 || kv[i].key != prev)
        {
            u++;
            out_rows[u] = (int)(kv[i].key >> 32);
            out_cols[u] = (int)(kv[i].key & 0xffffffffu);
            memcpy(out_blocks + 9 * (size_t)u, blocks + 9 * (size_t)kv[i].idx, 9 * sizeof(double));
            prev = kv[i].key;
        }
        else
        {
            for(int e = 0; e < 9; e++) out_blocks[9 * (size_t)u + e] += blocks[9 * (size_t)kv[i].idx + e];
        }
    }
    free(kv);
    return u + 1;
}

/* ------------------------------------------------------------------------------------ */
/* srbk_spmv: y = a*A*x + b*y with A symmetric, stored as unique upper blocks           */
/* (spmv.cu:188-313).  Diagonal block: H x_j.  Off-diagonal: H x_j into row i and       */
/* H^T x_i into row j.                                                                  */
/* ------------------------------------------------------------------------------------ */
void orc_spmv(double a, int nnzb, const int* rows, const int* cols, const double* blocks,
              const double* x, double b, double* y, int n)
{
    for(int i = 0; i < n; i++) y[i] = (b != 0.0) ? b * y[i] : 0.0;
    for(int k = 0; k < nnzb; k++)
    {
        int i = rows[k], j = cols[k];
        const double* H = blocks + 9 * (size_t)k;
        for(int r = 0; r < 3; r++)
        {
            double s = 0;
            for(int c = 0; c < 3; c++) s += bget(H, r, c) * x[3 * j + c];
            y[3 * i + r] += a * s;
        }
        if(i != j)
        {
            for(int r = 0; r < 3; r++)
            {
                double s = 0;
                for(int c = 0; c < 3; c++) s += bget(H, c, r) * x[3 * i + c];
                y[3 * j + r] += a * s;
            }
        }
    }
}

/* ------------------------------------------------------------------------------------ */
/* MAS                                                                                  */
/* ------------------------------------------------------------------------------------ */
typedef struct
{
    int bank;            /* BANKSIZE (16 or 32)                     */
    int V;               /* totalNodes (FEM vertices)               */
    int M;               /* totalMapNodes = part_offset * bank      */
    int L;               /* levelnum                                */
    int node_offset;     /* collision_node_Offset                   */
    int nlist_size;
    unsigned* nstart;    /* neighbour CSR (init copies)             */
    unsigned* nnum_init;
    unsigned* nlist_init;
    unsigned* nnum;      /* working copies                          */
    unsigned* nlist;
    int* part_map;       /* partId_map_real [M]                     */
    int* real_map;       /* real_map_partId [V]                     */
    /* hierarchy */
    unsigned* fine_mask;       /* [V]                */
    unsigned* next_mask;       /* [V]                */
    int* prefix_orig;          /* [M/bank]           */
    int* prefix_sum_orig;      /* [M/bank]           */
    unsigned* next_prefix;     /* [V]                */
    unsigned* next_prefix_sum; /* [V]                */
    int* coarse_tables;        /* [L*V]              */
    int* going_next;           /* [L*V + M]          */
    int* coarse_table;         /* [V*(L-1)] (itable) */
    unsigned* closed;          /* [total_clusters] closure masks of the coarse nodes (levels >= 1) */
    int level_size[2 * (ORC_MAX_LEVELS + 1)];
    int total_clusters;
    int order;                 /* ORC_ORDER_FIXED (default) or ORC_ORDER_WALK */
    /* matrices */
    int nbanks;                /* total_clusters / bank */
    double* mat;               /* [nbanks * nsym * 9] FP64 packed upper (column-major 3x3) */
    float* inv;                /* [nbanks * nsym * 9] FP32                                 */
} orc_mas;

static inline int nsym(int bank) { return bank * (bank + 1) / 2; }
static inline int upper_index(int bank, int r, int c) { return bank * r - r * (r + 1) / 2 + c; }
static inline unsigned lanemask_lt(int lane) { return (lane >= 32) ? 0xffffffffu : ((1u << lane) - 1u); }
static inline int ffs32(unsigned m) { return m ? __builtin_ctz(m) + 1 : 0; }

/* computeNumLevels (MASPreconditioner.cu:1731-1750) */
int orc_mas_num_levels(int n, int bank)
{
    int nLevel = 1;
    int levelSz = (n + bank - 1) / bank * bank;
    while(levelSz > bank)
    {
        levelSz /= bank;
        nLevel++;
        levelSz = (levelSz + bank - 1) / bank * bank;
    }
    nLevel = nLevel + 1;
    return nLevel > ORC_MAX_LEVELS ? ORC_MAX_LEVELS : nLevel;
}

void orc_mas_destroy(orc_mas* m)
{
    if(!m) return;
    free(m->nstart); free(m->nnum_init); free(m->nlist_init); free(m->nnum); free(m->nlist);
    free(m->part_map); free(m->real_map); free(m->fine_mask); free(m->next_mask);
    free(m->prefix_orig); free(m->prefix_sum_orig); free(m->next_prefix); free(m->next_prefix_sum);
    free(m->coarse_tables); free(m->going_next); free(m->coarse_table); free(m->mat); free(m->inv);
    free(m->closed);
    free(m);
}

/* initPreconditioner_Neighbor (MASPreconditioner.cu:2291-2328) + the uploads of
 * sim_bootstrap.cpp:276-306 */
orc_mas* orc_mas_create(int bank, int V, const unsigned* nstart, const unsigned* nnum,
                        const unsigned* nlist, int nlist_size, const int* part_map, int M,
                        const int* real_map, int node_offset)
{
    orc_mas* m = (orc_mas*)calloc(1, sizeof(orc_mas));
    m->bank = bank; m->V = V; m->M = M; m->node_offset = node_offset; m->nlist_size = nlist_size;
    m->L = orc_mas_num_levels(M > V ? M : V, bank);
    m->nstart = (unsigned*)malloc(sizeof(unsigned) * V);
    m->nnum_init = (unsigned*)malloc(sizeof(unsigned) * V);
    m->nnum = (unsigned*)malloc(sizeof(unsigned) * V);
    m->nlist_init = (unsigned*)malloc(sizeof(unsigned) * (nlist_size > 0 ? nlist_size : 1));
    m->nlist = (unsigned*)malloc(sizeof(unsigned) * (nlist_size > 0 ? nlist_size : 1));
    memcpy(m->nstart, nstart, sizeof(unsigned) * V);
    memcpy(m->nnum_init, nnum, sizeof(unsigned) * V);
    if(nlist_size > 0) memcpy(m->nlist_init, nlist, sizeof(unsigned) * nlist_size);
    m->part_map = (int*)malloc(sizeof(int) * M);
    m->real_map = (int*)malloc(sizeof(int) * V);
    memcpy(m->part_map, part_map, sizeof(int) * M);
    memcpy(m->real_map, real_map, sizeof(int) * V);
    m->fine_mask = (unsigned*)calloc(V, sizeof(unsigned));
    m->next_mask = (unsigned*)calloc(V, sizeof(unsigned));
    int nb0 = M / bank + 1;
    m->prefix_orig = (int*)calloc(nb0, sizeof(int));
    m->prefix_sum_orig = (int*)calloc(nb0, sizeof(int));
    m->next_prefix = (unsigned*)calloc(V + 1, sizeof(unsigned));
    m->next_prefix_sum = (unsigned*)calloc(V + 1, sizeof(unsigned));
    m->coarse_tables = (int*)calloc((size_t)m->L * V, sizeof(int));
    m->going_next = (int*)calloc((size_t)m->L * V + M, sizeof(int));
    m->coarse_table = (int*)calloc((size_t)V * (m->L > 1 ? m->L - 1 : 1), sizeof(int));
    m->order = ORC_ORDER_FIXED;
    return m;
}

void orc_mas_set_order(orc_mas* m, int order) { m->order = order; }

int orc_mas_levels(const orc_mas* m) { return m->L; }
int orc_mas_total_clusters(const orc_mas* m) { return m->total_clusters; }

/* Decode one sign-encoded collision pair (MASPreconditioner.cu:1141-1548) into up to four
 * FEM-local vertex ids (-1 = absent or ABD).  Returns the vertex count. */
static int decode_pair(const int* cp, int node_offset, int out[4])
{
    int v[4] = {cp[0], cp[1], cp[2], cp[3]};
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
                v[1] = -v[1] - 1; v[2] = -v[2] - 1; v[3] = -v[3] - 1;
            }
            else
                cnt = 2;
        }
        else if(v[3] < 0)
        {
            if(v[1] < 0)
            {
                v[1] = -v[1] - 1; v[3] = -v[3] - 1;
            }
            else
                cnt = 3;
        }
    }
    for(int i = 0; i < 4; i++) out[i] = -1;
    for(int i = 0; i < cnt; i++)
    {
        int id = v[i] - node_offset;
        out[i] = id >= 0 ? id : -1;
    }
    return cnt;
}

/* _buildCollisionConnection_new for one level (level 0: coarse == NULL). */
static void collision_connection(orc_mas* m, unsigned* conn, const int* coarse, const int* pairs, int ncp)
{
    const int B = m->bank;
    for(int p = 0; p < ncp; p++)
    {
        int vid[4];
        int cnt = decode_pair(pairs + 4 * p, m->node_offset, vid);
        int cpv[4];
        for(int i = 0; i < cnt; i++)
            cpv[i] = vid[i] >= 0 ? (coarse ? coarse[vid[i]] : m->real_map[vid[i]]) : -1;
        unsigned msk[4] = {0, 0, 0, 0};
        for(int i = 0; i < cnt; i++)
            for(int j = i + 1; j < cnt; j++)
            {
                int a = cpv[i], b = cpv[j];
                if(a == b || a < 0 || b < 0) continue;
                if(a / B == b / B)
                {
                    msk[i] |= 1u << (b % B);
                    msk[j] |= 1u << (a % B);
                }
            }
        for(int i = 0; i < cnt; i++)
        {
            if(coarse)
            {
                if(cpv[i] >= 0) conn[cpv[i]] |= msk[i];
            }
            else if(vid[i] >= 0)
                conn[vid[i]] |= msk[i];
        }
    }
}

/* closure of the in-bank graph: visit lanes reachable from `lane` through the original
 * masks `orig` of the bank (the loop of _preparePrefixSumL0_new / _nextLevelCluster) */
static unsigned closure(const unsigned* orig, int lane, unsigned start)
{
    unsigned conn = start;
    unsigned visited = 1u << lane;
    for(;;)
    {
        unsigned todo = visited ^ conn;
        if(!todo) break;
        int nv = ffs32(todo) - 1;
        visited |= 1u << nv;
        conn |= orig[nv];
    }
    return conn;
}

/* ReorderRealtime (MASPreconditioner.cu:1785-1826) with intended (race-free) semantics. */
int orc_mas_build(orc_mas* m, const int* pairs, int ncp)
{
    const int B = m->bank, V = m->V, M = m->M, L = m->L;
    const int nb0 = M / B;
    unsigned orig[32];
    memcpy(m->nlist, m->nlist_init, sizeof(unsigned) * (m->nlist_size > 0 ? m->nlist_size : 0));
    memcpy(m->nnum, m->nnum_init, sizeof(unsigned) * V);
    memset(m->level_size, 0, sizeof(m->level_size));

    /* BuildConnectMaskL0: _buildCML0_new (MASPreconditioner.cu:62-98) */
    for(int s = 0; s < M; s++)
    {
        int v = m->part_map[s];
        if(v < 0) continue;
        int bank = s / B, lane = s % B;
        unsigned msk = 1u << lane;
        unsigned nk = 0, st = m->nstart[v], num = m->nnum[v];
        for(unsigned i = 0; i < num; i++)
        {
            unsigned u = m->nlist[st + i];
            int su = m->real_map[u];
            if(su / B == bank)
                msk |= 1u << (su % B);
            else
                m->nlist[st + nk++] = u;
        }
        m->nnum[v] = nk;
        m->fine_mask[v] = msk;
    }
    if(ncp > 0) collision_connection(m, m->fine_mask, NULL, pairs, ncp);

    /* PreparePrefixSumL0: _preparePrefixSumL0_new (MASPreconditioner.cu:159-214) */
    for(int b = 0; b < nb0; b++)
    {
        for(int l = 0; l < B; l++)
        {
            int v = m->part_map[b * B + l];
            orig[l] = v >= 0 ? m->fine_mask[v] : 0u;
        }
        int comps = 0;
        for(int l = 0; l < B; l++)
        {
            int v = m->part_map[b * B + l];
            if(v < 0) continue;
            unsigned c = closure(orig, l, orig[l]);
            m->fine_mask[v] = c;
            if(__builtin_popcount(c & lanemask_lt(l)) == 0) comps++;
        }
        m->prefix_orig[b] = comps;
    }

    /* BuildLevel1: exclusive scan + _buildLevel1_new (MASPreconditioner.cu:270-328) */
    {
        int acc = 0;
        for(int b = 0; b < nb0; b++) { m->prefix_sum_orig[b] = acc; acc += m->prefix_orig[b]; }
        m->level_size[2 * 1 + 0] = acc;
        m->level_size[2 * 1 + 1] = M;
        for(int b = 0; b < nb0; b++)
        {
            unsigned elected = 0;
            for(int l = 0; l < B; l++)
            {
                int v = m->part_map[b * B + l];
                if(v < 0) continue;
                if(__builtin_popcount(m->fine_mask[v] & lanemask_lt(l)) == 0) elected |= 1u << l;
            }
            for(int l = 0; l < B; l++)
            {
                int v = m->part_map[b * B + l];
                if(v < 0) continue;
                int lead = ffs32(m->fine_mask[v]) - 1;
                int id = __builtin_popcount(elected & lanemask_lt(lead)) + m->prefix_sum_orig[b];
                m->coarse_tables[v] = id;
                m->going_next[v] = id + M;
            }
        }
    }

    free(m->closed);
    m->closed = (unsigned*)calloc((size_t)(m->L + 1) * (M > V ? M : V) + 64, sizeof(unsigned));
    for(int level = 1; level < L; level++)
    {
        memset(m->next_mask, 0, sizeof(unsigned) * V);
        const int* prev = m->coarse_tables + (size_t)(level - 1) * V;
        /* _buildConnectMaskLx_new (MASPreconditioner.cu:401-470), union semantics */
        for(int s = 0; s < M; s++)
        {
            int v = m->part_map[s];
            if(v < 0) continue;
            unsigned c = (unsigned)prev[v];
            unsigned msk = 0, nk = 0, st = m->nstart[v], num = m->nnum[v];
            for(unsigned i = 0; i < num; i++)
            {
                unsigned u = m->nlist[st + i];
                unsigned cu = (unsigned)prev[u];
                if(c / B == cu / B)
                    msk |= 1u << (cu % B);
                else
                    m->nlist[st + nk++] = u;
            }
            m->nnum[v] = nk;
            m->next_mask[c] |= msk;
        }
        if(ncp > 0) collision_connection(m, m->next_mask, prev, pairs, ncp);

        int number = m->level_size[2 * level + 0];
        int level_begin = m->level_size[2 * level + 1];
        int nb = (number + B - 1) / B;
        /* _nextLevelCluster (MASPreconditioner.cu:473-520) */
        for(int b = 0; b < nb; b++)
        {
            int cnt = (b == nb - 1) ? number - b * B : B;
            for(int l = 0; l < B; l++) orig[l] = (l < cnt) ? ((1u << l) | m->next_mask[b * B + l]) : 0u;
            int comps = 0;
            for(int l = 0; l < cnt; l++)
            {
                unsigned c = closure(orig, l, orig[l]);
                m->next_mask[b * B + l] = c;
                m->closed[level_begin + b * B + l] = c;
                if(__builtin_popcount(c & lanemask_lt(l)) == 0) comps++;
            }
            m->next_prefix[b] = (unsigned)comps;
        }
        /* exclusive scan + _prefixSumLx (MASPreconditioner.cu:522-566) */
        unsigned acc = 0;
        for(int b = 0; b < nb; b++) { m->next_prefix_sum[b] = acc; acc += m->next_prefix[b]; }
        int rounded = (number + B - 1) / B * B;
        m->level_size[2 * (level + 1) + 0] = (int)acc;
        m->level_size[2 * (level + 1) + 1] = level_begin + rounded;
        for(int b = 0; b < nb; b++)
        {
            int cnt = (b == nb - 1) ? number - b * B : B;
            unsigned elected = 0;
            for(int l = 0; l < cnt; l++)
                if(__builtin_popcount(m->next_mask[b * B + l] & lanemask_lt(l)) == 0) elected |= 1u << l;
            int ids[32];
            for(int l = 0; l < cnt; l++)
            {
                int lead = ffs32(m->next_mask[b * B + l]) - 1;
                ids[l] = __builtin_popcount(elected & lanemask_lt(lead)) + (int)m->next_prefix_sum[b];
            }
            for(int l = 0; l < cnt; l++)
            {
                m->next_mask[b * B + l] = (unsigned)ids[l];
                m->going_next[b * B + l + level_begin] = ids[l] + level_begin + rounded;
            }
        }
        /* _computeNextLevel (MASPreconditioner.cu:568-579) */
        int* cur = m->coarse_tables + (size_t)level * V;
        for(int v = 0; v < V; v++) cur[v] = (int)m->next_mask[prev[v]];
    }
    m->total_clusters = m->level_size[2 * L + 1];

    /* _aggregationKernel (MASPreconditioner.cu:581-608) */
    for(int v = 0; v < V; v++)
    {
        int cur = v;
        for(int l = 0; l < L - 1; l++)
        {
            cur = m->going_next[cur];
            m->coarse_table[(size_t)v * (L - 1) + l] = cur;
        }
    }
    return m->total_clusters;
}

/* Copies of the hierarchy for bit-exact comparisons.  Any pointer may be NULL. */
void orc_mas_export(const orc_mas* m, unsigned* fine_mask, int* prefix_orig, int* coarse_tables,
                    int* going_next, int* coarse_table, int* level_size, unsigned* nlist, unsigned* nnum)
{
    const int V = m->V, L = m->L;
    if(fine_mask) memcpy(fine_mask, m->fine_mask, sizeof(unsigned) * V);
    if(prefix_orig) memcpy(prefix_orig, m->prefix_orig, sizeof(int) * (m->M / m->bank));
    if(coarse_tables) memcpy(coarse_tables, m->coarse_tables, sizeof(int) * (size_t)L * V);
    if(going_next)
    {
        /* entries [0, V) for vertices and [M, total) for coarse nodes */
        memcpy(going_next, m->going_next, sizeof(int) * (size_t)((m->total_clusters > V) ? m->total_clusters : V));
    }
    if(coarse_table) memcpy(coarse_table, m->coarse_table, sizeof(int) * (size_t)V * (L > 1 ? L - 1 : 1));
    if(level_size) memcpy(level_size, m->level_size, sizeof(int) * 2 * (L + 1));
    if(nlist) memcpy(nlist, m->nlist, sizeof(unsigned) * m->nlist_size);
    if(nnum) memcpy(nnum, m->nnum, sizeof(unsigned) * V);
}

/* calculate_subsystem_bcoo_indices (i_preconditioner.cu:32-73): entries whose row and col
 * both lie in [offset, end), in BCOO order. */
int orc_select_range(int nnzb, const int* rows, const int* cols, int offset, int end, int* out)
{
    int c = 0;
    for(int k = 0; k < nnzb; k++)
        if(rows[k] >= offset && rows[k] < end && cols[k] >= offset && cols[k] < end) out[c++] = k;
    return c;
}

static inline double* mblk(orc_mas* m, int gid_bank, int idx) { return m->mat + ((size_t)gid_bank * nsym(m->bank) + idx) * 9; }

/* In-place Gauss-Jordan inverse of one bank (__inverse6_P96x96, MASPreconditioner.cu:630-726).
 * The pivot row is divided by the pivot (ORC_ORDER_WALK, `/= rt` as in the reference) or
 * multiplied by its correctly rounded reciprocal (ORC_ORDER_FIXED); the elimination is
 * fma(-colm[k], A[j][i], A[k][i]), the contraction of the reference's `+= rate * ...`. */
static void invert_bank(orc_mas* m, int bk, double* A, double* colm)
{
    const int B = m->bank, N = 3 * B;
    for(int j = 0; j < N; j++)
        for(int i = 0; i < N; i++)
        {
            int rowId = j / 3, colId = i / 3;
            double v;
            if(colId >= rowId)
                v = bget(mblk(m, bk, upper_index(B, rowId, colId)), j % 3, i % 3);
            else
                v = bget(mblk(m, bk, upper_index(B, colId, rowId)), i % 3, j % 3);
            if(i == j && v == 0.0) v = 1.0;
            A[(size_t)j * N + i] = v;
        }
    for(int j = 0; j < N; j++)
    {
        double rt = A[(size_t)j * N + j];
        for(int i = 0; i < N; i++) colm[i] = A[(size_t)i * N + j];
        for(int i = 0; i < N; i++) A[(size_t)i * N + j] = (i == j) ? 1.0 : 0.0;
        if(m->order == ORC_ORDER_FIXED)
        {
            const double rinv = 1.0 / rt;
            for(int i = 0; i < N; i++) A[(size_t)j * N + i] *= rinv;
        }
        else
            for(int i = 0; i < N; i++) A[(size_t)j * N + i] /= rt;
        for(int k = 0; k < N; k++)
        {
            if(k == j) continue;
            double rate = -colm[k];
            for(int i = 0; i < N; i++) A[(size_t)k * N + i] = fma(rate, A[(size_t)j * N + i], A[(size_t)k * N + i]);
        }
    }
    for(int i = 0; i < N; i++)
    {
        if(i % 3 < 2)
            A[(size_t)(i + 1) * N + i] = A[(size_t)i * N + i + 1];
        else
            A[(size_t)i * N + i - 2] = A[(size_t)(i - 2) * N + i];
    }
    float* P = m->inv + (size_t)bk * nsym(B) * 9;
    for(int j = 0; j < N; j++)
        for(int i = 0; i < N; i++)
        {
            int rowId = j / 3, colId = i / 3;
            if(colId >= rowId)
                P[(size_t)upper_index(B, rowId, colId) * 9 + (i % 3) * 3 + (j % 3)] = (float)A[(size_t)j * N + i];
        }
}

/* An upper entry (u <= v) with value H mapped to the coarse pair (a, b) and oriented upper:
 * a < b: H; a > b: H^T at (b, a); a == b: H (u == v) or H + H^T (u < v).  The level-(l+1)
 * Galerkin entry P^T A P sums these over the level-l entries. */
static void coarse_triplet(int u, int v, int a, int b, const double* H, int* orow, int* ocol, double* oblk)
{
    if(a < b || (a == b && u == v))
        memcpy(oblk, H, 9 * sizeof(double));
    else if(a > b)
    {
        for(int i = 0; i < 3; i++)
            for(int j = 0; j < 3; j++) oblk[j * 3 + i] = H[i * 3 + j];
        int t = a; a = b; b = t;
    }
    else
        for(int i = 0; i < 3; i++)
            for(int j = 0; j < 3; j++) oblk[j * 3 + i] = H[j * 3 + i] + H[i * 3 + j];
    *orow = a;
    *ocol = b;
}

/* ORC_ORDER_FIXED assembly: the bank-diagonal blocks of every level's Galerkin operator, one
 * level at a time (A_1 from the fine entries, A_(l+1) from A_l).  The level-0 in-bank entries
 * with slot(col) < slot(row) are left out of A_0 as lambda 1 leaves them out of the bank
 * matrix (MASPreconditioner.cu:1849-1944), which lambda 2 then propagates (:1946-2075). */
static void assemble_levels(orc_mas* m, const int* rows, const int* cols, const double* blocks,
                            const int* sel, int nsel, int offset)
{
    const int B = m->bank, L = m->L;
    int* trow = (int*)malloc(sizeof(int) * (size_t)(nsel > 0 ? nsel : 1));
    int* tcol = (int*)malloc(sizeof(int) * (size_t)(nsel > 0 ? nsel : 1));
    double* tblk = (double*)malloc(sizeof(double) * 9 * (size_t)(nsel > 0 ? nsel : 1));
    int* arow = (int*)malloc(sizeof(int) * (size_t)(nsel > 0 ? nsel : 1));
    int* acol = (int*)malloc(sizeof(int) * (size_t)(nsel > 0 ? nsel : 1));
    double* ablk = (double*)malloc(sizeof(double) * 9 * (size_t)(nsel > 0 ? nsel : 1));
    int nt = 0;
    for(int I = 0; I < nsel; I++)
    {
        const int k = sel[I];
        const double* H = blocks + 9 * (size_t)k;
        const int rr = rows[k] - offset, cc = cols[k] - offset;
        const int sc = m->real_map[cc], sr = m->real_map[rr];
        if(sc / B == sr / B)
        {
            if(sc < sr) continue;
            memcpy(mblk(m, sc / B, upper_index(B, sr % B, sc % B)), H, 9 * sizeof(double));
        }
        if(L > 1)
        {
            coarse_triplet(rr, cc, m->coarse_tables[rr], m->coarse_tables[cc], H, trow + nt, tcol + nt,
                           tblk + 9 * (size_t)nt);
            nt++;
        }
    }
    for(int level = 1; level < L && nt > 0; level++)
    {
        const int begin = m->level_size[2 * level + 1];
        const int na = orc_convert(nt, trow, tcol, tblk, arow, acol, ablk);
        for(int e = 0; e < na; e++)
        {
            const int ga = begin + arow[e], gb = begin + acol[e];
            if(ga / B != gb / B) continue;
            memcpy(mblk(m, ga / B, upper_index(B, ga % B, gb % B)), ablk + 9 * (size_t)e, 9 * sizeof(double));
        }
        if(level + 1 >= L) break;
        const int begin_next = m->level_size[2 * (level + 1) + 1];
        for(int e = 0; e < na; e++)
            coarse_triplet(arow[e], acol[e], m->going_next[begin + arow[e]] - begin_next,
                           m->going_next[begin + acol[e]] - begin_next, ablk + 9 * (size_t)e, trow + e, tcol + e,
                           tblk + 9 * (size_t)e);
        nt = na;
    }
    free(trow); free(tcol); free(tblk); free(arow); free(acol); free(ablk);
}

/* setPreconditioner_bcoo after ReorderRealtime: PrepareHessian_bcoo + inverse
 * (MASPreconditioner.cu:1829-2075, 2207-2245).  `sel` lists the BCOO entries of the FEM
 * range (orc_select_range); `offset` is the FEM block offset. */
void orc_mas_assemble(orc_mas* m, const int* rows, const int* cols, const double* blocks,
                      const int* sel, int nsel, int offset)
{
    const int B = m->bank, L = m->L, NS = nsym(B);
    m->nbanks = m->total_clusters / B;
    free(m->mat); free(m->inv);
    m->mat = (double*)calloc((size_t)m->nbanks * NS * 9, sizeof(double));
    m->inv = (float*)calloc((size_t)m->nbanks * NS * 9, sizeof(float));
    if(m->order == ORC_ORDER_FIXED)
    {
        assemble_levels(m, rows, cols, blocks, sel, nsel, offset);
        goto invert;
    }

    /* lambda 1 (MASPreconditioner.cu:1849-1944) */
    for(int I = 0; I < nsel; I++)
    {
        int k = sel[I];
        const double* H = blocks + 9 * (size_t)k;
        int rr = rows[k] - offset, cc = cols[k] - offset;
        int sc = m->real_map[cc], sr = m->real_map[rr];
        if(sc / B == sr / B)
        {
            if(sc >= sr) memcpy(mblk(m, sc / B, upper_index(B, sr % B, sc % B)), H, 9 * sizeof(double));
            continue;
        }
        int gc = cc, gr = rr;
        for(int level = 1; level < L; level++)
        {
            gc = m->going_next[gc];
            gr = m->going_next[gr];
            if(gc / B != gr / B) continue;
            if(gc >= gr)
            {
                double* D = mblk(m, gc / B, upper_index(B, gr % B, gc % B));
                for(int i = 0; i < 3; i++)
                    for(int j = 0; j < 3; j++)
                    {
                        D[j * 3 + i] += bget(H, i, j);
                        if(gc == gr) D[j * 3 + i] += bget(H, j, i);
                    }
            }
            else
            {
                double* D = mblk(m, gc / B, upper_index(B, gc % B, gr % B));
                for(int i = 0; i < 3; i++)
                    for(int j = 0; j < 3; j++) D[j * 3 + i] += bget(H, j, i);
            }
        }
    }

    /* lambda 2 (MASPreconditioner.cu:1946-2075) */
    const int nb0 = m->M / B;
    for(int b = 0; b < nb0; b++)
    {
        double S[9] = {0};
        int any = -1;
        for(int LR = 0; LR < B; LR++)
            for(int LC = 0; LC < B; LC++)
            {
                int rdx = m->part_map[b * B + LR], cdx = m->part_map[b * B + LC];
                if(rdx < 0 || cdx < 0) continue;
                double mat3[9];
                if(LC >= LR)
                    memcpy(mat3, mblk(m, b, upper_index(B, LR, LC)), sizeof(mat3));
                else
                {
                    const double* src = mblk(m, b, upper_index(B, LC, LR));
                    for(int i = 0; i < 3; i++)
                        for(int j = 0; j < 3; j++) mat3[j * 3 + i] = src[i * 3 + j];
                }
                if(m->prefix_orig[b] == 1)
                {
                    for(int e = 0; e < 9; e++) S[e] += mat3[e];
                    any = rdx;
                }
                else
                {
                    for(int level = 1; level < L; level++)
                    {
                        rdx = m->going_next[rdx];
                        cdx = m->going_next[cdx];
                        if(rdx / B == cdx / B && cdx >= rdx)
                        {
                            double* D = mblk(m, cdx / B, upper_index(B, rdx % B, cdx % B));
                            for(int e = 0; e < 9; e++) D[e] += mat3[e];
                        }
                    }
                }
            }
        if(m->prefix_orig[b] == 1 && any >= 0)
        {
            int nid = m->going_next[any];
            for(int level = 1; level < L; level++)
            {
                double* D = mblk(m, nid / B, upper_index(B, nid % B, nid % B));
                for(int e = 0; e < 9; e++) D[e] += S[e];
                nid = m->going_next[nid];
            }
        }
    }

    /* __inverse6_P96x96 over every bank of every level */
invert:
    {
        const int N = 3 * B;
        double* A = (double*)malloc(sizeof(double) * N * N);
        double* colm = (double*)malloc(sizeof(double) * N);
        for(int bk = 0; bk < m->nbanks; bk++) invert_bank(m, bk, A, colm);
        free(A); free(colm);
    }
}

int orc_mas_nbanks(const orc_mas* m) { return m->nbanks; }

void orc_mas_export_matrices(const orc_mas* m, double* mat, float* inv)
{
    size_t cnt = (size_t)m->nbanks * nsym(m->bank) * 9;
    if(mat) memcpy(mat, m->mat, cnt * sizeof(double));
    if(inv) memcpy(inv, m->inv, cnt * sizeof(float));
}

/* ORC_ORDER_FIXED: sum, from 0 and in lane order, of the lanes of `msk` in the bank whose
 * values start at R + 3 * base */
static void lane_sum(const float* R, int base, unsigned msk, int B, float out[3])
{
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    for(int b = 0; b < B; b++)
        if(msk & (1u << b))
        {
            a0 += R[3 * (size_t)(base + b)];
            a1 += R[3 * (size_t)(base + b) + 1];
            a2 += R[3 * (size_t)(base + b) + 2];
        }
    out[0] = a0; out[1] = a1; out[2] = a2;
}

/* element (i, k) of block (a, c) of a packed upper bank inverse (column-major 3x3 blocks;
 * a lower block is the transpose of its mirror) */
static inline float pblk(const float* P, int B, int a, int c, int i, int k)
{
    return c >= a ? P[(size_t)upper_index(B, a, c) * 9 + k * 3 + i] : P[(size_t)upper_index(B, c, a) * 9 + i * 3 + k];
}

/* ORC_ORDER_FIXED bank solve z_a = sum_c P_ac r_c of one bank (see the order notes above) */
static void bank_solve_fixed(const float* P, const float* R, int B, float* Z)
{
    for(int a = 0; a < B; a++)
    {
        float z[3];
        if(B == 16)
        {
            float zh[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
            for(int h = 0; h < 2; h++)
                for(int j = 0; j < 8; j++)
                {
                    const int c = 8 * h + ((j + a) & 7);
                    const float* x = R + 3 * c;
                    for(int i = 0; i < 3; i++)
                    {
                        float acc = zh[h][i];
                        acc = fmaf(pblk(P, B, a, c, i, 0), x[0], acc);
                        acc = fmaf(pblk(P, B, a, c, i, 1), x[1], acc);
                        acc = fmaf(pblk(P, B, a, c, i, 2), x[2], acc);
                        zh[h][i] = acc;
                    }
                }
            for(int i = 0; i < 3; i++) z[i] = zh[0][i] + zh[1][i];
        }
        else
        {
            float v[32][3];
            for(int c = 0; c < 32; c++)
            {
                const float* x = R + 3 * c;
                for(int i = 0; i < 3; i++)
                    v[c][i] = fmaf(pblk(P, B, a, c, i, 2), x[2], fmaf(pblk(P, B, a, c, i, 1), x[1], pblk(P, B, a, c, i, 0) * x[0]));
            }
            for(int o = 16; o > 0; o >>= 1)
            {
                float w[32][3];
                for(int l = 0; l < 32; l++)
                    for(int i = 0; i < 3; i++) w[l][i] = v[l][i] + v[l ^ o][i];
                memcpy(v, w, sizeof(v));
            }
            for(int i = 0; i < 3; i++) z[i] = v[0][i];
        }
        for(int i = 0; i < 3; i++) Z[3 * a + i] = z[i];
    }
}

static void mas_apply_fixed(const orc_mas* m, const double* r, double* z)
{
    const int B = m->bank, V = m->V, M = m->M, L = m->L, T = m->total_clusters, NS = nsym(B);
    float* R = (float*)calloc((size_t)T * 3 + 3 * 32, sizeof(float));
    float* Zc = (float*)calloc((size_t)T * 3 + 3 * 32, sizeof(float));
    for(int s = 0; s < M; s++)
    {
        int v = m->part_map[s];
        if(v < 0) continue;
        for(int c = 0; c < 3; c++) R[3 * (size_t)s + c] = (float)r[3 * v + c];
    }
    if(L > 1)
        for(int s = 0; s < M; s++)
        {
            const int v = m->part_map[s];
            if(v < 0) continue;
            const unsigned msk = m->fine_mask[v];
            if(__builtin_popcount(msk & lanemask_lt(s % B)) != 0) continue;
            lane_sum(R, s / B * B, msk, B, R + 3 * (size_t)m->going_next[v]);
        }
    for(int level = 1; level < L - 1; level++)
    {
        const int number = m->level_size[2 * level], begin = m->level_size[2 * level + 1];
        for(int i = 0; i < number; i++)
        {
            const unsigned msk = m->closed[begin + i];
            if(__builtin_popcount(msk & lanemask_lt(i % B)) != 0) continue;
            lane_sum(R, begin + i / B * B, msk, B, R + 3 * (size_t)m->going_next[begin + i]);
        }
    }
    for(int bk = 0; bk < T / B; bk++)
        bank_solve_fixed(m->inv + (size_t)bk * NS * 9, R + 3 * (size_t)bk * B, B, Zc + 3 * (size_t)bk * B);
    for(int v = 0; v < V; v++)
    {
        const int s = m->real_map[v];
        float cz[3] = {Zc[3 * (size_t)s], Zc[3 * (size_t)s + 1], Zc[3 * (size_t)s + 2]};
        for(int l = 1; l < L; l++)
        {
            const int now = m->coarse_table[(size_t)v * (L - 1) + l - 1];
            for(int c = 0; c < 3; c++) cz[c] += Zc[3 * (size_t)now + c];
        }
        for(int c = 0; c < 3; c++) z[3 * v + c] = (double)cz[c];
    }
    free(R); free(Zc);
}

/* preconditioning (MASPreconditioner.cu:2248-2289): restrict (729-847), local solves
 * (957-1027), prolong (850-879).  r, z: FEM sub-range, 3V doubles. */
void orc_mas_apply(const orc_mas* m, const double* r, double* z)
{
    if(m->order == ORC_ORDER_FIXED)
    {
        mas_apply_fixed(m, r, z);
        return;
    }
    const int B = m->bank, V = m->V, M = m->M, L = m->L, T = m->total_clusters;
    float* R = (float*)calloc((size_t)T * 3, sizeof(float));
    float* Zc = (float*)calloc((size_t)T * 3, sizeof(float));
    for(int s = 0; s < M; s++)
    {
        int v = m->part_map[s];
        if(v < 0) continue;
        float rv[3] = {(float)r[3 * v], (float)r[3 * v + 1], (float)r[3 * v + 2]};
        for(int c = 0; c < 3; c++) R[3 * s + c] = rv[c];
        int id = v;
        for(int level = 1; level < L; level++)
        {
            id = m->going_next[id];
            for(int c = 0; c < 3; c++) R[3 * (size_t)id + c] += rv[c];
        }
    }
    const int NS = nsym(B);
    for(int bk = 0; bk < T / B; bk++)
    {
        const float* P = m->inv + (size_t)bk * NS * 9;
        for(int a = 0; a < B; a++)
        {
            float acc[3] = {0, 0, 0};
            for(int c = 0; c < B; c++)
            {
                const float* rc = R + 3 * ((size_t)bk * B + c);
                if(c >= a)
                {
                    const float* Pb = P + (size_t)upper_index(B, a, c) * 9;
                    for(int i = 0; i < 3; i++)
                        acc[i] += Pb[0 * 3 + i] * rc[0] + Pb[1 * 3 + i] * rc[1] + Pb[2 * 3 + i] * rc[2];
                }
                else
                {
                    const float* Pb = P + (size_t)upper_index(B, c, a) * 9;
                    for(int i = 0; i < 3; i++)
                        acc[i] += Pb[i * 3 + 0] * rc[0] + Pb[i * 3 + 1] * rc[1] + Pb[i * 3 + 2] * rc[2];
                }
            }
            for(int i = 0; i < 3; i++) Zc[3 * ((size_t)bk * B + a) + i] = acc[i];
        }
    }
    for(int v = 0; v < V; v++)
    {
        int s = m->real_map[v];
        float cz[3] = {Zc[3 * (size_t)s], Zc[3 * (size_t)s + 1], Zc[3 * (size_t)s + 2]};
        for(int l = 1; l < L; l++)
        {
            int now = m->coarse_table[(size_t)v * (L - 1) + l - 1];
            for(int c = 0; c < 3; c++) cz[c] += Zc[3 * (size_t)now + c];
        }
        for(int c = 0; c < 3; c++) z[3 * v + c] = (double)cz[c];
    }
    free(R); free(Zc);
}

/* ------------------------------------------------------------------------------------ */
/* Preconditioner composition + PCG                                                      */
/* ------------------------------------------------------------------------------------ */
typedef struct
{
    int iterations;
    double rz0, rz_final;
    double rel_residual;      /* ||b - A x|| / ||b||, FP64 */
} orc_pcg_stats;

/* 3x3 inverse of a column-major block (cofactor / determinant) */
static void inv3(const double* H, double* D)
{
    double a = bget(H, 0, 0), b = bget(H, 0, 1), c = bget(H, 0, 2);
    double d = bget(H, 1, 0), e = bget(H, 1, 1), f = bget(H, 1, 2);
    double g = bget(H, 2, 0), h = bget(H, 2, 1), i = bget(H, 2, 2);
    double A = e * i - f * h, Bc = -(d * i - f * g), C = d * h - e * g;
    double det = a * A + b * Bc + c * C;
    double inv_det = 1.0 / det;
    double R[9] = {A, -(b * i - c * h), b * f - c * e, Bc, a * i - c * g, -(a * f - c * d), C, -(a * h - b * g), a * e - b * d};
    /* R row-major adjugate */
    for(int r = 0; r < 3; r++)
        for(int col = 0; col < 3; col++) D[col * 3 + r] = R[r * 3 + col] * inv_det;
}

typedef struct
{
    int nnzb;
    const int* rows;
    const int* cols;
    const double* blocks;
    int n;
    /* global block-Jacobi (DiagPreconditioner) when nonzero */
    int use_diag;
    double* diag_inv;          /* [n/3 * 9] */
    /* ABD 12x12 block-Jacobi over the first abd_bodies*12 dofs */
    int abd_bodies;
    const double* abd_inv;     /* [bodies * 144] row-major */
    /* MAS over [fem_offset, fem_offset + V) blocks */
    const orc_mas* mas;
    int fem_offset;
} orc_system;

static void apply_preconditioner(const orc_system* s, const double* r, double* z)
{
    /* GlobalLinearSystem::apply_preconditioner (global_linear_system.cu:167-180) */
    if(s->use_diag)
    {
        for(int bi = 0; bi < s->n / 3; bi++)
        {
            const double* D = s->diag_inv + 9 * (size_t)bi;
            for(int rr = 0; rr < 3; rr++)
                z[3 * bi + rr] = bget(D, rr, 0) * r[3 * bi] + bget(D, rr, 1) * r[3 * bi + 1] + bget(D, rr, 2) * r[3 * bi + 2];
        }
    }
    else
        memcpy(z, r, sizeof(double) * s->n);
    for(int body = 0; body < s->abd_bodies; body++)
    {
        const double* J = s->abd_inv + 144 * (size_t)body;
        for(int rr = 0; rr < 12; rr++)
        {
            double acc = 0;
            for(int c = 0; c < 12; c++) acc += J[rr * 12 + c] * r[12 * body + c];
            z[12 * body + rr] = acc;
        }
    }
    if(s->mas) orc_mas_apply(s->mas, r + 3 * s->fem_offset, z + 3 * s->fem_offset);
}

static double dot(const double* a, const double* b, int n)
{
    double s = 0;
    for(int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* PCGSolver::solve + pcg (pcg_solver.cu:158-332).  max_iter = (SizeT)(ratio * n).
 * stop_rule 0: |r.z| <= tol * r0.z0 (the reference); 1: ||r||/||b|| <= tol.
 * budget_s > 0 bounds the iteration loop in wall time (CPU baseline sampling); *t_iter gets
 * the mean seconds per iteration and *done whether the stop rule (or max_iter) ended it. */
int orc_pcg_ex(const int* rows, const int* cols, const double* blocks, int nnzb, int n,
               const double* b, double* x, const orc_mas* mas, int fem_offset, int use_diag,
               int abd_bodies, const double* abd_inv, double tol, double max_iter_ratio,
               int stop_rule, double budget_s, orc_pcg_stats* st, double* t_iter, int* done);

int orc_pcg(const int* rows, const int* cols, const double* blocks, int nnzb, int n,
            const double* b, double* x, const orc_mas* mas, int fem_offset, int use_diag,
            int abd_bodies, const double* abd_inv, double tol, double max_iter_ratio,
            orc_pcg_stats* st)
{
    return orc_pcg_ex(rows, cols, blocks, nnzb, n, b, x, mas, fem_offset, use_diag, abd_bodies, abd_inv, tol,
                      max_iter_ratio, 0, 0.0, st, NULL, NULL);
}

int orc_pcg_ex(const int* rows, const int* cols, const double* blocks, int nnzb, int n,
               const double* b, double* x, const orc_mas* mas, int fem_offset, int use_diag,
               int abd_bodies, const double* abd_inv, double tol, double max_iter_ratio,
               int stop_rule, double budget_s, orc_pcg_stats* st, double* t_iter, int* done)
{
    orc_system s = {nnzb, rows, cols, blocks, n, use_diag, NULL, abd_bodies, abd_inv, mas, fem_offset};
    if(use_diag)
    {
        s.diag_inv = (double*)calloc((size_t)n / 3 * 9, sizeof(double));
        for(int k = 0; k < nnzb; k++)
            if(rows[k] == cols[k]) inv3(blocks + 9 * (size_t)k, s.diag_inv + 9 * (size_t)rows[k]);
    }
    double* r = (double*)malloc(sizeof(double) * n);
    double* z = (double*)malloc(sizeof(double) * n);
    double* p = (double*)malloc(sizeof(double) * n);
    double* Ap = (double*)malloc(sizeof(double) * n);
    long max_iter = (long)(max_iter_ratio * (double)n);
    for(int i = 0; i < n; i++) { x[i] = 0; r[i] = b[i]; }
    apply_preconditioner(&s, r, z);
    double rz = dot(r, z, n);
    memcpy(p, z, sizeof(double) * n);
    double rz0 = rz;
    const double bb = dot(b, b, n);
    long k;
    int finished = 0;
    double t0 = now_s();
    long counted = 0;
    for(k = 1; k < max_iter; ++k)
    {
        orc_spmv(1.0, nnzb, rows, cols, blocks, p, 0.0, Ap, n);
        double alpha = rz / dot(p, Ap, n);
        for(int i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * Ap[i]; }
        counted = k;
        if(stop_rule == 0 ? (fabs(rz) <= tol * rz0) : (dot(r, r, n) <= tol * tol * bb))
        {
            finished = 1;
            break;
        }
        if(budget_s > 0 && now_s() - t0 > budget_s) break;
        apply_preconditioner(&s, r, z);
        double rz_new = dot(r, z, n);
        double beta = rz_new / rz;
        for(int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz = rz_new;
    }
    if(k >= max_iter) finished = 1;
    if(t_iter) *t_iter = counted > 0 ? (now_s() - t0) / (double)counted : 0.0;
    if(done) *done = finished;
    if(st)
    {
        st->iterations = (int)k;
        st->rz0 = rz0;
        st->rz_final = rz;
        orc_spmv(1.0, nnzb, rows, cols, blocks, x, 0.0, Ap, n);
        double nr = 0, nb = 0;
        for(int i = 0; i < n; i++) { double d = b[i] - Ap[i]; nr += d * d; nb += b[i] * b[i]; }
        st->rel_residual = nb > 0 ? sqrt(nr / nb) : 0.0;
    }
    free(r); free(z); free(p); free(Ap); free(s.diag_inv);
    return (int)k;
}

/* ------------------------------------------------------------------------------------ */
/* Multithreaded timing variant (CPU baseline only)                                      */
/* ------------------------------------------------------------------------------------ */
/* The same MAS-PCG recurrence as orc_pcg_ex (stop rule 1: ||r|| <= tol ||b||), spread over
 * the host's threads with OpenMP: the SpMV on a full symmetric CSR copy built once (rows in
 * parallel), the bank solves of the MAS apply in parallel over banks, the prolongation over
 * vertices, and the vector updates and dot products over entries.  The restriction to the
 * coarse levels stays serial (it accumulates into shared coarse nodes).  Used to time the
 * reference algorithm on all host cores; the serial functions above are the checker. */
#include <omp.h>

typedef struct
{
    int n3;          /* block rows */
    int* ptr;        /* [n3 + 1] */
    int* col;
    double* val;     /* 9 per entry, column-major */
} orc_csr;

static void csr_build(orc_csr* A, int nnzb, const int* rows, const int* cols, const double* blocks, int n3)
{
    A->n3 = n3;
    A->ptr = (int*)calloc((size_t)n3 + 1, sizeof(int));
    for(int k = 0; k < nnzb; k++)
    {
        A->ptr[rows[k] + 1]++;
        if(rows[k] != cols[k]) A->ptr[cols[k] + 1]++;
    }
    for(int i = 0; i < n3; i++) A->ptr[i + 1] += A->ptr[i];
    const int nnz = A->ptr[n3];
    A->col = (int*)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    A->val = (double*)malloc(sizeof(double) * 9 * (size_t)(nnz > 0 ? nnz : 1));
    int* cur = (int*)malloc(sizeof(int) * (size_t)n3);
    memcpy(cur, A->ptr, sizeof(int) * (size_t)n3);
    for(int k = 0; k < nnzb; k++)
    {
        const int i = rows[k], j = cols[k];
        const double* H = blocks + 9 * (size_t)k;
        int e = cur[i]++;
        A->col[e] = j;
        memcpy(A->val + 9 * (size_t)e, H, 9 * sizeof(double));
        if(i != j)
        {
            e = cur[j]++;
            A->col[e] = i;
            for(int r = 0; r < 3; r++)
                for(int c = 0; c < 3; c++) A->val[9 * (size_t)e + c * 3 + r] = bget(H, c, r);  /* H^T */
        }
    }
    free(cur);
}

static void csr_spmv(const orc_csr* A, const double* x, double* y)
{
#pragma omp parallel for schedule(static)
    for(int i = 0; i < A->n3; i++)
    {
        double s0 = 0, s1 = 0, s2 = 0;
        for(int e = A->ptr[i]; e < A->ptr[i + 1]; e++)
        {
            const double* H = A->val + 9 * (size_t)e;
            const double* xj = x + 3 * (size_t)A->col[e];
            s0 += H[0] * xj[0] + H[3] * xj[1] + H[6] * xj[2];
            s1 += H[1] * xj[0] + H[4] * xj[1] + H[7] * xj[2];
            s2 += H[2] * xj[0] + H[5] * xj[1] + H[8] * xj[2];
        }
        y[3 * i] = s0;
        y[3 * i + 1] = s1;
        y[3 * i + 2] = s2;
    }
}

static void mas_apply_mt(const orc_mas* m, const double* r, double* z, float* R, float* Zc)
{
    const int B = m->bank, V = m->V, M = m->M, L = m->L, T = m->total_clusters;
    memset(R, 0, sizeof(float) * 3 * (size_t)T);
    for(int s = 0; s < M; s++)
    {
        int v = m->part_map[s];
        if(v < 0) continue;
        float rv[3] = {(float)r[3 * v], (float)r[3 * v + 1], (float)r[3 * v + 2]};
        for(int c = 0; c < 3; c++) R[3 * s + c] = rv[c];
        int id = v;
        for(int level = 1; level < L; level++)
        {
            id = m->going_next[id];
            for(int c = 0; c < 3; c++) R[3 * (size_t)id + c] += rv[c];
        }
    }
    const int NS = nsym(B);
#pragma omp parallel for schedule(static)
    for(int bk = 0; bk < T / B; bk++)
    {
        const float* P = m->inv + (size_t)bk * NS * 9;
        for(int a = 0; a < B; a++)
        {
            float acc[3] = {0, 0, 0};
            for(int c = 0; c < B; c++)
            {
                const float* rc = R + 3 * ((size_t)bk * B + c);
                if(c >= a)
                {
                    const float* Pb = P + (size_t)upper_index(B, a, c) * 9;
                    for(int i = 0; i < 3; i++) acc[i] += Pb[i] * rc[0] + Pb[3 + i] * rc[1] + Pb[6 + i] * rc[2];
                }
                else
                {
                    const float* Pb = P + (size_t)upper_index(B, c, a) * 9;
                    for(int i = 0; i < 3; i++) acc[i] += Pb[i * 3] * rc[0] + Pb[i * 3 + 1] * rc[1] + Pb[i * 3 + 2] * rc[2];
                }
            }
            for(int i = 0; i < 3; i++) Zc[3 * ((size_t)bk * B + a) + i] = acc[i];
        }
    }
#pragma omp parallel for schedule(static)
    for(int v = 0; v < V; v++)
    {
        int s = m->real_map[v];
        float cz[3] = {Zc[3 * (size_t)s], Zc[3 * (size_t)s + 1], Zc[3 * (size_t)s + 2]};
        for(int l = 1; l < L; l++)
        {
            int now = m->coarse_table[(size_t)v * (L - 1) + l - 1];
            for(int c = 0; c < 3; c++) cz[c] += Zc[3 * (size_t)now + c];
        }
        for(int c = 0; c < 3; c++) z[3 * v + c] = (double)cz[c];
    }
}

static double dot_mt(const double* a, const double* b, int n)
{
    double s = 0;
#pragma omp parallel for schedule(static) reduction(+ : s)
    for(int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

/* MAS-PCG (FEM-only system, MAS over the whole range) with all host threads; returns the
 * iterations, *t_setup the seconds of the CSR build, *t_iter the seconds per iteration,
 * *threads the OpenMP thread count, *rel the last ||r|| / ||b||.  The loop stops at ||r|| <= tol ||b||, max_iter or
 * after budget_s seconds (*done = 0). */
int orc_pcg_mt(const int* rows, const int* cols, const double* blocks, int nnzb, int n, const double* b, double* x,
               const orc_mas* mas, double tol, double max_iter_ratio, double budget_s, double* t_setup,
               double* t_iter, int* done, int* threads, double* rel)
{
    const double ts = now_s();
    orc_csr A;
    csr_build(&A, nnzb, rows, cols, blocks, n / 3);
    *t_setup = now_s() - ts;
    *threads = omp_get_max_threads();
    double* r = (double*)malloc(sizeof(double) * n);
    double* z = (double*)malloc(sizeof(double) * n);
    double* p = (double*)malloc(sizeof(double) * n);
    double* Ap = (double*)malloc(sizeof(double) * n);
    float* R = (float*)malloc(sizeof(float) * 3 * (size_t)mas->total_clusters);
    float* Zc = (float*)malloc(sizeof(float) * 3 * (size_t)mas->total_clusters);
    const long max_iter = (long)(max_iter_ratio * (double)n);
#pragma omp parallel for schedule(static)
    for(int i = 0; i < n; i++)
    {
        x[i] = 0;
        r[i] = b[i];
    }
    mas_apply_mt(mas, r, z, R, Zc);
    double rz = dot_mt(r, z, n);
    memcpy(p, z, sizeof(double) * n);
    const double bb = dot_mt(b, b, n);
    const double t0 = now_s();
    long k, counted = 0;
    int finished = 0;
    for(k = 1; k < max_iter; ++k)
    {
        csr_spmv(&A, p, Ap);
        const double alpha = rz / dot_mt(p, Ap, n);
#pragma omp parallel for schedule(static)
        for(int i = 0; i < n; i++)
        {
            x[i] += alpha * p[i];
            r[i] -= alpha * Ap[i];
        }
        counted = k;
        const double rr = dot_mt(r, r, n);
        *rel = bb > 0 ? sqrt(rr / bb) : 0.0;
        if(rr <= tol * tol * bb)
        {
            finished = 1;
            break;
        }
        if(budget_s > 0 && now_s() - t0 > budget_s) break;
        mas_apply_mt(mas, r, z, R, Zc);
        const double rz_new = dot_mt(r, z, n);
        const double beta = rz_new / rz;
#pragma omp parallel for schedule(static)
        for(int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz = rz_new;
    }
    if(k >= max_iter) finished = 1;
    *t_iter = counted > 0 ? (now_s() - t0) / (double)counted : 0.0;
    *done = finished;
    free(r); free(z); free(p); free(Ap); free(R); free(Zc);
    free(A.ptr); free(A.col); free(A.val);
    return (int)k;
}

/* Block-Jacobi CG on all host threads, for the CPU baseline the metric names (Eigen's
 * ConjugateGradient with a 3x3 block-Jacobi preconditioner, restated without Eigen): the
 * same CSR product as orc_pcg_mt, z = D_i^-1 r_i with the inverses of the diagonal blocks,
 * stop at ||r|| <= tol ||b||, max_iter or after budget_s seconds (*done = 0).  Returns the
 * iterations; *t_setup covers the CSR build and the block inverses. */
int orc_cg_bj_mt(const int* rows, const int* cols, const double* blocks, int nnzb, int n, const double* b, double* x,
                 double tol, double max_iter_ratio, double budget_s, double* t_setup, double* t_iter, int* done,
                 int* threads, double* rel)
{
    const double ts = now_s();
    orc_csr A;
    csr_build(&A, nnzb, rows, cols, blocks, n / 3);
    const int nb = n / 3;
    double* Dinv = (double*)calloc((size_t)nb * 9, sizeof(double));
#pragma omp parallel for schedule(static)
    for(int i = 0; i < nb; i++)
    {
        double D[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  /* column-major diagonal block */
        for(int e = A.ptr[i]; e < A.ptr[i + 1]; e++)
            if(A.col[e] == i)
                for(int q = 0; q < 9; q++) D[q] += A.val[9 * (size_t)e + q];
        /* inverse of a 3x3 by cofactors (column-major in and out) */
        const double a = D[0], bq = D[3], c = D[6], d = D[1], ee = D[4], f = D[7], g = D[2], h = D[5], k = D[8];
        const double det = a * (ee * k - f * h) - bq * (d * k - f * g) + c * (d * h - ee * g);
        double* O = Dinv + 9 * (size_t)i;
        if(det != 0.0)
        {
            const double id = 1.0 / det;
            O[0] = (ee * k - f * h) * id;
            O[3] = (c * h - bq * k) * id;
            O[6] = (bq * f - c * ee) * id;
            O[1] = (f * g - d * k) * id;
            O[4] = (a * k - c * g) * id;
            O[7] = (c * d - a * f) * id;
            O[2] = (d * h - ee * g) * id;
            O[5] = (bq * g - a * h) * id;
            O[8] = (a * ee - bq * d) * id;
        }
        else
            O[0] = O[4] = O[8] = 1.0;
    }
    *t_setup = now_s() - ts;
    *threads = omp_get_max_threads();
    double* r = (double*)malloc(sizeof(double) * n);
    double* z = (double*)malloc(sizeof(double) * n);
    double* p = (double*)malloc(sizeof(double) * n);
    double* Ap = (double*)malloc(sizeof(double) * n);
    const long max_iter = (long)(max_iter_ratio * (double)n);
#pragma omp parallel for schedule(static)
    for(int i = 0; i < n; i++)
    {
        x[i] = 0;
        r[i] = b[i];
    }
#define BJ_APPLY()                                                                         \
    do                                                                                     \
    {                                                                                      \
        _Pragma("omp parallel for schedule(static)") for(int i = 0; i < nb; i++)           \
        {                                                                                  \
            const double* O = Dinv + 9 * (size_t)i;                                        \
            const double* ri = r + 3 * (size_t)i;                                          \
            for(int q = 0; q < 3; q++) z[3 * i + q] = O[q] * ri[0] + O[3 + q] * ri[1] + O[6 + q] * ri[2]; \
        }                                                                                  \
    } while(0)
    BJ_APPLY();
    double rz = dot_mt(r, z, n);
    memcpy(p, z, sizeof(double) * n);
    const double bb = dot_mt(b, b, n);
    const double t0 = now_s();
    long k, counted = 0;
    int finished = 0;
    for(k = 1; k < max_iter; ++k)
    {
        csr_spmv(&A, p, Ap);
        const double alpha = rz / dot_mt(p, Ap, n);
#pragma omp parallel for schedule(static)
        for(int i = 0; i < n; i++)
        {
            x[i] += alpha * p[i];
            r[i] -= alpha * Ap[i];
        }
        counted = k;
        const double rr = dot_mt(r, r, n);
        *rel = bb > 0 ? sqrt(rr / bb) : 0.0;
        if(rr <= tol * tol * bb)
        {
            finished = 1;
            break;
        }
        if(budget_s > 0 && now_s() - t0 > budget_s) break;
        BJ_APPLY();
        const double rz_new = dot_mt(r, z, n);
        const double beta = rz_new / rz;
#pragma omp parallel for schedule(static)
        for(int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz = rz_new;
    }
#undef BJ_APPLY
    if(k >= max_iter) finished = 1;
    *t_iter = counted > 0 ? (now_s() - t0) / (double)counted : 0.0;
    *done = finished;
    free(r); free(z); free(p); free(Ap); free(Dinv);
    free(A.ptr); free(A.col); free(A.val);
    return (int)k;
}

/* ---- contact barrier Hessians ----------------------------------------------------------
 * Restates _calBarrierGradientAndHessian (StiffGIPC/GIPC.cu:3149-4988, NEWF and RANK 2) for
 * the unmollified pair encodings: E(s) = kappa dHat^2 (s^2 - 1)^2 ln^2(s^2), s = d / sqrt(dHat),
 * gradient E'(s) ds/dx (flatten_pk1, GIPC.cu:3258-3262), Hessian lambda0 ds/dx ds/dx^T with
 * lambda0 = E''(s) (GIPC.cu:3310-3327), frozen at s^2 = 1e-6 below it.  ds/dx is written here
 * in closed form from the squared distances of mlbvh.cu:229-257 (the reference's PFPx last
 * column, GIPC_PDerivative.cuh, is the same derivative generated symbolically).  The output
 * layout is 10 upper 3x3 blocks per pair (SymGH order, GIPC.cu:117-175) plus 12 gradient
 * entries; unused slots hold a zero block on the first vertex's diagonal.  Returns the number
 * of pairs skipped (mollified encodings, out-of-range or repeated vertices). */
static void v3sub(const double* a, const double* b, double* r) { r[0] = a[0] - b[0], r[1] = a[1] - b[1], r[2] = a[2] - b[2]; }
static double v3dot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void v3cross(const double* a, const double* b, double* r)
{
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}

/* d^2 and its gradient (12 entries, 3 per local vertex) for type 0 PP, 1 PE, 2 PT, 3 EE */
static double contact_d2(int type, const double* v, double* g)
{
    const double *p0 = v, *p1 = v + 3, *p2 = v + 6, *p3 = v + 9;
    memset(g, 0, 12 * sizeof(double));
    if(type == 0)
    {
        double r[3];
        v3sub(p0, p1, r);
        for(int k = 0; k < 3; k++) g[k] = 2 * r[k], g[3 + k] = -2 * r[k];
        return v3dot(r, r);
    }
    if(type == 1)
    {
        /* d^2 = |c|^2 / |e|^2, c = (p1 - p0) x (p2 - p0), e = p2 - p1 */
        double a[3], b[3], c[3], e[3], bc[3], ca[3];
        v3sub(p1, p0, a), v3sub(p2, p0, b), v3sub(p2, p1, e), v3cross(a, b, c);
        v3cross(b, c, bc), v3cross(c, a, ca);
        const double C2 = v3dot(c, c), E2 = v3dot(e, e), d2 = C2 / E2;
        for(int k = 0; k < 3; k++)
        {
            const double ga = 2 * bc[k], gb = 2 * ca[k]; /* d|c|^2 / da, d|c|^2 / db */
            g[3 + k] = (ga + d2 * 2 * e[k]) / E2;
            g[6 + k] = (gb - d2 * 2 * e[k]) / E2;
            g[k] = -(ga + gb) / E2;
        }
        return d2;
    }
    /* PT: b = (p2 - p1) x (p3 - p1), r = p0 - p1, u = p2 - p1, w = p3 - p1, moving (r, u, w);
     * EE: b = (p1 - p0) x (p3 - p2), r = p2 - p0, u = p1 - p0, w = p3 - p2.
     * d^2 = A^2 / |b|^2 with A = r . b */
    double r[3], u[3], w[3], b[3], wr[3], ru[3], wb[3], bu[3];
    if(type == 2)
        v3sub(p0, p1, r), v3sub(p2, p1, u), v3sub(p3, p1, w);
    else
        v3sub(p2, p0, r), v3sub(p1, p0, u), v3sub(p3, p2, w);
    v3cross(u, w, b), v3cross(w, r, wr), v3cross(r, u, ru), v3cross(w, b, wb), v3cross(b, u, bu);
    const double A = v3dot(r, b), B2 = v3dot(b, b), d2 = A * A / B2;
    for(int k = 0; k < 3; k++)
    {
        /* d(d^2) = (2 A dA - d^2 d|b|^2) / |b|^2; dA/dr = b, dA/du = w x r, dA/dw = r x u;
         * d|b|^2/du = 2 w x b, d|b|^2/dw = 2 b x u */
        const double gr = 2 * A * b[k] / B2;
        const double gu = (2 * A * wr[k] - d2 * 2 * wb[k]) / B2;
        const double gw = (2 * A * ru[k] - d2 * 2 * bu[k]) / B2;
        if(type == 2)
            g[k] = gr, g[6 + k] = gu, g[9 + k] = gw, g[3 + k] = -(gr + gu + gw);
        else
            g[k] = -(gr + gu), g[3 + k] = gu, g[6 + k] = gr - gw, g[9 + k] = gw;
    }
    return d2;
}

int orc_contact_barrier(int ncp, const int32_t* pairs, const double* x, int nv, int block_offset, double dhat,
                        double kappa, int32_t* rows, int32_t* cols, double* blocks, double* grad)
{
    int skipped = 0;
    for(int p = 0; p < ncp; p++)
    {
        const int32_t* q = pairs + 4 * (size_t)p;
        int vid[4] = {0, 0, 0, 0}, cnt = 0, type = -1;
        if(q[0] >= 0)
        {
            if(q[3] >= 0) type = 3, vid[0] = q[0], vid[1] = q[1], vid[2] = q[2], vid[3] = q[3], cnt = 4;
        }
        else if(q[1] >= 0)
        {
            vid[0] = -q[0] - 1, vid[1] = q[1];
            if(q[2] < 0)
                type = 0, cnt = 2;
            else if(q[3] < 0)
                type = 1, vid[2] = q[2], cnt = 3;
            else
                type = 2, vid[2] = q[2], vid[3] = q[3], cnt = 4;
        }
        int ok = type >= 0;
        for(int i = 0; i < cnt; i++) ok = ok && vid[i] >= 0 && vid[i] < nv;
        for(int i = 0; i < cnt; i++)
            for(int j = i + 1; j < cnt; j++) ok = ok && vid[i] != vid[j];
        double h[12] = {0}, lam = 0, e1 = 0;
        if(ok)
        {
            double v[12] = {0}, g2[12];
            for(int i = 0; i < cnt; i++) memcpy(v + 3 * i, x + 3 * (size_t)vid[i], 3 * sizeof(double));
            const double d2 = contact_d2(type, v, g2), d = sqrt(d2), s = d / sqrt(dhat);
            if(s > 0 && s < 1)
            {
                const double I = s * s, lI = log(I), D2 = dhat * dhat;
                e1 = s * 2 * (2 * kappa * D2 * lI * (I - 1) * (I + I * lI - 1)) / I;
                const double Ic = I < 1e-6 ? 1e-6 : I, l = log(Ic);
                lam = -(4 * kappa * D2 *
                        (4 * Ic + l - 3 * Ic * Ic * l * l + 6 * Ic * l - 2 * Ic * Ic + Ic * l * l - 7 * Ic * Ic * l - 2)) /
                      Ic;
                for(int k = 0; k < 12; k++) h[k] = g2[k] / (2 * d) / sqrt(dhat);
            }
        }
        else
            skipped++;
        for(int k = 0; k < 12; k++) grad[12 * (size_t)p + k] = e1 * h[k];
        int slot = 0;
        for(int i = 0; i < 4; i++)
            for(int j = i; j < 4; j++, slot++)
            {
                const size_t o = 10 * (size_t)p + slot;
                double* B = blocks + 9 * o;
                if(!ok || i >= cnt || j >= cnt)
                {
                    rows[o] = cols[o] = block_offset + (ok ? vid[0] : 0);
                    memset(B, 0, 9 * sizeof(double));
                    continue;
                }
                const int gi = vid[i], gj = vid[j], sw = gi > gj;
                rows[o] = block_offset + (sw ? gj : gi);
                cols[o] = block_offset + (sw ? gi : gj);
                for(int a = 0; a < 3; a++)
                    for(int b = 0; b < 3; b++)
                    {
                        const double val = lam * h[3 * i + a] * h[3 * j + b];
                        B[sw ? a * 3 + b : b * 3 + a] = val;
                    }
            }
    }
    return skipped;
}

/* d^2 of one pair of type 0 PP, 1 PE, 2 PT, 3 EE and its gradient g[12] (test access) */
double orc_contact_d2(int type, const double* v, double* g) { return contact_d2(type, v, g); }

/* ---- additive CCD (line-search step bound) ----------------------------------------------
 * Restates the reference's conservative-advancement CCD (StiffGIPC/ACCD.cu:15-262 distance
 * classification, :264-371 unclassified squared distances, :373-534 edge_edge_ccd /
 * point_triangle_ccd) and the step bound of GIPC::self_largestFeasibleStepSize
 * (GIPC.cu:7095-7180, 9010-9047): per pair the time of impact toc along the displacement,
 * eta = 1 - slackness, thickness 0 in the reference's call; alpha = 1 / max(1 / toc).
 * Every expression keeps the operand order of the reference's vector helpers
 * (gpu_eigen_libs.cu: dot and squared norm summed x, y, z; the 3x3 determinant as a sum of six
 * triple products), so that the device restatement (ccd.cu, compiled without FMA contraction)
 * can be compared bit for bit. */
typedef struct { double x, y, z; } cv3;
static cv3 c3(double x, double y, double z) { cv3 r = {x, y, z}; return r; }
static cv3 c3sub(cv3 a, cv3 b) { return c3(a.x - b.x, a.y - b.y, a.z - b.z); }
static cv3 c3add(cv3 a, cv3 b) { return c3(a.x + b.x, a.y + b.y, a.z + b.z); }
static cv3 c3mul(cv3 a, double s) { return c3(a.x * s, a.y * s, a.z * s); }
static double c3dot(cv3 a, cv3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static double c3sq(cv3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static cv3 c3cross(cv3 a, cv3 b) { return c3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
/* det of the matrix with columns (c0, c1, c2) given row-wise as m[r][k] = ck.r */
static double cdet(const double m[3][3])
{
    return m[0][0] * m[1][1] * m[2][2] + m[1][0] * m[2][1] * m[0][2] + m[2][0] * m[0][1] * m[1][2] -
           m[2][0] * m[1][1] * m[0][2] - m[0][0] * m[1][2] * m[2][1] - m[0][1] * m[1][0] * m[2][2];
}
static void cset(double m[3][3], cv3 a, cv3 b, cv3 c)
{
    m[0][0] = a.x, m[0][1] = b.x, m[0][2] = c.x;
    m[1][0] = a.y, m[1][1] = b.y, m[1][2] = c.y;
    m[2][0] = a.z, m[2][1] = b.z, m[2][2] = c.z;
}
/* barycentric-like parameters of p against edge (a, b) of a triangle with normal n */
static void pt_param(cv3 p, cv3 a, cv3 b, cv3 n, double* px, double* py)
{
    const cv3 b0 = c3sub(b, a), b1 = c3cross(b0, n), b2 = c3sub(p, a);
    double D[3][3], D1[3][3], D2[3][3];
    cset(D, b0, b1, n), cset(D1, b2, b1, n), cset(D2, b0, b2, n);
    *px = cdet(D1) / cdet(D);
    *py = cdet(D2) / cdet(D);
}
/* 0..2 vertex t_k, 3..5 edges (t0 t1), (t1 t2), (t2 t0), 6 interior */
static int pt_type(cv3 p, cv3 t0, cv3 t1, cv3 t2)
{
    const cv3 n = c3cross(c3sub(t1, t0), c3sub(t2, t0));
    double x0, y0, x1, y1, x2, y2;
    pt_param(p, t0, t1, n, &x0, &y0);
    if(x0 > 0 && x0 < 1 && y0 >= 0) return 3;
    pt_param(p, t1, t2, n, &x1, &y1);
    if(x1 > 0.0 && x1 < 1.0 && y1 >= 0.0) return 4;
    pt_param(p, t2, t0, n, &x2, &y2);
    if(x2 > 0.0 && x2 < 1.0 && y2 >= 0.0) return 5;
    if(x0 <= 0.0 && x2 >= 1.0) return 0;
    if(x1 <= 0.0 && x0 >= 1.0) return 1;
    if(x2 <= 0.0 && x1 >= 1.0) return 2;
    return 6;
}
/* 0..8: (a0 b0) (a0 b1) (a0 | b) (a1 b0) (a1 b1) (a1 | b) (b0 | a) (b1 | a) (a | b) */
static int ee_type(cv3 v0, cv3 v1, cv3 v2, cv3 v3)
{
    const cv3 u = c3sub(v1, v0), v = c3sub(v3, v2), w = c3sub(v0, v2);
    const double a = c3sq(u), b = c3dot(u, v), c = c3sq(v), d = c3dot(u, w), e = c3dot(v, w);
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
        if(tN > 0.0 && tN < tD && (c3dot(w, c3cross(u, v)) == 0.0 || c3sq(c3cross(u, v)) < 1.0e-20 * a * c))
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
static double d_pp(cv3 a, cv3 b) { return c3sq(c3sub(a, b)); }
static double d_pe(cv3 p, cv3 e0, cv3 e1) { return c3sq(c3cross(c3sub(e0, p), c3sub(e1, p))) / c3sq(c3sub(e1, e0)); }
static double d_pt(cv3 p, cv3 t0, cv3 t1, cv3 t2)
{
    const cv3 b = c3cross(c3sub(t1, t0), c3sub(t2, t0));
    const double aTb = c3dot(c3sub(p, t0), b);
    return aTb * aTb / c3sq(b);
}
static double d_ee(cv3 a0, cv3 a1, cv3 b0, cv3 b1)
{
    const cv3 b = c3cross(c3sub(a1, a0), c3sub(b1, b0));
    const double aTb = c3dot(c3sub(b0, a0), b);
    return aTb * aTb / c3sq(b);
}
static double ee_dist2(cv3 a0, cv3 a1, cv3 b0, cv3 b1)
{
    switch(ee_type(a0, a1, b0, b1))
    {
        case 0: return d_pp(a0, b0);
        case 1: return d_pp(a0, b1);
        case 2: return d_pe(a0, b0, b1);
        case 3: return d_pp(a1, b0);
        case 4: return d_pp(a1, b1);
        case 5: return d_pe(a1, b0, b1);
        case 6: return d_pe(b0, a0, a1);
        case 7: return d_pe(b1, a0, a1);
        default: return d_ee(a0, a1, b0, b1);
    }
}
static double pt_dist2(cv3 p, cv3 t0, cv3 t1, cv3 t2)
{
    switch(pt_type(p, t0, t1, t2))
    {
        case 0: return d_pp(p, t0);
        case 1: return d_pp(p, t1);
        case 2: return d_pp(p, t2);
        case 3: return d_pe(p, t0, t1);
        case 4: return d_pe(p, t1, t2);
        case 5: return d_pe(p, t2, t0);
        default: return d_pt(p, t0, t1, t2);
    }
}
static double ee_floor(cv3 a0, cv3 a1, cv3 b0, cv3 b1)
{
    const double s0 = c3sq(c3sub(a0, b0)), s1 = c3sq(c3sub(a0, b1)), s2 = c3sq(c3sub(a1, b0)),
                 s3 = c3sq(c3sub(a1, b1));
    return fmin(fmin(s0, s1), fmin(s2, s3));
}

/* time of impact of points x[0..3] moving by dx[0..3]: type 0 point-triangle (p, t0, t1, t2),
 * 1 edge-edge (a0, a1, b0, b1) */
double orc_accd(int type, const double* x, const double* dx, double eta, double thickness)
{
    cv3 v[4], d[4];
    for(int i = 0; i < 4; i++) v[i] = c3(x[3 * i], x[3 * i + 1], x[3 * i + 2]), d[i] = c3(dx[3 * i], dx[3 * i + 1], dx[3 * i + 2]);
    const double th2 = thickness * thickness;
    if(type == 1)
    {
        const cv3 mov = c3mul(c3add(c3add(d[0], d[1]), c3add(d[2], d[3])), -0.25);
        for(int i = 0; i < 4; i++) d[i] = c3add(d[i], mov);
        const double mdm = sqrt(fmax(c3sq(d[0]), c3sq(d[1]))) + sqrt(fmax(c3sq(d[2]), c3sq(d[3])));
        if(mdm == 0) return 1.0;
        double dist2 = ee_dist2(v[0], v[1], v[2], v[3]);
        double dF = dist2 - th2;
        if(dF <= 0)
        {
            dist2 = ee_floor(v[0], v[1], v[2], v[3]);
            dF = dist2 - th2;
        }
        double dist = sqrt(dist2);
        const double gap = eta * dF / (dist + thickness);
        double toc = 0.0;
        for(int count = 1;; count++)
        {
            if(count > 50000) return toc;
            const double lb = (1 - eta) * dF / ((dist + thickness) * mdm);
            for(int i = 0; i < 4; i++) v[i] = c3add(v[i], c3mul(d[i], lb));
            dist2 = ee_dist2(v[0], v[1], v[2], v[3]);
            dF = dist2 - th2;
            if(dF <= 0)
            {
                dist2 = ee_floor(v[0], v[1], v[2], v[3]);
                dF = dist2 - th2;
            }
            dist = sqrt(dist2);
            if(toc != 0.0 && (dF / (dist + thickness) < gap)) break;
            toc += lb;
            if(toc > 1.0) return 1.0;
        }
        return toc;
    }
    const cv3 mov = c3mul(c3add(c3add(d[1], d[2]), c3add(d[3], d[0])), -0.25);
    for(int i = 0; i < 4; i++) d[i] = c3add(d[i], mov);
    const double mdm = sqrt(c3sq(d[0])) + sqrt(fmax(c3sq(d[1]), fmax(c3sq(d[2]), c3sq(d[3]))));
    if(mdm == 0) return 1.0;
    double dist2 = pt_dist2(v[0], v[1], v[2], v[3]);
    double dist = sqrt(dist2);
    const double gap = eta * (dist2 - th2) / (dist + thickness);
    double toc = 0.0;
    for(int count = 1;; count++)
    {
        if(count > 50000) return toc;
        const double lb = (1 - eta) * (dist2 - th2) / ((dist + thickness) * mdm);
        for(int i = 0; i < 4; i++) v[i] = c3add(v[i], c3mul(d[i], lb));
        dist2 = pt_dist2(v[0], v[1], v[2], v[3]);
        dist = sqrt(dist2);
        if(toc != 0.0 && ((dist2 - th2) / (dist + thickness) < gap)) break;
        toc += lb;
        if(toc > 1.0) return 1.0;
    }
    return toc;
}

/* the largest feasible step of displacement dx for the CCD pairs (x < 0: point -x-1 and
 * triangle (y, z, w); else edges (x, y), (z, w)): 1 / max over pairs of 1 / toc, or 1 */
double orc_ccd_step_size(int npairs, const int32_t* pairs, const double* x, const double* dx, double slackness)
{
    if(npairs < 1) return 1.0;
    double mx = 0.0;
    for(int p = 0; p < npairs; p++)
    {
        const int32_t* q = pairs + 4 * (size_t)p;
        const int id[4] = {q[0] < 0 ? -q[0] - 1 : q[0], q[1], q[2], q[3]};
        double xs[12], ds[12];
        for(int i = 0; i < 4; i++)
            for(int k = 0; k < 3; k++) xs[3 * i + k] = x[3 * (size_t)id[i] + k], ds[3 * i + k] = dx[3 * (size_t)id[i] + k];
        const double t = 1.0 / orc_accd(q[0] < 0 ? 0 : 1, xs, ds, 1.0 - slackness, 0.0);
        if(!(t <= mx)) mx = t;
    }
    return 1.0 / mx;
}

/* the barrier energy of each pair (kappa dhat^2 (s^2 - 1)^2 ln^2(s^2), s^2 = d^2 / dhat < 1) */
void orc_contact_energy(int ncp, const int32_t* pairs, const double* x, int nv, double dhat, double kappa,
                        double* energy)
{
    for(int p = 0; p < ncp; p++)
    {
        const int32_t* q = pairs + 4 * (size_t)p;
        int vid[4] = {0, 0, 0, 0}, cnt = 0, type = -1;
        if(q[0] >= 0)
        {
            if(q[3] >= 0) type = 3, vid[0] = q[0], vid[1] = q[1], vid[2] = q[2], vid[3] = q[3], cnt = 4;
        }
        else if(q[1] >= 0)
        {
            vid[0] = -q[0] - 1, vid[1] = q[1];
            if(q[2] < 0)
                type = 0, cnt = 2;
            else if(q[3] < 0)
                type = 1, vid[2] = q[2], cnt = 3;
            else
                type = 2, vid[2] = q[2], vid[3] = q[3], cnt = 4;
        }
        int ok = type >= 0;
        for(int i = 0; i < cnt; i++) ok = ok && vid[i] >= 0 && vid[i] < nv;
        for(int i = 0; i < cnt; i++)
            for(int j = i + 1; j < cnt; j++) ok = ok && vid[i] != vid[j];
        double e = 0.0;
        if(ok)
        {
            double v[12] = {0}, g[12];
            for(int i = 0; i < cnt; i++) memcpy(v + 3 * i, x + 3 * (size_t)vid[i], 3 * sizeof(double));
            const double I = contact_d2(type, v, g) / dhat;
            if(I < 1.0)
            {
                const double l = log(I);
                e = kappa * dhat * dhat * (I - 1.0) * (I - 1.0) * l * l;
            }
        }
        energy[p] = e;
    }
}
