// solver.hpp -- internal state of one libstgipc handle.
//
// A handle mirrors the reference's GlobalLinearSystem (global_linear_system.h:15-113)
// holding one IterativeSolver (PCGSolver, pcg_solver.h:19-52), the MAS preconditioner
// (MASPreconditioner.cuh) and the converted BCOO, all on one CUDA stream.
#pragma once
#include "common.cuh"
#include "pcg_dev.cuh"
#include "learned.cuh"
#include "../../include/stgipc.h"

#include <algorithm>

namespace stg
{

constexpr int kMaxLevels = 6;
constexpr int kSMs = 148;

// Sorted unique upper BCOO plus the derived row / transpose structure the SpMV uses.
struct Bcoo
{
    int nnzb = 0;
    int nrows = 0;
    bool external = false;       // blocks/rows/cols point at caller memory
    bool row_ptr_valid = false;
    const double* ext_blocks = nullptr;
    const int* ext_rows = nullptr;
    const int* ext_cols = nullptr;
    DBuf<int> rows, cols;        // owned copies (converter output)
    DBuf<double> blocks;
    DBuf<int> row_ptr;           // [nrows+1]
    // transpose references: for block row i, the strictly-upper blocks k with col(k) == i,
    // stored as (k, row(k)) pairs sorted by k
    DBuf<int> t_ptr;             // [nrows+1]
    DBuf<int> t_cnt;             // [nrows+1]
    DBuf<int2> t_ent;            // [offdiag]
    DBuf<double> blk64p;         // FP64 blocks padded to 80 B (5 x double2), residual replacement
    // full symmetric row-sliced copy for the PCG SpMV in 16-byte planes (FullPlanes in
    // spmv_core.cuh, built by k_build_full in pcg.cu)
    DBuf<unsigned char> fent;
    DBuf<int> frow;              // [nrows+1] first entry of each row (row_ptr + t_ptr)
    size_t fstride = 0;          // entries per plane
    // per-tile operand windows of the halo SpMV phase (k_tile_halo / k_phase_a_halo in pcg.cu)
    DBuf<unsigned char> htail;   // {h8, slot} plane replacing {h8, col}
    DBuf<int> hcnt, hlist;       // [tiles], [tiles * HCAP] halo columns, sorted
    bool halo_ok = false;        // every tile fits a stage
    // upper copy for the upper SpMV phase (UpperPlanes in spmv_core.cuh, k_build_upper)
    DBuf<unsigned char> uent;
    DBuf<int> urow;              // [nrows+1] row_ptr, padded for the tiles' row-bound copies
    size_t ustride = 0;          // entries per plane
    bool upper_built = false;    // built for the current matrix
    DBuf<double> diag_inv;       // 3x3 block-Jacobi inverses [nrows*9]
    int offdiag = 0;

    const double* B() const { return external ? ext_blocks : blocks.data(); }
    const int* R() const { return external ? ext_rows : rows.data(); }
    const int* C() const { return external ? ext_cols : cols.data(); }
};

// The fine convert's fused level-0 pass (stg_solve_linear_system with MAS): every unique block
// in the FEM range [offset, offset + V) is also written into its level-0 bank matrix (same
// bank, upper) and, when c1 is given, turned into its level-1 Galerkin triplet at its own
// index (row -1 where it is masked), as k_mas_store_l0 and k_mas_agg_l0 would from the BCOO.
struct ConvFuse
{
    int B = 0, NS = 0, offset = 0, V = 0;
    const int* real_map = nullptr;
    const int* c1 = nullptr;
    double* mat = nullptr;
    int* trow = nullptr;
    int* tcol = nullptr;
    double* tblk = nullptr;
};

struct ConvertScratch
{
    DBuf<int> row_cnt, row_start, cursor, perm, perm2, pcol, scol, uniq, scratch, long_rows;
};

struct MasState
{
    bool inited = false, built = false, assembled = false;
    bool l0_fused = false;        // the last convert wrote level 0 and the level-1 triplets
    int l0_offset = 0;            // ... for this FEM block offset
    bool identity = false;        // part_map[s] == s for s < V (Morton order): no slot indirection
    int bank = 16, V = 0, M = 0, L = 0, node_offset = 0, nlist_size = 0;
    int total_clusters = 0, nbanks = 0, nb0 = 0;
    int level_size[2 * (kMaxLevels + 1)] = {};
    int gn_size = 0;
    DBuf<unsigned> nstart, nnum_init, nlist_init, nnum, nlist;
    DBuf<int> part_map, real_map;
    DBuf<unsigned> fine_mask, next_mask;
    DBuf<unsigned> closed;        // closed masks of coarse nodes, by global id
    DBuf<int> prefix_orig, prefix_sum_orig;
    DBuf<int> next_prefix, next_prefix_sum;
    DBuf<int> coarse_tables;      // [L*V]
    DBuf<int> going_next;         // [L*V + M]
    DBuf<int> coarse_table;       // [V*(L-1)]
    DBuf<int2> level_size_d;      // [kMaxLevels+1]
    DBuf<int> scratch;
    DBuf<double> mat;             // [nbanks * NS * 9]
    DBuf<float> inv;              // [nbanks * NS * 9]
    DBuf<float> R, Z;             // [total_clusters * 4], float4 per node
    // Galerkin assembly: coarse triplets and the current / next level operator (upper BCOO)
    ConvertScratch gcv;
    DBuf<int> tr_rows, tr_cols, ga_rows, ga_cols, gb_rows, gb_cols, g_rowptr;
    DBuf<double> tr_blocks, ga_blocks, gb_blocks;
};

struct PcgState
{
    DBuf<double> r;                // FP64 residual
    DBuf<double> vbuf;             // zp0, zp1, q slots in the iteration precision
    DBuf<double> q;                // scratch for the true residual
    DBuf<double> partials;         // per-block partial sums, 6 sites
    DBuf<double> scal;             // device scalars, see enum below
    DBuf<unsigned> counters;       // last-block counters
    DBuf<int> flags;               // [0] done, [1] status, [2] replacements
    DBuf<unsigned> bar;            // persistent grid barrier
    DBuf<unsigned char> flush;     // 256 MiB written between timed SpMV launches (L2 flush)
    DBuf<double> abd_inv;          // ABD 12x12 block-Jacobi built from the BCOO [bodies * 144]
    DBuf<double> spill;            // transposed products of the upper SpMV phase (4 T per slot)
    cudaGraphExec_t graph = nullptr;
    PcgDev graph_key{};            // parameter block of the captured graph (handles zeroed)
    PcgDev graph_dev{};            // the same with the graph's conditional handles
    int graph_variant = 0;         // element size * 1000 + bank size of the captured kernels
};

// device scalar slots
enum : int
{
    S_RZ = 0,      // current r.z
    S_RZ0 = 1,     // r0.z0
    S_PQ = 2,      // p.Aq
    S_ALPHA = 3,
    S_BETA = 4,
    S_RZNEW = 5,
    S_RR = 6,      // r.r
    S_BB = 7,      // b.b
    S_TOL = 8,     // stop threshold
    S_ITER = 9,    // completed iterations (as double)
    S_LRR = 10,    // true r.r at the last residual replacement (learned correction judge)
    S_COUNT = 16
};

// The learned coarse correction of one handle: its level, parameters, the level's graph
// (rebuilt by every MAS assembly), the in-loop forward buffers, and the sample recorder.
struct LearnedState
{
    int level = 0;                 // coarse level of the network; 0: not configured
    bool has_params = false;
    bool graph_ready = false;      // graph built from the current assembly
    int begin = 0;                 // first node of the level in R / Z
    DBuf<float> params;            // [P_COUNT] FP32
    DBuf<unsigned char> wbf;       // [P_COUNT] BF16 copy
    DBuf<unsigned char> scratch;   // forward buffers of one sample
    NetBuffers buf;
    NetGraphStore graph;
    DBuf<int> urow, ucol;          // the level's upper Galerkin BCOO, captured at assembly
    DBuf<double> ublk;
    int unnz = 0;
    float* rec_rc = nullptr;       // recorder (caller buffers): samples r_c, z_c
    float* rec_zc = nullptr;
    int rec_cap = 0, rec_every = 0;
    DBuf<int> rec_count;
};

struct Solver
{
    stg_config cfg{};
    cudaStream_t stream = nullptr;
    cudaStream_t capture_stream = nullptr;  // private stream used only to record graphs
    int launches = 0;
    Bcoo bcoo;
    ConvertScratch cv;
    MasState mas;
    PcgState pcg;
    LearnedState learned;
    cudaEvent_t ev[6] = {};
    bool events = false;
    int mas_fem_offset = 0;       // FEM block offset of the last MAS assembly
    long long generation = 0;     // bumped by every (re)assembly
    bool graph_dirty = true;
    int launches_per_batch = 0;   // kernels in one captured iteration
    cudaGraph_t pending_if_body = nullptr;
    PcgDev pcg_dev{};             // parameters of the last solve (measurement hook)
    bool pcg_ready = false;
    // SpMV kernel: spmv_rt > 0 fixes the rows per tile of the full-copy kernel, -2 the halo
    // kernel, -3 the upper kernel; spmv_rt == 0 with spmv_tune set times the candidates at the
    // next solve of a new shape and keeps the fastest
    // independent scenes on contiguous block-row ranges (stg_set_segments)
    int nseg = 0;
    std::vector<int> seg_off_host;    // [nseg + 1]
    std::vector<double> seg_host;     // [nseg][SEG_N] after the last solve
    DBuf<int> seg_off, seg_of_row;
    DBuf<double> seg_scal, seg_row;
    int spmv_rt = 0;
    bool spmv_tune = false;
    int tuned_rt = 0, tuned_prec = -1, tuned_nrows = -1, tuned_nnzb = -1;
    float tune_us[4] = {0.f, 0.f, 0.f, 0.f};

    ~Solver();

    // stages
    // fuse_offset >= 0 (MAS built): also the fused level-0 pass for that FEM block offset
    int convert(int count, const int* rows, const int* cols, const double* blocks, int nrows_hint,
                int fuse_offset = -1);
    int bind_bcoo(const double* blocks, const int* rows, const int* cols, int nnzb, int nrows);
    int prepare_spmv();   // row_ptr, transpose refs, FP32 copy, diag inverses
    int spmv(double a, const double* x, double b, double* y);
    int mas_init(int V, int node_offset, const uint32_t* ns, const uint32_t* nn, const uint32_t* nl, int nls,
                 const int* pm, int pms, const int* rm);
    int mas_build(const int* contacts, int ncp);
    int mas_assemble(int fem_block_offset);
    int mas_apply(const double* r, double* z);
    int pcg_solve(const double* b, double* x, int n, int abd_bodies, const double* abd_inv, stg_stats* st);
};

// ABD block-Jacobi (abd.cu): inverses of the bodies' diagonal 12x12 tiles of a sorted BCOO
int abd_block_jacobi(int nnzb, const int* rows, const int* cols, const double* blocks, int N, double* P,
                     int* singular, cudaStream_t s);

// Hessian producer (fem.cu): 10 T + V triplets and the gradient of one Newton iteration
size_t fem_scratch_bytes(int V, int T);
int fem_newton_system(cudaStream_t s, int V, const double* rest, const double* pos, const double* vel,
                      const double* xtilde, int T, const int* tets, const double* E, double nu, double rho, double dt,
                      double gy, int nplanes, const double* planes, int* rows, int* cols, double* blocks, double* b,
                      void* scratch, size_t bytes);
int fem_energy(cudaStream_t s, int V, const double* rest, const double* pos, const double* xtilde, int T,
               const int* tets, const double* E, double nu, double rho, double dt, int nplanes, const double* planes,
               void* scratch, size_t bytes, double* energy, int* violations);

}  // namespace stg
