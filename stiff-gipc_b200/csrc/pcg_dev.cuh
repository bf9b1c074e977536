// pcg_dev.cuh -- the by-value parameter block of the PCG phases (pcg.cu).
#pragma once
#include "reduce.cuh"

namespace stg
{
constexpr int kMaxLevelsDev = 6;
// per-scene scalar slots of PcgDev::seg
enum : int
{
    SG_RZ = 0, SG_PQ = 1, SG_ALPHA = 2, SG_BETA = 3, SG_RR = 4, SG_BB = 5, SG_DONE = 6, SG_ITER = 7, SEG_N = 8
};

// Everything a phase needs, passed by value.
struct PcgDev
{
    // SpMV structure (padded blocks: FP32 48 B = 3 x float4, FP64 80 B = 5 x double2)
    const int* row_ptr;
    const int* cols;
    const int* t_ptr;
    const int2* t_ent;
    const unsigned char* fent;  // full symmetric row-sliced copy in 16-byte planes (phase A)
    const int* frow;          // [nrows+1] first entry of each row in fent
    size_t fstride;           // entries per plane
    const unsigned char* htail;  // halo SpMV: {h8, slot} plane, per-tile halo columns
    const int* hcnt;
    const int* hlist;
    int halo;                 // the SpMV phase runs the halo kernel
    // upper SpMV phase (UpperPlanes in spmv_core.cuh): the upper copy, its row bounds padded
    // for the tiles' copies, and the spill slots of the transposed products (4 T per
    // strictly upper block, in transpose-list order).  spill == null: the full-copy kernels,
    // and q holds the whole product
    const unsigned char* uent;
    const int* urow;
    size_t ustride;
    void* spill;
    int upper;
    const double2* blk64;     // FP64 padded upper blocks (residual replacement)
    int nrows, n;
    // vectors in the iteration precision T, one 4-wide (16 B FP32 / 32 B FP64) slot per block
    // row; z and p of a row share one 32 / 64-byte slot, so that a neighbour gather is one
    // (FP32) or two (FP64) 32-byte loads:
    //   zp[2]: per block row {z0 z1 z2 -, p0 p1 p2 -} (8 T); double-buffered across iterations
    //   q    : per block row {q0 q1 q2 -} (4 T)
    // x, r, b stay FP64 in the caller's [3n] layout
    void* zp0;
    void* zp1;
    void* q;
    double* x;
    double* r;
    const double* b;
    // MAS
    const int* part_map;
    const unsigned* fine_mask;
    const int* going_next;
    const unsigned* closed;
    float* R;
    float* Z;
    const float* inv;
    const int* real_map;
    const int* coarse_table;
    int M, V, L, nbanks, fem_dof;
    int identity;                     // part_map[s] == s for s < V, -1 after
    int ls[2 * (kMaxLevelsDev + 1)];  // level (count, begin) pairs; constant indices only
    const int* ls_dev;                // the same pairs in device memory (runtime indices)
    // non-MAS preconditioners
    const double* diag_inv;   // null: identity
    int abd_bodies;
    const double* abd_inv;
    // reductions / control
    double* partials;         // [8][slots]
    unsigned* counters;       // [8]
    double* scal;
    int* flags;
    int slots;
    int grid_a;               // CTAs of the SpMV phase: its p.q partials, summed by phase B
    int grid_e;               // CTAs of phase E: its r.z partials, summed by phases A and B
    PcgParams prm;
    cudaGraphConditionalHandle h_while, h_if;
    int use_cond;
    unsigned* bar;            // persistent barrier: [0] count, [1] generation
    // learned coarse correction: flexible PCG (beta from r_(k+1).(z_(k+1) - z_k), phase E's
    // r.z_old partials at SITE_F); the rest only keys the captured graph
    int a_rt;                 // rows per tile of the SpMV phase (one of the compiled shapes)
    // independent systems (scenes) on contiguous block-row ranges, each with its own PCG
    // scalars and stop test; null seg_of_row: one system
    const int* seg_of_row;    // [nrows] scene of each block row
    const int* seg_row_off;   // [nseg + 1] first block row of each scene
    double* seg;              // [nseg][SEG_N] per-scene scalars (SG_* slots)
    double* seg_row;          // [3][nrows] per-row p.q, r.r, r.z contributions
    int nseg;
    double seg_tol2;          // per-scene stop: r.r <= seg_tol2 * b.b
    int flex;
    int net_mode;             // bit 0: network applied, bit 1: samples recorded
    int net_n, net_rec_cap, net_rec_every;
    const void* net_ptrs[6];
};

}  // namespace stg
