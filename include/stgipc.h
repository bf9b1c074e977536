/*
 * stgipc.h -- C ABI of the B200 (sm_100a) Newton linear solve for StiffGIPC.
 *
 * One handle = one GlobalLinearSystem + PCGSolver + MAS preconditioner instance, bound to
 * one CUDA stream and one host thread (the reference is single-threaded per simulation;
 * its statistics are thread_local, gipc/statistics.h:14-16).  Handles share no state.
 *
 * Pointer conventions
 *   - stg_mas_init() takes HOST arrays: they are the mesh-side tables that the reference
 *     uploads from host vectors once per scene (app/common/sim_bootstrap.cpp:276-306).
 *   - every other entry point takes DEVICE pointers on the handle's stream, as the
 *     reference's GIPCTripletMatrix / DenseVectorView buffers live on the device
 *     (linear_system/linear_system/global_matrix.h:52-253).
 *   - 3x3 blocks are FP64, column-major (Eigen::Matrix3d): element (i,j) at [j*3+i].
 *   - block indices: ABD bodies own [0, 4*abd_bodies), FEM vertex v owns
 *     4*abd_bodies + v (GIPC.cu:10329-10330, 10482-10483).  n = 3 * block rows.
 *
 * Error convention
 *   The reference aborts on CUDA errors (CUDA_SAFE_CALL, cuda_tools/cuda_tools.h:36-46) or
 *   exit(0)s on launch errors (:52-96).  Here every entry point returns an int status
 *   (STG_OK or a code below) and never aborts; stg_last_error() gives a message.
 */
#ifndef STGIPC_H
#define STGIPC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STGIPC_VERSION 1

/* ---- status codes ---------------------------------------------------------------- */
enum
{
    STG_OK = 0,
    STG_ERR_INVALID = 1,        /* bad argument / size                                */
    STG_ERR_CUDA = 2,           /* a CUDA call failed (message in stg_last_error)       */
    STG_ERR_NOT_READY = 3,      /* stg_mas_init / assemble not called yet              */
    STG_MAX_ITER = 4,           /* PCG stopped at max_iter; x holds the last iterate   */
    STG_BREAKDOWN = 5,          /* p^T A p <= 0 or non-finite                          */
    STG_ERR_TIMEOUT = 6,        /* a bounded device wait gave up                       */
    STG_ERR_NO_DEVICE = 7       /* no usable CUDA device                               */
};

/* ---- configuration ---------------------------------------------------------------- */
enum { STG_PREC_FP64 = 0, STG_PREC_FP32 = 1 };
enum { STG_PRECOND_DIAG = 0, STG_PRECOND_MAS = 1, STG_PRECOND_NONE = 2 };
enum { STG_STOP_REFERENCE = 0, STG_STOP_RELATIVE_RESIDUAL = 1 };
enum { STG_LOOP_HOST = 0, STG_LOOP_GRAPH = 1, STG_LOOP_PERSISTENT = 2 };

typedef struct stg_config
{
    int bank_size;          /* MAS partition size: 16 (CEMAS as shipped) or 32         */
    int precision;          /* STG_PREC_FP64: FP64 SpMV/vectors, FP32 MAS apply (as the
                               reference); STG_PREC_FP32: FP32 blocks/vectors for SpMV and
                               MAS, FP64 dots, FP64 residual replacement               */
    int preconditioner;     /* STG_PRECOND_MAS (P_type==1) / STG_PRECOND_DIAG / NONE   */
    int stop_rule;          /* STG_STOP_REFERENCE: |r.z| <= tol * r0.z0 (pcg_solver.cu:279-280)
                               STG_STOP_RELATIVE_RESIDUAL: ||r||/||b|| <= tol            */
    double tol;             /* PCGSolverConfig::global_tol_rate (1e-4)                 */
    double max_iter_ratio;  /* PCGSolverConfig::max_iter_ratio (0.3): max_iter = ratio*n */
    int refine_interval;    /* FP32 mode: recompute r = b - A x in FP64 every k iters    */
    int loop_mode;          /* STG_LOOP_HOST / STG_LOOP_GRAPH / STG_LOOP_PERSISTENT      */
    int graph_batch;        /* iterations per captured graph launch (STG_LOOP_GRAPH)     */
    int learned;            /* 1: apply the learned coarse correction (stg_net_*) inside a
                               flexible PCG, MAS only, host or graph loop; 0: off        */
    void* stream;           /* cudaStream_t (NULL = legacy default stream)               */
} stg_config;

/* Fills `cfg` with the reference defaults: bank 16, FP64, MAS, reference stop rule,
 * tol 1e-4, ratio 0.3, refine 32, graph loop, batch 8, learned off, default stream. */
void stg_config_default(stg_config* cfg);

typedef struct stg_stats
{
    int status;             /* same value the call returned                          */
    int iterations;         /* PCG iteration count as returned by PCGSolver::pcg     */
    double rz0;             /* r0 . z0                                               */
    double rz_final;        /* last r . z                                            */
    double rel_residual;    /* ||b - A x|| / ||b|| recomputed in FP64 after the solve */
    double rel_residual_recursive; /* ||r_k|| / ||b|| of the recurrence at exit      */
    int nnzb;               /* unique upper blocks after convert                     */
    int levels;             /* MAS levelnum                                          */
    int total_clusters;     /* MAS totalNumberClusters                               */
    int replacements;       /* FP64 residual replacements (FP32 mode)                */
    int learned_accepted;   /* checks (residual replacements, or every refine_interval
                               FP64 iterations) at which the FP64 residual had fallen since
                               the previous one with the learned correction on          */
    int learned_rejected;   /* ... had not: the correction was switched off (0 or 1)   */
    float ms_convert;       /* device time per phase (CUDA events; 0 if not timed)   */
    float ms_mas_build;
    float ms_mas_assemble;
    float ms_pcg;
    float ms_total;
    int kernel_launches;    /* kernels this call launched                            */
} stg_stats;

typedef struct stg_solver* stg_handle;

/* Latest error message of this thread (never NULL). */
const char* stg_last_error(void);

/* ---- lifetime ---------------------------------------------------------------------- */
/* Replaces: GIPC::create_LinearSystem (StiffGIPC/gipc/gipc.cu:46-75) building
 * GlobalLinearSystem + PCGSolver(PCGSolverConfig) (linear_system/solver/pcg_solver.h:6-16)
 * + MAS_Preconditioner / DiagPreconditioner. */
int stg_create(const stg_config* cfg, stg_handle* out);
int stg_destroy(stg_handle h);

/* Replaces: MASPreconditioner::initPreconditioner_Neighbor + initPreconditioner_Matrix
 * (MASPreconditioner.cu:2291-2358) with the uploads of sim_bootstrap.cpp:276-306.
 * HOST arrays: neighbour CSR (load_mesh.cpp:934-1040), partId_map_real (part_map_size =
 * part_offset * bank_size, -1 padding) and real_map_partId (vert_num), set_mas_partition
 * (sim_bootstrap.cpp:90-113).  collision_node_offset = first FEM vertex in the contact
 * pair numbering (tet_mesh.abd_vertexOffset). */
int stg_mas_init(stg_handle h, int vert_num, int collision_node_offset,
                 const uint32_t* neighbor_start, const uint32_t* neighbor_num,
                 const uint32_t* neighbor_list, int neighbor_list_size,
                 const int32_t* part_map, int part_map_size, const int32_t* real_map);

/* ---- individual stages ------------------------------------------------------------- */
/* Replaces: Converter::srbk_convert (linear_system/utils/converter.cu:32-51, 88-238).
 * Sorts `count` triplets by (row<<32)+col, merges duplicates (summing blocks) and writes
 * the unique sorted BCOO back into the first *unique_count entries of the same arrays,
 * as the reference does in place. */
int stg_convert(stg_handle h, int count, int32_t* rows, int32_t* cols, double* blocks,
                int* unique_count);

/* Replaces: Spmv::srbk_spmv (linear_system/utils/spmv.cu:188-313):
 * y = a * A * x + b * y, A symmetric given by its unique upper blocks sorted by (row,col). */
int stg_spmv(stg_handle h, double a, const double* blocks, const int32_t* rows,
             const int32_t* cols, int nnzb, const double* x, double b, double* y, int n);

/* Replaces: MAS_Preconditioner::assemble (preconditioner/fem_mas_preconditioner.cu:18-31):
 * calculate_subsystem_bcoo_indices (i_preconditioner.cu:32-73) + setPreconditioner_bcoo
 * (MASPreconditioner.cu:2207-2245: ReorderRealtime + PrepareHessian_bcoo + inverse).
 * `contacts` is the device int4 array _collisonPairs (GIPC.cuh:49-66), `ncp` = h_cpNum[0]. */
int stg_mas_assemble(stg_handle h, const double* blocks, const int32_t* rows,
                     const int32_t* cols, int nnzb, int fem_block_offset,
                     const int32_t* contacts, int ncp);

/* Replaces: MAS_Preconditioner::apply -> MASPreconditioner::preconditioning
 * (fem_mas_preconditioner.cu:33-37, MASPreconditioner.cu:2248-2289).  r, z: the FEM
 * sub-range, 3 * vert_num doubles. */
int stg_mas_apply(stg_handle h, const double* r, double* z);

/* Replaces: PCGSolver::solve / pcg (linear_system/solver/pcg_solver.cu:158-332) with the
 * preconditioner composition of GlobalLinearSystem::apply_preconditioner
 * (global_linear_system.cu:167-180).  Requires the BCOO to be the one last assembled
 * (stg_mas_assemble or stg_solve_linear_system).  x is overwritten (x0 = 0). */
int stg_pcg_solve(stg_handle h, const double* blocks, const int32_t* rows, const int32_t* cols,
                  int nnzb, const double* b, double* x, int n, stg_stats* stats);

/* ---- the whole Newton linear solve ------------------------------------------------- */
typedef struct stg_system
{
    /* triplets as GIPCTripletMatrix holds them before convert (global_triplet_offset) */
    int triplet_count;
    const int32_t* rows;
    const int32_t* cols;
    const double* blocks;
    int n;                      /* 3 * block rows                                      */
    const double* b;            /* right-hand side (gradient), n doubles              */
    /* MAS inputs */
    int fem_block_offset;       /* 4 * abd_bodies                                      */
    const int32_t* contacts;    /* int4 collision pairs or NULL                        */
    int ncp;
    /* ABD 12x12 block-Jacobi (abd_preconditioner.cu:20-38): row-major inverses, or NULL to
     * invert the bodies' diagonal 12x12 tiles of the converted BCOO on the device, as
     * ABDSystem::_cal_abd_system_preconditioner does (setup_abd_system_gradient_and_hessian.cu:
     * 612-655; FP64 Gauss-Jordan with partial pivoting) */
    int abd_bodies;
    const double* abd_inv;
} stg_system;

/* Replaces: GlobalLinearSystem::solve_linear_system (global_linear_system.cu:136-148):
 * convert_new -> preconditioner assemble -> PCG -> solution.  Writes x (n doubles).
 * Returns STG_OK, STG_MAX_ITER or an error. */
int stg_solve_linear_system(stg_handle h, const stg_system* sys, double* x, stg_stats* stats);

/* ---- introspection (tests) ---------------------------------------------------------- */
/* Level count and cluster count of the last MAS build. */
int stg_mas_info(stg_handle h, int* levels, int* total_clusters, int* level_size /* 2*(L+1) */);

/* Copies the last MAS hierarchy to HOST arrays (any may be NULL):
 * fine_mask[V], prefix_orig[M/bank], coarse_tables[L*V], going_next[max(total,V)],
 * coarse_table[V*(L-1)]. */
int stg_mas_export_hierarchy(stg_handle h, uint32_t* fine_mask, int32_t* prefix_orig,
                             int32_t* coarse_tables, int32_t* going_next,
                             int32_t* coarse_table);

/* Copies the assembled FP64 bank matrices and FP32 inverses to HOST arrays
 * (nbanks * bank*(bank+1)/2 * 9 values each; either may be NULL). */
int stg_mas_export_matrices(stg_handle h, double* mat, float* inv, int* nbanks);

/* Measurement hook (no counterpart in the reference, whose PCG times phases with
 * cudaEventSynchronize, pcg_solver.cu:204-323): times `reps` back-to-back launches of the
 * PCG's SpMV kernel (q = A p with p.q fused) on the system of the last solve, with CUDA
 * events on the handle's stream.  avg_ms = mean duration per launch; bytes = algorithmic
 * bytes per launch, nnzb*(block + 8) + 3*n*vec with block = 72 (FP64) or 36 (FP32) and
 * vec = 8 or 4 (each array counted once). */
int stg_profile_spmv(stg_handle h, int reps, float* avg_ms, double* bytes);

/* Diagnostic (no counterpart in the reference) for the bounded waits of the bulk-copy
 * pipelines: one thread waits, with the same bounded poll, on an mbarrier that nothing
 * completes.  *status receives what the kernel recorded (STG_ERR_TIMEOUT when the wait
 * gave up, as it must) and *seconds how long the wait took.  Nothing is left in flight;
 * the device stays usable.  Returns STG_OK when the diagnostic ran. */
int stg_selftest_wait_timeout(int* status, double* seconds);

/* ---- Morton keys ----------------------------------------------------------------------- */
/* Replaces _calcVertMChash (StiffGIPC/GIPC.cu:453-502) with hash_code type -1 and expand_bits
 * (GIPC.cu:183-208): keys[i] = (code << 32) | i, code the 30-bit interleave (x << 2 | y << 1 | z)
 * of the position's cell at 1024 cells per axis of the bounding box of all n positions
 * (normalised, clamped to [0, 1023], truncated).  Ascending keys give the Morton vertex
 * order of the MAS banks.  pos: device double[3n]; keys: device uint64[n]; stream: a
 * cudaStream_t (NULL: the legacy default stream).  Asynchronous on the stream. */
int stg_morton_keys(int n, const double* pos, uint64_t* keys, void* stream);

/* ---- Hessian producer ------------------------------------------------------------------ */
/* The triplets and gradient of one implicit-Euler Newton iteration of a tet mesh, on the
 * GPU: what GIPC hands to GlobalLinearSystem::solve_linear_system (femEnergy.cu:1719-1855
 * for the elastic part, GIPC.cu:6524-6551 for the plane barrier).  Per tet: stable
 * Neo-Hookean psi = mu/2 (|F|^2 - 3) + lam/2 (J - 1 - mu/lam)^2 (E per tet, nu), its 9x9
 * Hessian in F projected to PSD (negative eigenvalues clamped, FP64 Jacobi), times
 * vol dt^2, as the tet's 10 upper 3x3 blocks (column-major) at triplets 10 t .. 10 t + 9.
 * Per vertex (triplet 10 tets + v): lumped mass rho vol / 4 plus the barrier Hessians of
 * the planes it is within dhat of.  b = dt^2 vol P : dF/dx + M (x - x - dt v - dt^2 g) +
 * barrier gradients, with g = (0, gravity_y, 0).  When xtilde (the inertial target
 * x_n + dt v_n + dt^2 g of the step) is given, the kinetic gradient is M (x - xtilde) and
 * vel is not read; later Newton iterations of a step pass it.  planes: [nplanes][6] =
 * normal xyz, offset (plane n.x = offset), dhat, kappa.  All arrays are device arrays;
 * rows / cols / blocks hold 10 tets + verts triplets, b 3 verts doubles. */
size_t stg_fem_scratch_bytes(int verts, int tets);
int stg_fem_newton_system(int verts, const double* rest, const double* pos, const double* vel,
                          const double* xtilde, int tets, const int32_t* tet_verts, const double* youngs,
                          double poisson, double density, double dt, double gravity_y, int nplanes,
                          const double* planes, int32_t* rows, int32_t* cols, double* blocks, double* b,
                          void* scratch, size_t scratch_bytes, void* stream);
/* The objective those triplets are the Hessian of (the incremental potential):
 * sum_tets dt^2 vol psi(F) + 1/2 sum_v m_v |x_v - xtilde_v|^2 + sum kappa b(d^2) over the
 * (vertex, plane) pairs within dhat, b(s) = -(s - dhat^2)^2 log(s / dhat^2).  *violations
 * (may be NULL) counts vertices on or behind a plane, where the potential is infinite. */
int stg_fem_energy(int verts, const double* rest, const double* pos, const double* xtilde, int tets,
                   const int32_t* tet_verts, const double* youngs, double poisson, double density, double dt,
                   int nplanes, const double* planes, void* scratch, size_t scratch_bytes, double* energy,
                   int* violations, void* stream);

/* ---- contact barriers ------------------------------------------------------------------- */
/* Replaces _calBarrierGradientAndHessian (StiffGIPC/GIPC.cu:3149-4988, built with NEWF and
 * RANK 2) for the unmollified encodings of the int4 pairs (GIPC.cuh:49-66): edge-edge
 * (x, y | z, w), point-point (-x-1, y; z < 0), point-edge (-x-1 | y, z; w < 0) and
 * point-triangle (-x-1 | y, z, w).  With s = d / sqrt(dhat) (d the pair's distance, dhat the
 * squared activation distance) the barrier is kappa dhat^2 (s^2 - 1)^2 ln^2(s^2) for s < 1;
 * per pair: gradient E'(s) ds/dx (12 doubles, 3 per local vertex, zero for unused vertices)
 * and the 10 upper 3x3 blocks (column-major, row <= col, plus block_offset) of the rank-one
 * Hessian E''(s) ds/dx ds/dx^T, with E'' frozen at s^2 = 1e-6 below it (GIPC.cu:3171,
 * 3310-3327).  Slot k of pair p is triplet 10 p + k in the order (0,0) (0,1) (0,2) (0,3)
 * (1,1) (1,2) (1,3) (2,2) (2,3) (3,3) of local vertices; a slot past the pair's vertex count
 * holds a zero block on its first vertex.  A mollified, out-of-range or degenerate pair gets
 * zero blocks and a zero gradient and is counted in *skipped (device int, may be NULL; added
 * to, not reset).  pairs: device int32[4 ncp]; x: device double[3 num_verts]; rows / cols:
 * device int32[10 ncp]; blocks: device double[90 ncp]; grad: device double[12 ncp].
 * Asynchronous on `stream` (a cudaStream_t; NULL: the legacy default stream). */
int stg_contact_barrier(int ncp, const int32_t* pairs, const double* x, int num_verts, int block_offset,
                        double dhat, double kappa, int32_t* rows, int32_t* cols, double* blocks,
                        double* grad, int* skipped, void* stream);
/* The energies of the same pairs: energy[p] = kappa dhat^2 (s^2 - 1)^2 ln^2(s^2) for s < 1,
 * else 0 (also 0 for the pairs stg_contact_barrier skips) -- the barrier term of the
 * incremental potential the line search evaluates (GIPC::computeEnergy, the RANK 2 barrier).
 * energy: device double[ncp]; asynchronous. */
int stg_contact_energy(int ncp, const int32_t* pairs, const double* x, int num_verts, double dhat,
                       double kappa, double* energy, void* stream);

/* ---- cloth ------------------------------------------------------------------------------ */
/* Replaces _calculate_triangle_fem_gradient_hessian (StiffGIPC/femEnergy.cu:2146-2216): per
 * triangle, the Baraff-Witkin membrane energy area dt^2 [stretch ((su - 1)^2 + (sv - 1)^2 +
 * strain_rate ((su - 1)^3_+ + (sv - 1)^3_+)) + shear I6^2], su = |F u|, sv = |F v|,
 * I6 = F u . F v, F = Ds Dm^-1; gradient (9 doubles per triangle, 3 per vertex) and the 6 upper
 * 3x3 blocks (column-major, row <= col, plus block_offset) of its Hessian, whose stretch part is
 * projected per direction and shear part to PSD as the reference does (:535-706).
 * tri_verts: int32[3 tris]; dminv: double[4 tris] row-major 2x2 inverse of the rest edges in
 * the reference's triangle frame (__calculateDm2D_double); area: double[tris], rest area times
 * thickness.  *bad (device, may be NULL) counts triangles with an index out of range or a
 * repeated vertex (zero terms).  Device arrays; asynchronous. */
int stg_cloth_membrane(int tris, const int32_t* tri_verts, const double* dminv, const double* area,
                       const double* x, int num_verts, double stretch, double shear, double strain_rate,
                       double dt, int block_offset, int32_t* rows, int32_t* cols, double* blocks,
                       double* grad, int* bad, void* stream);
/* Replaces _calculate_quad_bending_gradient_hessian (femEnergy.cu:2620-2755,
 * USE_QUADRATIC_BENDING): per edge stencil (v0, v1, opposite vertex of each triangle;
 * int32[4 edges], the last -1 for a boundary edge, which gets zero terms), c = rest_length
 * bend_stiff dt^2, gradient c Q x (12 doubles) and the 10 upper blocks of c Q (x) I3.  Q:
 * double[16 edges], row-major 4x4 (PrepareQuadBendingQ).  Device arrays; asynchronous. */
int stg_cloth_bending(int edges, const int32_t* stencil, const double* Q, const double* rest_length,
                      const double* x, int num_verts, double bend_stiff, double dt, int block_offset,
                      int32_t* rows, int32_t* cols, double* blocks, double* grad, int* bad, void* stream);

/* ---- affine bodies (ABD) ---------------------------------------------------------------- */
/* Body b owns block rows 4 b .. 4 b + 3; q[12 b ..] = (t, a1, a2, a3) with a_i the rows of A
 * (x = A xbar + t, abd_jacobi_matrix.inl); FEM vertices follow at block row 4 bodies + v.
 *
 * Replaces ABDSystem::_cal_abd_body_gradient_and_hessian + write_abd_body_hessian
 * (abd_system/abd_system_function/setup_abd_system_gradient_and_hessian.cu:129-139, 200-262)
 * for free and fixed bodies: per body, the 10 upper 3x3 blocks (column-major, triplets
 * 10 b .. 10 b + 9 in (0,0) (0,1) .. (3,3) order) of H = M + kappa vol dt^2 PSD(d2S/da2) and
 * the gradient g = M (q - q_tilde) + kappa vol dt^2 dS/da, S = sum (a_i.a_i - 1)^2 +
 * sum_{i != j} (a_i.a_j)^2 (abd_energy.inl:9-140), PSD by clamping negative eigenvalues of the
 * 9x9 a-block (FP64 Jacobi).  mass: 13 doubles per body, the dyadic mass m, m xbar (3),
 * m xbar xbar^T (9, row-major) summed over the body's points (ABDJacobiDyadicMass).  fixed
 * (may be NULL): nonzero marks a fixed body (H = M, g = 0).  Device arrays; asynchronous. */
int stg_abd_body_system(int bodies, const double* q, const double* q_tilde, const double* mass,
                        const double* volume, const int32_t* fixed, double kappa, double dt,
                        int32_t* rows, int32_t* cols, double* blocks, double* grad, void* stream);
/* Replaces write_barrier_hessian and the ABD-FEM coupling kernel
 * (setup_abd_system_gradient_and_hessian.cu:89-126, 510-551) and the FEM contact shift
 * (GIPC.cu:10328-10362): maps `count` point-level 3x3 triplets (i, j) of a symmetric matrix
 * given by its upper blocks (a block with i > j is read as the transpose at (j, i)) onto the
 * global block index space, 16 output triplets per input at 16 t .. 16 t + 15.  Points
 * [0, abd_points) belong to bodies point_body[i] with rest coordinates xbar[3 i ..]; points
 * from abd_points on are FEM vertex i - abd_points.  Two FEM vertices: the block at
 * (4 bodies + i - P, 4 bodies + j - P).  Body point and FEM vertex: the 4 blocks of J_i^T B.
 * Two body points of different bodies: the 16 blocks of J_i^T B J_j (JT_H_J).  Of one body:
 * the 10 upper blocks of J_i^T B J_i (i == j) or of J_i^T B J_j + (J_i^T B J_j)^T (i != j).
 * Unused slots hold zero blocks on the first row written.  *bad (device, may be NULL) counts
 * inputs with a negative index or a body id outside [0, bodies); they get zero blocks. */
int stg_abd_map_triplets(int count, const int32_t* rows, const int32_t* cols, const double* blocks,
                         int abd_points, const int32_t* point_body, const double* xbar, int bodies,
                         int32_t* out_rows, int32_t* out_cols, double* out_blocks, int* bad, void* stream);
/* x[3 i ..] = A xbar_i + t of point i's body (cal_x_from_q); device arrays. */
int stg_abd_points(int abd_points, const int32_t* point_body, const double* xbar, const double* q,
                   double* x, void* stream);
/* body_grad[12 b ..] += sum over the body's points i in [start[b], start[b + 1]) of J_i^T g_i,
 * in point order (_cal_abd_system_barrier_gradient, :362-396); device arrays. */
int stg_abd_gather_gradient(int bodies, const int32_t* body_point_start, const double* xbar,
                            const double* point_grad, double* body_grad, void* stream);

/* ---- continuous collision detection (line-search step bound) ------------------------------ */
/* Replaces GIPC::self_largestFeasibleStepSize and _reduct_min_selfTimeStep_to_double
 * (StiffGIPC/GIPC.cu:7095-7180, 9010-9047) with the reference's additive CCD per pair
 * (point_triangle_ccd, edge_edge_ccd and their distance classification, ACCD.cu:15-534).
 * pairs: device int32[4 npairs], point-triangle as (-p-1, t0, t1, t2), edge-edge as
 * (a0, a1, b0, b1); x, dx: device double[3 num_verts], positions and the step's displacement
 * (the reference passes -moveDir).  Each pair's time of impact toc in [0, 1] uses
 * eta = 1 - slackness (the reference calls it with slackness 0.8) and `thickness` (0 there);
 * *alpha (device double) = 1 / max over pairs of 1 / toc, 1 with no pairs.  toc (device
 * double[npairs], may be NULL) receives every pair's value; *bad (device int, may be NULL;
 * added to) counts pairs with a vertex outside [0, num_verts), which impose no bound.
 * scratch: one device unsigned long long the call owns until it completes.  Asynchronous. */
int stg_ccd_step_size(int npairs, const int32_t* pairs, const double* x, const double* dx, int num_verts,
                      double slackness, double thickness, double* alpha, double* toc, int* bad,
                      unsigned long long* scratch, void* stream);

/* ---- independent scenes in one solve ---------------------------------------------------- */
/* No counterpart in the reference.  The system of the following solves is a block-diagonal
 * batch of independent scenes on contiguous block-row ranges [row_offsets[s],
 * row_offsets[s + 1]) (host array of nseg + 1 entries, the last one the block-row count).
 * Every scene runs its own PCG recurrence (its own alpha, beta and stop test
 * ||r_s|| <= tol ||b_s||) inside the one graph-captured loop, which ends when every scene
 * is done; a finished scene's rows stop changing.  Needs the relative-residual stop rule,
 * the host or graph loop, no ABD bodies and no learned correction.  nseg = 0: one system. */
int stg_set_segments(stg_handle h, const int32_t* row_offsets, int nseg);
/* Per scene of the last solve (host arrays of nseg): iterations until its stop test held
 * (0 if it never did) and ||r_s|| / ||b_s|| of its recurrence at the end. */
int stg_segment_stats(stg_handle h, int* iterations, double* rel_residual);

/* ---- BCOO tile autotuner -------------------------------------------------------------- */
/* No counterpart in the reference.  Kernel of the in-loop SpMV: rows_per_tile rows per
 * tile of the row-sliced full copy, with 256 / rows_per_tile lanes per row (FP32: 64 or 32;
 * FP64: 32 or 16); -2: the halo kernel (fixed tiles whose column operands are staged in
 * shared memory); -3: the upper kernel (each upper block streamed once, its transposed
 * product spilled to the column's row and added there in a fixed order).  0 = autotune: the
 * next solve of a new shape class (precision, block rows, unique blocks) times every
 * candidate (both tile shapes, the upper kernel, and the halo kernel when its windows fit)
 * on that system; the choice is kept for that shape class by every handle of the process.
 * -1 = the default kernel.  The persistent loop always runs the full-copy SpMV.  Results
 * differ between candidates in the last bits (summation order); a fixed choice keeps solves
 * bitwise reproducible across processes. */
int stg_spmv_tiles(stg_handle h, int rows_per_tile);
/* Kernel of the last solve (rows per tile; -2: the halo kernel; -3: the upper kernel), and
 * the autotuner's mean time per launch of each candidate in microseconds (0 when it has not
 * run or the candidate did not fit). */
int stg_spmv_tiles_info(stg_handle h, int* rows_per_tile, float* us_default, float* us_alternative,
                        float* us_halo, float* us_upper);

/* ---- allocation-free SpMV ---------------------------------------------------------- */
/* No counterpart in the reference.  The same y = a * A * x + b * y as stg_spmv (same
 * kernel, same result bit for bit), for callers that cannot allocate device memory: a host
 * simulator that has reserved the GPU's memory for its own pool and forbids allocations
 * outside it, or a step loop that cannot take cudaMalloc's implicit device synchronisation.
 * It takes no handle and allocates nothing: its row pointers and transpose lists live in
 * one fixed device array of STG_NOALLOC_SCRATCH_BYTES (about 9.5 MiB) inside the library,
 * held by every GPU that loads the library until the process exits.  Systems larger than
 * STG_NOALLOC_MAX_ROWS block rows (n / 3) or STG_NOALLOC_MAX_BLOCKS upper blocks are
 * rejected with STG_ERR_INVALID.  All calls share that array: calls that overlap on the
 * GPU (two host threads, or two streams) race and give wrong results.  Every pointer must
 * be memory of the current device (STG_ERR_INVALID otherwise).  The first call on each
 * device resolves the array's address on that device; under lazy module loading (the
 * CUDA 12 default) that first call may also be when the array is reserved, so a caller
 * that hands the rest of HBM to its own pool makes a call with n == 0 first (it does only
 * this set-up), or sets CUDA_MODULE_LOADING=EAGER.  `stream` is a cudaStream_t (NULL: the
 * legacy default stream).  The call is synchronous: it reads the input check back to the
 * host and returns after the stream has finished the product, so it cannot be called
 * inside a stream capture. */
#define STG_NOALLOC_MAX_ROWS 131072
#define STG_NOALLOC_MAX_BLOCKS 1048576
#define STG_NOALLOC_SCRATCH_BYTES (256 + 3 * 4 * 131136 + 8 * 1048576)
int stg_spmv_noalloc(double a, const double* blocks, const int32_t* rows,
                     const int32_t* cols, int nnzb, const double* x, double b, double* y,
                     int n, void* stream);

/* ---- learned coarse correction ------------------------------------------------------ */
/* No counterpart in the reference (its MAS is the fallback).  A 3-layer message-passing
 * network (hidden width 64, BF16 weights, FP32 accumulation) over the nodes of one coarse
 * MAS level predicts a correction of that level's bank solve: z_l = D_l^-1 r_l + s d(r_l),
 * inside a flexible PCG (beta = r_k.(z_k - z_(k-1)) / r_(k-1).z_(k-1)).  At every FP64
 * residual replacement (FP32 path), or every refine_interval iterations of the FP64
 * recurrence (FP64 path), the FP64 residual must have fallen since the previous check,
 * else the solve continues with plain MAS (stg_stats.learned_*).
 * Parameters are one FP32 vector of STG_NET_PARAMS floats, every weight matrix stored
 * [out][in]: W0 [64][16] at 0, b0 [64] at 1024, W1..W3 [64][128] at 1088 + 8192 k, b1..b3
 * [64] at 25664 + 64 k, Wo [8][64] at 25856, bo [8] at 26368 (outputs 3..7 unused). */
#define STG_NET_PARAMS 26376

/* The coarse level the network works on (1 .. levels-1; 0 = none).  Takes effect at the
 * next MAS assembly, which then builds the level's graph from its Galerkin operator. */
int stg_net_configure(stg_handle h, int level);
/* Nodes and directed neighbour entries of the level's graph (after an assembly). */
int stg_net_graph_info(stg_handle h, int* nodes, int* entries);
/* Copies the graph to caller device buffers: row [nodes+1], col [entries] (both directions,
 * sorted by column), w [entries] = |A_ij|_F / sqrt(|A_ii|_F |A_jj|_F), oblk [9 entries]
 * (A_(i,col) row-major), dblk [9 nodes], feat [nodes] (centred log trace of A_ii); FP32. */
int stg_net_export_graph(stg_handle h, int32_t* row, int32_t* col, float* w, float* oblk, float* dblk,
                         float* feat);
/* Arms the sample recorder for the following solves (capacity 0 disarms): at iterations
 * 0, every, 2 every, ... the level's restricted residual and bank solve (float4 per node,
 * before any correction) go to rc / zc [capacity][nodes][4]. */
int stg_net_record(stg_handle h, float* rc, float* zc, int capacity, int every);
int stg_net_recorded(stg_handle h, int* count);
/* Parameters for the in-loop network (device pointer, STG_NET_PARAMS floats, copied). */
int stg_net_set_params(stg_handle h, const float* params);

/* Training, handle-free, on `stream`, through the project's own kernels. */
typedef struct stg_net_graph
{
    int nodes, entries;
    const int32_t* row;
    const int32_t* col;
    const float* w;
    const float* oblk;
    const float* dblk;
    const float* feat;
} stg_net_graph;
/* Bytes of the 256-byte aligned device scratch a forward / training step over `samples`
 * samples of a `nodes`-node graph needs. */
size_t stg_net_scratch_bytes(int nodes, int samples);
/* delta [samples][nodes][4] = the network's output d for samples rc / zc. */
int stg_net_forward(const stg_net_graph* g, const float* rc, const float* zc, int samples, const float* params,
                    float* delta, void* scratch, size_t scratch_bytes, void* stream);
/* The in-loop application on one sample, in place: z += theta s_z d(rc, z), theta <= 1 the
 * largest step that keeps rc.z at least half its value before.  The fused single-launch
 * kernel (one thread-block cluster) when the graph fits it, else the layered kernels;
 * *fused (may be NULL) receives the cluster size used, 0 for the layered kernels. */
int stg_net_apply(const stg_net_graph* g, const float* rc, float* z, const float* params, void* scratch,
                  size_t scratch_bytes, int* fused, void* stream);
/* One step: loss[s] = J(z + s_z d) / |J(z)| per sample (J(v) = v.A v / 2 - v.r), grad =
 * gradient of the mean loss; with lr > 0 an Adam step (beta 0.9 / 0.999, eps 1e-8, bias
 * corrections of step `step` >= 1) on params with moments m, v.  All device pointers. */
int stg_net_train_step(const stg_net_graph* g, const float* rc, const float* zc, int samples, float* params,
                       float* grad, float* adam_m, float* adam_v, int step, float lr, float* loss, void* scratch,
                       size_t scratch_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* STGIPC_H */
