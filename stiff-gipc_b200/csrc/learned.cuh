// learned.cuh -- the learned coarse correction: a 3-layer message-passing network over the
// nodes of one MAS coarse level, predicting a correction of that level's bank solve inside a
// flexible PCG (pcg.cu).  Kernels in learned.cu; this header is shared with pcg.cu / capi.cu.
//
// Network (hidden width 64, BF16 weights and activations, FP32 accumulation on the tensor
// cores with mma.sync m16n8k16):
//   input   x_i = [r_i / s_r, z_i / s_z, f_i, 1, 0 ...] (16 wide), r = the level's restricted
//           residual, z = its bank solve, s_r / s_z their RMS over the level's nodes, f_i a
//           static node feature (log of the trace of the diagonal block, centred)
//   embed   h0 = relu(W0 x + b0)
//   layer k h_k = relu(W_k [h_(k-1), m_k] + b_k), m_k,i = sum_j w_ij h_(k-1),j over the
//           coarse operator's off-diagonal neighbours, w_ij = |A_ij|_F / sqrt(|A_ii|_F |A_jj|_F)
//   head    d_i = Wo h3 + bo (3 of 8 outputs used)
//   output  g_i = z_i + s_z d_i replaces the bank solve z_i of the level
// Training minimises J(g) / |J(z)| with J(g) = 1/2 g.A g - g.r (A the level's Galerkin
// operator): J(g) = 1/2 |e - P^T g|_A^2 - 1/2 |e|_A^2 for the fine error e with A e = r, so
// the loss is the energy-norm error left after the coarse correction, relative to the bank
// solve's.
#pragma once
#include "common.cuh"

namespace stg
{
constexpr int NET_IN = 16, NET_H = 64, NET_OUT = 8, NET_LAYERS = 3;
// flat FP32 parameter vector; every weight matrix stored [out][in] (the mma B operand layout)
constexpr int P_W0 = 0;                                // [64][16]
constexpr int P_B0 = P_W0 + NET_H * NET_IN;            // [64]
constexpr int P_W1 = P_B0 + NET_H;                     // 3 x [64][128]
constexpr int P_B1 = P_W1 + NET_LAYERS * NET_H * 2 * NET_H;  // 3 x [64]
constexpr int P_WO = P_B1 + NET_LAYERS * NET_H;        // [8][64]
constexpr int P_BO = P_WO + NET_OUT * NET_H;           // [8]
constexpr int P_COUNT = P_BO + NET_OUT;                // 26,376

// One coarse level as a graph (device pointers).  Neighbour lists are full symmetric (both
// directions, no self entry), sorted by column; oblk[e] is the 3x3 block A_(i, col[e])
// row-major, dblk[i] the diagonal block.  FP32.
struct NetGraph
{
    int n = 0, nnz = 0;
    const int* row = nullptr;     // [n+1]
    const int* col = nullptr;     // [nnz]
    const float* w = nullptr;     // [nnz]
    const float* oblk = nullptr;  // [nnz*9]
    const float* dblk = nullptr;  // [n*9]
    const float* feat = nullptr;  // [n]
};

// Activations of one forward pass over S samples of the same graph (rows = S n, padded to
// 16).  Device pointers into one scratch block.
struct NetBuffers
{
    int S = 0, rows = 0, rows_pad = 0, wg_blocks = 0;
    void* x0 = nullptr;        // bf16 [rows_pad][16]
    void* h[4] = {};           // bf16 [rows_pad][64]: h0 .. h3
    void* m[3] = {};           // bf16 [rows_pad][64]: m1 .. m3
    float* delta = nullptr;    // [rows_pad][4]
    float* scale = nullptr;    // [S][2]: s_r, s_z
    float* ddelta = nullptr;   // [rows_pad][4]
    float* du = nullptr;       // [rows_pad][64]
    float* dha = nullptr;      // [rows_pad][64]
    float* dm = nullptr;       // [rows_pad][64]
    float* part = nullptr;     // [wg_blocks][64*128 + 64]
    float* loss = nullptr;     // [S]
    void* wbf = nullptr;       // bf16 [P_COUNT]
};

// kernel attributes of the forward pass (call once per thread before a graph capture)
int net_prepare();
size_t net_scratch_bytes(int n, int S);
int net_carve(void* scratch, size_t bytes, int n, int S, NetBuffers& b);

// forward over S samples: rc / zc are float4 per node, sample stride 4 n floats.  When
// `apply` is set (S == 1, inside the PCG loop), Z_level += theta s_z d with theta <= 1
// chosen so that r.z stays >= half the bank solve's r.z; flags (if set) gate the launch:
// nothing runs when flags[0] (done) is set or flags[3] (learned on) is clear.
int net_forward(cudaStream_t s, const NetGraph& g, const float* rc, const float* zc, int S, const NetBuffers& b,
                const void* wbf, const float* params, float* apply, const int* flags, int* launches);
// one training step: forward, loss, backward into grad; Adam update of params (and the
// BF16 copy) when lr > 0
int net_train_step(cudaStream_t s, const NetGraph& g, const float* rc, const float* zc, int S, const NetBuffers& b,
                   float* params, float* grad, float* adam_m, float* adam_v, int step, float lr, int* launches);
int net_to_bf16(cudaStream_t s, const float* params, void* wbf);
// one launch of the sample recorder (see k_net_record)
int net_record(cudaStream_t s, const float* R, const float* Z, int n, const double* scal, const int* flags, float* rc,
               float* zc, int* count, int cap, int every);

// the level's graph from its upper Galerkin BCOO (level-local ids, FP64 column-major blocks)
struct NetGraphStore
{
    int level = 0, n = 0, nnz = 0;
    int fu_cl = 0, fu_rpc = 0;    // fused forward: cluster size and rows per CTA (0: layered)
    DBuf<int> row, col, cnt, cur;
    DBuf<float> w, oblk, dblk, feat;
    DBuf<long long> key;
    DBuf<int2> fu_nb;             // neighbour entries packed for the fused forward
    NetGraph view() const
    {
        NetGraph g;
        g.n = n;
        g.nnz = nnz;
        g.row = row.data();
        g.col = col.data();
        g.w = w.data();
        g.oblk = oblk.data();
        g.dblk = dblk.data();
        g.feat = feat.data();
        return g;
    }
};
int net_build_graph(cudaStream_t s, NetGraphStore& G, int n, int nnzu, const int* urow, const int* ucol,
                    const double* ublk, int* launches);
// the fused single-launch forward + apply (one thread-block cluster, see k_net_fused)
int net_fused_plan(const int* row, int n, int* cl, int* rpc);
int net_forward_fused(cudaStream_t s, const NetGraph& g, const int2* nbp, const float* rc, float* Z, const void* wbf,
                      const float* params, const int* flags, int cl, int rpc);

}  // namespace stg
