// capi.cu -- the C ABI (include/stgipc.h) over the solver stages.
//
// The orchestration follows GlobalLinearSystem::solve_linear_system / build_linear_system
// (StiffGIPC/linear_system/linear_system/global_linear_system.cu:8-148): convert the triplets,
// assemble the preconditioner(s), run the iterative solver, hand back x.
#include "solver.hpp"
#include "reduce.cuh"

#include <cmath>
#include <new>

using stg::Solver;

// the opaque handle type of the C ABI
struct stg_solver : stg::Solver
{
};

namespace stg
{
Solver::~Solver()
{
    if(pcg.graph) cudaGraphExecDestroy(pcg.graph);
    if(capture_stream) cudaStreamDestroy(capture_stream);
    for(auto& e : ev)
        if(e) cudaEventDestroy(e);
}

// ||b - y||^2 and ||b||^2 into out[0], out[1] (deterministic, one CTA)
__global__ void __launch_bounds__(256) k_resid_norms(const double* __restrict__ b, const double* __restrict__ y, int n,
                                                     double* out)
{
    __shared__ double red[8];
    double rr = 0, bb = 0;
    for(int i = threadIdx.x; i < n; i += 256)
    {
        const double d = b[i] - y[i];
        rr += d * d;
        bb += b[i] * b[i];
    }
    rr = block_sum<256>(rr, red);
    bb = block_sum<256>(bb, red);
    if(threadIdx.x == 0)
    {
        out[0] = rr;
        out[1] = bb;
    }
}

static int true_residual(Solver& S, const double* b, const double* x, int n, double* rel)
{
    STG_TRY(S.pcg.q.resize(n));
    STG_TRY(S.pcg.partials.resize(std::max<size_t>(S.pcg.partials.size, 2)));
    STG_TRY(S.spmv(1.0, x, 0.0, S.pcg.q.data()));
    k_resid_norms<<<1, 256, 0, S.stream>>>(b, S.pcg.q.data(), n, S.pcg.partials.data());
    STG_LAUNCH_CHECK();
    S.launches++;
    double h[2];
    STG_CUDA_TRY(cudaMemcpyAsync(h, S.pcg.partials.data(), sizeof(h), cudaMemcpyDeviceToHost, S.stream));
    STG_CUDA_TRY(cudaStreamSynchronize(S.stream));
    *rel = h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
    return 0;
}
}  // namespace stg

#define CHECK_HANDLE(h)                                   \
    do                                                    \
    {                                                     \
        if(!(h))                                          \
        {                                                 \
            stg::set_error("null stg_handle");            \
            return STG_ERR_INVALID;                       \
        }                                                 \
    } while(0)

#define GUARD(...)                                        \
    try                                                   \
    {                                                     \
        __VA_ARGS__                                       \
    }                                                     \
    catch(const std::bad_alloc&)                          \
    {                                                     \
        stg::set_error("host allocation failed");         \
        return STG_ERR_INVALID;                           \
    }                                                     \
    catch(...)                                            \
    {                                                     \
        stg::set_error("unexpected C++ exception");       \
        return STG_ERR_INVALID;                           \
    }

extern "C" {

const char* stg_last_error(void) { return stg::last_error(); }

void stg_config_default(stg_config* c)
{
    if(!c) return;
    c->bank_size = 16;
    c->precision = STG_PREC_FP64;
    c->preconditioner = STG_PRECOND_MAS;
    c->stop_rule = STG_STOP_REFERENCE;
    c->tol = 1e-4;
    c->max_iter_ratio = 0.3;
    c->refine_interval = 32;
    c->loop_mode = STG_LOOP_GRAPH;
    c->graph_batch = 8;
    c->learned = 0;
    c->stream = nullptr;
}

int stg_create(const stg_config* cfg, stg_handle* out)
{
    GUARD({
        if(!out)
        {
            stg::set_error("stg_create: out is null");
            return STG_ERR_INVALID;
        }
        *out = nullptr;
        stg_config c;
        stg_config_default(&c);
        if(cfg) c = *cfg;
        if(c.bank_size != 16 && c.bank_size != 32)
        {
            stg::set_error("stg_create: bank_size must be 16 or 32");
            return STG_ERR_INVALID;
        }
        if(c.precision != STG_PREC_FP64 && c.precision != STG_PREC_FP32)
        {
            stg::set_error("stg_create: unknown precision");
            return STG_ERR_INVALID;
        }
        if(c.preconditioner < STG_PRECOND_DIAG || c.preconditioner > STG_PRECOND_NONE || c.stop_rule < 0 ||
           c.stop_rule > 1 || !(c.tol > 0) || !(c.max_iter_ratio > 0) || c.loop_mode < 0 || c.loop_mode > 2)
        {
            stg::set_error("stg_create: invalid configuration value");
            return STG_ERR_INVALID;
        }
        if(c.learned != 0 && c.learned != 1)
        {
            stg::set_error("stg_create: learned must be 0 or 1");
            return STG_ERR_INVALID;
        }
        if(c.learned && c.preconditioner != STG_PRECOND_MAS)
        {
            stg::set_error("stg_create: the learned coarse correction needs the MAS preconditioner");
            return STG_ERR_INVALID;
        }
        if(c.learned && c.loop_mode == STG_LOOP_PERSISTENT)
        {
            stg::set_error("stg_create: the learned coarse correction runs in the host and graph loops only");
            return STG_ERR_INVALID;
        }
        int ndev = 0;
        if(cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        {
            cudaGetLastError();
            stg::set_error("stg_create: no CUDA device");
            return STG_ERR_NO_DEVICE;
        }
        stg_solver* S = new stg_solver();
        S->cfg = c;
        S->stream = (cudaStream_t)c.stream;
        for(auto& e : S->ev)
            if(cudaEventCreate(&e) != cudaSuccess)
            {
                delete S;
                stg::set_error("stg_create: cudaEventCreate failed");
                return STG_ERR_CUDA;
            }
        *out = S;
        return STG_OK;
    })
}

int stg_destroy(stg_handle h)
{
    GUARD({
        if(h) delete h;
        return STG_OK;
    })
}

int stg_mas_init(stg_handle h, int vert_num, int collision_node_offset, const uint32_t* neighbor_start,
                 const uint32_t* neighbor_num, const uint32_t* neighbor_list, int neighbor_list_size,
                 const int32_t* part_map, int part_map_size, const int32_t* real_map)
{
    CHECK_HANDLE(h);
    GUARD({
        if(!neighbor_start || !neighbor_num || (!neighbor_list && neighbor_list_size > 0) || !part_map || !real_map)
        {
            stg::set_error("stg_mas_init: null array");
            return STG_ERR_INVALID;
        }
        return h->mas_init(vert_num, collision_node_offset, neighbor_start, neighbor_num, neighbor_list,
                           neighbor_list_size, part_map, part_map_size, real_map);
    })
}

int stg_convert(stg_handle h, int count, int32_t* rows, int32_t* cols, double* blocks, int* unique_count)
{
    CHECK_HANDLE(h);
    GUARD({
        if(count < 0 || (count > 0 && (!rows || !cols || !blocks)))
        {
            stg::set_error("stg_convert: invalid arguments");
            return STG_ERR_INVALID;
        }
        if(count == 0)
        {
            if(unique_count) *unique_count = 0;
            return STG_OK;
        }
        Solver& S = *h;
        STG_TRY(S.convert(count, rows, cols, blocks, 0));
        const int u = S.bcoo.nnzb;
        STG_CUDA_TRY(cudaMemcpyAsync(rows, S.bcoo.rows.data(), sizeof(int) * u, cudaMemcpyDeviceToDevice, S.stream));
        STG_CUDA_TRY(cudaMemcpyAsync(cols, S.bcoo.cols.data(), sizeof(int) * u, cudaMemcpyDeviceToDevice, S.stream));
        STG_CUDA_TRY(
            cudaMemcpyAsync(blocks, S.bcoo.blocks.data(), sizeof(double) * 9 * u, cudaMemcpyDeviceToDevice, S.stream));
        STG_CUDA_TRY(cudaStreamSynchronize(S.stream));
        if(unique_count) *unique_count = u;
        S.graph_dirty = true;
        return STG_OK;
    })
}

int stg_spmv(stg_handle h, double a, const double* blocks, const int32_t* rows, const int32_t* cols, int nnzb,
             const double* x, double b, double* y, int n)
{
    CHECK_HANDLE(h);
    GUARD({
        if(nnzb < 0 || n < 0 || n % 3 != 0 || (nnzb > 0 && (!blocks || !rows || !cols)) || (n > 0 && (!x || !y)))
        {
            stg::set_error("stg_spmv: invalid arguments");
            return STG_ERR_INVALID;
        }
        Solver& S = *h;
        STG_TRY(S.bind_bcoo(blocks, rows, cols, nnzb, n / 3));
        STG_TRY(S.prepare_spmv());
        STG_TRY(S.spmv(a, x, b, y));
        STG_CUDA_TRY(cudaStreamSynchronize(S.stream));
        S.graph_dirty = true;
        return STG_OK;
    })
}

int stg_mas_assemble(stg_handle h, const double* blocks, const int32_t* rows, const int32_t* cols, int nnzb,
                     int fem_block_offset, const int32_t* contacts, int ncp)
{
    CHECK_HANDLE(h);
    GUARD({
        Solver& S = *h;
        if(nnzb < 0 || ncp < 0 || (ncp > 0 && !contacts) || fem_block_offset < 0)
        {
            stg::set_error("stg_mas_assemble: invalid arguments");
            return STG_ERR_INVALID;
        }
        STG_TRY(S.bind_bcoo(blocks, rows, cols, nnzb, 0));
        STG_TRY(S.mas_build(contacts, ncp));
        STG_TRY(S.mas_assemble(fem_block_offset));
        S.mas_fem_offset = fem_block_offset;
        STG_CUDA_TRY(cudaStreamSynchronize(S.stream));
        S.generation++;
        S.graph_dirty = true;
        return STG_OK;
    })
}

int stg_mas_apply(stg_handle h, const double* r, double* z)
{
    CHECK_HANDLE(h);
    GUARD({
        if(!r || !z)
        {
            stg::set_error("stg_mas_apply: null vector");
            return STG_ERR_INVALID;
        }
        Solver& S = *h;
        STG_TRY(S.mas_apply(r, z));
        STG_CUDA_TRY(cudaStreamSynchronize(S.stream));
        return STG_OK;
    })
}

int stg_pcg_solve(stg_handle h, const double* blocks, const int32_t* rows, const int32_t* cols, int nnzb, const double* b,
                  double* x, int n, stg_stats* stats)
{
    CHECK_HANDLE(h);
    GUARD({
        if(nnzb < 1 || n < 3 || n % 3 != 0 || !blocks || !rows || !cols || !b || !x)
        {
            stg::set_error("stg_pcg_solve: invalid arguments");
            return STG_ERR_INVALID;
        }
        Solver& S = *h;
        if(stats) *stats = stg_stats{};
        STG_TRY(S.bind_bcoo(blocks, rows, cols, nnzb, n / 3));
        STG_TRY(S.prepare_spmv());
        S.generation++;
        const int l0 = S.launches;
        int st = S.pcg_solve(b, x, n, 0, nullptr, stats);
        if(st != STG_OK && st != STG_MAX_ITER) return st;
        if(stats)
        {
            double rel = 0;
            STG_TRY(stg::true_residual(S, b, x, n, &rel));
            stats->rel_residual = rel;
            stats->status = st;
            stats->nnzb = nnzb;
            stats->levels = S.mas.L;
            stats->total_clusters = S.mas.total_clusters;
            stats->kernel_launches = S.launches - l0;
        }
        return st;
    })
}

int stg_solve_linear_system(stg_handle h, const stg_system* sys, double* x, stg_stats* stats)
{
    CHECK_HANDLE(h);
    GUARD({
        Solver& S = *h;
        if(!sys || !x || sys->triplet_count < 1 || !sys->rows || !sys->cols || !sys->blocks || !sys->b || sys->n < 3 ||
           sys->n % 3 != 0 || sys->abd_bodies < 0 || sys->ncp < 0 ||
           (sys->ncp > 0 && !sys->contacts))
        {
            stg::set_error("stg_solve_linear_system: invalid arguments");
            return STG_ERR_INVALID;
        }
        if(stats) *stats = stg_stats{};
        const bool timed = stats != nullptr;
        cudaStream_t s = S.stream;
        const int l0 = S.launches;
        const bool use_mas = S.cfg.preconditioner == STG_PRECOND_MAS;
        if(timed) STG_CUDA_TRY(cudaEventRecord(S.ev[0], s));
        // the MAS hierarchy depends on the mesh and the contacts only: built first, so that the
        // convert can store level 0 and emit the level-1 triplets in the same pass
        if(use_mas) STG_TRY(S.mas_build(sys->contacts, sys->ncp));
        if(timed) STG_CUDA_TRY(cudaEventRecord(S.ev[5], s));
        STG_TRY(S.convert(sys->triplet_count, sys->rows, sys->cols, sys->blocks, sys->n / 3,
                          use_mas ? sys->fem_block_offset : -1));
        STG_TRY(S.prepare_spmv());
        if(timed) STG_CUDA_TRY(cudaEventRecord(S.ev[1], s));
        if(use_mas)
        {
            STG_TRY(S.mas_assemble(sys->fem_block_offset));
            S.mas_fem_offset = sys->fem_block_offset;
        }
        if(timed) STG_CUDA_TRY(cudaEventRecord(S.ev[2], s));
        S.generation++;
        if(timed) STG_CUDA_TRY(cudaEventRecord(S.ev[3], s));
        int st = S.pcg_solve(sys->b, x, sys->n, sys->abd_bodies, sys->abd_inv, stats);
        if(st != STG_OK && st != STG_MAX_ITER) return st;
        if(timed)
        {
            STG_CUDA_TRY(cudaEventRecord(S.ev[4], s));
            double rel = 0;
            STG_TRY(stg::true_residual(S, sys->b, x, sys->n, &rel));
            STG_CUDA_TRY(cudaEventSynchronize(S.ev[4]));
            float t05 = 0, t51 = 0, t13 = 0, t34 = 0, t04 = 0;
            cudaEventElapsedTime(&t05, S.ev[0], S.ev[5]);
            cudaEventElapsedTime(&t51, S.ev[5], S.ev[1]);
            cudaEventElapsedTime(&t13, S.ev[1], S.ev[3]);
            cudaEventElapsedTime(&t34, S.ev[3], S.ev[4]);
            cudaEventElapsedTime(&t04, S.ev[0], S.ev[4]);
            stats->ms_convert = t51;
            stats->ms_mas_build = t05;
            stats->ms_mas_assemble = t13;
            stats->ms_pcg = t34;
            stats->ms_total = t04;
            stats->rel_residual = rel;
            stats->status = st;
            stats->nnzb = S.bcoo.nnzb;
            stats->levels = S.mas.L;
            stats->total_clusters = S.mas.total_clusters;
            stats->kernel_launches = S.launches - l0;
        }
        return st;
    })
}

int stg_mas_info(stg_handle h, int* levels, int* total_clusters, int* level_size)
{
    CHECK_HANDLE(h);
    if(!h->mas.built)
    {
        stg::set_error("MAS hierarchy not built");
        return STG_ERR_NOT_READY;
    }
    if(levels) *levels = h->mas.L;
    if(total_clusters) *total_clusters = h->mas.total_clusters;
    if(level_size) memcpy(level_size, h->mas.level_size, sizeof(int) * 2 * (h->mas.L + 1));
    return STG_OK;
}

int stg_mas_export_hierarchy(stg_handle h, uint32_t* fine_mask, int32_t* prefix_orig, int32_t* coarse_tables,
                             int32_t* going_next, int32_t* coarse_table)
{
    CHECK_HANDLE(h);
    GUARD({
        stg::MasState& m = h->mas;
        if(!m.built)
        {
            stg::set_error("MAS hierarchy not built");
            return STG_ERR_NOT_READY;
        }
        cudaStream_t s = h->stream;
        const int V = m.V, L = m.L;
        if(fine_mask) STG_CUDA_TRY(cudaMemcpyAsync(fine_mask, m.fine_mask.data(), sizeof(unsigned) * V, cudaMemcpyDeviceToHost, s));
        if(prefix_orig)
            STG_CUDA_TRY(cudaMemcpyAsync(prefix_orig, m.prefix_orig.data(), sizeof(int) * m.nb0, cudaMemcpyDeviceToHost, s));
        if(coarse_tables)
            STG_CUDA_TRY(cudaMemcpyAsync(coarse_tables, m.coarse_tables.data(), sizeof(int) * (size_t)L * V,
                                         cudaMemcpyDeviceToHost, s));
        if(going_next)
            STG_CUDA_TRY(cudaMemcpyAsync(going_next, m.going_next.data(), sizeof(int) * (size_t)std::max(m.total_clusters, V),
                                         cudaMemcpyDeviceToHost, s));
        if(coarse_table && L > 1)
            STG_CUDA_TRY(cudaMemcpyAsync(coarse_table, m.coarse_table.data(), sizeof(int) * (size_t)V * (L - 1),
                                         cudaMemcpyDeviceToHost, s));
        STG_CUDA_TRY(cudaStreamSynchronize(s));
        return STG_OK;
    })
}

int stg_mas_export_matrices(stg_handle h, double* mat, float* inv, int* nbanks)
{
    CHECK_HANDLE(h);
    GUARD({
        stg::MasState& m = h->mas;
        if(!m.assembled)
        {
            stg::set_error("MAS not assembled");
            return STG_ERR_NOT_READY;
        }
        const size_t cnt = (size_t)m.nbanks * (m.bank * (m.bank + 1) / 2) * 9;
        if(nbanks) *nbanks = m.nbanks;
        if(mat) STG_CUDA_TRY(cudaMemcpyAsync(mat, m.mat.data(), sizeof(double) * cnt, cudaMemcpyDeviceToHost, h->stream));
        if(inv) STG_CUDA_TRY(cudaMemcpyAsync(inv, m.inv.data(), sizeof(float) * cnt, cudaMemcpyDeviceToHost, h->stream));
        STG_CUDA_TRY(cudaStreamSynchronize(h->stream));
        return STG_OK;
    })
}

}  // extern "C"

namespace stg
{
int profile_spmv(Solver& S, int reps, float* avg_ms, double* bytes);
}

namespace stg
{
int selftest_wait(int* status, double* seconds);
}

extern "C" int stg_selftest_wait_timeout(int* status, double* seconds)
{
    GUARD({
        int dev = 0;
        if(cudaGetDeviceCount(&dev) != cudaSuccess || dev < 1)
        {
            cudaGetLastError();
            stg::set_error("no CUDA device");
            return STG_ERR_NO_DEVICE;
        }
        return stg::selftest_wait(status, seconds);
    })
}

extern "C" int stg_profile_spmv(stg_handle h, int reps, float* avg_ms, double* bytes)
{
    CHECK_HANDLE(h);
    GUARD({
        if(reps < 1)
        {
            stg::set_error("stg_profile_spmv: reps must be >= 1");
            return STG_ERR_INVALID;
        }
        return stg::profile_spmv(*h, reps, avg_ms, bytes);
    })
}

// ---- learned coarse correction ------------------------------------------------------------
namespace
{
int net_graph_of(const stg_net_graph* g, stg::NetGraph& out)
{
    if(!g || g->nodes < 1 || g->entries < 0 || !g->row || (g->entries > 0 && (!g->col || !g->w || !g->oblk)) ||
       !g->dblk || !g->feat)
    {
        stg::set_error("stg_net: invalid graph");
        return STG_ERR_INVALID;
    }
    out.n = g->nodes;
    out.nnz = g->entries;
    out.row = g->row;
    out.col = g->col;
    out.w = g->w;
    out.oblk = g->oblk;
    out.dblk = g->dblk;
    out.feat = g->feat;
    return STG_OK;
}
}  // namespace

int stg_net_configure(stg_handle h, int level)
{
    CHECK_HANDLE(h);
    GUARD({
        if(level < 0 || level >= stg::kMaxLevels)
        {
            stg::set_error("stg_net_configure: level out of range");
            return STG_ERR_INVALID;
        }
        h->learned.level = level;
        h->learned.graph_ready = false;
        h->graph_dirty = true;
        return STG_OK;
    })
}

int stg_net_graph_info(stg_handle h, int* nodes, int* entries)
{
    CHECK_HANDLE(h);
    if(!h->learned.graph_ready)
    {
        stg::set_error("stg_net_graph_info: no graph: configure a level and assemble MAS first");
        return STG_ERR_NOT_READY;
    }
    if(nodes) *nodes = h->learned.graph.n;
    if(entries) *entries = h->learned.graph.nnz;
    return STG_OK;
}

int stg_net_export_graph(stg_handle h, int32_t* row, int32_t* col, float* w, float* oblk, float* dblk, float* feat)
{
    CHECK_HANDLE(h);
    GUARD({
        const stg::NetGraphStore& G = h->learned.graph;
        if(!h->learned.graph_ready)
        {
            stg::set_error("stg_net_export_graph: no graph: configure a level and assemble MAS first");
            return STG_ERR_NOT_READY;
        }
        if(!row || !dblk || !feat || (G.nnz > 0 && (!col || !w || !oblk)))
        {
            stg::set_error("stg_net_export_graph: null buffer");
            return STG_ERR_INVALID;
        }
        cudaStream_t s = h->stream;
        STG_CUDA_TRY(cudaMemcpyAsync(row, G.row.data(), sizeof(int) * (G.n + 1), cudaMemcpyDeviceToDevice, s));
        STG_CUDA_TRY(cudaMemcpyAsync(dblk, G.dblk.data(), sizeof(float) * 9 * G.n, cudaMemcpyDeviceToDevice, s));
        STG_CUDA_TRY(cudaMemcpyAsync(feat, G.feat.data(), sizeof(float) * G.n, cudaMemcpyDeviceToDevice, s));
        if(G.nnz > 0)
        {
            STG_CUDA_TRY(cudaMemcpyAsync(col, G.col.data(), sizeof(int) * G.nnz, cudaMemcpyDeviceToDevice, s));
            STG_CUDA_TRY(cudaMemcpyAsync(w, G.w.data(), sizeof(float) * G.nnz, cudaMemcpyDeviceToDevice, s));
            STG_CUDA_TRY(cudaMemcpyAsync(oblk, G.oblk.data(), sizeof(float) * 9 * G.nnz, cudaMemcpyDeviceToDevice, s));
        }
        return STG_OK;
    })
}

int stg_net_record(stg_handle h, float* rc, float* zc, int capacity, int every)
{
    CHECK_HANDLE(h);
    GUARD({
        if(capacity < 0 || (capacity > 0 && (!rc || !zc || every < 1)))
        {
            stg::set_error("stg_net_record: invalid buffers, capacity or interval");
            return STG_ERR_INVALID;
        }
        stg::LearnedState& L = h->learned;
        STG_TRY(L.rec_count.resize(1));
        STG_CUDA_TRY(cudaMemsetAsync(L.rec_count.data(), 0, sizeof(int), h->stream));
        L.rec_rc = capacity > 0 ? rc : nullptr;
        L.rec_zc = capacity > 0 ? zc : nullptr;
        L.rec_cap = capacity;
        L.rec_every = capacity > 0 ? every : 0;
        return STG_OK;
    })
}

int stg_net_recorded(stg_handle h, int* count)
{
    CHECK_HANDLE(h);
    GUARD({
        if(!count)
        {
            stg::set_error("stg_net_recorded: count is null");
            return STG_ERR_INVALID;
        }
        *count = 0;
        if(h->learned.rec_count.data())
        {
            STG_CUDA_TRY(cudaMemcpyAsync(count, h->learned.rec_count.data(), sizeof(int), cudaMemcpyDeviceToHost, h->stream));
            STG_CUDA_TRY(cudaStreamSynchronize(h->stream));
        }
        return STG_OK;
    })
}

int stg_net_set_params(stg_handle h, const float* params)
{
    CHECK_HANDLE(h);
    GUARD({
        if(!params)
        {
            stg::set_error("stg_net_set_params: params is null");
            return STG_ERR_INVALID;
        }
        stg::LearnedState& L = h->learned;
        STG_TRY(L.params.resize(stg::P_COUNT));
        STG_TRY(L.wbf.resize(2 * stg::P_COUNT));
        STG_CUDA_TRY(cudaMemcpyAsync(L.params.data(), params, sizeof(float) * stg::P_COUNT, cudaMemcpyDeviceToDevice,
                                     h->stream));
        STG_TRY(stg::net_to_bf16(h->stream, L.params.data(), L.wbf.data()));
        L.has_params = true;
        return STG_OK;
    })
}

size_t stg_net_scratch_bytes(int nodes, int samples)
{
    if(nodes < 1 || samples < 1) return 0;
    return stg::net_scratch_bytes(nodes, samples);
}

int stg_net_forward(const stg_net_graph* g, const float* rc, const float* zc, int samples, const float* params,
                    float* delta, void* scratch, size_t scratch_bytes, void* stream)
{
    GUARD({
        stg::NetGraph G;
        STG_TRY(net_graph_of(g, G));
        if(!rc || !zc || !params || !delta || samples < 1)
        {
            stg::set_error("stg_net_forward: invalid arguments");
            return STG_ERR_INVALID;
        }
        stg::NetBuffers b;
        STG_TRY(stg::net_carve(scratch, scratch_bytes, G.n, samples, b));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        int l = 0;
        STG_TRY(stg::net_to_bf16(s, params, b.wbf));
        STG_TRY(stg::net_forward(s, G, rc, zc, samples, b, b.wbf, params, nullptr, nullptr, &l));
        STG_CUDA_TRY(cudaMemcpyAsync(delta, b.delta, sizeof(float) * 4 * (size_t)G.n * samples, cudaMemcpyDeviceToDevice, s));
        return STG_OK;
    })
}

int stg_net_train_step(const stg_net_graph* g, const float* rc, const float* zc, int samples, float* params,
                       float* grad, float* adam_m, float* adam_v, int step, float lr, float* loss, void* scratch,
                       size_t scratch_bytes, void* stream)
{
    GUARD({
        stg::NetGraph G;
        STG_TRY(net_graph_of(g, G));
        if(!rc || !zc || !params || !grad || samples < 1 || !(lr >= 0.f) || (lr > 0.f && (!adam_m || !adam_v || step < 1)))
        {
            stg::set_error("stg_net_train_step: invalid arguments");
            return STG_ERR_INVALID;
        }
        stg::NetBuffers b;
        STG_TRY(stg::net_carve(scratch, scratch_bytes, G.n, samples, b));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        int l = 0;
        STG_TRY(stg::net_train_step(s, G, rc, zc, samples, b, params, grad, adam_m, adam_v, step, lr, &l));
        if(loss) STG_CUDA_TRY(cudaMemcpyAsync(loss, b.loss, sizeof(float) * samples, cudaMemcpyDeviceToDevice, s));
        return STG_OK;
    })
}

int stg_net_apply(const stg_net_graph* g, const float* rc, float* z, const float* params, void* scratch,
                  size_t scratch_bytes, int* fused, void* stream)
{
    GUARD({
        stg::NetGraph G;
        STG_TRY(net_graph_of(g, G));
        if(!rc || !z || !params)
        {
            stg::set_error("stg_net_apply: invalid arguments");
            return STG_ERR_INVALID;
        }
        stg::NetBuffers b;
        STG_TRY(stg::net_carve(scratch, scratch_bytes, G.n, 1, b));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        std::vector<int> row(G.n + 1);
        STG_CUDA_TRY(cudaMemcpyAsync(row.data(), G.row, sizeof(int) * (G.n + 1), cudaMemcpyDeviceToHost, s));
        STG_CUDA_TRY(cudaStreamSynchronize(s));
        int cl = 0, rpc = 0;
        STG_TRY(stg::net_fused_plan(row.data(), G.n, &cl, &rpc));
        STG_TRY(stg::net_prepare());
        STG_TRY(stg::net_to_bf16(s, params, b.wbf));
        int l = 0;
        if(cl > 0)
            STG_TRY(stg::net_forward_fused(s, G, nullptr, rc, z, b.wbf, params, nullptr, cl, rpc));
        else
            STG_TRY(stg::net_forward(s, G, rc, z, 1, b, b.wbf, params, z, nullptr, &l));
        if(fused) *fused = cl;
        return STG_OK;
    })
}

int stg_spmv_tiles(stg_handle h, int rows_per_tile)
{
    CHECK_HANDLE(h);
    const bool fp32 = h->cfg.precision == STG_PREC_FP32;
    const bool ok = rows_per_tile == 0 || rows_per_tile == -1 || rows_per_tile == -2 || rows_per_tile == -3 ||
                    (fp32 ? (rows_per_tile == 64 || rows_per_tile == 32) : (rows_per_tile == 32 || rows_per_tile == 16));
    if(!ok)
    {
        stg::set_error("stg_spmv_tiles: rows per tile must be 0 (autotune), -1 (default), -2 (halo kernel), -3 (upper "
                       "kernel), 64 or 32 (FP32), 32 or 16 (FP64)");
        return STG_ERR_INVALID;
    }
    h->spmv_rt = (rows_per_tile == -2 || rows_per_tile == -3) ? rows_per_tile : (rows_per_tile > 0 ? rows_per_tile : 0);
    h->spmv_tune = rows_per_tile == 0;
    h->tuned_prec = -1;
    return STG_OK;
}

int stg_spmv_tiles_info(stg_handle h, int* rows_per_tile, float* us_default, float* us_alternative, float* us_halo,
                        float* us_upper)
{
    CHECK_HANDLE(h);
    if(rows_per_tile)
        *rows_per_tile = h->pcg_ready ? (h->pcg_dev.upper ? -3 : (h->pcg_dev.halo ? -2 : h->pcg_dev.a_rt)) : -1;
    if(us_default) *us_default = h->tune_us[0];
    if(us_alternative) *us_alternative = h->tune_us[1];
    if(us_halo) *us_halo = h->tune_us[2];
    if(us_upper) *us_upper = h->tune_us[3];
    return STG_OK;
}

size_t stg_fem_scratch_bytes(int verts, int tets)
{
    if(verts < 1 || tets < 0) return 0;
    return stg::fem_scratch_bytes(verts, tets);
}

int stg_fem_newton_system(int verts, const double* rest, const double* pos, const double* vel,
                          const double* xtilde, int tets, const int32_t* tet_verts, const double* youngs,
                          double poisson, double density, double dt, double gravity_y, int nplanes,
                          const double* planes, int32_t* rows, int32_t* cols, double* blocks, double* b,
                          void* scratch, size_t scratch_bytes, void* stream)
{
    GUARD({
        return stg::fem_newton_system(static_cast<cudaStream_t>(stream), verts, rest, pos, vel, xtilde, tets, tet_verts,
                                      youngs, poisson, density, dt, gravity_y, nplanes, planes, rows, cols, blocks, b,
                                      scratch, scratch_bytes);
    })
}

int stg_fem_energy(int verts, const double* rest, const double* pos, const double* xtilde, int tets,
                   const int32_t* tet_verts, const double* youngs, double poisson, double density, double dt,
                   int nplanes, const double* planes, void* scratch, size_t scratch_bytes, double* energy,
                   int* violations, void* stream)
{
    GUARD({
        return stg::fem_energy(static_cast<cudaStream_t>(stream), verts, rest, pos, xtilde, tets, tet_verts, youngs,
                               poisson, density, dt, nplanes, planes, scratch, scratch_bytes, energy, violations);
    })
}

int stg_set_segments(stg_handle h, const int32_t* row_offsets, int nseg)
{
    CHECK_HANDLE(h);
    GUARD({
        if(nseg < 0 || (nseg > 0 && !row_offsets))
        {
            stg::set_error("stg_set_segments: invalid arguments");
            return STG_ERR_INVALID;
        }
        if(nseg == 0)
        {
            h->nseg = 0;
            h->seg_off_host.clear();
            return STG_OK;
        }
        if(row_offsets[0] != 0)
        {
            stg::set_error("stg_set_segments: the first offset must be 0");
            return STG_ERR_INVALID;
        }
        for(int q = 0; q < nseg; q++)
            if(row_offsets[q + 1] <= row_offsets[q])
            {
                stg::set_error("stg_set_segments: offsets must increase");
                return STG_ERR_INVALID;
            }
        const int nrows = row_offsets[nseg];
        std::vector<int> of(nrows);
        for(int q = 0; q < nseg; q++)
            for(int r = row_offsets[q]; r < row_offsets[q + 1]; r++) of[r] = q;
        STG_TRY(h->seg_off.resize(nseg + 1));
        STG_TRY(h->seg_of_row.resize(nrows));
        STG_CUDA_TRY(cudaMemcpyAsync(h->seg_off.data(), row_offsets, sizeof(int) * (nseg + 1), cudaMemcpyHostToDevice, h->stream));
        STG_CUDA_TRY(cudaMemcpyAsync(h->seg_of_row.data(), of.data(), sizeof(int) * nrows, cudaMemcpyHostToDevice, h->stream));
        STG_CUDA_TRY(cudaStreamSynchronize(h->stream));
        h->seg_off_host.assign(row_offsets, row_offsets + nseg + 1);
        h->nseg = nseg;
        h->graph_dirty = true;
        return STG_OK;
    })
}

int stg_segment_stats(stg_handle h, int* iterations, double* rel_residual)
{
    CHECK_HANDLE(h);
    if(h->nseg == 0 || h->seg_host.size() < (size_t)stg::SEG_N * h->nseg)
    {
        stg::set_error("stg_segment_stats: no scenes solved");
        return STG_ERR_NOT_READY;
    }
    for(int q = 0; q < h->nseg; q++)
    {
        const double* S = h->seg_host.data() + (size_t)stg::SEG_N * q;
        if(iterations) iterations[q] = (int)S[stg::SG_ITER];
        if(rel_residual) rel_residual[q] = S[stg::SG_BB] > 0 ? std::sqrt(S[stg::SG_RR] / S[stg::SG_BB]) : 0.0;
    }
    return STG_OK;
}
