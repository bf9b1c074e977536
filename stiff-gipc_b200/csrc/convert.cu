// convert.cu -- triplets -> sorted unique upper BCOO on sm_100a.
//
// Replaces Converter::srbk_convert (StiffGIPC/linear_system/utils/converter.cu:32-51,88-238):
// the reference builds a 64-bit key (row<<32)+col, radix-sorts key/index pairs with cub,
// flags segment heads, scans, scatters row/col and sums each segment with a warp
// segmented reduce plus FP64 atomics (fast_segmental_reduce.inl:20-94), then copies the
// unique count to the host.
//
// Here the same result is produced by a counting sort on the row (histogram -> scan ->
// scatter), a per-row sort on (col, original index) (a warp per row of up to 128 entries, a
// CTA per longer row), and a per-row emit that sums duplicate blocks in original triplet
// order.  No atomics touch the values, so the output
// is bitwise deterministic; the summation order (input order) equals that of a stable
// sort followed by a sequential sum.
#include "solver.hpp"
#include "mas_index.cuh"

namespace stg
{

// largest block index among rows and cols (the block dimension when the caller gives none)
__global__ void k_conv_max_row(const int* rows, const int* cols, int count, int* max_row)
{
    int m = -1;
    for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        m = max(m, max(rows[i], cols[i]));
#pragma unroll
    for(int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if((threadIdx.x & 31) == 0) atomicMax(max_row, m);
}

// Row histogram.  Triplets whose row or col lies outside [0, nrows) are counted in *bad
// (the caller gets STG_ERR_INVALID) and never used as an index.
__global__ void k_conv_hist(const int* rows, const int* cols, int count, int nrows, bool skip_negative, int* row_cnt,
                            int* bad)
{
    for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    {
        const int r = rows[i], c = cols[i];
        if(skip_negative && r < 0) continue;
        if(r < 0 || r >= nrows || c < 0 || c >= nrows)
            atomicAdd(bad, 1);
        else
            atomicAdd(row_cnt + r, 1);
    }
}

// counting-sort scatter by row; each slot gets the triplet's index and its column, so the
// per-row sort reads its keys contiguously
__global__ void k_conv_scatter(const int* rows, const int* cols, int count, int nrows, const int* row_start, int* cursor,
                               int* perm, int* pcol)
{
    for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    {
        const int r = rows[i], c = cols[i];
        if(r < 0 || r >= nrows || c < 0 || c >= nrows) continue;
        const int pos = row_start[r] + atomicAdd(cursor + r, 1);
        perm[pos] = i;
        pcol[pos] = c;
    }
}

// One warp per row: order every entry by (col, original index), write the sorted permutation
// and sorted cols, and count distinct cols.  Rows of up to 128 entries are sorted by a
// bitonic network on 64-bit keys (col << 32 | index; 4 keys per lane, position 4 * lane + h);
// longer rows are listed for k_conv_sort_long, which sorts each with a whole CTA.  The keys
// are unique, so every path gives the same permutation.
constexpr int CONV_WARPS = 8;

__device__ __forceinline__ unsigned long long shfl_xor_u64(unsigned long long v, int m)
{
    const unsigned lo = __shfl_xor_sync(0xffffffffu, (unsigned)v, m);
    const unsigned hi = __shfl_xor_sync(0xffffffffu, (unsigned)(v >> 32), m);
    return ((unsigned long long)hi << 32) | lo;
}

__global__ void __launch_bounds__(32 * CONV_WARPS) k_conv_sort_rows(const int* pcol, const int* row_start,
                                                                    const int* perm_in, int* perm_out, int* scol,
                                                                    int* uniq, int nrows, int* long_rows,
                                                                    int* long_cnt)
{
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for(int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nrows; r += warps)
    {
        const int s = row_start[r], e = row_start[r + 1], n = e - s;
        if(n <= 128)
        {
            unsigned long long k[4];
#pragma unroll
            for(int h = 0; h < 4; h++)
            {
                const int p = 4 * lane + h;
                k[h] = ~0ull;
                if(p < n) k[h] = ((unsigned long long)(unsigned)pcol[s + p] << 32) | (unsigned)perm_in[s + p];
            }
#pragma unroll
            for(int kk = 2; kk <= 128; kk <<= 1)
            {
#pragma unroll
                for(int d = kk >> 1; d >= 1; d >>= 1)
                {
                    if(d >= 4)
                    {
#pragma unroll
                        for(int h = 0; h < 4; h++)
                        {
                            const int p = 4 * lane + h;
                            const unsigned long long o = shfl_xor_u64(k[h], d >> 2);
                            const bool up = (p & kk) == 0, lower = (p & d) == 0;
                            k[h] = (up == lower) ? (k[h] < o ? k[h] : o) : (k[h] < o ? o : k[h]);
                        }
                    }
                    else
                    {
#pragma unroll
                        for(int h = 0; h < 4; h++)
                        {
                            if(h & d) continue;
                            const int p = 4 * lane + h;
                            const bool up = (p & kk) == 0;
                            const unsigned long long x = k[h], y = k[h + d];
                            const bool sw = up ? (x > y) : (x < y);
                            k[h] = sw ? y : x;
                            k[h + d] = sw ? x : y;
                        }
                    }
                }
            }
#pragma unroll
            for(int h = 0; h < 4; h++)
            {
                const int p = 4 * lane + h;
                if(p < n)
                {
                    perm_out[s + p] = (int)(unsigned)k[h];
                    scol[s + p] = (int)(k[h] >> 32);
                }
            }
        }
        else
        {
            if(lane == 0) long_rows[atomicAdd(long_cnt, 1)] = r;
            continue;
        }
        __syncwarp();
        int heads = 0;
        for(int a = lane; a < n; a += 32) heads += (a == 0 || scol[s + a] != scol[s + a - 1]);
#pragma unroll
        for(int o = 16; o > 0; o >>= 1) heads += __shfl_xor_sync(0xffffffffu, heads, o);
        if(lane == 0) uniq[r] = heads;
        __syncwarp();
    }
}

// Rows of more than 128 entries, one CTA each: a bitonic sort of the 64-bit keys in shared
// memory (up to CONV_LONG_CAP entries), else ranking against the row in global memory;
// then the distinct cols are counted.
constexpr int CONV_LONG_THREADS = 256;
constexpr int CONV_LONG_CAP = 4096;

__global__ void __launch_bounds__(CONV_LONG_THREADS) k_conv_sort_long(const int* pcol, const int* row_start,
                                                                      const int* perm_in, int* perm_out, int* scol,
                                                                      int* uniq, const int* long_rows,
                                                                      const int* long_cnt)
{
    __shared__ unsigned long long key[CONV_LONG_CAP];
    __shared__ int heads;
    const int nl = *long_cnt, t = threadIdx.x;
    for(int i = blockIdx.x; i < nl; i += gridDim.x)
    {
        const int r = long_rows[i];
        const int s = row_start[r], n = row_start[r + 1] - s;
        if(t == 0) heads = 0;
        if(n <= CONV_LONG_CAP)
        {
            int P = 1;
            while(P < n) P <<= 1;
            for(int a = t; a < P; a += CONV_LONG_THREADS)
                key[a] = a < n ? ((unsigned long long)(unsigned)pcol[s + a] << 32) | (unsigned)perm_in[s + a] : ~0ull;
            __syncthreads();
            for(int k = 2; k <= P; k <<= 1)
                for(int j = k >> 1; j > 0; j >>= 1)
                {
                    for(int a = t; a < P; a += CONV_LONG_THREADS)
                    {
                        const int b = a ^ j;
                        if(b > a)
                        {
                            const unsigned long long x = key[a], y = key[b];
                            if((x > y) == ((a & k) == 0)) key[a] = y, key[b] = x;
                        }
                    }
                    __syncthreads();
                }
            int h = 0;
            for(int a = t; a < n; a += CONV_LONG_THREADS)
            {
                perm_out[s + a] = (int)(unsigned)key[a];
                scol[s + a] = (int)(key[a] >> 32);
                h += a == 0 || (key[a] >> 32) != (key[a - 1] >> 32);
            }
            atomicAdd(&heads, h);
        }
        else
        {
            for(int a = t; a < n; a += CONV_LONG_THREADS)
            {
                const int ia = perm_in[s + a], ca = pcol[s + a];
                int rank = 0;
                for(int b = 0; b < n; b++)
                {
                    const int ib = perm_in[s + b], cb = pcol[s + b];
                    rank += (cb < ca) || (cb == ca && ib < ia);
                }
                perm_out[s + rank] = ia;
                scol[s + rank] = ca;
            }
            __syncthreads();
            int h = 0;
            for(int a = t; a < n; a += CONV_LONG_THREADS) h += a == 0 || scol[s + a] != scol[s + a - 1];
            atomicAdd(&heads, h);
        }
        __syncthreads();
        if(t == 0) uniq[r] = heads;
        __syncthreads();
    }
}

// One warp per row: each lane owns a run of equal cols (a unique block) and sums it in
// sorted (= original) order.  Rows of up to CONV_EMIT_CAP entries first stage their blocks
// (in sorted order) in shared memory with independent loads, so the sequential sums read
// shared memory; longer rows sum from global memory.  The sums are the same either way.
constexpr int CONV_EMIT_WARPS = 4;
constexpr int CONV_EMIT_CAP = 128;

// the fused level-0 pass for unique block o = (r, c) with sum acc (ConvFuse)
__device__ __forceinline__ void fuse_block(const ConvFuse& F, int r, int c, const double* acc, int o)
{
    const int rr = r - F.offset, cc = c - F.offset;
    const bool in = rr >= 0 && rr < F.V && cc >= 0 && cc < F.V;
    bool lower_in_bank = false;
    if(in)
    {
        const int sc = F.real_map[cc], sr = F.real_map[rr];
        if(sc / F.B == sr / F.B)
        {
            if(sc >= sr)
            {
                double* D = F.mat + ((size_t)(sc / F.B) * F.NS + upper_index(F.B, sr % F.B, sc % F.B)) * 9;
#pragma unroll
                for(int e = 0; e < 9; e++) D[e] = acc[e];
            }
            else
                lower_in_bank = true;
        }
    }
    if(F.c1)
    {
        if(!in || lower_in_bank)
        {
            F.trow[o] = -1;
            F.tcol[o] = 0;
        }
        else
            coarse_triplet(rr, cc, F.c1[rr], F.c1[cc], acc, F.trow + o, F.tcol + o, F.tblk + 9 * (size_t)o);
    }
}

__global__ void __launch_bounds__(32 * CONV_EMIT_WARPS) k_conv_emit(const double* blocks, const int* row_start,
                                                                    const int* perm, const int* scol,
                                                                    const int* ustart, int* out_rows, int* out_cols,
                                                                    double* out_blocks, int nrows, ConvFuse F)
{
    extern __shared__ double ebuf[];  // [CONV_EMIT_WARPS][CONV_EMIT_CAP * 9]
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double* sb = ebuf + (size_t)w * CONV_EMIT_CAP * 9;
    for(int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nrows; r += warps)
    {
        const int s = row_start[r], e = row_start[r + 1], n = e - s;
        const bool staged = n <= CONV_EMIT_CAP;
        if(staged)
        {
            for(int a = lane; a < n; a += 32)
            {
                const double* b0 = blocks + 9 * (size_t)perm[s + a];
#pragma unroll
                for(int t = 0; t < 9; t++) sb[9 * a + t] = b0[t];
            }
            __syncwarp();
        }
        if(!staged)
        {
            // a long row: the warp loads 32 entries at a time and every lane accumulates the
            // runs in sorted order from the shuffled values (the same sums as one lane walking
            // the run); lane 0 writes each finished run
            double acc[9];
            int cur = -1, o = ustart[r] - 1;
            for(int a0 = 0; a0 < n; a0 += 32)
            {
                const int a = a0 + lane;
                int col = -1;
                double v[9];
#pragma unroll
                for(int t = 0; t < 9; t++) v[t] = 0.0;
                if(a < n)
                {
                    col = scol[s + a];
                    const double* b0 = blocks + 9 * (size_t)perm[s + a];
#pragma unroll
                    for(int t = 0; t < 9; t++) v[t] = b0[t];
                }
                const int m = min(32, n - a0);
                for(int j = 0; j < m; j++)
                {
                    const int cj = __shfl_sync(0xffffffffu, col, j);
                    if(cj != cur)
                    {
                        if(cur >= 0 && lane == 0)
                        {
                            out_rows[o] = r;
                            out_cols[o] = cur;
#pragma unroll
                            for(int t = 0; t < 9; t++) out_blocks[9 * (size_t)o + t] = acc[t];
                            if(F.B) fuse_block(F, r, cur, acc, o);
                        }
                        o++;
                        cur = cj;
#pragma unroll
                        for(int t = 0; t < 9; t++) acc[t] = __shfl_sync(0xffffffffu, v[t], j);
                    }
                    else
                    {
#pragma unroll
                        for(int t = 0; t < 9; t++) acc[t] += __shfl_sync(0xffffffffu, v[t], j);
                    }
                }
            }
            if(cur >= 0 && lane == 0)
            {
                out_rows[o] = r;
                out_cols[o] = cur;
#pragma unroll
                for(int t = 0; t < 9; t++) out_blocks[9 * (size_t)o + t] = acc[t];
                if(F.B) fuse_block(F, r, cur, acc, o);
            }
            __syncwarp();
            continue;
        }
        int base = 0;
        for(int a0 = 0; a0 < n; a0 += 32)
        {
            const int a = a0 + lane;
            const bool head = a < n && (a == 0 || scol[s + a] != scol[s + a - 1]);
            const unsigned hm = __ballot_sync(0xffffffffu, head);
            if(head)
            {
                const int o = ustart[r] + base + __popc(hm & lanemask_lt(lane));
                double acc[9];
#pragma unroll
                for(int t = 0; t < 9; t++) acc[t] = sb[9 * a + t];
                for(int c = a + 1; c < n && scol[s + c] == scol[s + a]; c++)
                {
#pragma unroll
                    for(int t = 0; t < 9; t++) acc[t] += sb[9 * c + t];
                }
                out_rows[o] = r;
                out_cols[o] = scol[s + a];
#pragma unroll
                for(int t = 0; t < 9; t++) out_blocks[9 * (size_t)o + t] = acc[t];
                if(F.B) fuse_block(F, r, scol[s + a], acc, o);
            }
            base += __popc(hm);
        }
        __syncwarp();
    }
}

// Sort/merge `count` triplets into unique (row, col) blocks written to out_* (row_ptr gets the
// CSR offsets).  Triplets with row < 0 are skipped when skip_negative is set (used to mask
// entries); any other row or col outside [0, nrows) is an error.  Returns the unique count
// through *unique (one device->host read).
int convert_into(Solver& S, ConvertScratch& cv, int count, const int* rows, const int* cols, const double* blocks,
                 int nrows, bool skip_negative, DBuf<int>& out_rows, DBuf<int>& out_cols, DBuf<double>& out_blocks,
                 DBuf<int>& row_ptr, int* unique, bool fuse)
{
    cudaStream_t s = S.stream;
    *unique = 0;
    STG_TRY(row_ptr.resize(nrows + 1));
    STG_TRY(cv.scratch.resize(4));
    if(count < 1 || nrows < 1)
    {
        STG_CUDA_TRY(cudaMemsetAsync(row_ptr.data(), 0, sizeof(int) * (nrows + 1), s));
        return 0;
    }
    STG_TRY(cv.row_cnt.resize(nrows + 1));
    STG_TRY(cv.row_start.resize(nrows + 1));
    STG_TRY(cv.cursor.resize(nrows + 1));
    STG_TRY(cv.perm.resize(count));
    STG_TRY(cv.perm2.resize(count));
    STG_TRY(cv.scol.resize(count));
    STG_TRY(cv.pcol.resize(count));
    STG_TRY(cv.uniq.resize(nrows + 1));
    STG_TRY(cv.long_rows.resize(nrows + 1));
    STG_TRY(out_rows.resize(count));
    STG_TRY(out_cols.resize(count));
    STG_TRY(out_blocks.resize((size_t)count * 9));

    STG_CUDA_TRY(cudaMemsetAsync(cv.row_cnt.data(), 0, sizeof(int) * (nrows + 1), s));
    STG_CUDA_TRY(cudaMemsetAsync(cv.cursor.data(), 0, sizeof(int) * (nrows + 1), s));
    STG_CUDA_TRY(cudaMemsetAsync(cv.scratch.data() + 2, 0, 2 * sizeof(int), s));
    const int g = std::min(div_up(count, 256), kSMs * 16);
    k_conv_hist<<<g, 256, 0, s>>>(rows, cols, count, nrows, skip_negative, cv.row_cnt.data(), cv.scratch.data() + 2);
    STG_LAUNCH_CHECK();
    k_scan_exclusive<<<1, 1024, 0, s>>>(cv.row_cnt.data(), cv.row_start.data(), nullptr, nrows + 1, cv.scratch.data());
    STG_LAUNCH_CHECK();
    k_conv_scatter<<<g, 256, 0, s>>>(rows, cols, count, nrows, cv.row_start.data(), cv.cursor.data(), cv.perm.data(),
                                     cv.pcol.data());
    STG_LAUNCH_CHECK();
    const int gw = std::min(div_up((long)nrows * 32, 32 * CONV_WARPS), kSMs * 16);
    k_conv_sort_rows<<<gw, 32 * CONV_WARPS, 0, s>>>(cv.pcol.data(), cv.row_start.data(), cv.perm.data(), cv.perm2.data(),
                                                    cv.scol.data(), cv.uniq.data(), nrows, cv.long_rows.data(),
                                                    cv.scratch.data() + 3);
    STG_LAUNCH_CHECK();
    k_conv_sort_long<<<kSMs, CONV_LONG_THREADS, 0, s>>>(cv.pcol.data(), cv.row_start.data(), cv.perm.data(),
                                                        cv.perm2.data(), cv.scol.data(), cv.uniq.data(),
                                                        cv.long_rows.data(), cv.scratch.data() + 3);
    STG_LAUNCH_CHECK();
    STG_CUDA_TRY(cudaMemsetAsync(cv.uniq.data() + nrows, 0, sizeof(int), s));
    k_scan_exclusive<<<1, 1024, 0, s>>>(cv.uniq.data(), row_ptr.data(), nullptr, nrows + 1, cv.scratch.data() + 1);
    STG_LAUNCH_CHECK();
    int h[2] = {0, 0};
    ConvFuse F;
    if(fuse)
    {
        // the fused level-0 pass needs the unique count first (its level-1 triplet arrays)
        STG_CUDA_TRY(cudaMemcpyAsync(h, cv.scratch.data() + 1, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
        STG_CUDA_TRY(cudaStreamSynchronize(s));
        if(h[1] != 0)
        {
            set_error("convert: " + std::to_string(h[1]) + " triplets have a row or col outside [0, " +
                      std::to_string(nrows) + ")");
            return STG_ERR_INVALID;
        }
        MasState& m = S.mas;
        F.B = m.bank;
        F.NS = nsym(m.bank);
        F.offset = m.l0_offset;
        F.V = m.V;
        F.real_map = m.real_map.data();
        const size_t nvals = (size_t)m.nbanks * F.NS * 9;
        STG_TRY(m.mat.resize(nvals));
        STG_CUDA_TRY(cudaMemsetAsync(m.mat.data(), 0, nvals * sizeof(double), s));
        F.mat = m.mat.data();
        if(m.L > 1 && h[0] > 0)
        {
            STG_TRY(m.tr_rows.resize(h[0]));
            STG_TRY(m.tr_cols.resize(h[0]));
            STG_TRY(m.tr_blocks.resize((size_t)h[0] * 9));
            F.c1 = m.coarse_tables.data();
            F.trow = m.tr_rows.data();
            F.tcol = m.tr_cols.data();
            F.tblk = m.tr_blocks.data();
        }
    }
    const int ge = std::min(div_up((long)nrows * 32, 32 * CONV_EMIT_WARPS), kSMs * 32);
    k_conv_emit<<<ge, 32 * CONV_EMIT_WARPS, sizeof(double) * CONV_EMIT_WARPS * CONV_EMIT_CAP * 9, s>>>(
        blocks, cv.row_start.data(), cv.perm2.data(), cv.scol.data(), row_ptr.data(), out_rows.data(), out_cols.data(),
        out_blocks.data(), nrows, F);
    STG_LAUNCH_CHECK();
    S.launches += 7;
    if(!fuse)
    {
        STG_CUDA_TRY(cudaMemcpyAsync(h, cv.scratch.data() + 1, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
        STG_CUDA_TRY(cudaStreamSynchronize(s));
        if(h[1] != 0)
        {
            set_error("convert: " + std::to_string(h[1]) + " triplets have a row or col outside [0, " +
                      std::to_string(nrows) + ")");
            return STG_ERR_INVALID;
        }
    }
    *unique = h[0];
    return 0;
}

int Solver::convert(int count, const int* rows, const int* cols, const double* blocks, int nrows_hint, int fuse_offset)
{
    cudaStream_t s = stream;
    bcoo.nnzb = 0;
    if(count < 1) return 0;
    int nrows = nrows_hint;
    if(nrows <= 0)
    {
        STG_TRY(cv.scratch.resize(4));
        STG_CUDA_TRY(cudaMemsetAsync(cv.scratch.data(), 0xff, sizeof(int), s));
        k_conv_max_row<<<std::min(div_up(count, 256), 1184), 256, 0, s>>>(rows, cols, count, cv.scratch.data());
        STG_LAUNCH_CHECK();
        int mr = -1;
        STG_CUDA_TRY(cudaMemcpyAsync(&mr, cv.scratch.data(), sizeof(int), cudaMemcpyDeviceToHost, s));
        STG_CUDA_TRY(cudaStreamSynchronize(s));
        nrows = mr + 1;
        launches += 1;
    }
    int total = 0;
    const bool fuse = fuse_offset >= 0 && mas.built && mas.V > 0;
    mas.l0_fused = false;
    if(fuse) mas.l0_offset = fuse_offset;
    STG_TRY(convert_into(*this, cv, count, rows, cols, blocks, nrows, false, bcoo.rows, bcoo.cols, bcoo.blocks,
                         bcoo.row_ptr, &total, fuse));
    mas.l0_fused = fuse;
    bcoo.nnzb = total;
    bcoo.nrows = nrows;
    bcoo.external = false;
    bcoo.row_ptr_valid = true;
    return 0;
}

}  // namespace stg
