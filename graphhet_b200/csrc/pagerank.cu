// PageRank, pull form over the in-CSR (replaces GPU_PR_csr.cuh:34-197;
// semantics of CPU_PageRank.hpp:12-56):
//   S       = sum of rank[u] over vertices with no out-edges
//   rank'[v] = (1-d)/N + d*S/N + d * sum_{u in in(v)} rank[u] / outdeg(u)
//
// Per iteration one pass reads in_rowptr and in_col once and gathers
// contrib[u] = rank[u] / outdeg(u) (precomputed once per vertex, so the
// per-entry division of the CPU path becomes a per-vertex one with the same
// FP64 result).  The same pass writes rank' and the next contrib, and block
// partials of the next S and of the L1 change; a one-block kernel reduces the
// partials in a fixed order (deterministic S and norm, FP64 in both modes).
//
// Rows of up to 32 entries are summed by one thread each; longer rows are
// cut into 256-entry chunks summed by one warp each and combined per row in
// chunk order.  Both kernels serve the hubs' contributions from a shared-
// memory cache (a degree-relabelled graph puts the hubs first).
//
// FP32 mode: ranks and contributions are stored as float (half the gather
// footprint: 64 MiB at n = 2^24, resident in the 126 MB L2); each lane keeps
// a Kahan-compensated FP32 sum and lanes are merged with an error-free
// TwoSum; the row total, S and the L1 norm are FP64.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "scan.cuh"

namespace ghb {
namespace {

constexpr int kPrThreads = 256;

template <class T>
struct KSum;  // per-lane accumulator

template <>
struct KSum<double> {
    double s = 0.0;
    __device__ __forceinline__ void add(double x) { s += x; }
    __device__ __forceinline__ void merge_from_lane(int offset, int width) {
        s += __shfl_down_sync(0xffffffffu, s, offset, width);
    }
    __device__ __forceinline__ double value() const { return s; }
};

template <>
struct KSum<float> {
    float s = 0.f, c = 0.f;  // true sum ~= s - c
    __device__ __forceinline__ void add(float x) {
        const float y = x - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ void merge_from_lane(int offset, int width) {
        const float s2 = __shfl_down_sync(0xffffffffu, s, offset, width);
        const float c2 = __shfl_down_sync(0xffffffffu, c, offset, width);
        // TwoSum: t + err == s + s2 exactly.
        const float t = s + s2;
        const float bp = t - s;
        const float err = (s - (t - bp)) + (s2 - bp);
        s = t;
        c = c + c2 - err;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

template <class T>
__device__ __forceinline__ T load_contrib(const T* p, uint64_t pol);
template <>
__device__ __forceinline__ double load_contrib<double>(const double* p, uint64_t pol) {
    return ld_keep_f64(p, pol);
}
template <>
__device__ __forceinline__ float load_contrib<float>(const float* p, uint64_t pol) {
    return ld_keep_f32(p, pol);
}

struct PrScalars {
    double base;  // (1-d)/N + d*S/N for the current iteration
    double l1;    // L1 change of the last iteration
    double sink;  // S of the current ranks
};

// rank0 = 1/N, contrib0 = rank0/outdeg, block partials of S0.
template <class T>
__global__ void __launch_bounds__(kPrThreads) pr_init_kernel(int32_t n, const int32_t* __restrict__ out_rp,
                                                             int32_t* __restrict__ outdeg, T* rank,
                                                             T* contrib, double* part_sink) {
    __shared__ double red[kPrThreads / 32];
    double sink = 0.0;
    const double r0 = 1.0 / (double)n;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = out_rp[v + 1] - out_rp[v];
        outdeg[v] = d;
        rank[v] = (T)r0;
        contrib[v] = d > 0 ? (T)(r0 / (double)d) : (T)0;
        if (d == 0) sink += (double)(T)r0;
    }
    sink = warp_sum(sink);
    if (lane_id() == 0) red[threadIdx.x >> 5] = sink;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < kPrThreads / 32; ++i) s += red[i];
        part_sink[blockIdx.x] = s;
    }
}

template <class T>
__device__ __forceinline__ void pr_finish_row(int64_t v, double sum, const PrScalars* sc, double damping,
                                              const int32_t* __restrict__ outdeg, const T* rank_old,
                                              T* rank_new, T* contrib_new, int track_l1, double& sink,
                                              double& l1) {
    const double r = sc->base + damping * sum;
    const T rt = (T)r;
    const int32_t d = outdeg[v];
    rank_new[v] = rt;
    contrib_new[v] = d > 0 ? (T)(r / (double)d) : (T)0;
    if (d == 0) sink += (double)rt;
    if (track_l1) l1 += fabs((double)rt - (double)rank_old[v]);
}

template <class T>
__device__ __forceinline__ void block_partials(double sink, double l1, double* part_sink, double* part_l1,
                                               int slot) {
    __shared__ double red_s[32], red_l[32];
    sink = warp_sum(sink);
    l1 = warp_sum(l1);
    if (lane_id() == 0) {
        red_s[threadIdx.x >> 5] = sink;
        red_l[threadIdx.x >> 5] = l1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0, l = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            s += red_s[i];
            l += red_l[i];
        }
        part_sink[slot] = s;
        part_l1[slot] = l;
    }
}

// Shared-memory cache of the first K contributions (K from the workspace's
// pr_cache_kb, 192 KB by default).
// On a degree-relabelled graph these are the hubs' (the top 32K vertices of
// an RMAT scale-22 graph hold half of all entries), so about half of the
// gathers are served from shared memory instead of L2 sectors.  The kernels
// that use it run persistent blocks (pr_threads x pr_blocks_per_sm per SM,
// 1024 x 1 by default), so each block fills the cache once per launch.
constexpr int kPrPersistThreads = 1024;

template <class T>
__device__ __forceinline__ int32_t fill_hub_cache(T* cache, const T* __restrict__ contrib_old, int32_t n,
                                                  int32_t cache_elems) {
    const int32_t K = min(cache_elems, n);
    for (int32_t i = threadIdx.x; i < K; i += blockDim.x) cache[i] = contrib_old[i];
    __syncthreads();
    return K;
}

template <class T>
__device__ __forceinline__ T gather(const T* cache, int32_t K, const T* __restrict__ contrib_old, int32_t u,
                                    uint64_t pol) {
    return u < K ? cache[u] : load_contrib<T>(contrib_old + u, pol);
}

// Rows of up to `short_max` entries: one thread per row, gathers four at a time
// (independent loads), Kahan-summed in row order.  Longer rows are skipped
// here (chunk path).
template <class T>
__global__ void __launch_bounds__(kPrPersistThreads) pr_rows_short_kernel(
    int32_t n, const int32_t* __restrict__ in_rp, const int32_t* __restrict__ in_col,
    const int32_t* __restrict__ outdeg, const T* __restrict__ contrib_old, const T* rank_old,
    T* rank_new, T* contrib_new, const PrScalars* sc, double damping, int track_l1, double* part_sink,
    double* part_l1, int32_t short_max, int32_t cache_elems) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* cache = reinterpret_cast<T*>(smem_raw);
    const int32_t K = fill_hub_cache<T>(cache, contrib_old, n, cache_elems);
    const uint64_t pol_stream = policy_evict_first();
    const uint64_t pol_keep = policy_evict_last();
    double sink = 0.0, l1 = 0.0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = in_rp[r], e = in_rp[r + 1];
        if (e - b > short_max) continue;
        KSum<T> acc;
        for (int32_t j = b; j < e; j += 4) {
            int32_t u[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) u[k] = (j + k < e) ? ld_stream(in_col + j + k, pol_stream) : -1;
            T x[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) x[k] = u[k] >= 0 ? gather<T>(cache, K, contrib_old, u[k], pol_keep) : (T)0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (u[k] >= 0) acc.add(x[k]);
        }
        pr_finish_row<T>(r, acc.value(), sc, damping, outdeg, rank_old, rank_new, contrib_new, track_l1, sink, l1);
    }
    block_partials<T>(sink, l1, part_sink, part_l1, blockIdx.x);
}

__global__ void pr_long_flags_kernel(int32_t n, const int32_t* __restrict__ in_rp, int32_t* flag, int32_t short_max) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        flag[v] = (in_rp[v + 1] - in_rp[v]) > short_max ? 1 : 0;
}

// Long rows in ascending order, and their chunk counts.
__global__ void pr_long_compact_kernel(int32_t n, const int32_t* __restrict__ in_rp, const int32_t* __restrict__ flag,
                                       const int32_t* __restrict__ pos, int32_t* long_rows, int32_t* nchunks,
                                       int32_t chunk) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        if (!flag[v]) continue;
        const int32_t i = pos[v];
        long_rows[i] = (int32_t)v;
        nchunks[i] = (in_rp[v + 1] - in_rp[v] + chunk - 1) / chunk;
    }
}

// chunk_row[c] = index (in long_rows) of the row chunk c belongs to.
__global__ void pr_chunk_rows_kernel(int32_t nlong, const int32_t* __restrict__ chunk_prefix, int32_t* chunk_row) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < nlong; i += nwarps)
        for (int32_t c = chunk_prefix[i] + lane_id(); c < chunk_prefix[i + 1]; c += 32) chunk_row[c] = (int32_t)i;
}

// One warp per chunk of `chunk` entries: a partial sum, G independent
// 32-wide loads in flight per lane (4 or 8: the workspace's pr_gathers),
// hub contributions from shared memory.
template <class T, int G>
__global__ void __launch_bounds__(kPrPersistThreads) pr_chunk_kernel(
    int32_t n, const int32_t* __restrict__ in_rp, const int32_t* __restrict__ in_col,
    const int32_t* __restrict__ long_rows, const int32_t* __restrict__ chunk_prefix,
    const int32_t* __restrict__ chunk_row, int32_t nchunks, const T* __restrict__ contrib_old, double* chunk_sum,
    int32_t chunk, int32_t cache_elems) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* cache = reinterpret_cast<T*>(smem_raw);
    const int32_t K = fill_hub_cache<T>(cache, contrib_old, n, cache_elems);
    const uint64_t pol_stream = policy_evict_first();
    const uint64_t pol_keep = policy_evict_last();
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t ch = warp; ch < nchunks; ch += nwarps) {
        const int32_t i = chunk_row[ch];
        const int32_t u = long_rows[i];
        const int32_t rb = in_rp[u], re = in_rp[u + 1];
        const int32_t b = rb + (int32_t)(ch - chunk_prefix[i]) * chunk;
        const int32_t e = min(re, b + chunk);
        KSum<T> acc;
        for (int32_t j0 = b; j0 < e; j0 += 32 * G) {
            int32_t x[G];
#pragma unroll
            for (int k = 0; k < G; ++k) {
                const int32_t j = j0 + lane + 32 * k;
                x[k] = j < e ? ld_stream(in_col + j, pol_stream) : -1;
            }
            T y[G];
#pragma unroll
            for (int k = 0; k < G; ++k) y[k] = x[k] >= 0 ? gather<T>(cache, K, contrib_old, x[k], pol_keep) : (T)0;
#pragma unroll
            for (int k = 0; k < G; ++k)
                if (x[k] >= 0) acc.add(y[k]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc.merge_from_lane(o, 32);
        if (lane == 0) chunk_sum[ch] = acc.value();
    }
}

// Long rows: the chunk partials summed in chunk order, then the row update.
template <class T>
__global__ void __launch_bounds__(kPrThreads) pr_long_finish_kernel(
    int32_t nlong, const int32_t* __restrict__ long_rows, const int32_t* __restrict__ chunk_prefix,
    const double* __restrict__ chunk_sum, const int32_t* __restrict__ outdeg, const T* rank_old, T* rank_new,
    T* contrib_new, const PrScalars* sc, double damping, int track_l1, double* part_sink, double* part_l1,
    int slot0) {
    double sink = 0.0, l1 = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nlong;
         i += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int32_t c = chunk_prefix[i]; c < chunk_prefix[i + 1]; ++c) s += chunk_sum[c];
        pr_finish_row<T>(long_rows[i], s, sc, damping, outdeg, rank_old, rank_new, contrib_new, track_l1, sink, l1);
    }
    block_partials<T>(sink, l1, part_sink, part_l1, slot0 + blockIdx.x);
}

// One block: S and L1 from the partials (fixed order), next base.
__global__ void __launch_bounds__(1024) pr_reduce_kernel(const double* part_sink, const double* part_l1,
                                                         int nparts, int32_t n, double damping,
                                                         PrScalars* sc, double* l1_hist, int iter,
                                                         int has_l1) {
    __shared__ double rs[1024], rl[1024];
    double s = 0.0, l = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        s += part_sink[i];
        if (has_l1) l += part_l1[i];
    }
    rs[threadIdx.x] = s;
    rl[threadIdx.x] = l;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            rs[threadIdx.x] += rs[threadIdx.x + o];
            rl[threadIdx.x] += rl[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double S = rs[0];
        sc->sink = S;
        sc->base = (1.0 - damping) / (double)n + S * damping / (double)n;
        if (has_l1) {
            sc->l1 = rl[0];
            if (l1_hist) l1_hist[iter] = rl[0];
        }
    }
}

template <class T>
__global__ void pr_to_f64_kernel(const T* src, double* dst, int32_t n) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x)
        dst[v] = (double)src[v];
}

template <class T>
int pagerank_impl(ghb_workspace* ws, int32_t n, const int32_t* in_rp, const int32_t* in_col,
                  const int32_t* out_rp, const ghb_pr_options* o, double* rank_out, int32_t* iters_run) {
    cudaStream_t st = ws->stream;
    const Tuning& tu = ws->tune;
    const int32_t short_max = tu.pr_short, chunk = tu.pr_chunk;
    const int pthreads = tu.pr_threads;
    const size_t cache_bytes = (size_t)tu.pr_cache_kb * 1024;
    const int32_t cache_elems = (int32_t)(cache_bytes / sizeof(T));
    const unsigned grid_rows = ws->num_sms * tu.pr_blocks_per_sm;  // persistent blocks
    const unsigned grid_long = ws->num_sms * 2;
    const int nparts = grid_rows + grid_long;
    int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned);
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, in_rp + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t m = hp[0];
    // Upper bounds: long rows <= min(n, m / (short_max + 1)), chunks <= m / chunk + long rows.
    const int64_t max_long = std::min<int64_t>(n, m / (short_max + 1) + 1);
    const int64_t max_chunks = m / chunk + max_long + 1;
    auto carve = [&](Carver& c, T** ra, T** rb, T** ca, T** cb, int32_t** outdeg, int32_t** flag, int32_t** pos,
                     int32_t** long_rows, int32_t** nch, int32_t** cpre, int32_t** crow, double** csum, int64_t** bs,
                     double** ps, double** pl, PrScalars** sc, double** hist) {
        *ra = c.take<T>(n);
        *rb = c.take<T>(n);
        *ca = c.take<T>(n);
        *cb = c.take<T>(n);
        *outdeg = c.take<int32_t>(n);
        *flag = c.take<int32_t>(n);
        *pos = c.take<int32_t>((size_t)n + 1);
        *long_rows = c.take<int32_t>(max_long);
        *nch = c.take<int32_t>(max_long);
        *cpre = c.take<int32_t>(max_long + 1);
        *crow = c.take<int32_t>(max_chunks);
        *csum = c.take<double>(max_chunks);
        *bs = c.take<int64_t>(scan_scratch_words(n > max_long ? n : max_long));
        *ps = c.take<double>(nparts);
        *pl = c.take<double>(nparts);
        *sc = c.take<PrScalars>(1);
        *hist = c.take<double>(o->iterations > 0 ? o->iterations : 1);
    };
    T *ra, *rb, *ca, *cb;
    int32_t *outdeg, *flag, *pos, *long_rows, *nch, *cpre, *crow;
    double *csum, *ps, *pl, *hist;
    int64_t* bs;
    PrScalars* sc;
    Carver sizing(nullptr);
    carve(sizing, &ra, &rb, &ca, &cb, &outdeg, &flag, &pos, &long_rows, &nch, &cpre, &crow, &csum, &bs, &ps, &pl, &sc,
          &hist);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &ra, &rb, &ca, &cb, &outdeg, &flag, &pos, &long_rows, &nch, &cpre, &crow, &csum, &bs, &ps, &pl, &sc,
          &hist);

    const double d = o->damping;
    const unsigned g = ws->num_sms * 8;
    GHB_CUDA_TRY(cudaFuncSetAttribute(pr_rows_short_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)cache_bytes));
    GHB_CUDA_TRY(cudaFuncSetAttribute(pr_chunk_kernel<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)cache_bytes));
    GHB_CUDA_TRY(cudaFuncSetAttribute(pr_chunk_kernel<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)cache_bytes));
    GHB_CUDA_TRY(cudaMemsetAsync(ps, 0, sizeof(double) * nparts, st));
    GHB_CUDA_TRY(cudaMemsetAsync(pl, 0, sizeof(double) * nparts, st));
    GHB_TRY(launch(ws, pr_init_kernel<T>, dim3(grid_rows), dim3(kPrThreads), 0, n, out_rp, outdeg, ra, ca, ps));
    GHB_TRY(launch(ws, pr_reduce_kernel, dim3(1), dim3(1024), 0, (const double*)ps, (const double*)pl, nparts, n, d,
                   sc, (double*)nullptr, 0, 0));
    // Long-row list (ascending) and its chunks.
    GHB_TRY(launch(ws, pr_long_flags_kernel, dim3(grid_for(n, 256, g)), dim3(256), 0, n, in_rp, flag, short_max));
    GHB_TRY(scan_exclusive_i32(ws, flag, pos, n, bs));
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, pos + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const int32_t nlong = hp[0];
    int32_t nchunks = 0;
    if (nlong > 0) {
        GHB_TRY(launch(ws, pr_long_compact_kernel, dim3(grid_for(n, 256, g)), dim3(256), 0, n, in_rp,
                       (const int32_t*)flag, (const int32_t*)pos, long_rows, nch, chunk));
        GHB_TRY(scan_exclusive_i32(ws, nch, cpre, nlong, bs));
        GHB_CUDA_TRY(cudaMemcpyAsync(hp, cpre + nlong, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        nchunks = hp[0];
        GHB_TRY(launch(ws, pr_chunk_rows_kernel, dim3(grid_for((int64_t)nlong * 32, 256, g)), dim3(256), 0, nlong,
                       (const int32_t*)cpre, crow));
    }

    T *r_cur = ra, *r_nxt = rb, *c_cur = ca, *c_nxt = cb;
    const bool track = o->tolerance > 0 || o->l1_history != nullptr;
    int it = 0;
    for (; it < o->iterations; ++it) {
        GHB_TRY(launch(ws, pr_rows_short_kernel<T>, dim3(grid_rows), dim3(pthreads), cache_bytes, n, in_rp, in_col,
                       (const int32_t*)outdeg, (const T*)c_cur, (const T*)r_cur, r_nxt, c_nxt, (const PrScalars*)sc, d,
                       track ? 1 : 0, ps, pl, short_max, cache_elems));
        if (nlong > 0) {
            GHB_TRY(launch(ws, ws->tune.pr_gathers == 8 ? pr_chunk_kernel<T, 8> : pr_chunk_kernel<T, 4>,
                           dim3(grid_rows), dim3(pthreads), cache_bytes, n, in_rp, in_col,
                           (const int32_t*)long_rows, (const int32_t*)cpre, (const int32_t*)crow, nchunks,
                           (const T*)c_cur, csum, chunk, cache_elems));
        }
        GHB_TRY(launch(ws, pr_long_finish_kernel<T>, dim3(grid_long), dim3(kPrThreads), 0, nlong,
                       (const int32_t*)long_rows, (const int32_t*)cpre, (const double*)csum, (const int32_t*)outdeg,
                       (const T*)r_cur, r_nxt, c_nxt, (const PrScalars*)sc, d, track ? 1 : 0, ps, pl,
                       (int)grid_rows));
        GHB_TRY(launch(ws, pr_reduce_kernel, dim3(1), dim3(1024), 0, (const double*)ps, (const double*)pl, nparts, n,
                       d, sc, hist, it, track ? 1 : 0));
        std::swap(r_cur, r_nxt);
        std::swap(c_cur, c_nxt);
        if (o->tolerance > 0) {
            GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, sc, sizeof(PrScalars), cudaMemcpyDeviceToHost, st));
            GHB_CUDA_TRY(cudaStreamSynchronize(st));
            const PrScalars* h = reinterpret_cast<const PrScalars*>(ws->host_pinned);
            if (h->l1 <= o->tolerance) {
                ++it;
                break;
            }
        }
    }
    GHB_TRY(launch(ws, pr_to_f64_kernel<T>, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0, (const T*)r_cur,
                   rank_out, n));
    if (o->l1_history && it > 0) {
        GHB_CUDA_TRY(cudaMemcpyAsync(o->l1_history, hist, sizeof(double) * it, cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
    }
    if (iters_run) *iters_run = it;
    return GHB_OK;
}

}  // namespace

int pagerank_run(ghb_workspace* ws, int32_t n, const int32_t* in_rp, const int32_t* in_col, const int32_t* out_rp,
                 const ghb_pr_options* o, double* rank, int32_t* iters_run) {
    if (o->precision == GHB_PR_FP64) return pagerank_impl<double>(ws, n, in_rp, in_col, out_rp, o, rank, iters_run);
    return pagerank_impl<float>(ws, n, in_rp, in_col, out_rp, o, rank, iters_run);
}

}  // namespace ghb

using namespace ghb;

extern "C" int ghb_pagerank(ghb_workspace* ws, int32_t n, const int32_t* in_rowptr, const int32_t* in_col,
                            const int32_t* out_rowptr, const ghb_pr_options* options, double* rank,
                            int32_t* iterations_run) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(in_rowptr && out_rowptr && rank && options, "NULL argument");
    GHB_REQUIRE(options->iterations >= 0, "iterations < 0");
    GHB_REQUIRE(options->precision == GHB_PR_FP64 || options->precision == GHB_PR_FP32_KAHAN,
                "bad precision");
    if (options->precision == GHB_PR_FP64)
        return pagerank_impl<double>(ws, n, in_rowptr, in_col, out_rowptr, options, rank, iterations_run);
    return pagerank_impl<float>(ws, n, in_rowptr, in_col, out_rowptr, options, rank, iterations_run);
}
