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
// Rows are summed by groups of VW lanes (VW picked from the mean in-degree);
// rows with >= kPrBig entries are split into kPrChunk-entry chunks summed by
// one warp each and combined per row in chunk order.
//
// FP32 mode: ranks and contributions are stored as float (half the gather
// footprint: 64 MiB at n = 2^24, resident in the 126 MB L2); each lane keeps
// a Kahan-compensated FP32 sum and lanes are merged with an error-free
// TwoSum; the row total, S and the L1 norm are FP64.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace ghb {
namespace {

constexpr int32_t kPrBig = 8192;
constexpr int32_t kPrChunk = 2048;
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
                                              T* rank_new, T* contrib_new, double& sink, double& l1) {
    const double r = sc->base + damping * sum;
    const T rt = (T)r;
    const int32_t d = outdeg[v];
    const double old = (double)rank_old[v];
    rank_new[v] = rt;
    contrib_new[v] = d > 0 ? (T)(r / (double)d) : (T)0;
    if (d == 0) sink += (double)rt;
    l1 += fabs((double)rt - old);
}

template <class T>
__device__ __forceinline__ void block_partials(double sink, double l1, double* part_sink, double* part_l1,
                                               int slot) {
    __shared__ double red_s[kPrThreads / 32], red_l[kPrThreads / 32];
    sink = warp_sum(sink);
    l1 = warp_sum(l1);
    if (lane_id() == 0) {
        red_s[threadIdx.x >> 5] = sink;
        red_l[threadIdx.x >> 5] = l1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0, l = 0.0;
        for (int i = 0; i < kPrThreads / 32; ++i) {
            s += red_s[i];
            l += red_l[i];
        }
        part_sink[slot] = s;
        part_l1[slot] = l;
    }
}

// Rows with < kPrBig entries: VW lanes per row.
template <class T, int VW>
__global__ void __launch_bounds__(kPrThreads) pr_rows_kernel(
    int32_t n, const int32_t* __restrict__ in_rp, const int32_t* __restrict__ in_col,
    const int32_t* __restrict__ outdeg, const T* __restrict__ contrib_old, const T* rank_old,
    T* rank_new, T* contrib_new, const PrScalars* sc, double damping, double* part_sink,
    double* part_l1) {
    const uint64_t pol_stream = policy_evict_first();
    const uint64_t pol_keep = policy_evict_last();
    const int sub = threadIdx.x % VW;
    const int64_t group = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / VW;
    const int64_t ngroups = ((int64_t)gridDim.x * blockDim.x) / VW;
    double sink = 0.0, l1 = 0.0;
    // Every lane of a warp runs the same trip count so the shuffles stay
    // converged.
    const int64_t rounds = ((int64_t)n + ngroups - 1) / ngroups;
    for (int64_t r = 0; r < rounds; ++r) {
        const int64_t v = group + r * ngroups;
        int32_t b = 0, e = 0;
        if (v < n) {
            b = in_rp[v];
            e = in_rp[v + 1];
            if (e - b >= kPrBig) e = b - 1;  // handled by the chunk kernels
        }
        KSum<T> acc;
        for (int32_t j = b + sub; j < e; j += VW) {
            const int32_t u = ld_stream(in_col + j, pol_stream);
            acc.add(load_contrib<T>(contrib_old + u, pol_keep));
        }
#pragma unroll
        for (int o = VW / 2; o > 0; o >>= 1) acc.merge_from_lane(o, VW);
        if (sub == 0 && v < n && e >= b)
            pr_finish_row<T>(v, acc.value(), sc, damping, outdeg, rank_old, rank_new, contrib_new, sink, l1);
    }
    block_partials<T>(sink, l1, part_sink, part_l1, blockIdx.x);
}

__global__ void pr_find_big_kernel(int32_t n, const int32_t* __restrict__ in_rp, int32_t* big,
                                   int32_t* big_tail) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = in_rp[v + 1] - in_rp[v];
        if (d >= kPrBig) big[atomicAdd(big_tail, 1)] = (int32_t)v;
    }
}

// chunk_prefix[i] = chunks before big row i (one block, few rows).
__global__ void __launch_bounds__(1024) pr_chunk_scan_kernel(const int32_t* __restrict__ in_rp,
                                                             const int32_t* __restrict__ big,
                                                             const int32_t* big_tail,
                                                             int32_t* chunk_prefix) {
    __shared__ int32_t carry;
    if (threadIdx.x == 0) {
        // Sequential: the list is short (rows >= kPrBig entries).
        int32_t acc = 0;
        const int32_t count = *big_tail;
        for (int32_t i = 0; i < count; ++i) {
            const int32_t u = big[i];
            chunk_prefix[i] = acc;
            acc += (in_rp[u + 1] - in_rp[u] + kPrChunk - 1) / kPrChunk;
        }
        chunk_prefix[count] = acc;
        carry = acc;
    }
}

template <class T>
__global__ void __launch_bounds__(kPrThreads) pr_chunk_kernel(
    const int32_t* __restrict__ in_rp, const int32_t* __restrict__ in_col, const int32_t* __restrict__ big,
    const int32_t* big_tail, const int32_t* __restrict__ chunk_prefix, const T* __restrict__ contrib_old,
    double* chunk_sum) {
    const uint64_t pol_stream = policy_evict_first();
    const uint64_t pol_keep = policy_evict_last();
    const int32_t count = *big_tail;
    if (count == 0) return;
    const int32_t nchunks = chunk_prefix[count];
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t ch = warp; ch < nchunks; ch += nwarps) {
        int32_t lo = 0, hi = count - 1;
        while (lo < hi) {
            const int32_t mid = (lo + hi + 1) >> 1;
            if (chunk_prefix[mid] <= ch) lo = mid;
            else hi = mid - 1;
        }
        const int32_t u = big[lo];
        const int32_t rb = in_rp[u], re = in_rp[u + 1];
        const int32_t b = rb + (int32_t)(ch - chunk_prefix[lo]) * kPrChunk;
        const int32_t e = min(re, b + kPrChunk);
        KSum<T> acc;
        for (int32_t j = b + lane_id(); j < e; j += 32) {
            const int32_t x = ld_stream(in_col + j, pol_stream);
            acc.add(load_contrib<T>(contrib_old + x, pol_keep));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc.merge_from_lane(o, 32);
        if (lane_id() == 0) chunk_sum[ch] = acc.value();
    }
}

template <class T>
__global__ void __launch_bounds__(kPrThreads) pr_big_finish_kernel(
    const int32_t* __restrict__ big, const int32_t* big_tail, const int32_t* __restrict__ chunk_prefix,
    const double* __restrict__ chunk_sum, const int32_t* __restrict__ outdeg, const T* rank_old,
    T* rank_new, T* contrib_new, const PrScalars* sc, double damping, double* part_sink,
    double* part_l1, int slot0) {
    const int32_t count = *big_tail;
    double sink = 0.0, l1 = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int32_t c = chunk_prefix[i]; c < chunk_prefix[i + 1]; ++c) s += chunk_sum[c];
        pr_finish_row<T>(big[i], s, sc, damping, outdeg, rank_old, rank_new, contrib_new, sink, l1);
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

template <class T, int VW>
int launch_rows(ghb_workspace* ws, unsigned grid, int32_t n, const int32_t* in_rp, const int32_t* in_col,
                const int32_t* outdeg, const T* c_old, const T* r_old, T* r_new, T* c_new,
                const PrScalars* sc, double d, double* ps, double* pl) {
    return launch(ws, pr_rows_kernel<T, VW>, dim3(grid), dim3(kPrThreads), 0, n, in_rp, in_col, outdeg,
                  c_old, r_old, r_new, c_new, sc, d, ps, pl);
}

template <class T>
int pagerank_impl(ghb_workspace* ws, int32_t n, const int32_t* in_rp, const int32_t* in_col,
                  const int32_t* out_rp, const ghb_pr_options* o, double* rank_out, int32_t* iters_run) {
    cudaStream_t st = ws->stream;
    const unsigned grid_rows = ws->num_sms * 8;
    const unsigned grid_big = ws->num_sms * 2;
    const int nparts = grid_rows + grid_big;
    Carver sizing(nullptr);
    auto carve = [&](Carver& c, T** ra, T** rb, T** ca, T** cb, int32_t** outdeg, int32_t** big,
                     int32_t** big_tail, int32_t** chunk_prefix, double** chunk_sum, double** ps,
                     double** pl, PrScalars** sc, double** hist) {
        *ra = c.take<T>(n);
        *rb = c.take<T>(n);
        *ca = c.take<T>(n);
        *cb = c.take<T>(n);
        *outdeg = c.take<int32_t>(n);
        const int64_t max_big = 1 + (int64_t)n / 1;  // bounded by n
        *big = c.take<int32_t>(max_big);
        *big_tail = c.take<int32_t>(8);
        *chunk_prefix = c.take<int32_t>(max_big + 1);
        // chunk count <= m / kPrChunk + big rows; m < 2^31.
        *chunk_sum = c.take<double>(((int64_t)1 << 31) / kPrChunk + max_big + 1);
        *ps = c.take<double>(nparts);
        *pl = c.take<double>(nparts);
        *sc = c.take<PrScalars>(1);
        *hist = c.take<double>(o->iterations > 0 ? o->iterations : 1);
    };
    T *ra, *rb, *ca, *cb;
    int32_t *outdeg, *big, *big_tail, *chunk_prefix;
    double *chunk_sum, *ps, *pl, *hist;
    PrScalars* sc;
    carve(sizing, &ra, &rb, &ca, &cb, &outdeg, &big, &big_tail, &chunk_prefix, &chunk_sum, &ps, &pl, &sc,
          &hist);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &ra, &rb, &ca, &cb, &outdeg, &big, &big_tail, &chunk_prefix, &chunk_sum, &ps, &pl, &sc, &hist);

    const double d = o->damping;
    GHB_CUDA_TRY(cudaMemsetAsync(ps, 0, sizeof(double) * nparts, st));
    GHB_CUDA_TRY(cudaMemsetAsync(pl, 0, sizeof(double) * nparts, st));
    GHB_CUDA_TRY(cudaMemsetAsync(big_tail, 0, sizeof(int32_t), st));
    GHB_TRY(launch(ws, pr_init_kernel<T>, dim3(grid_rows), dim3(kPrThreads), 0, n, out_rp, outdeg, ra, ca, ps));
    GHB_TRY(launch(ws, pr_reduce_kernel, dim3(1), dim3(1024), 0, (const double*)ps, (const double*)pl,
                   nparts, n, d, sc, (double*)nullptr, 0, 0));
    GHB_TRY(launch(ws, pr_find_big_kernel, dim3(grid_for(n, 256, ws->num_sms * 4)), dim3(256), 0, n, in_rp,
                   big, big_tail));
    GHB_TRY(launch(ws, pr_chunk_scan_kernel, dim3(1), dim3(32), 0, in_rp, (const int32_t*)big,
                   (const int32_t*)big_tail, chunk_prefix));

    // Mean in-degree picks the lanes per row.
    int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned);
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, in_rp + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const double mean = (double)hp[0] / (double)n;
    const int vw = mean >= 24 ? 16 : mean >= 10 ? 8 : mean >= 4 ? 4 : 2;

    T *r_cur = ra, *r_nxt = rb, *c_cur = ca, *c_nxt = cb;
    const bool track = o->tolerance > 0 || o->l1_history != nullptr;
    int it = 0;
    for (; it < o->iterations; ++it) {
        int s;
        switch (vw) {
            case 16: s = launch_rows<T, 16>(ws, grid_rows, n, in_rp, in_col, outdeg, c_cur, r_cur, r_nxt, c_nxt, sc, d, ps, pl); break;
            case 8: s = launch_rows<T, 8>(ws, grid_rows, n, in_rp, in_col, outdeg, c_cur, r_cur, r_nxt, c_nxt, sc, d, ps, pl); break;
            case 4: s = launch_rows<T, 4>(ws, grid_rows, n, in_rp, in_col, outdeg, c_cur, r_cur, r_nxt, c_nxt, sc, d, ps, pl); break;
            default: s = launch_rows<T, 2>(ws, grid_rows, n, in_rp, in_col, outdeg, c_cur, r_cur, r_nxt, c_nxt, sc, d, ps, pl); break;
        }
        GHB_TRY(s);
        GHB_TRY(launch(ws, pr_chunk_kernel<T>, dim3(ws->num_sms * 4), dim3(kPrThreads), 0, in_rp, in_col,
                       (const int32_t*)big, (const int32_t*)big_tail, (const int32_t*)chunk_prefix,
                       (const T*)c_cur, chunk_sum));
        GHB_TRY(launch(ws, pr_big_finish_kernel<T>, dim3(grid_big), dim3(kPrThreads), 0, (const int32_t*)big,
                       (const int32_t*)big_tail, (const int32_t*)chunk_prefix, (const double*)chunk_sum,
                       (const int32_t*)outdeg, (const T*)r_cur, r_nxt, c_nxt, (const PrScalars*)sc, d, ps, pl,
                       (int)grid_rows));
        GHB_TRY(launch(ws, pr_reduce_kernel, dim3(1), dim3(1024), 0, (const double*)ps, (const double*)pl,
                       nparts, n, d, sc, hist, it, track ? 1 : 0));
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
    GHB_TRY(launch(ws, pr_to_f64_kernel<T>, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0,
                   (const T*)r_cur, rank_out, n));
    if (o->l1_history && it > 0) {
        GHB_CUDA_TRY(cudaMemcpyAsync(o->l1_history, hist, sizeof(double) * it, cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
    }
    if (iters_run) *iters_run = it;
    return GHB_OK;
}

}  // namespace
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
