// Single-source shortest paths, FP64, by delta-stepping in its near/far form
// (replaces the reference's frontier Bellman-Ford, GPU_SSSP_csr.cuh:23-327,
// which materialises an 8-byte entry per improving edge and syncs the host
// every round).  Semantics: the CPU Dijkstra (CPU_shortest_paths.hpp:19-64).
//
// Both compute, for every vertex, the minimum over paths of the
// left-to-right FP64 sum of the path's weights: a relaxation only ever
// lowers dist[v] to fl(dist[u] + w), fl is monotone and fl(x + w) >= x for
// w >= 0, so any relaxation order reaches the same least fixpoint, bit for
// bit.  dist is updated with a 64-bit atomicMin on the bit pattern, which
// orders non-negative doubles like the values themselves.
//
// Phase loop: vertices whose tentative distance is below the threshold form
// the near queue and are relaxed until the queue is empty (one load-balanced
// pass over their out-rows per round, edge_walk.cuh); improvements at or
// above the threshold go to the far list.  Then the threshold moves up by
// delta and the far list is split.  A vertex enters a queue at most once per
// round (stamp arrays).
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "edge_walk.cuh"
#include "graph.cuh"
#include "policy.cuh"

namespace ghb {

bool sssp_persistent_available(ghb_workspace* ws, int* blocks);
int sssp_persistent_run(ghb_workspace* ws, int32_t n, const int32_t* rp, const int32_t* le, const int32_t* col,
                        const double* wt, int32_t src, double inf, double delta, double* dist, const int32_t* perm,
                        double* out, ghb_traversal_stats* stats);
int graph_light_ends(ghb_workspace* ws, ghb_graph* g, double delta, const int32_t** le);

namespace {

struct SsspCounters {
    int32_t near_tail;
    int32_t far_tail;
    int32_t split_near;
    int32_t pad;
    unsigned long long examined;
    unsigned long long improved;
};

__device__ __forceinline__ double ld_dist(const unsigned long long* d, int32_t v) {
    return __longlong_as_double((long long)__ldcg(d + v));
}

struct RelaxVisitor {
    const double* w;
    unsigned long long* dist;
    double threshold;
    int32_t* near_next;
    int32_t* near_stamp;
    int32_t round;
    int32_t* far;
    int32_t* far_stamp;
    int32_t phase;
    SsspCounters* cnt;
    unsigned long long examined;
    __device__ bool want_row(int32_t) const { return true; }
    __device__ void operator()(int32_t u, int32_t v, int32_t j) {
        ++examined;
        const double nd = ld_dist(dist, u) + w[j];
        if (nd < ld_dist(dist, v)) {
            const unsigned long long nb = (unsigned long long)__double_as_longlong(nd);
            const unsigned long long old = atomicMin(dist + v, nb);
            if (nb < old) {
                if (nd < threshold) {
                    if (atomicExch(near_stamp + v, round) != round) {
                        const int32_t pos = atomicAdd(&cnt->near_tail, 1);
                        near_next[pos] = v;
                    }
                } else {
                    if (atomicExch(far_stamp + v, phase) != phase) {
                        const int32_t pos = atomicAdd(&cnt->far_tail, 1);
                        far[pos] = v;
                    }
                }
            }
        }
    }
    __device__ void finish() {
        unsigned long long e = warp_sum(examined);
        if (lane_id() == 0 && e) atomicAdd(&cnt->examined, e);
    }
};

__global__ void sssp_init_kernel(int32_t n, int32_t src, double inf, unsigned long long* dist,
                                 int32_t* near_stamp, int32_t* far_stamp, int32_t* near_q) {
    const unsigned long long ib = (unsigned long long)__double_as_longlong(inf);
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        dist[v] = (v == src) ? 0ull : ib;
        near_stamp[v] = -1;
        far_stamp[v] = -1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) near_q[0] = src;
}

// Split the far list at a new threshold: entries already settled (below the
// old threshold) are dropped, entries below the new one go to the near
// queue, the rest to the next far list.
__global__ void sssp_split_kernel(const int32_t* __restrict__ far, int32_t far_count,
                                  const unsigned long long* dist, double old_thr, double new_thr,
                                  int32_t* near_q, int32_t* near_stamp, int32_t round, int32_t* far_next,
                                  int32_t* far_stamp, int32_t phase, SsspCounters* cnt,
                                  double* min_far) {
    double mn = INFINITY;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < far_count;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = far[i];
        const double d = ld_dist(dist, v);
        if (d < old_thr) continue;
        if (d < new_thr) {
            if (atomicExch(near_stamp + v, round) != round) near_q[atomicAdd(&cnt->split_near, 1)] = v;
        } else {
            if (atomicExch(far_stamp + v, phase) != phase) far_next[atomicAdd(&cnt->far_tail, 1)] = v;
            mn = d < mn ? d : mn;
        }
    }
    // Smallest distance left in the far list, to skip empty buckets.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double x = __shfl_xor_sync(0xffffffffu, mn, o);
        mn = x < mn ? x : mn;
    }
    if (lane_id() == 0 && mn < INFINITY)
        atomicMin(reinterpret_cast<unsigned long long*>(min_far), (unsigned long long)__double_as_longlong(mn));
}

__global__ void mean_weight_kernel(const double* __restrict__ w, int64_t m, int64_t stride, double* out) {
    double s = 0.0;
    int64_t c = 0;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) * stride; i < m;
         i += (int64_t)gridDim.x * blockDim.x * stride) {
        s += w[i];
        ++c;
    }
    s = warp_sum(s);
    double cd = warp_sum((double)c);
    if (lane_id() == 0) {
        atomicAdd(out, s);
        atomicAdd(out + 1, cd);
    }
}

// Graph statistics for the width choice: degree sum of squares, maximum and
// vertices with entries (all rows); weight sum, count, min, max (every
// stride-th entry).  out: [0] deg2 sum, [1] w sum, [2] w count,
// [3] degmax (as u64), [4] active (u64), [5] w min bits, [6] w max bits.
__global__ void sssp_stats_kernel(int32_t n, const int32_t* __restrict__ rp, const double* __restrict__ w, int64_t m,
                                  int64_t stride, double* out) {
    unsigned long long* u = reinterpret_cast<unsigned long long*>(out);
    double d2 = 0.0, ws = 0.0, wc = 0.0;
    unsigned long long dmax = 0, act = 0;
    long long wmin = 0x7fefffffffffffffll, wmax = 0;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, nt = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = tid; v < n; v += nt) {
        const unsigned long long d = (unsigned long long)(rp[v + 1] - rp[v]);
        d2 += (double)d * (double)d;
        dmax = d > dmax ? d : dmax;
        act += d > 0 ? 1 : 0;
    }
    for (int64_t i = tid * stride; i < m; i += nt * stride) {
        const double x = w[i];
        ws += x;
        wc += 1.0;
        const long long b = __double_as_longlong(x);  // weights are >= 0: bits order as values
        wmin = b < wmin ? b : wmin;
        wmax = b > wmax ? b : wmax;
    }
    d2 = warp_sum(d2);
    ws = warp_sum(ws);
    wc = warp_sum(wc);
    act = warp_sum(act);
    dmax = warp_max(dmax);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const long long a = __shfl_xor_sync(0xffffffffu, wmin, o), b = __shfl_xor_sync(0xffffffffu, wmax, o);
        wmin = a < wmin ? a : wmin;
        wmax = b > wmax ? b : wmax;
    }
    if (lane_id() == 0) {
        atomicAdd(out, d2);
        atomicAdd(out + 1, ws);
        atomicAdd(out + 2, wc);
        atomicMax(u + 3, dmax);
        atomicAdd(u + 4, act);
        atomicMin(reinterpret_cast<long long*>(u + 5), wmin);
        atomicMax(reinterpret_cast<long long*>(u + 6), wmax);
    }
}

// Predecessors after the distances are final: the smallest-id u in v's
// in-row with dist[u] + w(u, v) == dist[v] exactly.
__global__ void sssp_pred_pull_kernel(int32_t n, int32_t src, const int32_t* __restrict__ in_rp,
                                      const int32_t* __restrict__ in_col, const double* __restrict__ in_w,
                                      const double* __restrict__ dist, double inf, int32_t* __restrict__ pred) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = warp; v < n; v += nwarps) {
        const double dv = dist[v];
        int32_t p = -1;
        if (v != src && dv != inf) {
            const int32_t b = in_rp[v], e = in_rp[v + 1];
            for (int32_t k0 = b; k0 < e; k0 += 32) {
                const int32_t k = k0 + lane;
                bool h = false;
                int32_t u = -1;
                if (k < e) {
                    u = in_col[k];
                    const double du = dist[u];
                    h = du != inf && du + in_w[k] == dv;
                }
                const unsigned hm = __ballot_sync(0xffffffffu, h);
                if (hm) {
                    p = __shfl_sync(0xffffffffu, u, __ffs(hm) - 1);
                    break;
                }
            }
        }
        if (lane == 0) pred[v] = p;
    }
}

__global__ void sssp_pred_push_kernel(int32_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                                      const double* __restrict__ w, const double* __restrict__ dist, double inf,
                                      int32_t* pred) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = warp; u < n; u += nwarps) {
        const double du = dist[u];
        if (du == inf) continue;
        for (int32_t k = rp[u] + lane; k < rp[u + 1]; k += 32) {
            const int32_t v = col[k];
            if (du + w[k] == dist[v]) atomicMin(pred + v, (int32_t)u);
        }
    }
}

__global__ void sssp_pred_finish_kernel(int32_t n, int32_t src, int32_t* pred) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x)
        if (v == src || pred[v] == 0x7fffffff) pred[v] = -1;
}

__global__ void reached_edges_kernel(int32_t n, const int32_t* __restrict__ rp, const double* __restrict__ dist,
                                     double inf, unsigned long long* out) {
    unsigned long long e = 0, r = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        if (dist[v] != inf) {
            e += (unsigned long long)(rp[v + 1] - rp[v]);
            ++r;
        }
    }
    e = warp_sum(e);
    r = warp_sum(r);
    if (lane_id() == 0) {
        atomicAdd(out, e);
        atomicAdd(out + 1, r);
    }
}

// ---- delta-stepping with a light/heavy split (resident graphs)

// Sort key of entry j of row u: row, then the weight's top 39 bits (sign,
// exponent and 28 mantissa bits).  Rows must fit in 25 bits.
__global__ void weight_key_kernel(int32_t n, const int32_t* __restrict__ rp, const double* __restrict__ w,
                                  uint64_t* keys, uint32_t* vals) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = warp; u < n; u += nwarps) {
        for (int32_t j = rp[u] + lane_id(); j < rp[u + 1]; j += 32) {
            const uint64_t wb = (uint64_t)__double_as_longlong(w[j]);
            keys[j] = ((uint64_t)u << 39) | (wb >> 25);
            vals[j] = (uint32_t)j;
        }
    }
}

__global__ void weight_gather_kernel(int64_t m, const uint32_t* __restrict__ vals, const int32_t* __restrict__ col,
                                     const double* __restrict__ w, int32_t* sw_col, double* sw_w) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t j = vals[i];
        sw_col[i] = col[j];
        sw_w[i] = w[j];
    }
}

// light_end[u] = first entry of row u with weight >= delta (rows sorted by
// the truncated weight, and delta itself has no bits below the truncation,
// so the comparison is exact).
__global__ void light_end_kernel(int32_t n, const int32_t* __restrict__ rp, const double* __restrict__ sw_w,
                                 double delta, int32_t* light_end) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
        int32_t lo = rp[u], hi = rp[u + 1];
        while (lo < hi) {
            const int32_t mid = (lo + hi) >> 1;
            if (sw_w[mid] < delta) lo = mid + 1;
            else hi = mid;
        }
        light_end[u] = lo;
    }
}

// Adds the vertices of the near queue to the settled list R (once per phase).
__global__ void mark_settled_kernel(const int32_t* __restrict__ q, int32_t count, int32_t* r_stamp, int32_t phase,
                                    int32_t* R, int32_t* r_tail) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = q[i];
        if (atomicExch(r_stamp + u, phase) != phase) R[atomicAdd(r_tail, 1)] = u;
    }
}

__global__ void fill_i32(int32_t* p, int64_t count, int32_t value) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = value;
}

}  // namespace

// Bucket width from a weight sample when the caller gives none: the mean
// weight times 32 over the mean degree (wider buckets on sparse graphs,
// where rounds are latency-bound).
int sssp_pick_delta(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const double* w, double* delta) {
    cudaStream_t st = ws->stream;
    int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned);
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, rowptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t m = hp[0];
    if (m == 0) {
        *delta = 1.0;
        return GHB_OK;
    }
    double* acc = reinterpret_cast<double*>(ws->dev_small);
    GHB_CUDA_TRY(cudaMemsetAsync(acc, 0, 2 * sizeof(double), st));
    const int64_t stride = std::max<int64_t>(1, m / (1 << 20));
    GHB_TRY(launch(ws, mean_weight_kernel, dim3(64), dim3(256), 0, w, m, stride, acc));
    GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, acc, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const double* h = reinterpret_cast<const double*>(ws->host_pinned);
    const double mean_w = h[1] > 0 ? h[0] / h[1] : 1.0;
    const double mean_d = (double)m / (double)n;
    double d = mean_w * 32.0 / std::max(1.0, mean_d);
    if (!(d > 0)) d = 1.0;
    *delta = d;
    return GHB_OK;
}

// The width for one SSSP call: the caller's, else the weight rule above,
// scaled by the policy network's bin when the learned policy is asked for
// and a network is installed.  With record_trace, trace row 0 gets the
// features, then 12 the width used, 13 -1, 14 the rule's width, 15 1 when
// the network chose it; the caller's driver fills 13 (device ms).
int sssp_choose_delta(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const double* w, int32_t src,
                      const ghb_sssp_options* opt, double* delta) {
    if (opt && opt->delta > 0) {
        *delta = opt->delta;
        return GHB_OK;
    }
    GHB_TRY(sssp_pick_delta(ws, n, rowptr, w, delta));
    const bool learned = opt && opt->policy == GHB_POLICY_LEARNED;
    const bool tracing = opt && opt->record_trace && opt->trace && opt->trace_cap > 0;
    if (!learned && !tracing) return GHB_OK;
    cudaStream_t st = ws->stream;
    int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned);
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, rowptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaMemcpyAsync(hp + 1, rowptr + src, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t m = hp[0];
    const double deg_src = (double)(hp[2] - hp[1]);
    double* acc = reinterpret_cast<double*>(ws->dev_small);
    double init[7] = {0, 0, 0, 0, 0, 0, 0};
    const long long big = 0x7fefffffffffffffll;
    std::memcpy(&init[5], &big, sizeof(double));
    std::memcpy(ws->host_pinned, init, sizeof(init));
    GHB_CUDA_TRY(cudaMemcpyAsync(acc, ws->host_pinned, sizeof(init), cudaMemcpyHostToDevice, st));
    const int64_t stride = std::max<int64_t>(1, m / (1 << 20));
    GHB_TRY(launch(ws, sssp_stats_kernel, dim3(grid_for(n, 256, ws->num_sms * 4)), dim3(256), 0, n, rowptr, w, m,
                   stride, acc));
    GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, acc, sizeof(init), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    double h[7];
    std::memcpy(h, ws->host_pinned, sizeof(h));
    unsigned long long dmax, act;
    long long bmin, bmax;
    std::memcpy(&dmax, &h[3], 8);
    std::memcpy(&act, &h[4], 8);
    std::memcpy(&bmin, &h[5], 8);
    std::memcpy(&bmax, &h[6], 8);
    double wmin, wmax;
    std::memcpy(&wmin, &bmin, 8);
    std::memcpy(&wmax, &bmax, 8);
    const double wmean = h[2] > 0 ? h[1] / h[2] : 1.0;
    float f[GHB_TRACE_FEATURES];
    sssp_features(f, (double)n, (double)m, (double)act, deg_src, h[0], (double)dmax, wmean, wmin, wmax, *delta);
    const double base = *delta;
    bool by_net = false;
    if (learned) {
        const double d = policy_pick_delta(f, base);
        if (d > 0) {
            *delta = d;
            by_net = true;
        }
    }
    if (tracing) {
        float* row = opt->trace;
        for (int k = 0; k < GHB_TRACE_COLS; ++k) row[k] = -1.f;
        for (int k = 0; k < GHB_TRACE_FEATURES; ++k) row[k] = f[k];
        row[12] = (float)*delta;
        row[14] = (float)base;
        row[15] = by_net ? 1.f : 0.f;
    }
    return GHB_OK;
}

int sssp_run(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, const double* w,
             int32_t src, double inf, double* dist_out, const ghb_sssp_options* opt,
             ghb_traversal_stats* stats) {
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(rowptr && dist_out, "NULL argument");
    GHB_REQUIRE(src >= 0 && src < n, "source outside [0, n)");
    GHB_REQUIRE(inf >= 0, "inf must be >= 0");
    ghb_sssp_options defaults = {};
    if (!opt) opt = &defaults;
    cudaStream_t st = ws->stream;
    double delta = 0.0;
    GHB_TRY(sssp_choose_delta(ws, n, rowptr, w, src, opt, &delta));
    int blocks = 0;
    if (ws->tune.sssp_persistent && sssp_persistent_available(ws, &blocks))
        return sssp_persistent_run(ws, n, rowptr, nullptr, col, w, src, inf, delta, dist_out, nullptr, nullptr,
                                   stats);

    Carver sizing(nullptr);
    auto carve = [&](Carver& c, WalkBuffers* wb, int32_t** qa, int32_t** qb, int32_t** fa, int32_t** fb,
                     int32_t** ns, int32_t** fs, SsspCounters** cnt, double** minfar) {
        *wb = WalkBuffers::carve(c, n);
        *qa = c.take<int32_t>(n);
        *qb = c.take<int32_t>(n);
        *fa = c.take<int32_t>(n);
        *fb = c.take<int32_t>(n);
        *ns = c.take<int32_t>(n);
        *fs = c.take<int32_t>(n);
        *cnt = c.take<SsspCounters>(1);
        *minfar = c.take<double>(1);
    };
    WalkBuffers wb;
    int32_t *qa, *qb, *fa, *fb, *ns, *fs;
    SsspCounters* cnt;
    double* minfar;
    carve(sizing, &wb, &qa, &qb, &fa, &fb, &ns, &fs, &cnt, &minfar);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &wb, &qa, &qb, &fa, &fb, &ns, &fs, &cnt, &minfar);

    unsigned long long* dist = reinterpret_cast<unsigned long long*>(dist_out);
    const unsigned g = grid_for(n, 256, ws->num_sms * 8);
    if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
    GHB_TRY(launch(ws, sssp_init_kernel, dim3(g), dim3(256), 0, n, src, inf, dist, ns, fs, qa));
    GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(SsspCounters), st));
    int64_t near_count = 1, far_count = 0, examined = 0, rounds = 0;
    int32_t round = 0, phase = 0;
    double thr = delta;
    const SsspCounters* hc = reinterpret_cast<const SsspCounters*>(ws->host_pinned);
    // Budget: every productive round lowers some distance; n rounds per phase
    // and n phases with work bound any correct run.
    const int64_t round_budget = 64ll * n + 1024;
    while (true) {
        while (near_count > 0) {
            if (++rounds > round_budget) {
                set_error("SSSP round budget exhausted");
                return GHB_ERR_LIMIT;
            }
            ++round;
            GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, offsetof(SsspCounters, far_tail), st));
            GHB_CUDA_TRY(cudaMemsetAsync(&cnt->examined, 0, sizeof(unsigned long long), st));
            RelaxVisitor f{w, dist, thr, qb, ns, round, fa, fs, phase, cnt, 0ull};
            GHB_TRY(walk(ws, rowptr, col, (const int32_t*)qa, (const int32_t*)nullptr, near_count, near_count,
                         wb, f));
            GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, cnt, sizeof(SsspCounters), cudaMemcpyDeviceToHost, st));
            GHB_CUDA_TRY(cudaStreamSynchronize(st));
            near_count = hc->near_tail;
            far_count = hc->far_tail;
            examined += (int64_t)hc->examined;
            std::swap(qa, qb);
        }
        if (far_count == 0) break;
        // Advance the threshold past empty buckets: to the first multiple of
        // delta above the smallest far distance.
        ++phase;
        ++round;
        const double old_thr = thr;
        GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(SsspCounters), st));
        const double big = INFINITY;
        GHB_CUDA_TRY(cudaMemcpyAsync(minfar, &big, sizeof(double), cudaMemcpyHostToDevice, st));
        // Two steps: find the minimum (no moves: new_thr = old_thr), then split.
        GHB_TRY(launch(ws, sssp_split_kernel, dim3(grid_for(far_count, 256, ws->num_sms * 8)), dim3(256), 0,
                       (const int32_t*)fa, (int32_t)far_count, (const unsigned long long*)dist, old_thr, old_thr,
                       qa, ns, round, fb, fs, phase, cnt, minfar));
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, cnt, sizeof(SsspCounters), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char*>(ws->host_pinned) + 256, minfar, sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        const int64_t kept = hc->far_tail;
        const double mn = *reinterpret_cast<const double*>(reinterpret_cast<const char*>(ws->host_pinned) + 256);
        if (kept == 0) break;
        double nthr = old_thr + delta;
        if (mn >= nthr) nthr = old_thr + delta * std::floor((mn - old_thr) / delta + 1.0);
        if (!(nthr > mn)) nthr = mn + delta;  // guards rounding
        ++phase;
        ++round;
        GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(SsspCounters), st));
        GHB_TRY(launch(ws, sssp_split_kernel, dim3(grid_for(kept, 256, ws->num_sms * 8)), dim3(256), 0,
                       (const int32_t*)fb, (int32_t)kept, (const unsigned long long*)dist, old_thr, nthr, qa, ns,
                       round, fa, fs, phase, cnt, minfar));
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, cnt, sizeof(SsspCounters), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        near_count = hc->split_near;
        far_count = hc->far_tail;
        thr = nthr;
    }
    if (stats) {
        GHB_CUDA_TRY(cudaEventRecord(ws->ev_stop, st));
        unsigned long long* acc = reinterpret_cast<unsigned long long*>(ws->dev_small);
        GHB_CUDA_TRY(cudaMemsetAsync(acc, 0, 2 * sizeof(unsigned long long), st));
        GHB_TRY(launch(ws, reached_edges_kernel, dim3(g), dim3(256), 0, n, rowptr, (const double*)dist_out, inf, acc));
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, acc, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaEventSynchronize(ws->ev_stop));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        float ms = 0.f;
        GHB_CUDA_TRY(cudaEventElapsedTime(&ms, ws->ev_start, ws->ev_stop));
        const unsigned long long* ha = reinterpret_cast<const unsigned long long*>(ws->host_pinned);
        stats->levels = (int32_t)rounds;
        stats->pull_levels = phase;
        stats->edges_reached = (int64_t)ha[0];
        stats->reached = (int64_t)ha[1];
        stats->edges_examined = examined;
        stats->device_ms = ms;
    }
    return GHB_OK;
}

// Weight-sorted copy of a resident graph's rows (once per handle).
int graph_weight_sorted(ghb_workspace* ws, ghb_graph* g) {
    if (g->sw_col || g->m == 0) return GHB_OK;
    const int64_t m = g->m;
    size_t sort_tmp = 0;
    {
        cub::DoubleBuffer<uint64_t> dk(nullptr, nullptr);
        cub::DoubleBuffer<uint32_t> dv(nullptr, nullptr);
        cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, dk, dv, m, 0, 64);
    }
    Carver sizing(nullptr);
    sizing.take<uint64_t>(m);
    sizing.take<uint64_t>(m);
    sizing.take<uint32_t>(m);
    sizing.take<uint32_t>(m);
    sizing.take<char>(sort_tmp);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    uint64_t* k0 = c.take<uint64_t>(m);
    uint64_t* k1 = c.take<uint64_t>(m);
    uint32_t* v0 = c.take<uint32_t>(m);
    uint32_t* v1 = c.take<uint32_t>(m);
    void* tmp = c.take<char>(sort_tmp);
    GHB_CUDA_TRY(cudaMalloc(&g->sw_col, sizeof(int32_t) * m));
    GHB_CUDA_TRY(cudaMalloc(&g->sw_w, sizeof(double) * m));
    g->device_bytes += (int64_t)(12 * m);
    const unsigned gr = ws->num_sms * 8;
    GHB_TRY(launch(ws, weight_key_kernel, dim3(gr), dim3(256), 0, g->n, (const int32_t*)g->rowptr,
                   (const double*)g->w, k0, v0));
    cub::DoubleBuffer<uint64_t> dk(k0, k1);
    cub::DoubleBuffer<uint32_t> dv(v0, v1);
    size_t tb = sort_tmp;
    GHB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, dk, dv, m, 0, 64, ws->stream));
    ws->launches++;
    return launch(ws, weight_gather_kernel, dim3(gr), dim3(256), 0, m, (const uint32_t*)dv.Current(),
                  (const int32_t*)g->col, (const double*)g->w, g->sw_col, g->sw_w);
}

// Delta-stepping on a resident graph: each bucket's rounds relax only the
// light entries (w < delta) of its near queue; once the bucket is empty the
// heavy entries of every vertex it settled are relaxed once.  Rows are read
// from the weight-sorted copy, so a light pass reads only a row prefix.
int sssp_delta_run(ghb_workspace* ws, ghb_graph* g, int32_t src, double inf, double delta, double* dist_out,
                   ghb_traversal_stats* stats) {
    const int32_t n = g->n;
    cudaStream_t st = ws->stream;
    GHB_TRY(graph_weight_sorted(ws, g));
    // Clear the mantissa bits below the sort key's precision.
    {
        uint64_t b;
        std::memcpy(&b, &delta, sizeof(b));
        b &= ~((1ull << 25) - 1);
        std::memcpy(&delta, &b, sizeof(b));
        if (!(delta > 0)) delta = 1.0;
    }
    {
        int blocks = 0;
        if (ws->tune.sssp_persistent && sssp_persistent_available(ws, &blocks)) {
            const int32_t* le = nullptr;
            GHB_TRY(graph_light_ends(ws, g, delta, &le));
            return sssp_persistent_run(ws, n, g->rowptr, le, g->sw_col, g->sw_w, src, inf, delta, dist_out, nullptr,
                                       nullptr, stats);
        }
    }
    auto carve = [&](Carver& c, WalkBuffers* wb, int32_t** qa, int32_t** qb, int32_t** fa, int32_t** fb, int32_t** ns,
                     int32_t** fs, int32_t** rs, int32_t** R, int32_t** le, SsspCounters** cnt, double** minfar,
                     int32_t** rtail) {
        *wb = WalkBuffers::carve(c, n);
        *qa = c.take<int32_t>(n);
        *qb = c.take<int32_t>(n);
        *fa = c.take<int32_t>(n);
        *fb = c.take<int32_t>(n);
        *ns = c.take<int32_t>(n);
        *fs = c.take<int32_t>(n);
        *rs = c.take<int32_t>(n);
        *R = c.take<int32_t>(n);
        *le = c.take<int32_t>(n);
        *cnt = c.take<SsspCounters>(1);
        *minfar = c.take<double>(1);
        *rtail = c.take<int32_t>(8);
    };
    WalkBuffers wb;
    int32_t *qa, *qb, *fa, *fb, *ns, *fs, *rs, *R, *le, *rtail;
    SsspCounters* cnt;
    double* minfar;
    Carver sizing(nullptr);
    carve(sizing, &wb, &qa, &qb, &fa, &fb, &ns, &fs, &rs, &R, &le, &cnt, &minfar, &rtail);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &wb, &qa, &qb, &fa, &fb, &ns, &fs, &rs, &R, &le, &cnt, &minfar, &rtail);

    unsigned long long* dist = reinterpret_cast<unsigned long long*>(dist_out);
    const unsigned gsz = grid_for(n, 256, ws->num_sms * 8);
    if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
    GHB_TRY(launch(ws, sssp_init_kernel, dim3(gsz), dim3(256), 0, n, src, inf, dist, ns, fs, qa));
    GHB_TRY(launch(ws, fill_i32, dim3(gsz), dim3(256), 0, rs, (int64_t)n, (int32_t)-1));
    GHB_TRY(launch(ws, light_end_kernel, dim3(gsz), dim3(256), 0, n, (const int32_t*)g->rowptr,
                   (const double*)g->sw_w, delta, le));
    GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(SsspCounters), st));
    const int32_t* rp = g->rowptr;
    const int32_t* rp1 = g->rowptr + 1;
    int64_t near_count = 1, far_count = 0, examined = 0, rounds = 0;
    int32_t round = 0, phase = 0;
    double thr = delta;
    const SsspCounters* hc = reinterpret_cast<const SsspCounters*>(ws->host_pinned);
    const int64_t round_budget = 64ll * n + 1024;
    while (true) {
        int32_t r_count = 0;
        GHB_CUDA_TRY(cudaMemsetAsync(rtail, 0, sizeof(int32_t), st));
        while (true) {
            while (near_count > 0) {
                if (++rounds > round_budget) {
                    set_error("SSSP round budget exhausted");
                    return GHB_ERR_LIMIT;
                }
                ++round;
                GHB_TRY(launch(ws, mark_settled_kernel, dim3(grid_for(near_count, 256, ws->num_sms * 8)), dim3(256), 0,
                               (const int32_t*)qa, (int32_t)near_count, rs, phase, R, rtail));
                GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, offsetof(SsspCounters, far_tail), st));
                GHB_CUDA_TRY(cudaMemsetAsync(&cnt->examined, 0, sizeof(unsigned long long), st));
                RelaxVisitor f{g->sw_w, dist, thr, qb, ns, round, fa, fs, phase, cnt, 0ull};
                GHB_TRY(walk_range(ws, rp, (const int32_t*)le, g->sw_col, (const int32_t*)qa, (const int32_t*)nullptr,
                                   near_count, near_count, wb, f));
                GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, cnt, sizeof(SsspCounters), cudaMemcpyDeviceToHost, st));
                GHB_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char*>(ws->host_pinned) + 128, rtail, sizeof(int32_t),
                                             cudaMemcpyDeviceToHost, st));
                GHB_CUDA_TRY(cudaStreamSynchronize(st));
                near_count = hc->near_tail;
                far_count = hc->far_tail;
                r_count = *reinterpret_cast<const int32_t*>(reinterpret_cast<const char*>(ws->host_pinned) + 128);
                examined += (int64_t)hc->examined;
                std::swap(qa, qb);
            }
            if (r_count == 0) break;
            // Heavy entries of the vertices this bucket settled, once.
            ++round;
            GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, offsetof(SsspCounters, far_tail), st));
            GHB_CUDA_TRY(cudaMemsetAsync(&cnt->examined, 0, sizeof(unsigned long long), st));
            RelaxVisitor f{g->sw_w, dist, thr, qa, ns, round, fa, fs, phase, cnt, 0ull};
            GHB_TRY(walk_range(ws, (const int32_t*)le, rp1, g->sw_col, (const int32_t*)R, (const int32_t*)nullptr,
                               r_count, r_count, wb, f));
            GHB_CUDA_TRY(cudaMemsetAsync(rtail, 0, sizeof(int32_t), st));
            GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, cnt, sizeof(SsspCounters), cudaMemcpyDeviceToHost, st));
            GHB_CUDA_TRY(cudaStreamSynchronize(st));
            near_count = hc->near_tail;  // heavy entries landing in this bucket (rounding)
            far_count = hc->far_tail;
            examined += (int64_t)hc->examined;
            r_count = 0;
            if (near_count == 0) break;
        }
        if (far_count == 0) break;
        ++phase;
        ++round;
        const double old_thr = thr;
        GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(SsspCounters), st));
        const double big = INFINITY;
        GHB_CUDA_TRY(cudaMemcpyAsync(minfar, &big, sizeof(double), cudaMemcpyHostToDevice, st));
        GHB_TRY(launch(ws, sssp_split_kernel, dim3(grid_for(far_count, 256, ws->num_sms * 8)), dim3(256), 0,
                       (const int32_t*)fa, (int32_t)far_count, (const unsigned long long*)dist, old_thr, old_thr, qa, ns,
                       round, fb, fs, phase, cnt, minfar));
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, cnt, sizeof(SsspCounters), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char*>(ws->host_pinned) + 256, minfar, sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        const int64_t kept = hc->far_tail;
        const double mn = *reinterpret_cast<const double*>(reinterpret_cast<const char*>(ws->host_pinned) + 256);
        if (kept == 0) break;
        double nthr = old_thr + delta;
        if (mn >= nthr) nthr = old_thr + delta * std::floor((mn - old_thr) / delta + 1.0);
        if (!(nthr > mn)) nthr = mn + delta;
        ++phase;
        ++round;
        GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(SsspCounters), st));
        GHB_TRY(launch(ws, sssp_split_kernel, dim3(grid_for(kept, 256, ws->num_sms * 8)), dim3(256), 0,
                       (const int32_t*)fb, (int32_t)kept, (const unsigned long long*)dist, old_thr, nthr, qa, ns, round,
                       fa, fs, phase, cnt, minfar));
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, cnt, sizeof(SsspCounters), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        near_count = hc->split_near;
        far_count = hc->far_tail;
        thr = nthr;
    }
    if (stats) {
        GHB_CUDA_TRY(cudaEventRecord(ws->ev_stop, st));
        unsigned long long* acc = reinterpret_cast<unsigned long long*>(ws->dev_small);
        GHB_CUDA_TRY(cudaMemsetAsync(acc, 0, 2 * sizeof(unsigned long long), st));
        GHB_TRY(launch(ws, reached_edges_kernel, dim3(gsz), dim3(256), 0, n, (const int32_t*)g->rowptr,
                       (const double*)dist_out, inf, acc));
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, acc, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaEventSynchronize(ws->ev_stop));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        float ms = 0.f;
        GHB_CUDA_TRY(cudaEventElapsedTime(&ms, ws->ev_start, ws->ev_stop));
        const unsigned long long* ha = reinterpret_cast<const unsigned long long*>(ws->host_pinned);
        stats->levels = (int32_t)rounds;
        stats->pull_levels = phase;
        stats->edges_reached = (int64_t)ha[0];
        stats->reached = (int64_t)ha[1];
        stats->edges_examined = examined;
        stats->device_ms = ms;
    }
    return GHB_OK;
}

int sssp_pred_run(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, const double* w,
                  const int32_t* in_rp, const int32_t* in_col, const double* in_w, int32_t src, double inf,
                  const double* dist, int32_t* pred) {
    const unsigned g = ws->num_sms * 8;
    if (in_rp && in_w) {
        return launch(ws, sssp_pred_pull_kernel, dim3(grid_for((int64_t)n * 32, 256, g)), dim3(256), 0, n, src,
                      in_rp, in_col, in_w, dist, inf, pred);
    }
    GHB_TRY(launch(ws, fill_i32, dim3(grid_for(n, 256, g)), dim3(256), 0, pred, (int64_t)n, (int32_t)0x7fffffff));
    GHB_TRY(launch(ws, sssp_pred_push_kernel, dim3(grid_for((int64_t)n * 32, 256, g)), dim3(256), 0, n, rowptr, col,
                   w, dist, inf, pred));
    return launch(ws, sssp_pred_finish_kernel, dim3(grid_for(n, 256, g)), dim3(256), 0, n, src, pred);
}

}  // namespace ghb

using namespace ghb;

extern "C" {

int ghb_sssp(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, const double* w,
             int32_t src, double inf, double* dist, const ghb_sssp_options* options, ghb_traversal_stats* stats) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    return sssp_run(ws, n, rowptr, col, w, src, inf, dist, options, stats);
}

int ghb_sssp_pred(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, const double* w,
                  const int32_t* in_rowptr, const int32_t* in_col, const double* in_w, int32_t src, double inf,
                  double* dist, int32_t* pred, const ghb_sssp_options* options, ghb_traversal_stats* stats) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(pred, "NULL pred");
    GHB_TRY(sssp_run(ws, n, rowptr, col, w, src, inf, dist, options, stats));
    return sssp_pred_run(ws, n, rowptr, col, w, in_rowptr, in_col, in_w, src, inf, dist, pred);
}

}  // extern "C"
