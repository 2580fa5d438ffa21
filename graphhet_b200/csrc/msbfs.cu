// Multi-source BFS: up to 64 sources share one traversal, one bit per source
// in a uint64 word per vertex (the bit-parallel multi-source BFS of Then et
// al., VLDB 2014).  Every CSR entry read serves all 64 sources at once.
// Output: depth[s * n + v] = hops from srcs[s] to v (INT32_MAX unreached),
// the same values as n_src single-source runs (CPU_BFS.hpp:10-41).
//
// Per level, either
//   push: for each active v, for each out-neighbour u, atomicOr(next[u],
//         front[v] & ~seen[u]) (load-balanced walk over the active queue),
//         then a pass that turns next into the new frontier; or
//   pull: for each vertex v not yet seen by all sources, OR the frontier
//         words of its in-neighbours, stopping once every missing source
//         bit is found.
// New bits write their depths row by row, so a warp's stores to one source
// row cover 32 consecutive vertices.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "edge_walk.cuh"

namespace ghb {
namespace {

struct MsCounters {
    int32_t active;              // vertices in the new frontier
    int32_t pad;
    unsigned long long m_f;      // their out-entries
    unsigned long long examined;
};

__global__ void ms_init_kernel(int32_t n, int64_t total, int32_t* depth, uint64_t* seen, uint64_t* front,
                               uint64_t* next) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x)
        depth[i] = kInfDepth;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        seen[v] = 0;
        front[v] = 0;
        next[v] = 0;
    }
}

__global__ void ms_seed_kernel(int32_t n, const int32_t* __restrict__ srcs, int32_t k, int32_t* depth,
                               uint64_t* seen, uint64_t* front) {
    const int s = threadIdx.x;
    if (s < k) {
        const int32_t v = srcs[s];
        atomicOr((unsigned long long*)(seen + v), 1ull << s);
        atomicOr((unsigned long long*)(front + v), 1ull << s);
        depth[(int64_t)s * n + v] = 0;
    }
}

// Active queue from the seeded frontier.
__global__ void ms_queue_kernel(int32_t n, const uint64_t* __restrict__ front, const int32_t* __restrict__ rp,
                                int32_t* queue, MsCounters* cnt) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        if (front[v]) {
            const int32_t pos = warp_append_active(&cnt->active);
            queue[pos] = (int32_t)v;
            atomicAdd(&cnt->m_f, (unsigned long long)(rp[v + 1] - rp[v]));
        }
    }
}

struct MsPushVisitor {
    const uint64_t* front;
    const uint64_t* seen;
    uint64_t* next;
    unsigned long long examined;
    __device__ bool want_row(int32_t) const { return true; }
    __device__ void operator()(int32_t v, int32_t u, int32_t) {
        ++examined;
        const uint64_t bits = front[v] & ~__ldcg((const unsigned long long*)(seen + u));
        if (bits && (bits & ~__ldcg((const unsigned long long*)(next + u))))
            atomicOr((unsigned long long*)(next + u), (unsigned long long)bits);
    }
    __device__ void finish() {}
};

// Writes the depth of every new bit: a warp covers 32 consecutive vertices,
// so its stores to one source row are contiguous.
__device__ __forceinline__ void ms_write_depths(uint64_t nb, int64_t v, bool valid, int32_t n, int32_t k,
                                                int32_t lvl, int32_t* depth) {
    uint64_t any = nb;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) any |= __shfl_xor_sync(0xffffffffu, any, o);
    while (any) {
        const int s = __ffsll((long long)any) - 1;
        any &= any - 1;
        if (valid && ((nb >> s) & 1ull) && s < k) depth[(int64_t)s * n + v] = lvl;
    }
}

// After a push level: new = next & ~seen for every vertex.
__global__ void __launch_bounds__(256) ms_settle_kernel(int32_t n, int32_t k, int32_t lvl,
                                                        const int32_t* __restrict__ rp, uint64_t* seen,
                                                        uint64_t* front_new, uint64_t* next, int32_t* depth,
                                                        int32_t* queue, MsCounters* cnt) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t rounds = ((int64_t)n + stride - 1) / stride;
    unsigned long long mf = 0;
    for (int64_t r = 0; r < rounds; ++r) {
        const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x + r * stride;
        const bool valid = v < n;
        uint64_t nb = 0;
        if (valid) {
            const uint64_t x = next[v];
            const uint64_t s = seen[v];
            nb = x & ~s;
            if (x) next[v] = 0;
            front_new[v] = nb;
            if (nb) {
                seen[v] = s | nb;
                mf += (unsigned long long)(rp[v + 1] - rp[v]);
            }
        }
        if (valid && nb) queue[warp_append_active(&cnt->active)] = (int32_t)v;
        ms_write_depths(nb, v, valid, n, k, lvl, depth);
    }
    mf = warp_sum(mf);
    if (lane_id() == 0 && mf) atomicAdd(&cnt->m_f, mf);
}

// Pull level: thread per vertex over its in-row, early exit when complete.
__global__ void __launch_bounds__(256) ms_pull_kernel(int32_t n, int32_t k, int32_t lvl, uint64_t all,
                                                      const int32_t* __restrict__ in_rp,
                                                      const int32_t* __restrict__ in_col,
                                                      const int32_t* __restrict__ out_rp,
                                                      const uint64_t* __restrict__ front, uint64_t* seen,
                                                      uint64_t* front_new, int32_t* depth, int32_t* queue,
                                                      MsCounters* cnt) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t rounds = ((int64_t)n + stride - 1) / stride;
    unsigned long long mf = 0, ex = 0;
    for (int64_t r = 0; r < rounds; ++r) {
        const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x + r * stride;
        const bool valid = v < n;
        uint64_t nb = 0;
        if (valid) {
            const uint64_t s = seen[v];
            const uint64_t missing = all & ~s;
            if (missing) {
                uint64_t acc = 0;
                const int32_t b = in_rp[v], e = in_rp[v + 1];
                int32_t j = b;
                for (; j < e; ++j) {
                    acc |= front[in_col[j]];
                    if ((acc & missing) == missing) {
                        ++j;
                        break;
                    }
                }
                ex += (unsigned long long)(j - b);
                nb = acc & missing;
                if (nb) {
                    seen[v] = s | nb;
                    mf += (unsigned long long)(out_rp[v + 1] - out_rp[v]);
                }
            }
            front_new[v] = nb;
        }
        if (valid && nb) queue[warp_append_active(&cnt->active)] = (int32_t)v;
        ms_write_depths(nb, v, valid, n, k, lvl, depth);
    }
    mf = warp_sum(mf);
    ex = warp_sum(ex);
    if (lane_id() == 0) {
        if (mf) atomicAdd(&cnt->m_f, mf);
        if (ex) atomicAdd(&cnt->examined, ex);
    }
}

}  // namespace

int msbfs_batch(ghb_workspace* ws, int32_t n, const int32_t* out_rp, const int32_t* out_col, const int32_t* in_rp,
                const int32_t* in_col, const int32_t* srcs_dev, int32_t k, int32_t* depth, int64_t* levels_out,
                int64_t* examined_out) {
    cudaStream_t st = ws->stream;
    Carver sizing(nullptr);
    auto carve = [&](Carver& c, uint64_t** seen, uint64_t** fa, uint64_t** fb, uint64_t** next, int32_t** qa,
                     int32_t** qb, WalkBuffers* wb, MsCounters** cnt) {
        *seen = c.take<uint64_t>(n);
        *fa = c.take<uint64_t>(n);
        *fb = c.take<uint64_t>(n);
        *next = c.take<uint64_t>(n);
        *qa = c.take<int32_t>(n);
        *qb = c.take<int32_t>(n);
        *wb = WalkBuffers::carve(c, n);
        *cnt = c.take<MsCounters>(1);
    };
    uint64_t *seen, *fa, *fb, *next;
    int32_t *qa, *qb;
    WalkBuffers wb;
    MsCounters* cnt;
    carve(sizing, &seen, &fa, &fb, &next, &qa, &qb, &wb, &cnt);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &seen, &fa, &fb, &next, &qa, &qb, &wb, &cnt);

    const unsigned g = ws->num_sms * 8;
    const int64_t total = (int64_t)k * n;
    GHB_TRY(launch(ws, ms_init_kernel, dim3(grid_for(total, 256, g)), dim3(256), 0, n, total, depth, seen, fa, next));
    GHB_TRY(launch(ws, ms_seed_kernel, dim3(1), dim3(64), 0, n, srcs_dev, k, depth, seen, fa));
    GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(MsCounters), st));
    GHB_TRY(launch(ws, ms_queue_kernel, dim3(grid_for(n, 256, g)), dim3(256), 0, n, (const uint64_t*)fa, out_rp, qa, cnt));
    GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, cnt, sizeof(MsCounters), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const MsCounters* hc = reinterpret_cast<const MsCounters*>(ws->host_pinned);
    int64_t active = hc->active, m_f = (int64_t)hc->m_f;
    int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned) + 64;
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, out_rp + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t m = hp[0];
    const uint64_t all = (k == 64) ? ~0ull : ((1ull << k) - 1ull);
    const bool can_pull = in_rp != nullptr && in_col != nullptr;
    int32_t lvl = 0;
    int64_t examined = 0;
    uint64_t *f_cur = fa, *f_new = fb;
    int32_t *q_cur = qa, *q_new = qb;
    while (active > 0 && lvl < n) {
        ++lvl;
        GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(MsCounters), st));
        // Pull when the frontier's out-entries are a large share of the graph.
        const bool pull = can_pull && (double)m_f * 8.0 > (double)m;
        if (pull) {
            GHB_TRY(launch(ws, ms_pull_kernel, dim3(grid_for(n, 256, g)), dim3(256), 0, n, k, lvl, all, in_rp, in_col,
                           out_rp, (const uint64_t*)f_cur, seen, f_new, depth, q_new, cnt));
        } else {
            MsPushVisitor f{f_cur, seen, next, 0ull};
            GHB_TRY(walk(ws, out_rp, out_col, (const int32_t*)q_cur, (const int32_t*)nullptr, active, active, wb, f));
            examined += m_f;
            GHB_TRY(launch(ws, ms_settle_kernel, dim3(grid_for(n, 256, g)), dim3(256), 0, n, k, lvl, out_rp, seen,
                           f_new, next, depth, q_new, cnt));
        }
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, cnt, sizeof(MsCounters), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        active = hc->active;
        m_f = (int64_t)hc->m_f;
        examined += (int64_t)hc->examined;
        std::swap(f_cur, f_new);
        std::swap(q_cur, q_new);
    }
    if (levels_out) *levels_out += lvl;
    if (examined_out) *examined_out += examined;
    return GHB_OK;
}

}  // namespace ghb

using namespace ghb;

extern "C" int ghb_msbfs(ghb_workspace* ws, int32_t n, const int32_t* out_rowptr, const int32_t* out_col,
                         const int32_t* in_rowptr, const int32_t* in_col, const int32_t* srcs, int32_t n_src,
                         int32_t* depth, ghb_traversal_stats* stats) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(out_rowptr && depth && srcs, "NULL argument");
    GHB_REQUIRE(n_src >= 0, "n_src < 0");
    cudaStream_t st = ws->stream;
    // Validate the sources on the host (they are a device array).
    std::vector<int32_t> hs(n_src > 0 ? n_src : 1);
    if (n_src > 0) {
        GHB_CUDA_TRY(cudaMemcpyAsync(hs.data(), srcs, sizeof(int32_t) * n_src, cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
    }
    for (int32_t i = 0; i < n_src; ++i) GHB_REQUIRE(hs[i] >= 0 && hs[i] < n, "source outside [0, n)");
    if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
    int64_t levels = 0, examined = 0;
    for (int32_t s0 = 0; s0 < n_src; s0 += 64) {
        const int32_t k = std::min<int32_t>(64, n_src - s0);
        GHB_TRY(msbfs_batch(ws, n, out_rowptr, out_col, in_rowptr, in_col, srcs + s0, k, depth + (int64_t)s0 * n,
                            &levels, &examined));
    }
    if (stats) {
        GHB_CUDA_TRY(cudaEventRecord(ws->ev_stop, st));
        GHB_CUDA_TRY(cudaEventSynchronize(ws->ev_stop));
        float ms = 0.f;
        GHB_CUDA_TRY(cudaEventElapsedTime(&ms, ws->ev_start, ws->ev_stop));
        stats->levels = (int32_t)levels;
        stats->pull_levels = 0;
        stats->reached = -1;
        stats->edges_reached = -1;
        stats->edges_examined = examined;
        stats->device_ms = ms;
    }
    return GHB_OK;
}
