// Multi-source BFS: up to 256 sources share one traversal, one bit per source
// in W = 1, 2 or 4 uint64 words per vertex (the bit-parallel multi-source
// BFS of Then et al., VLDB 2014).  Every CSR entry read serves all the
// pass's sources at once; with W = 4 a vertex's frontier words are one
// 32-byte sector, so a gather costs what it costs for 64 sources.
// Output: depth[s * n + v] = hops from srcs[s] to v (INT32_MAX unreached),
// the same values as n_src single-source runs (CPU_BFS.hpp:10-41).
//
// Per level, either
//   push: for each active v, for each out-neighbour u, atomicOr(next[u],
//         front[v] & ~seen[u]) (load-balanced walk over the active queue),
//         then a pass that turns next into the new frontier; or
//   pull: for each vertex v not yet seen by all sources, OR the frontier
//         words of its in-neighbours, stopping once every missing source
//         bit is found.  The first 16 entries are probed by the vertex's
//         own thread (4 gathers in flight); rows with up to ms_warp_rest
//         more entries (a workspace tunable, 256 by default) are finished by
//         the whole warp, 32 entries a step; longer
//         ones by a block each (ms_pull_hub_kernel), so the hubs that a
//         degree-ordered graph puts side by side never serialise one warp.
// Every level writes its new-bit words densely (front_new); the words of the
// last chunk of levels are kept, and after every chunk (and at the end)
// ms_flush_kernel turns them into depths, thread per output vertex in the
// caller's ids, so a warp's stores to one source row cover 32 consecutive
// vertices and a relabelled graph needs no separate mapping pass.  Each depth
// entry is written once: at the flush of the level that reached it, or as
// INT32_MAX by the final flush.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "edge_walk.cuh"

namespace ghb {
namespace {

struct MsCounters {
    int32_t active;              // vertices in the new frontier
    int32_t hubs;                // pull rows deferred to ms_pull_hub_kernel
    unsigned long long m_f;      // their out-entries
    unsigned long long examined;
};

// Levels of new-bit words kept between flushes: up to kMsChunkMax, fewer when
// kMsMaskBudget bytes do not hold that many (n x W words each).
constexpr int kMsChunkMax = 16;
constexpr size_t kMsMaskBudget = size_t(8) << 30;

__global__ void ms_init_kernel(int64_t words, uint64_t* seen, uint64_t* front, uint64_t* next) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < words; i += (int64_t)gridDim.x * blockDim.x) {
        seen[i] = 0;
        front[i] = 0;
        next[i] = 0;
    }
}

template <int W>
__global__ void ms_seed_kernel(const int32_t* __restrict__ srcs, int32_t k, uint64_t* seen, uint64_t* front) {
    const int s = threadIdx.x;
    if (s < k) {
        const int32_t v = srcs[s];
        const unsigned long long bit = 1ull << (s & 63);
        atomicOr((unsigned long long*)(seen + (int64_t)v * W + (s >> 6)), bit);
        atomicOr((unsigned long long*)(front + (int64_t)v * W + (s >> 6)), bit);
    }
}

// Active queue from the seeded frontier.
template <int W>
__global__ void ms_queue_kernel(int32_t n, const uint64_t* __restrict__ front, const int32_t* __restrict__ rp,
                                int32_t* queue, MsCounters* cnt) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        uint64_t any = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) any |= front[v * W + w];
        if (any) {
            const int32_t pos = warp_append_active(&cnt->active);
            queue[pos] = (int32_t)v;
            atomicAdd(&cnt->m_f, (unsigned long long)(rp[v + 1] - rp[v]));
        }
    }
}

template <int W>
struct MsPushVisitor {
    const uint64_t* front;
    const uint64_t* seen;
    uint64_t* next;
    __device__ bool want_row(int32_t) const { return true; }
    __device__ void operator()(int32_t v, int32_t u, int32_t) {
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const int64_t iu = (int64_t)u * W + w;
            const uint64_t bits = front[(int64_t)v * W + w] & ~__ldcg((const unsigned long long*)(seen + iu));
            if (bits && (bits & ~__ldcg((const unsigned long long*)(next + iu))))
                atomicOr((unsigned long long*)(next + iu), (unsigned long long)bits);
        }
    }
    __device__ void finish() {}
};

// After a push level: new = next & ~seen for every vertex of [0, n_scan).
template <int W>
__global__ void __launch_bounds__(256) ms_settle_kernel(int32_t n_scan, const int32_t* __restrict__ rp,
                                                        uint64_t* seen, uint64_t* front_new, uint64_t* next,
                                                        int32_t* queue, MsCounters* cnt) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t rounds = ((int64_t)n_scan + stride - 1) / stride;
    unsigned long long mf = 0;
    for (int64_t r = 0; r < rounds; ++r) {
        const int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x + r * stride;
        const bool valid = v < n_scan;
        uint64_t nb[W];
        bool anyb = false;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            nb[w] = 0;
            if (valid) {
                const uint64_t x = next[v * W + w];
                const uint64_t s = seen[v * W + w];
                nb[w] = x & ~s;
                if (x) next[v * W + w] = 0;
                front_new[v * W + w] = nb[w];
                if (nb[w]) seen[v * W + w] = s | nb[w];
            }
            anyb |= nb[w] != 0;
        }
        if (anyb) {
            mf += (unsigned long long)(rp[v + 1] - rp[v]);
            queue[warp_append_active(&cnt->active)] = (int32_t)v;
        }
    }
    mf = warp_sum(mf);
    if (lane_id() == 0 && mf) atomicAdd(&cnt->m_f, mf);
}

template <int W>
__device__ __forceinline__ bool ms_covers(const uint64_t* acc, const uint64_t* missing) {
    bool ok = true;
#pragma unroll
    for (int w = 0; w < W; ++w) ok &= (acc[w] & missing[w]) == missing[w];
    return ok;
}

// Pull level over [0, n_scan): a warp owns 32 consecutive vertices.
template <int W>
__global__ void __launch_bounds__(256) ms_pull_kernel(int32_t n_scan, const uint64_t* __restrict__ all,
                                                      const int32_t* __restrict__ in_rp,
                                                      const int32_t* __restrict__ in_col,
                                                      const int32_t* __restrict__ out_rp,
                                                      const uint64_t* __restrict__ front, uint64_t* seen,
                                                      uint64_t* front_new, int32_t* queue, int32_t* hubs,
                                                      MsCounters* cnt, int32_t warp_rest) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long mf = 0, ex = 0;
    for (int64_t base = warp * 32; base < n_scan; base += nwarps * 32) {
        const int64_t v = base + lane;
        const bool valid = v < n_scan;
        uint64_t s[W], missing[W], acc[W];
        bool anym = false;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            s[w] = valid ? seen[v * W + w] : ~0ull;
            missing[w] = all[w] & ~s[w];
            acc[w] = 0;
            anym |= missing[w] != 0;
        }
        int32_t j = 0, e = 0;
        bool done = !anym;
        if (anym) {
            j = in_rp[v];
            e = in_rp[v + 1];
            const int32_t b = j;
            const int32_t lim = min(e, b + 16);
            while (j < lim && !done) {
                int32_t u[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) u[q] = (j + q < lim) ? in_col[j + q] : -1;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (u[q] >= 0) {
#pragma unroll
                        for (int w = 0; w < W; ++w) acc[w] |= front[(int64_t)u[q] * W + w];
                    }
                j = min(j + 4, lim);
                done = ms_covers<W>(acc, missing);
            }
            ex += (unsigned long long)(j - b);
            if (!done && e - j > warp_rest) {
                // Long row: a block of ms_pull_hub_kernel settles it.  Here
                // it stays as it is (no new bits; front_new is rewritten there).
                hubs[atomicAdd(&cnt->hubs, 1)] = (int32_t)v;
                done = true;
#pragma unroll
                for (int w = 0; w < W; ++w) missing[w] = 0;
            }
        }
        // Rows not covered by their first 16 entries: the whole warp walks
        // the rest, 32 entries per step, one row at a time.
        unsigned rest = __ballot_sync(0xffffffffu, !done && j < e);
        while (rest) {
            const int leader = __ffs(rest) - 1;
            const int32_t lj = __shfl_sync(0xffffffffu, j, leader);
            const int32_t le = __shfl_sync(0xffffffffu, e, leader);
            uint64_t lm[W], la[W];
#pragma unroll
            for (int w = 0; w < W; ++w) {
                lm[w] = __shfl_sync(0xffffffffu, missing[w], leader);
                la[w] = __shfl_sync(0xffffffffu, acc[w], leader);
            }
            int32_t scanned = 0;
            for (int32_t k0 = lj; k0 < le; k0 += 32) {
                const int32_t kk = k0 + lane;
                uint64_t p[W];
#pragma unroll
                for (int w = 0; w < W; ++w) p[w] = 0;
                if (kk < le) {
                    const int64_t u = in_col[kk];
#pragma unroll
                    for (int w = 0; w < W; ++w) p[w] = front[u * W + w];
                }
#pragma unroll
                for (int w = 0; w < W; ++w) {
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) p[w] |= __shfl_xor_sync(0xffffffffu, p[w], o);
                    la[w] |= p[w];
                }
                scanned += min(32, le - k0);
                if (ms_covers<W>(la, lm)) break;
            }
            if (lane == leader) {
#pragma unroll
                for (int w = 0; w < W; ++w) acc[w] = la[w];
                ex += (unsigned long long)scanned;
            }
            rest &= rest - 1;
        }
        uint64_t nb[W];
        bool anyb = false;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            nb[w] = acc[w] & missing[w];
            anyb |= nb[w] != 0;
            if (valid) {
                front_new[v * W + w] = nb[w];
                if (nb[w]) seen[v * W + w] = s[w] | nb[w];
            }
        }
        if (anyb) {
            mf += (unsigned long long)(out_rp[v + 1] - out_rp[v]);
            queue[warp_append_active(&cnt->active)] = (int32_t)v;
        }
    }
    mf = warp_sum(mf);
    ex = warp_sum(ex);
    if (lane == 0) {
        if (mf) atomicAdd(&cnt->m_f, mf);
        if (ex) atomicAdd(&cnt->examined, ex);
    }
}

// Deferred pull rows: one block per row (round robin over the list).  The
// block's threads OR the frontier words of strided entries (4 gathers in
// flight each), re-check coverage every 4 x blockDim entries and stop early
// like the warp path; then the block settles the vertex.
template <int W>
__global__ void __launch_bounds__(256) ms_pull_hub_kernel(const uint64_t* __restrict__ all,
                                                          const int32_t* __restrict__ in_rp,
                                                          const int32_t* __restrict__ in_col,
                                                          const int32_t* __restrict__ out_rp,
                                                          const uint64_t* __restrict__ front, uint64_t* seen,
                                                          uint64_t* front_new, int32_t* queue,
                                                          const int32_t* __restrict__ hubs, MsCounters* cnt) {
    __shared__ unsigned long long s_acc[W];
    __shared__ int s_done;
    const int32_t count = *(volatile int32_t*)&cnt->hubs;
    unsigned long long ex = 0, mf = 0;
    for (int32_t r = blockIdx.x; r < count; r += gridDim.x) {
        const int32_t v = hubs[r];
        uint64_t missing[W], sv[W];
#pragma unroll
        for (int w = 0; w < W; ++w) {
            sv[w] = seen[(int64_t)v * W + w];
            missing[w] = all[w] & ~sv[w];
        }
        if (threadIdx.x < W) s_acc[threadIdx.x] = 0ull;
        if (threadIdx.x == 0) s_done = 0;
        __syncthreads();
        const int32_t b = in_rp[v], e = in_rp[v + 1];
        const int32_t step = 4 * (int32_t)blockDim.x;
        int32_t scanned = 0;
        for (int32_t c0 = b; c0 < e; c0 += step) {
            uint64_t p[W];
#pragma unroll
            for (int w = 0; w < W; ++w) p[w] = 0;
            int32_t u[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int32_t j = c0 + q * (int32_t)blockDim.x + (int32_t)threadIdx.x;
                u[q] = j < e ? in_col[j] : -1;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (u[q] >= 0) {
#pragma unroll
                    for (int w = 0; w < W; ++w) p[w] |= front[(int64_t)u[q] * W + w];
                }
#pragma unroll
            for (int w = 0; w < W; ++w) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) p[w] |= __shfl_xor_sync(0xffffffffu, p[w], o);
                if (lane_id() == 0 && (p[w] & missing[w])) atomicOr(&s_acc[w], (unsigned long long)(p[w] & missing[w]));
            }
            scanned += min(step, e - c0);
            __syncthreads();
            if (threadIdx.x == 0) {
                bool ok = true;
#pragma unroll
                for (int w = 0; w < W; ++w) ok &= (s_acc[w] & missing[w]) == missing[w];
                s_done = ok ? 1 : 0;
            }
            __syncthreads();
            if (s_done) break;
        }
        uint64_t nb[W];
        bool anyb = false;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            nb[w] = s_acc[w] & missing[w];
            anyb |= nb[w] != 0;
        }
        if (threadIdx.x == 0) {
            ex += (unsigned long long)scanned;
#pragma unroll
            for (int w = 0; w < W; ++w) {
                front_new[(int64_t)v * W + w] = nb[w];
                if (nb[w]) seen[(int64_t)v * W + w] = sv[w] | nb[w];
            }
            if (anyb) {
                mf += (unsigned long long)(out_rp[v + 1] - out_rp[v]);
                queue[atomicAdd(&cnt->active, 1)] = v;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (mf) atomicAdd(&cnt->m_f, mf);
        if (ex) atomicAdd(&cnt->examined, ex);
    }
}

// Depths of levels [l0, l1] (at most `chunk`, level l kept in slot l % chunk
// of `masks`), thread per output vertex v in the caller's ids (internal id
// p = perm[v], or v without perm).  The level of each bit inside the chunk
// is read from four bit-slices of the chunk's words (slice t ORs the levels
// whose index has bit t).  The final flush also writes INT32_MAX for every
// source bit that v never received.  Vertices p >= n_scan have no entries:
// only level 0 (a source) can reach them.
template <int W>
__global__ void __launch_bounds__(256) ms_flush_kernel(int32_t n, int32_t n_scan, int32_t k,
                                                       const int32_t* __restrict__ perm,
                                                       const uint64_t* __restrict__ masks, int32_t chunk, int32_t l0,
                                                       int32_t l1, bool final_flush,
                                                       const uint64_t* __restrict__ seen, int32_t* depth) {
    const int64_t slot = (int64_t)n * W;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = perm ? perm[v] : v;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            if (w * 64 >= k) break;
            uint64_t any = 0, sl0 = 0, sl1 = 0, sl2 = 0, sl3 = 0;
            for (int32_t l = l0; l <= l1; ++l) {
                if (p >= n_scan && l > 0) break;
                const uint64_t m = masks[(int64_t)(l % chunk) * slot + p * W + w];
                const int i = l - l0;
                any |= m;
                sl0 |= (i & 1) ? m : 0ull;
                sl1 |= (i & 2) ? m : 0ull;
                sl2 |= (i & 4) ? m : 0ull;
                sl3 |= (i & 8) ? m : 0ull;
            }
            const uint64_t unreached = final_flush ? ~seen[p * W + w] : 0ull;
            if (!(any | unreached)) continue;
            const int bmax = min(64, k - w * 64);
            for (int b = 0; b < bmax; ++b) {
                const int32_t d = l0 + (int32_t)((sl0 >> b) & 1ull) + 2 * (int32_t)((sl1 >> b) & 1ull) +
                                  4 * (int32_t)((sl2 >> b) & 1ull) + 8 * (int32_t)((sl3 >> b) & 1ull);
                if ((any >> b) & 1ull) depth[(int64_t)(w * 64 + b) * n + v] = d;
                else if ((unreached >> b) & 1ull) depth[(int64_t)(w * 64 + b) * n + v] = kInfDepth;
            }
        }
    }
}

template <int W>
int msbfs_pass(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* out_rp, const int32_t* out_col,
               const int32_t* in_rp, const int32_t* in_col, const int32_t* srcs_dev, int32_t k,
               const int32_t* perm, int32_t* depth, int64_t* levels_out, int64_t* examined_out) {
    cudaStream_t st = ws->stream;
    const int64_t words = (int64_t)n * W;
    const int32_t chunk = (int32_t)std::max<int64_t>(
        2, std::min<int64_t>(kMsChunkMax, (int64_t)(kMsMaskBudget / (size_t)(words * sizeof(uint64_t)))));
    Carver sizing(nullptr);
    auto carve = [&](Carver& c, uint64_t** seen, uint64_t** masks, uint64_t** next, int32_t** qa, int32_t** qb,
                     WalkBuffers* wb, MsCounters** cnt, uint64_t** all, int32_t** hubs) {
        *seen = c.take<uint64_t>(words);
        *masks = c.take<uint64_t>(words * chunk);
        *next = c.take<uint64_t>(words);
        *qa = c.take<int32_t>(n);
        *qb = c.take<int32_t>(n);
        *wb = WalkBuffers::carve(c, n);
        *cnt = c.take<MsCounters>(1);
        *all = c.take<uint64_t>(4);
        *hubs = c.take<int32_t>(n);
    };
    uint64_t *seen, *masks, *next, *all;
    int32_t *qa, *qb, *hubs;
    WalkBuffers wb;
    MsCounters* cnt;
    carve(sizing, &seen, &masks, &next, &qa, &qb, &wb, &cnt, &all, &hubs);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &seen, &masks, &next, &qa, &qb, &wb, &cnt, &all, &hubs);
    auto slot = [&](int32_t l) { return masks + (int64_t)(l % chunk) * words; };

    const unsigned g = ws->num_sms * 8;
    // Source masks per word (built on the host: k is known here).
    uint64_t* hall = reinterpret_cast<uint64_t*>(ws->host_pinned) + 32;
    for (int w = 0; w < 4; ++w) {
        const int b = k - 64 * w;
        hall[w] = b >= 64 ? ~0ull : (b <= 0 ? 0ull : ((1ull << b) - 1ull));
    }
    GHB_CUDA_TRY(cudaMemcpyAsync(all, hall, 4 * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    GHB_TRY(launch(ws, ms_init_kernel, dim3(grid_for(words, 256, g)), dim3(256), 0, words, seen, slot(0), next));
    GHB_TRY(launch(ws, ms_seed_kernel<W>, dim3(1), dim3(256), 0, srcs_dev, k, seen, slot(0)));
    GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(MsCounters), st));
    GHB_TRY(launch(ws, ms_queue_kernel<W>, dim3(grid_for(n, 256, g)), dim3(256), 0, n, (const uint64_t*)slot(0),
                   out_rp, qa, cnt));
    int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned) + 64;
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, out_rp + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, cnt, sizeof(MsCounters), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const MsCounters* hc = reinterpret_cast<const MsCounters*>(ws->host_pinned);
    int64_t active = hc->active, m_f = (int64_t)hc->m_f;
    const int64_t m = hp[0];
    const bool can_pull = in_rp != nullptr && in_col != nullptr;
    int32_t lvl = 0, flushed = 0;  // levels [flushed, lvl] not yet turned into depths
    int64_t examined = 0;
    int32_t *q_cur = qa, *q_new = qb;
    auto flush = [&](int32_t l1, bool final_flush) -> int {
        return launch(ws, ms_flush_kernel<W>, dim3(grid_for(n, 256, g)), dim3(256), 0, n, n_active, k, perm,
                      (const uint64_t*)masks, chunk, flushed, l1, final_flush, (const uint64_t*)seen, depth);
    };
    while (active > 0 && lvl < n) {
        ++lvl;
        uint64_t* f_cur = slot(lvl - 1);
        uint64_t* f_new = slot(lvl);
        GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(MsCounters), st));
        // Pull when the frontier's out-entries are a large share of the graph.
        const bool pull = can_pull && (double)m_f * (double)ws->tune.ms_pull_div > (double)m;
        if (pull) {
            GHB_TRY(launch(ws, ms_pull_kernel<W>, dim3(grid_for((int64_t)n_active, 256, g)), dim3(256), 0, n_active,
                           (const uint64_t*)all, in_rp, in_col, out_rp, (const uint64_t*)f_cur, seen, f_new, q_new,
                           hubs, cnt, ws->tune.ms_warp_rest));
            GHB_TRY(launch(ws, ms_pull_hub_kernel<W>, dim3(ws->num_sms * 4), dim3(256), 0, (const uint64_t*)all, in_rp,
                           in_col, out_rp, (const uint64_t*)f_cur, seen, f_new, q_new, (const int32_t*)hubs, cnt));
        } else {
            MsPushVisitor<W> f{f_cur, seen, next};
            GHB_TRY(walk(ws, out_rp, out_col, (const int32_t*)q_cur, (const int32_t*)nullptr, active, active, wb, f));
            examined += m_f;
            GHB_TRY(launch(ws, ms_settle_kernel<W>, dim3(grid_for((int64_t)n_active, 256, g)), dim3(256), 0, n_active,
                           out_rp, seen, f_new, next, q_new, cnt));
        }
        // The next level overwrites slot lvl + 1: flush a full chunk first.
        if ((lvl + 1) % chunk == 0) {
            GHB_TRY(flush(lvl, false));
            flushed = lvl + 1;
        }
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, cnt, sizeof(MsCounters), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        active = hc->active;
        m_f = (int64_t)hc->m_f;
        examined += (int64_t)hc->examined;
        std::swap(q_cur, q_new);
    }
    GHB_TRY(flush(lvl, true));
    if (levels_out) *levels_out += lvl;
    if (examined_out) *examined_out += examined;
    return GHB_OK;
}

}  // namespace

// One pass of up to kMsPass sources: W = ceil(k / 64) words per vertex (4 for
// 129..256).  n_active: vertices [n_active, n) have no entries (a relabelled
// graph puts them last); only sources can be reached there.  depth (k x n)
// is in the caller's ids: depth[s * n + v] belongs to internal vertex
// perm[v] (v itself when perm is NULL).
int msbfs_batch(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* out_rp, const int32_t* out_col,
                const int32_t* in_rp, const int32_t* in_col, const int32_t* srcs_dev, int32_t k,
                const int32_t* perm, int32_t* depth, int64_t* levels_out, int64_t* examined_out) {
    GHB_REQUIRE(k >= 1 && k <= kMsPass, "multi-source pass of 1..256 sources");
    if (k <= 64)
        return msbfs_pass<1>(ws, n, n_active, out_rp, out_col, in_rp, in_col, srcs_dev, k, perm, depth, levels_out,
                             examined_out);
    if (k <= 128)
        return msbfs_pass<2>(ws, n, n_active, out_rp, out_col, in_rp, in_col, srcs_dev, k, perm, depth, levels_out,
                             examined_out);
    return msbfs_pass<4>(ws, n, n_active, out_rp, out_col, in_rp, in_col, srcs_dev, k, perm, depth, levels_out,
                         examined_out);
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
    for (int32_t s0 = 0; s0 < n_src; s0 += kMsPass) {
        const int32_t k = std::min<int32_t>(kMsPass, n_src - s0);
        GHB_TRY(msbfs_batch(ws, n, n, out_rowptr, out_col, in_rowptr, in_col, srcs + s0, k, nullptr,
                            depth + (int64_t)s0 * n, &levels, &examined));
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
