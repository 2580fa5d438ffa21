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
#include <cmath>
#include <cstring>
#include <mutex>
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

// Each phase below is a __device__ body (grid-stride over the launch's
// grid) with a thin kernel around it: the host-driven pass launches the
// kernels, the whole-pass cooperative kernel calls the bodies between its
// grid barriers.
__device__ __forceinline__ void ms_init_body(int64_t words, uint64_t* seen, uint64_t* front, uint64_t* next) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < words; i += (int64_t)gridDim.x * blockDim.x) {
        seen[i] = 0;
        front[i] = 0;
        next[i] = 0;
    }
}
__global__ void ms_init_kernel(int64_t words, uint64_t* seen, uint64_t* front, uint64_t* next) {
    ms_init_body(words, seen, front, next);
}

// Loads of words that the whole-pass kernel writes in an earlier phase go
// through L2 (a line an SM cached before that write could be stale in its
// L1), and no such array is declared __restrict__ const.
__device__ __forceinline__ uint64_t ms_ld(const uint64_t* p) {
    return (uint64_t)__ldcg(reinterpret_cast<const unsigned long long*>(p));
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
__device__ __forceinline__ void ms_queue_body(int32_t n, const uint64_t* front, const int32_t* __restrict__ rp,
                                              int32_t* queue, MsCounters* cnt) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        uint64_t any = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) any |= ms_ld(front + v * W + w);
        if (any) {
            const int32_t pos = warp_append_active(&cnt->active);
            queue[pos] = (int32_t)v;
            atomicAdd(&cnt->m_f, (unsigned long long)(rp[v + 1] - rp[v]));
        }
    }
}
template <int W>
__global__ void ms_queue_kernel(int32_t n, const uint64_t* front, const int32_t* __restrict__ rp, int32_t* queue,
                                MsCounters* cnt) {
    ms_queue_body<W>(n, front, rp, queue, cnt);
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
            const uint64_t bits = ms_ld(front + (int64_t)v * W + w) & ~__ldcg((const unsigned long long*)(seen + iu));
            if (bits && (bits & ~__ldcg((const unsigned long long*)(next + iu))))
                atomicOr((unsigned long long*)(next + iu), (unsigned long long)bits);
        }
    }
    __device__ void finish() {}
};

// After a push level: new = next & ~seen for every vertex of [0, n_scan).
template <int W>
__device__ __forceinline__ void ms_settle_body(int32_t n_scan, const int32_t* __restrict__ rp, uint64_t* seen,
                                               uint64_t* front_new, uint64_t* next, int32_t* queue, MsCounters* cnt) {
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
                const uint64_t x = ms_ld(next + v * W + w);
                const uint64_t s = ms_ld(seen + v * W + w);
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
__global__ void __launch_bounds__(256) ms_settle_kernel(int32_t n_scan, const int32_t* __restrict__ rp,
                                                        uint64_t* seen, uint64_t* front_new, uint64_t* next,
                                                        int32_t* queue, MsCounters* cnt) {
    ms_settle_body<W>(n_scan, rp, seen, front_new, next, queue, cnt);
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
__device__ __forceinline__ void ms_pull_body(int32_t n_scan, const uint64_t* all, const int32_t* __restrict__ in_rp,
                                             const int32_t* __restrict__ in_col, const int32_t* __restrict__ out_rp,
                                             const uint64_t* front, uint64_t* seen, uint64_t* front_new,
                                             int32_t* queue, int32_t* hubs, MsCounters* cnt, int32_t warp_rest) {
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
            s[w] = valid ? ms_ld(seen + v * W + w) : ~0ull;
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
                        for (int w = 0; w < W; ++w) acc[w] |= ms_ld(front + (int64_t)u[q] * W + w);
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
                    for (int w = 0; w < W; ++w) p[w] = ms_ld(front + u * W + w);
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
template <int W>
__global__ void __launch_bounds__(256) ms_pull_kernel(int32_t n_scan, const uint64_t* all,
                                                      const int32_t* __restrict__ in_rp,
                                                      const int32_t* __restrict__ in_col,
                                                      const int32_t* __restrict__ out_rp, const uint64_t* front,
                                                      uint64_t* seen, uint64_t* front_new, int32_t* queue,
                                                      int32_t* hubs, MsCounters* cnt, int32_t warp_rest) {
    ms_pull_body<W>(n_scan, all, in_rp, in_col, out_rp, front, seen, front_new, queue, hubs, cnt, warp_rest);
}

// Deferred pull rows: one block per row (round robin over the list).  The
// block's threads OR the frontier words of strided entries (4 gathers in
// flight each), re-check coverage every 4 x blockDim entries and stop early
// like the warp path; then the block settles the vertex.
template <int W>
__device__ __forceinline__ void ms_pull_hub_body(const uint64_t* all, const int32_t* __restrict__ in_rp,
                                                 const int32_t* __restrict__ in_col,
                                                 const int32_t* __restrict__ out_rp, const uint64_t* front,
                                                 uint64_t* seen, uint64_t* front_new, int32_t* queue,
                                                 const int32_t* hubs, MsCounters* cnt) {
    __shared__ unsigned long long s_acc[W];
    __shared__ int s_done;
    const int32_t count = *(volatile int32_t*)&cnt->hubs;
    unsigned long long ex = 0, mf = 0;
    for (int32_t r = blockIdx.x; r < count; r += gridDim.x) {
        const int32_t v = __ldcg(hubs + r);
        uint64_t missing[W], sv[W];
#pragma unroll
        for (int w = 0; w < W; ++w) {
            sv[w] = ms_ld(seen + (int64_t)v * W + w);
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
                    for (int w = 0; w < W; ++w) p[w] |= ms_ld(front + (int64_t)u[q] * W + w);
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
template <int W>
__global__ void __launch_bounds__(256) ms_pull_hub_kernel(const uint64_t* all, const int32_t* __restrict__ in_rp,
                                                          const int32_t* __restrict__ in_col,
                                                          const int32_t* __restrict__ out_rp, const uint64_t* front,
                                                          uint64_t* seen, uint64_t* front_new, int32_t* queue,
                                                          const int32_t* hubs, MsCounters* cnt) {
    ms_pull_hub_body<W>(all, in_rp, in_col, out_rp, front, seen, front_new, queue, hubs, cnt);
}

// Depths of levels [l0, l1] (at most `chunk`, level l kept in slot l % chunk
// of `masks`), thread per output vertex v in the caller's ids (internal id
// p = perm[v], or v without perm).  The level of each bit inside the chunk
// is read from four bit-slices of the chunk's words (slice t ORs the levels
// whose index has bit t).  The final flush also writes INT32_MAX for every
// source bit that v never received.  Vertices p >= n_scan have no entries:
// only level 0 (a source) can reach them.
template <int W>
__device__ __forceinline__ void ms_flush_body(int32_t n, int32_t n_scan, int32_t k, const int32_t* __restrict__ perm,
                                              const uint64_t* masks, int32_t chunk, int32_t l0, int32_t l1,
                                              bool final_flush, const uint64_t* seen, int32_t* depth) {
    const int64_t slot = (int64_t)n * W;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = perm ? perm[v] : v;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            if (w * 64 >= k) break;
            uint64_t any = 0, sl0 = 0, sl1 = 0, sl2 = 0, sl3 = 0;
            for (int32_t l = l0; l <= l1; ++l) {
                if (p >= n_scan && l > 0) break;
                const uint64_t m = ms_ld(masks + (int64_t)(l % chunk) * slot + p * W + w);
                const int i = l - l0;
                any |= m;
                sl0 |= (i & 1) ? m : 0ull;
                sl1 |= (i & 2) ? m : 0ull;
                sl2 |= (i & 4) ? m : 0ull;
                sl3 |= (i & 8) ? m : 0ull;
            }
            const uint64_t unreached = final_flush ? ~ms_ld(seen + p * W + w) : 0ull;
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
__global__ void __launch_bounds__(256) ms_flush_kernel(int32_t n, int32_t n_scan, int32_t k,
                                                       const int32_t* __restrict__ perm, const uint64_t* masks,
                                                       int32_t chunk, int32_t l0, int32_t l1, bool final_flush,
                                                       const uint64_t* seen, int32_t* depth) {
    ms_flush_body<W>(n, n_scan, k, perm, masks, chunk, l0, l1, final_flush, seen, depth);
}

// ---------------------------------------------------------------------------
// The whole pass in one cooperative launch: set-up, every level (push: walk,
// deferred long-row chunks, settle; pull: rows, deferred hub rows), the
// flushes, separated by the bounded grid barrier.  The last block to arrive
// at a level's final barrier reads the level's counters and decides the
// next level's direction (the rule of the host-driven pass) or the end.
// Nothing goes back to the host, so the launch can be recorded in a CUDA
// graph.

constexpr int kMsThreads = 256;
constexpr int kMsPolicyFeatures = 8;
constexpr int kMsPolicyWeights = kMsPolicyFeatures + 1;

// Features of a multi-source level decision (the same definitions as the
// trainer's, graphhet_b200/policy.py ms_rows): the next frontier's share of
// the entries and of the vertices, the mean degree, the pass's source
// count, the level index, the frontier vertices visited so far, the last
// level's direction and the frontier's growth, all but two as log2.
__device__ __forceinline__ void ms_level_features(float* f, double mf, double active, double prev_active,
                                                  double visits, double n, double m, int k, int level,
                                                  int prev_pull) {
    const double tiny = 1.0 / 1073741824.0;
    f[0] = (float)log2(mf / m + tiny);
    f[1] = (float)log2(active / n + tiny);
    f[2] = (float)log2(m / n + tiny);
    f[3] = (float)log2((double)k);
    f[4] = (float)(level < 32 ? level : 32) * 0.125f;
    f[5] = (float)log2(visits / n + tiny);
    f[6] = (float)prev_pull;
    f[7] = (float)log2((active + 1.0) / (prev_active + 1.0));
}
constexpr int32_t kMsBigRow = 4096;   // push rows this long are cut into chunks
constexpr int32_t kMsRowChunk = 1024;

struct MsRunState {
    unsigned bar_count;  // barrier arrivals (own cache line)
    unsigned pad_a[31];
    unsigned bar_release;  // barrier epochs (own cache line)
    unsigned pad_b[31];
    int32_t status;
    int32_t lvl;      // last level expanded (0 after set-up)
    int32_t flushed;  // first level not yet turned into depths
    int32_t mode;     // next level: 0 push, 1 pull, 2 done
    int32_t qsel;     // queue holding the current frontier (0: qa)
    int32_t active;   // vertices of the current frontier
    int32_t c_tail;   // push: long-row chunks deferred by the walk
    int32_t bad_src;  // a source outside [0, n) was skipped
    unsigned long long m_f;       // out-entries of the current frontier
    unsigned long long examined;  // entries read over the pass
    long long pull_levels;
    unsigned long long t_prev;    // global timer at the previous decision
    long long visits;             // frontier vertices summed over the levels so far
};

// Directions forced per level and a per-level trace (device arrays; null:
// the rule decides, no trace).  Trace row L - 1 describes level L:
// direction, time (ms), frontier vertices and out-entries it expanded,
// vertices and out-entries it found.
struct MsSteer {
    const int8_t* schedule = nullptr;
    int32_t schedule_len = 0;
    float* trace = nullptr;
    int32_t trace_cap = 0;
    int32_t learned = 0;          // 1: the learned direction model below decides
    float w[kMsPolicyWeights] = {};  // bias, then one weight per ms_level_features entry
};

template <int W>
__device__ __forceinline__ void ms_push_walk(const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                                             const int32_t* queue, int32_t count, MsPushVisitor<W>& f, int4* chunks,
                                             int32_t* c_tail) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * 32; base < count; base += nwarps * 32) {
        const int64_t i = base + lane;
        int32_t v = -1, b = 0, e = 0;
        if (i < count) {
            v = __ldcg(queue + i);
            b = rp[v];
            e = rp[v + 1];
            if (e - b >= kMsBigRow) {
                const int32_t nc = (e - b + kMsRowChunk - 1) / kMsRowChunk;
                const int32_t pos = atomicAdd(c_tail, nc);
                for (int32_t c = 0; c < nc; ++c)
                    chunks[pos + c] = make_int4(v, b + c * kMsRowChunk, min(e, b + (c + 1) * kMsRowChunk), 0);
                e = b;
            }
        }
        unsigned med = __ballot_sync(0xffffffffu, e - b >= 32);
        while (med) {
            const int leader = __ffs(med) - 1;
            med &= med - 1;
            const int32_t lv = __shfl_sync(0xffffffffu, v, leader);
            const int32_t lb = __shfl_sync(0xffffffffu, b, leader);
            const int32_t le = __shfl_sync(0xffffffffu, e, leader);
            for (int32_t j = lb + lane; j < le; j += 32) f(lv, col[j], j);
        }
        if (e - b >= 32) e = b;
        const int32_t d = e - b;
        int32_t incl = d;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += x;
        }
        const int32_t excl = incl - d;
        const int32_t total = __shfl_sync(0xffffffffu, incl, 31);
        for (int32_t k0 = 0; k0 < total; k0 += 32) {
            const int32_t kk = k0 + lane;
            int owner = 0;
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1) {
                const int cand = owner + s;
                const int32_t ev = __shfl_sync(0xffffffffu, excl, cand);
                if (ev <= kk) owner = cand;
            }
            const int32_t ov = __shfl_sync(0xffffffffu, v, owner);
            const int32_t ob = __shfl_sync(0xffffffffu, b, owner);
            const int32_t oe = __shfl_sync(0xffffffffu, excl, owner);
            if (kk < total) {
                const int32_t j = ob + (kk - oe);
                f(ov, col[j], j);
            }
        }
    }
}

// Four blocks per SM (64 registers; the 4-word variant spills 76 bytes):
// 256 sources on RMAT-22 10.3-10.5 ms and 64 on RMAT-24 9.2-10.2 ms, against
// 10.5-10.7 and 10.2-10.7 ms at three blocks per SM with 80 registers.
template <int W>
__global__ void __launch_bounds__(kMsThreads, 4) ms_pass_kernel(
    int32_t n, int32_t n_active, int32_t k, int64_t m, const int32_t* __restrict__ out_rp,
    const int32_t* __restrict__ out_col, const int32_t* __restrict__ in_rp, const int32_t* __restrict__ in_col,
    const int32_t* srcs, const int32_t* __restrict__ perm, int32_t* depth, uint64_t* seen, uint64_t* masks,
    int32_t chunk, uint64_t* next, int32_t* qa, int32_t* qb, int4* chunks, uint64_t* all, int32_t* hubs,
    MsCounters* cnt, MsRunState* st, int32_t pull_div, int32_t warp_rest, unsigned long long bar_limit_ns,
    unsigned bar_extra, MsSteer steer) {
    const int64_t words = (int64_t)n * W;
    auto slot = [&](int32_t l) { return masks + (int64_t)(l % chunk) * words; };
    auto barrier = [&]() {
        return grid_sync_leader(&st->bar_count, &st->bar_release, &st->status, NoLeader(), bar_limit_ns, bar_extra);
    };
    const bool can_pull = in_rp != nullptr && in_col != nullptr;
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;

    // ---- set-up: clear, seed (sources in the caller's ids), first queue
    ms_init_body(words, seen, slot(0), next);
    if (blockIdx.x == 0 && threadIdx.x < 4) {
        const int b = k - 64 * (int)threadIdx.x;
        all[threadIdx.x] = b >= 64 ? ~0ull : (b <= 0 ? 0ull : ((1ull << b) - 1ull));
    }
    if (!barrier()) return;
    if (blockIdx.x == 0 && (int)threadIdx.x < k) {
        const int s = threadIdx.x;
        int32_t v = srcs[s];
        if (v >= 0 && v < n) {
            if (perm) v = perm[v];
            const unsigned long long bit = 1ull << (s & 63);
            atomicOr((unsigned long long*)(seen + (int64_t)v * W + (s >> 6)), bit);
            atomicOr((unsigned long long*)(slot(0) + (int64_t)v * W + (s >> 6)), bit);
        } else {
            st->bad_src = 1;
        }
    }
    if (!barrier()) return;
    ms_queue_body<W>(n, slot(0), out_rp, qa, cnt);
    // Level decision, run by the last block to reach a level's final barrier.
    auto decide = [&](int32_t L, bool pulled, bool flushed_now) {
        volatile MsCounters* vc = cnt;
        volatile MsRunState* vs = st;
        const int32_t active = vc->active;
        const unsigned long long mf = vc->m_f;
        const int32_t prev_active = vs->active;  // the frontier level L expanded
        const unsigned long long now = global_timer_ns();
        if (steer.trace && L >= 1 && L - 1 < steer.trace_cap) {
            float* row = steer.trace + (size_t)(L - 1) * GHB_MS_TRACE_COLS;
            row[0] = pulled ? 1.f : 0.f;
            row[1] = (float)((double)(now - vs->t_prev) * 1e-6);
            row[2] = (float)vs->active;
            row[3] = (float)vs->m_f;
            row[4] = (float)active;
            row[5] = (float)mf;
        }
        st->t_prev = now;
        unsigned long long ex = vs->examined + vc->examined;
        if (L > 0 && !pulled) ex += vs->m_f;  // a push level reads every entry of its frontier
        st->examined = ex;
        if (pulled) st->pull_levels = vs->pull_levels + 1;
        st->active = active;
        st->m_f = mf;
        st->lvl = L;
        if (flushed_now) st->flushed = L + 1;
        if (L > 0) st->qsel = vs->qsel ^ 1;
        cnt->active = 0;
        cnt->hubs = 0;
        cnt->m_f = 0;
        cnt->examined = 0;
        st->c_tail = 0;
        int32_t mode = 2;
        const long long visits = vs->visits + active;
        st->visits = visits;
        if (active > 0 && L < n) {
            if (steer.schedule && L < steer.schedule_len) {
                mode = can_pull ? (steer.schedule[L] & 1) : 0;
            } else if (steer.learned) {
                float f[kMsPolicyFeatures];
                ms_level_features(f, (double)mf, (double)active, (double)prev_active, (double)visits, (double)n,
                                  (double)m, k, L + 1, pulled ? 1 : 0);
                float z = steer.w[0];
#pragma unroll
                for (int i = 0; i < kMsPolicyFeatures; ++i) z += steer.w[1 + i] * f[i];
                mode = (can_pull && z > 0.f) ? 1 : 0;
            } else {
                mode = (can_pull && (double)mf * (double)pull_div > (double)m) ? 1 : 0;
            }
        }
        st->mode = mode;
    };
    if (!grid_sync_leader(&st->bar_count, &st->bar_release, &st->status, [&]() { decide(0, false, false); },
                          bar_limit_ns, bar_extra))
        return;

    __shared__ int32_t s_st[5];
    while (true) {
        if (threadIdx.x == 0) {
            volatile MsRunState* vs = st;
            s_st[0] = vs->mode;
            s_st[1] = vs->lvl;
            s_st[2] = vs->qsel;
            s_st[3] = vs->active;
            s_st[4] = vs->flushed;
        }
        __syncthreads();
        const int32_t mode = s_st[0];
        if (mode == 2) break;
        const int32_t L = s_st[1] + 1;
        const int32_t flushed = s_st[4];
        uint64_t* f_cur = slot(L - 1);
        uint64_t* f_new = slot(L);
        int32_t* q_cur = s_st[2] ? qb : qa;
        int32_t* q_new = s_st[2] ? qa : qb;
        if (mode == 1) {
            ms_pull_body<W>(n_active, all, in_rp, in_col, out_rp, f_cur, seen, f_new, q_new, hubs, cnt, warp_rest);
            if (!barrier()) return;
            ms_pull_hub_body<W>(all, in_rp, in_col, out_rp, f_cur, seen, f_new, q_new, hubs, cnt);
        } else {
            MsPushVisitor<W> f{f_cur, seen, next};
            ms_push_walk<W>(out_rp, out_col, q_cur, s_st[3], f, chunks, &st->c_tail);
            if (!barrier()) return;
            const int32_t nc = *(volatile int32_t*)&st->c_tail;
            for (int64_t i = warp; i < nc; i += nwarps) {
                const int4 ch = __ldcg(chunks + i);
                for (int32_t j = ch.y + lane; j < ch.z; j += 32) f(ch.x, out_col[j], j);
            }
            if (!barrier()) return;
            ms_settle_body<W>(n_active, out_rp, seen, f_new, next, q_new, cnt);
        }
        // The next level overwrites slot L + 1: flush a full chunk first.
        const bool flush_now = (L + 1) % chunk == 0;
        if (flush_now) {
            if (!barrier()) return;
            ms_flush_body<W>(n, n_active, k, perm, masks, chunk, flushed, L, false, seen, depth);
        }
        if (!grid_sync_leader(&st->bar_count, &st->bar_release, &st->status,
                              [&]() { decide(L, mode == 1, flush_now); }, bar_limit_ns, bar_extra))
            return;
    }
    // Final flush: the levels not flushed yet, and INT32_MAX where a source
    // never reached a vertex.
    ms_flush_body<W>(n, n_active, k, perm, masks, chunk, s_st[4], s_st[1], true, seen, depth);
}

int32_t ms_chunk_levels(int64_t words) {
    return (int32_t)std::max<int64_t>(
        2, std::min<int64_t>(kMsChunkMax, (int64_t)(kMsMaskBudget / (size_t)(words * sizeof(uint64_t)))));
}

// Scratch of one whole-pass launch, laid out by carve() (base == nullptr:
// sizing only).
template <int W>
struct MsPassScratch {
    uint64_t *seen, *masks, *next, *all;
    int32_t *qa, *qb, *hubs;
    int4* chunks;
    MsCounters* cnt;
    MsRunState* rs;
    int32_t chunk;
    size_t bytes;
    static MsPassScratch carve(void* base, int32_t n, int64_t m) {
        MsPassScratch s;
        const int64_t words = (int64_t)n * W;
        s.chunk = ms_chunk_levels(words);
        Carver c(base);
        s.seen = c.take<uint64_t>(words);
        s.masks = c.take<uint64_t>(words * s.chunk);
        s.next = c.take<uint64_t>(words);
        s.qa = c.take<int32_t>(n);
        s.qb = c.take<int32_t>(n);
        s.chunks = c.take<int4>(m / kMsRowChunk + m / kMsBigRow + 64);
        s.all = c.take<uint64_t>(4);
        s.hubs = c.take<int32_t>(n);
        s.cnt = c.take<MsCounters>(1);
        s.rs = c.take<MsRunState>(1);
        s.bytes = c.off;
        return s;
    }
};

template <int W>
int ms_pass_blocks(ghb_workspace* ws) {
    static int cached[64] = {0};
    const int dev = ws->device;
    if (dev < 0 || dev >= 64) return 0;
    if (!cached[dev]) {
        int coop = 0, per_sm = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        if (coop &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ms_pass_kernel<W>, kMsThreads, 0) == cudaSuccess)
            cached[dev] = std::max(0, std::min(per_sm, 4)) * ws->num_sms;
        if (!cached[dev]) cached[dev] = -1;
    }
    return cached[dev] > 0 ? cached[dev] : 0;
}

template <int W>
size_t ms_pass_bytes(int32_t n, int64_t m) {
    return MsPassScratch<W>::carve(nullptr, n, m).bytes;
}

// One whole-pass launch of k <= 256 sources (caller ids on the device; perm,
// when given, maps them and the outputs to the graph's ids).  Launch only:
// the workspace must already hold ms_pass_bytes<W>(n, m) bytes of scratch,
// and nothing is read back.
// The installed direction model of the multi-source pass (process-wide,
// ghb_ms_policy_load); used where the workspace's ms_learned is 1.
std::mutex g_ms_policy_mu;
bool g_ms_policy_set = false;
float g_ms_policy[kMsPolicyWeights];

template <int W>
int ms_pass_launch(ghb_workspace* ws, int32_t n, int32_t n_active, int64_t m, const int32_t* out_rp,
                   const int32_t* out_col, const int32_t* in_rp, const int32_t* in_col, const int32_t* srcs, int32_t k,
                   const int32_t* perm, int32_t* depth, MsSteer steer = MsSteer()) {
    const int blocks = ms_pass_blocks<W>(ws);
    if (blocks <= 0) {
        set_error("cooperative launch unavailable");
        return GHB_ERR_UNSUPPORTED;
    }
    if (ms_pass_bytes<W>(n, m) > ws->scratch_cap) {
        set_error("multi-source pass: workspace scratch not reserved (ghb_graph_msbfs_reserve)");
        return GHB_ERR_INVALID_ARGUMENT;
    }
    if (ws->tune.ms_learned && !steer.schedule) {
        std::lock_guard<std::mutex> lock(g_ms_policy_mu);
        if (g_ms_policy_set) {
            steer.learned = 1;
            std::memcpy(steer.w, g_ms_policy, sizeof(g_ms_policy));
        }
    }
    MsPassScratch<W> s = MsPassScratch<W>::carve(ws->scratch, n, m);
    GHB_CUDA_TRY(cudaMemsetAsync(s.cnt, 0, sizeof(MsCounters), ws->stream));
    GHB_CUDA_TRY(cudaMemsetAsync(s.rs, 0, sizeof(MsRunState), ws->stream));
    const bool pull = in_rp != nullptr && in_col != nullptr;
    return launch_coop(ws, ms_pass_kernel<W>, dim3(blocks), dim3(kMsThreads), (size_t)0, n, n_active, k, m, out_rp,
                       out_col, pull ? in_rp : (const int32_t*)nullptr, pull ? in_col : (const int32_t*)nullptr, srcs,
                       perm, depth, s.seen, s.masks, s.chunk, s.next, s.qa, s.qb, s.chunks, s.all, s.hubs, s.cnt,
                       s.rs, ws->tune.ms_pull_div, ws->tune.ms_warp_rest,
                       (unsigned long long)ws->tune.barrier_limit_us * 1000ull, (unsigned)ws->tune.barrier_extra,
                       steer);
}

// After a launch that was not captured: its status and counters.
template <int W>
int ms_pass_finish(ghb_workspace* ws, int32_t n, int64_t m, int64_t* levels_out, int64_t* examined_out) {
    MsPassScratch<W> s = MsPassScratch<W>::carve(ws->scratch, n, m);
    GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, s.rs, sizeof(MsRunState), cudaMemcpyDeviceToHost, ws->stream));
    GHB_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    MsRunState h;
    std::memcpy(&h, ws->host_pinned, sizeof(h));
    if (h.status != kDevOk) {
        set_error("multi-source BFS: grid barrier timed out");
        return GHB_ERR_TIMEOUT;
    }
    if (levels_out) *levels_out += h.lvl;
    if (examined_out) *examined_out += (int64_t)h.examined;
    return GHB_OK;
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

// Words per vertex of a pass of k sources.
static int ms_words_for(int32_t k) { return k <= 64 ? 1 : (k <= 128 ? 2 : 4); }

// Scratch of the whole-pass launches for n_src sources (their widest pass).
size_t msbfs_persistent_bytes(int32_t n, int64_t m, int32_t n_src) {
    const int w = ms_words_for(std::min<int32_t>(std::max<int32_t>(n_src, 1), kMsPass));
    return w == 1 ? ms_pass_bytes<1>(n, m) : (w == 2 ? ms_pass_bytes<2>(n, m) : ms_pass_bytes<4>(n, m));
}

bool msbfs_persistent_available(ghb_workspace* ws, int32_t n_src) {
    if (!ws->tune.ms_persistent) return false;
    const int w = ms_words_for(std::min<int32_t>(std::max<int32_t>(n_src, 1), kMsPass));
    return (w == 1 ? ms_pass_blocks<1>(ws) : (w == 2 ? ms_pass_blocks<2>(ws) : ms_pass_blocks<4>(ws))) > 0;
}

// n_src sources (caller ids, device array) in passes of up to kMsPass, one
// cooperative launch each.  With `finish` each pass's status and counters
// are read back after it; without, the calls only launch (the workspace
// must hold msbfs_persistent_bytes), so a stream capture can record them.
int msbfs_persistent(ghb_workspace* ws, int32_t n, int32_t n_active, int64_t m, const int32_t* out_rp,
                     const int32_t* out_col, const int32_t* in_rp, const int32_t* in_col, const int32_t* srcs,
                     int32_t n_src, const int32_t* perm, int32_t* depth, bool finish, int64_t* levels_out,
                     int64_t* examined_out, const MsSteer& steer) {
    for (int32_t s0 = 0; s0 < n_src; s0 += kMsPass) {
        const int32_t k = std::min<int32_t>(kMsPass, n_src - s0);
        const int w = ms_words_for(k);
        const int32_t* s = srcs + s0;
        int32_t* d = depth + (int64_t)s0 * n;
        MsSteer st = steer;
        if (s0 > 0) st.trace = nullptr;  // the trace describes the first pass
        if (w == 1) {
            GHB_TRY(ms_pass_launch<1>(ws, n, n_active, m, out_rp, out_col, in_rp, in_col, s, k, perm, d, st));
            if (finish) GHB_TRY(ms_pass_finish<1>(ws, n, m, levels_out, examined_out));
        } else if (w == 2) {
            GHB_TRY(ms_pass_launch<2>(ws, n, n_active, m, out_rp, out_col, in_rp, in_col, s, k, perm, d, st));
            if (finish) GHB_TRY(ms_pass_finish<2>(ws, n, m, levels_out, examined_out));
        } else {
            GHB_TRY(ms_pass_launch<4>(ws, n, n_active, m, out_rp, out_col, in_rp, in_col, s, k, perm, d, st));
            if (finish) GHB_TRY(ms_pass_finish<4>(ws, n, m, levels_out, examined_out));
        }
    }
    return GHB_OK;
}

int msbfs_persistent(ghb_workspace* ws, int32_t n, int32_t n_active, int64_t m, const int32_t* out_rp,
                     const int32_t* out_col, const int32_t* in_rp, const int32_t* in_col, const int32_t* srcs,
                     int32_t n_src, const int32_t* perm, int32_t* depth, bool finish, int64_t* levels_out,
                     int64_t* examined_out) {
    return msbfs_persistent(ws, n, n_active, m, out_rp, out_col, in_rp, in_col, srcs, n_src, perm, depth, finish,
                            levels_out, examined_out, MsSteer());
}

// Steered variant of ghb_graph_msbfs's one-launch path (schedule and trace
// are device arrays or null).
int msbfs_persistent_steered(ghb_workspace* ws, int32_t n, int32_t n_active, int64_t m, const int32_t* out_rp,
                             const int32_t* out_col, const int32_t* in_rp, const int32_t* in_col,
                             const int32_t* srcs, int32_t n_src, const int32_t* perm, int32_t* depth,
                             int64_t* levels_out, int64_t* examined_out, const int8_t* schedule,
                             int32_t schedule_len, float* trace, int32_t trace_cap) {
    MsSteer steer;
    steer.schedule = schedule;
    steer.schedule_len = schedule ? schedule_len : 0;
    steer.trace = trace;
    steer.trace_cap = trace ? trace_cap : 0;
    return msbfs_persistent(ws, n, n_active, m, out_rp, out_col, in_rp, in_col, srcs, n_src, perm, depth, true,
                            levels_out, examined_out, steer);
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
    int64_t levels = 0, examined = 0;
    if (n_src > 0 && msbfs_persistent_available(ws, n_src)) {
        int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned);
        GHB_CUDA_TRY(cudaMemcpyAsync(hp, out_rowptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        const int64_t m = hp[0];
        GHB_TRY(ws_reserve(ws, msbfs_persistent_bytes(n, m, n_src)));
        if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
        GHB_TRY(msbfs_persistent(ws, n, n, m, out_rowptr, out_col, in_rowptr, in_col, srcs, n_src, nullptr, depth,
                                 true, &levels, &examined));
    } else {
        if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
        for (int32_t s0 = 0; s0 < n_src; s0 += kMsPass) {
            const int32_t k = std::min<int32_t>(kMsPass, n_src - s0);
            GHB_TRY(msbfs_batch(ws, n, n, out_rowptr, out_col, in_rowptr, in_col, srcs + s0, k, nullptr,
                                depth + (int64_t)s0 * n, &levels, &examined));
        }
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

extern "C" int ghb_ms_policy_load(const float* weights, int32_t count) {
    std::lock_guard<std::mutex> lock(ghb::g_ms_policy_mu);
    if (!weights) {
        ghb::g_ms_policy_set = false;
        return GHB_OK;
    }
    GHB_REQUIRE(count == ghb::kMsPolicyWeights, "the multi-source direction model has 9 weights");
    for (int i = 0; i < count; ++i) GHB_REQUIRE(std::isfinite(weights[i]), "weights must be finite");
    std::memcpy(ghb::g_ms_policy, weights, sizeof(ghb::g_ms_policy));
    ghb::g_ms_policy_set = true;
    return GHB_OK;
}
