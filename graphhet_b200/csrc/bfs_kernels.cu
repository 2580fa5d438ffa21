// Top-down and bottom-up BFS level kernels.
//
// Top-down (push): a warp takes 32 queue vertices.  Lists of 32..kBigList-1
// entries are walked by the whole warp one list at a time; shorter lists are
// gathered warp-wide through an exclusive scan of their lengths, so each
// warp-wide step reads 32 consecutive CSR entries; lists of kBigList or more
// are deferred and expanded edge-parallel by the whole grid afterwards.
// A neighbour is claimed by atomicOr on the visited bitmap; the claimer
// writes its depth, appends it to the next queue and sets its bit in the next
// frontier bitmap (used if the next level runs bottom-up).
//
// Bottom-up (pull): one warp per 32-vertex bitmap word; each unvisited lane
// scans its in-row for a parent in the current frontier bitmap and stops at
// the first hit (rows are sorted, so the first hit is the smallest-id
// parent).  Lanes still searching after 32 entries continue warp-wide.  The
// warp owns its visited / next-frontier words, so no atomics are needed.
#include "bfs_kernels.cuh"

namespace ghb {

__global__ void fill_i32_kernel(int32_t* p, int64_t count, int32_t value) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = value;
}

__global__ void bfs_init_kernel(int32_t n, int64_t words, int32_t src, int32_t* depth,
                                uint32_t* visited, uint32_t* front, int32_t* queue) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (int64_t v = t0; v < n; v += stride) depth[v] = (v == src) ? 0 : kInfDepth;
    for (int64_t w = t0; w < words; w += stride) {
        uint32_t bit = (w == (src >> 5)) ? (1u << (src & 31)) : 0u;
        visited[w] = bit;
        front[w] = bit;
    }
    if (t0 == 0) queue[0] = src;
}

namespace {

struct LevelAcc {
    unsigned long long m_f = 0, examined = 0;
    double deg2 = 0.0;
    unsigned int degmax = 0;
};

// Block-level reduction of the level counters, then one atomic per counter
// per block (per-warp atomics on the same four addresses serialise at L2).
__device__ __forceinline__ void flush_acc(const LevelAcc& a, BfsCounters* cnt) {
    __shared__ unsigned long long s_mf[32], s_ex[32];
    __shared__ double s_d2[32];
    __shared__ unsigned int s_dm[32];
    unsigned long long mf = a.m_f, ex = a.examined;
    double d2 = a.deg2;
    unsigned int dm = a.degmax;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mf += __shfl_xor_sync(0xffffffffu, mf, o);
        ex += __shfl_xor_sync(0xffffffffu, ex, o);
        d2 += __shfl_xor_sync(0xffffffffu, d2, o);
        unsigned int x = __shfl_xor_sync(0xffffffffu, dm, o);
        dm = x > dm ? x : dm;
    }
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0) {
        s_mf[w] = mf;
        s_ex[w] = ex;
        s_d2[w] = d2;
        s_dm[w] = dm;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        for (int i = 1; i < nw; ++i) {
            mf += s_mf[i];
            ex += s_ex[i];
            d2 += s_d2[i];
            dm = s_dm[i] > dm ? s_dm[i] : dm;
        }
        if (mf) atomicAdd(&cnt->m_f, mf);
        if (ex) atomicAdd(&cnt->examined, ex);
        if (d2 != 0.0) atomicAdd(&cnt->deg2, d2);
        if (dm) atomicMax(&cnt->degmax, dm);
    }
}

// Claim v for the next level if nobody has.  With q_next (small levels) the
// claimer also appends v to the next queue and adds its degree to the level
// statistics; without it (large levels, where one queue counter would
// serialise millions of appends) only the frontier bitmap is written and
// bfs_queue_from_bitmap_kernel builds the queue and the statistics later.
__device__ __forceinline__ void visit(int32_t v, uint32_t* visited, uint32_t* f_next, int32_t* depth,
                                      int32_t next_depth, int32_t* q_next, int32_t* tail,
                                      const int32_t* __restrict__ rowptr, LevelAcc& acc) {
    const uint32_t bit = 1u << (v & 31);
    uint32_t* wp = visited + (v >> 5);
    if (*wp & bit) return;
    uint32_t old = atomicOr(wp, bit);
    if (old & bit) return;
    depth[v] = next_depth;
    atomicOr(f_next + (v >> 5), bit);
    if (q_next) {
        int32_t pos = warp_append_active(tail);
        q_next[pos] = v;
        uint32_t dv = (uint32_t)(rowptr[v + 1] - rowptr[v]);
        acc.m_f += dv;
        acc.deg2 += (double)dv * (double)dv;
        acc.degmax = dv > acc.degmax ? dv : acc.degmax;
    }
}

__global__ void __launch_bounds__(256) bfs_push_kernel(
    const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
    const int32_t* __restrict__ q_cur, int32_t n_f, int32_t next_depth, uint32_t* visited,
    uint32_t* f_next, int32_t* depth, int32_t* q_next, int32_t* big, BfsCounters* cnt) {
    LevelAcc acc;
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * 32; base < n_f; base += nwarps * 32) {
        const int64_t i = base + lane;
        int32_t b = 0, e = 0;
        if (i < n_f) {
            int32_t u = q_cur[i];
            b = rowptr[u];
            e = rowptr[u + 1];
            if (e - b >= kBigList) {
                int32_t pos = warp_append_active(&cnt->big_tail);
                big[pos] = u;
                atomicAdd(&cnt->big_edges, (unsigned long long)(e - b));
                e = b;
            }
        }
        // Medium lists: whole warp per list.
        unsigned med = __ballot_sync(0xffffffffu, e - b >= 32);
        while (med) {
            const int leader = __ffs(med) - 1;
            const int32_t lb = __shfl_sync(0xffffffffu, b, leader);
            const int32_t le = __shfl_sync(0xffffffffu, e, leader);
            for (int32_t j = lb + lane; j < le; j += 32)
                visit(col[j], visited, f_next, depth, next_depth, q_next, &cnt->tail, rowptr, acc);
            acc.examined += (lane == leader) ? (unsigned long long)(le - lb) : 0ull;
            med &= med - 1;
        }
        if (e - b >= 32) e = b;
        // Short lists: warp-wide gather over the scanned lengths.
        int32_t d = e - b;
        int32_t incl = d;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int32_t x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += x;
        }
        const int32_t excl = incl - d;
        const int32_t total = __shfl_sync(0xffffffffu, incl, 31);
        acc.examined += (lane == 0) ? (unsigned long long)total : 0ull;
        for (int32_t k0 = 0; k0 < total; k0 += 32) {
            const int32_t k = k0 + lane;
            int owner = 0;
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1) {
                int cand = owner + s;
                int32_t ev = __shfl_sync(0xffffffffu, excl, cand);
                if (ev <= k) owner = cand;
            }
            const int32_t ob = __shfl_sync(0xffffffffu, b, owner);
            const int32_t oe = __shfl_sync(0xffffffffu, excl, owner);
            if (k < total)
                visit(col[ob + (k - oe)], visited, f_next, depth, next_depth, q_next, &cnt->tail,
                      rowptr, acc);
        }
    }
    flush_acc(acc, cnt);
}

// Exclusive prefix of the deferred lists' lengths (one block; the lists are
// few because each holds >= kBigList entries).
__global__ void __launch_bounds__(1024) bfs_big_scan_kernel(const int32_t* __restrict__ rowptr,
                                                            const int32_t* __restrict__ big,
                                                            const BfsCounters* cnt,
                                                            int64_t* prefix) {
    __shared__ int64_t warp_tot[32];
    __shared__ int64_t carry;
    const int32_t count = cnt->big_tail;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int32_t base = 0; base < count; base += blockDim.x) {
        const int32_t i = base + threadIdx.x;
        int64_t d = 0;
        if (i < count) {
            int32_t u = big[i];
            d = rowptr[u + 1] - rowptr[u];
        }
        int64_t incl = d;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane_id() >= o) incl += x;
        }
        if (lane_id() == 31) warp_tot[threadIdx.x >> 5] = incl;
        __syncthreads();
        if (threadIdx.x < 32) {
            int64_t t = (threadIdx.x < (blockDim.x >> 5)) ? warp_tot[threadIdx.x] : 0;
            int64_t ti = t;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int64_t x = __shfl_up_sync(0xffffffffu, ti, o);
                if (lane_id() >= o) ti += x;
            }
            warp_tot[threadIdx.x] = ti - t;  // exclusive
        }
        __syncthreads();
        const int64_t c0 = carry;
        if (i < count) prefix[i] = c0 + warp_tot[threadIdx.x >> 5] + incl - d;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = c0 + warp_tot[threadIdx.x >> 5] + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) prefix[count] = carry;
}

// Edge-parallel expansion of the deferred lists.  Each warp takes 128
// consecutive entries; since every list holds >= kBigList >= 128 entries, a
// chunk crosses at most one list boundary.
__global__ void __launch_bounds__(256) bfs_big_kernel(
    const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
    const int32_t* __restrict__ big, const int64_t* __restrict__ prefix, int32_t next_depth,
    uint32_t* visited, uint32_t* f_next, int32_t* depth, int32_t* q_next, BfsCounters* cnt) {
    LevelAcc acc;
    const int32_t count = cnt->big_tail;
    if (count == 0) return;
    const int64_t total = prefix[count];
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c0 = warp * 128; c0 < total; c0 += nwarps * 128) {
        // owner of entry c0: last i with prefix[i] <= c0
        int32_t lo = 0, hi = count - 1;
        while (lo < hi) {
            int32_t mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= c0) lo = mid; else hi = mid - 1;
        }
        const int64_t next_start = prefix[lo + 1];
        const int32_t u0 = big[lo];
        const int32_t b0 = rowptr[u0];
        int32_t u1 = -1, b1 = 0;
        if (next_start < c0 + 128 && lo + 1 < count) {
            u1 = big[lo + 1];
            b1 = rowptr[u1];
        }
        int32_t vs[4];
        bool ok[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int64_t p = c0 + lane + 32 * k;
            ok[k] = p < total;
            int32_t idx;
            if (p < next_start) idx = b0 + (int32_t)(p - prefix[lo]);
            else idx = b1 + (int32_t)(p - next_start);
            vs[k] = ok[k] ? col[idx] : 0;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (ok[k]) visit(vs[k], visited, f_next, depth, next_depth, q_next, &cnt->tail, rowptr, acc);
        acc.examined += (unsigned long long)(ok[0] + ok[1] + ok[2] + ok[3]);
        (void)u1;
    }
    flush_acc(acc, cnt);
}

}  // namespace

__global__ void __launch_bounds__(256) bfs_pull_kernel(
    int32_t n, int64_t words, const int32_t* __restrict__ in_rp, const int32_t* __restrict__ in_col,
    const int32_t* __restrict__ out_rp, const uint32_t* __restrict__ f_cur, uint32_t* visited,
    uint32_t* f_next, int32_t* depth, int32_t next_depth, int32_t* q_next, BfsCounters* cnt) {
    (void)q_next;
    LevelAcc acc;
    unsigned long long found_total = 0;
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w = warp; w < words; w += nwarps) {
        const uint32_t vis = visited[w];
        if (vis == 0xffffffffu) continue;
        const int64_t v = w * 32 + lane;
        const bool todo = v < n && !((vis >> lane) & 1u);
        bool found = false;
        int32_t j = 0, e = 0;
        if (todo) {
            j = in_rp[v];
            e = in_rp[v + 1];
            const int32_t b = j;
            const int32_t lim = min(e, b + 32);
            // Probe four entries at a time: the four column loads and the four
            // frontier-word loads are independent, so they overlap.
            while (j < lim && !found) {
                int32_t u[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) u[k] = (j + k < lim) ? in_col[j + k] : -1;
                bool h[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) h[k] = u[k] >= 0 && ((f_cur[u[k] >> 5] >> (u[k] & 31)) & 1u);
                int hit = h[0] ? 0 : h[1] ? 1 : h[2] ? 2 : h[3] ? 3 : -1;
                if (hit >= 0) {
                    found = true;
                    j += hit + 1;
                } else {
                    j = min(j + 4, lim);
                }
            }
            acc.examined += (unsigned long long)(j - b);
        }
        unsigned rest = __ballot_sync(0xffffffffu, todo && !found && j < e);
        while (rest) {
            const int leader = __ffs(rest) - 1;
            const int32_t lj = __shfl_sync(0xffffffffu, j, leader);
            const int32_t le = __shfl_sync(0xffffffffu, e, leader);
            bool hit = false;
            int32_t scanned = 0;
            for (int32_t k0 = lj; k0 < le; k0 += 32) {
                const int32_t k = k0 + lane;
                bool h = false;
                if (k < le) {
                    const int32_t u = in_col[k];
                    h = (f_cur[u >> 5] >> (u & 31)) & 1u;
                }
                const unsigned hm = __ballot_sync(0xffffffffu, h);
                scanned += min(32, le - k0);
                if (hm) {
                    hit = true;
                    break;
                }
            }
            if (lane == leader) {
                found = hit;
                acc.examined += (unsigned long long)scanned;
            }
            rest &= rest - 1;
        }
        const unsigned fm = __ballot_sync(0xffffffffu, found);
        if (fm) {
            if (lane == 0) {
                visited[w] = vis | fm;
                f_next[w] = fm;
                found_total += (unsigned long long)__popc(fm);
            }
            if (found) {
                depth[v] = next_depth;
                const uint32_t dv = (uint32_t)(out_rp[v + 1] - out_rp[v]);
                acc.m_f += dv;
                acc.deg2 += (double)dv * (double)dv;
                acc.degmax = dv > acc.degmax ? dv : acc.degmax;
            }
        }
    }
    // New-frontier size: per-block total, one atomic per block.
    __shared__ unsigned long long s_found[32];
    found_total = warp_sum(found_total);
    if (lane == 0) s_found[threadIdx.x >> 5] = found_total;
    flush_acc(acc, cnt);  // contains __syncthreads
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += s_found[i];
        if (t) atomicAdd(&cnt->tail, (int32_t)t);
    }
}

// The frontier bitmap as a vertex queue (ascending within each warp's 32
// words), for a top-down level after a bottom-up one or after a large
// top-down level.  With cnt it also counts the frontier and its degree
// statistics.
__global__ void __launch_bounds__(256) bfs_queue_from_bitmap_kernel(int64_t words,
                                                                    const uint32_t* __restrict__ f,
                                                                    const int32_t* __restrict__ rowptr,
                                                                    int32_t* queue, int32_t* tail,
                                                                    BfsCounters* cnt) {
    LevelAcc acc;
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w0 = warp * 32; w0 < words; w0 += nwarps * 32) {
        const int64_t w = w0 + lane;
        uint32_t bits = w < words ? f[w] : 0u;
        const int32_t c = __popc(bits);
        int32_t incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += x;
        }
        const int32_t total = __shfl_sync(0xffffffffu, incl, 31);
        if (total == 0) continue;
        int32_t base = 0;
        if (lane == 0) base = atomicAdd(tail, total);
        base = __shfl_sync(0xffffffffu, base, 0);
        int32_t pos = base + incl - c;
        while (bits) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            const int32_t v = (int32_t)(w * 32 + b);
            queue[pos++] = v;
            if (cnt) {
                const uint32_t dv = (uint32_t)(rowptr[v + 1] - rowptr[v]);
                acc.m_f += dv;
                acc.deg2 += (double)dv * (double)dv;
                acc.degmax = dv > acc.degmax ? dv : acc.degmax;
            }
        }
    }
    if (cnt) flush_acc(acc, cnt);
}

__global__ void bfs_pred_pull_kernel(int32_t n, const int32_t* __restrict__ in_rp,
                                     const int32_t* __restrict__ in_col,
                                     const int32_t* __restrict__ depth, int32_t src,
                                     int32_t* __restrict__ pred) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = warp; v < n; v += nwarps) {
        const int32_t dv = depth[v];
        int32_t p = -1;
        if (v != src && dv != kInfDepth) {
            const int32_t b = in_rp[v], e = in_rp[v + 1];
            for (int32_t k0 = b; k0 < e; k0 += 32) {
                const int32_t k = k0 + lane;
                int32_t u = -1;
                bool h = false;
                if (k < e) {
                    u = in_col[k];
                    h = depth[u] == dv - 1;
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

__global__ void bfs_pred_push_kernel(int32_t n, const int32_t* __restrict__ out_rp,
                                     const int32_t* __restrict__ out_col,
                                     const int32_t* __restrict__ depth, int32_t* pred) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = warp; u < n; u += nwarps) {
        const int32_t du = depth[u];
        if (du == kInfDepth) continue;
        const int32_t b = out_rp[u], e = out_rp[u + 1];
        for (int32_t k = b + lane; k < e; k += 32) {
            const int32_t v = out_col[k];
            if (depth[v] == du + 1) atomicMin(&pred[v], (int32_t)u);
        }
    }
}

__global__ void bfs_pred_finish_kernel(int32_t n, int32_t src, int32_t* pred) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x)
        if (v == src || pred[v] == kInfDepth) pred[v] = -1;
}

int bfs_push_level(ghb_workspace* ws, const BfsBuffers& B, int32_t n, const int32_t* rowptr,
                   const int32_t* col, const int32_t* q_cur, int64_t n_f, int32_t next_depth,
                   int32_t* depth, int32_t* q_next, uint32_t* f_next) {
    // q_next == nullptr: bitmap mode (see visit()).
    (void)n;
    const unsigned gmax = ws->num_sms * 8;
    GHB_TRY(launch(ws, bfs_push_kernel, dim3(grid_for(n_f * 32, 256, gmax)), dim3(256), 0, rowptr,
                   col, q_cur, (int32_t)n_f, next_depth, B.visited, f_next, depth, q_next, B.big,
                   B.counters));
    GHB_TRY(launch(ws, bfs_big_scan_kernel, dim3(1), dim3(1024), 0, rowptr, (const int32_t*)B.big,
                   (const BfsCounters*)B.counters, B.big_prefix));
    GHB_TRY(launch(ws, bfs_big_kernel, dim3(gmax), dim3(256), 0, rowptr, col, (const int32_t*)B.big,
                   (const int64_t*)B.big_prefix, next_depth, B.visited, f_next, depth, q_next,
                   B.counters));
    return GHB_OK;
}

int bfs_time_both(ghb_workspace* ws, const BfsBuffers& B, int32_t n, int64_t words,
                  const int32_t* out_rowptr, const int32_t* out_col, const int32_t* in_rowptr,
                  const int32_t* in_col, const int32_t* q_cur, int64_t n_f, int64_t m_f, const uint32_t* f_cur,
                  int level, int32_t* depth, float* t_push, float* t_pull) {
    cudaStream_t st = ws->stream;
    const unsigned gmax = ws->num_sms * 8;
    // Scratch next-queue / next-frontier: the real ones are rewritten by the
    // level itself afterwards, so they can be used here.
    int32_t* q_tmp = (q_cur == B.queue_a) ? B.queue_b : B.queue_a;
    uint32_t* f_tmp = (f_cur == B.front_a) ? B.front_b : B.front_a;
    GHB_CUDA_TRY(cudaMemcpyAsync(B.depth_snap, depth, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
    GHB_CUDA_TRY(cudaMemcpyAsync(B.visited_snap, B.visited, sizeof(uint32_t) * words,
                                 cudaMemcpyDeviceToDevice, st));
    for (int pass = 0; pass < 2; ++pass) {
        GHB_CUDA_TRY(cudaMemsetAsync(B.counters, 0, sizeof(BfsCounters), st));
        GHB_CUDA_TRY(cudaMemsetAsync(f_tmp, 0, words * sizeof(uint32_t), st));
        GHB_CUDA_TRY(cudaEventRecord(ws->ev_a, st));
        if (pass == 0) {
            const bool append = m_f < kAppendMaxEdges;
            GHB_TRY(bfs_push_level(ws, B, n, out_rowptr, out_col, q_cur, n_f, level + 1, depth,
                                   append ? q_tmp : (int32_t*)nullptr, f_tmp));
            if (!append)
                GHB_TRY(launch(ws, bfs_queue_from_bitmap_kernel, dim3(grid_for(words * 32, 256, gmax)), dim3(256),
                               0, words, (const uint32_t*)f_tmp, out_rowptr, q_tmp, &B.counters->tail, B.counters));
        } else {
            GHB_TRY(launch(ws, bfs_pull_kernel, dim3(grid_for(words * 32, 256, gmax)), dim3(256), 0,
                           n, words, in_rowptr, in_col, out_rowptr, f_cur, B.visited, f_tmp, depth,
                           level + 1, q_tmp, B.counters));
        }
        GHB_CUDA_TRY(cudaEventRecord(ws->ev_b, st));
        GHB_CUDA_TRY(cudaEventSynchronize(ws->ev_b));
        float ms = 0.f;
        GHB_CUDA_TRY(cudaEventElapsedTime(&ms, ws->ev_a, ws->ev_b));
        if (pass == 0) *t_push = ms; else *t_pull = ms;
        GHB_CUDA_TRY(cudaMemcpyAsync(depth, B.depth_snap, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
        GHB_CUDA_TRY(cudaMemcpyAsync(B.visited, B.visited_snap, sizeof(uint32_t) * words,
                                     cudaMemcpyDeviceToDevice, st));
    }
    return GHB_OK;
}

}  // namespace ghb

namespace ghb {

// Consecutive small top-down levels in one cooperative launch.  Level L reads
// queue L%2 and appends to queue (L+1)%2; frontier counters are triple-
// buffered (level L appends to slot (L+1)%3 and block 0 clears slot (L+2)%3,
// which nobody reads or writes again before the next barrier), so one grid
// barrier per level suffices.  After each barrier every block reads the same
// settled counters and takes the same decision: continue, or stop when the
// frontier is empty, when its out-entries reach exit_edges, at max_depth, or
// when the direction rule (frontier entries > unexplored entries / alpha)
// asks for a bottom-up level.
// The barrier wait is bounded (grid_barrier): on timeout every block leaves
// and the host reports GHB_ERR_TIMEOUT.
__global__ void __launch_bounds__(1024) bfs_push_persistent_kernel(
    const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col, int32_t* qa, int32_t* qb,
    uint32_t* visited, int32_t* depth, int32_t start_level, int32_t max_depth, int64_t exit_edges,
    int64_t m_total, int64_t m_r_start, float alpha, BfsPersistState* ps) {
    __shared__ unsigned long long s_mf[32], s_ex[32];
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    int32_t level = start_level;
    int L = 0;  // levels done in this launch
    while (true) {
        volatile int32_t* vtail = ps->tail;
        const int32_t n_f = vtail[L % 3];
        const int32_t* q_cur = (L & 1) ? qb : qa;
        int32_t* q_next = (L & 1) ? qa : qb;
        int32_t* tail_next = &ps->tail[(L + 1) % 3];
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ps->tail[(L + 2) % 3] = 0;
            ps->mf[(L + 2) % 3] = 0;
            ps->dmax[(L + 2) % 3] = 0;
        }
        unsigned long long mf = 0, ex = 0;
        unsigned int dm = 0;
        for (int64_t base = warp * 32; base < n_f; base += nwarps * 32) {
            const int64_t i = base + lane;
            int32_t b = 0, e = 0;
            if (i < n_f) {
                const int32_t u = q_cur[i];
                b = rowptr[u];
                e = rowptr[u + 1];
            }
            ex += (unsigned long long)(e - b);
            // Whole warp per row, 32 entries per step.
            unsigned todo = __ballot_sync(0xffffffffu, e > b);
            while (todo) {
                const int leader = __ffs(todo) - 1;
                todo &= todo - 1;
                const int32_t lb = __shfl_sync(0xffffffffu, b, leader);
                const int32_t le = __shfl_sync(0xffffffffu, e, leader);
                for (int32_t j = lb + lane; j < le; j += 32) {
                    const int32_t v = col[j];
                    const uint32_t bit = 1u << (v & 31);
                    uint32_t* wp = visited + (v >> 5);
                    if ((*wp & bit) == 0 && (atomicOr(wp, bit) & bit) == 0) {
                        depth[v] = level + 1;
                        q_next[warp_append_active(tail_next)] = v;
                        const unsigned int dv = (unsigned int)(rowptr[v + 1] - rowptr[v]);
                        mf += dv;
                        dm = dv > dm ? dv : dm;
                    }
                }
            }
        }
        // Block totals of this level's counters.
        mf = warp_sum(mf);
        ex = warp_sum(ex);
        dm = warp_max(dm);
        if (lane == 0) {
            s_mf[threadIdx.x >> 5] = mf;
            s_ex[threadIdx.x >> 5] = ex;
            if (dm) atomicMax(&ps->dmax[(L + 1) % 3], dm);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long a = 0, c = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
                a += s_mf[k];
                c += s_ex[k];
            }
            if (a) atomicAdd(&ps->mf[(L + 1) % 3], a);
            if (c) atomicAdd(&ps->examined, c);
        }
        if (!grid_barrier(&ps->bar_count, &ps->bar_gen, &ps->status)) return;
        ++L;
        ++level;
        const int32_t nf_next = vtail[L % 3];
        const unsigned long long mf_next = ((volatile unsigned long long*)ps->mf)[L % 3];
        const unsigned int dmax_next = ((volatile unsigned int*)ps->dmax)[L % 3];
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ps->m_r += mf_next;
            ps->reached += nf_next;
            ps->levels_done = L;
        }
        // Stop for an empty frontier, at max_depth, when the frontier is too
        // big for one launch, or when the direction rule asks for bottom-up.
        const double m_u = (double)(m_total - m_r_start - (int64_t)ps->m_r);
        // Rows are walked by one warp each here, so a frontier holding a row of
        // kBigList entries or more goes back to the balanced host-driven path.
        if (nf_next == 0 || (int64_t)mf_next >= exit_edges || level >= max_depth || dmax_next >= (unsigned)kBigList ||
            (alpha > 0.f && (double)mf_next > m_u / alpha))
            return;
    }
}

__global__ void bfs_bitmap_from_queue_kernel(const int32_t* __restrict__ q, int32_t count, uint32_t* f) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = q[i];
        atomicOr(f + (v >> 5), 1u << (v & 31));
    }
}

}  // namespace ghb
