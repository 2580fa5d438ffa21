// Whole-traversal BFS in one cooperative launch.
//
// The host-driven BFS (bfs.cu) pays a host round trip per level; on an RMAT
// scale-24 graph that is most of a traversal's time, and on a 4096x4096 grid
// (4097 levels) it is all of it.  Here every level runs inside one launch:
//
//   level L:  expand   top-down (queue) or bottom-up (bitmap), claims write
//                      depth, the next frontier bitmap and level counters
//             barrier
//             [top-down only, if the frontier held rows of >= kBigList
//              entries: those rows, entry-parallel over the whole grid;
//              barrier]
//             block 0 decides the next level (direction rule, stop test)
//             barrier
//
// Frontier bitmaps and counters are triple-buffered by level: level L reads
// slot L%3, writes slot (L+1)%3 and clears slot (L+2)%3, which no block reads
// or writes during level L, so the clears need no extra barrier.  Queues are
// double-buffered (level L reads queue L%2, appends to queue (L+1)%2).
// Every grid barrier is bounded (grid_barrier): on timeout all blocks leave
// and the host reports GHB_ERR_TIMEOUT.
#include <algorithm>
#include <vector>

#include "bfs_kernels.cuh"
#include "common.cuh"
#include "policy.cuh"

namespace ghb {

// Deferred top-down rows (>= kBigList entries): up to kBigChunkRows of them
// are cut into kBigChunk-entry chunks spread over every warp of the grid.
constexpr int32_t kBigChunkRows = 2047;  // 4 per thread of a 512-thread block, plus the total
constexpr int32_t kBigChunk = 256;

struct BfsRunState {
    unsigned bar_count;            // barrier arrivals (own cache line)
    unsigned pad_a[31];
    unsigned long long bar_release; // barrier epoch (low 16 bits) and the next level's state (own cache line)
    unsigned pad_b[30];
    int32_t status;
    int32_t level;       // current level
    int32_t dir;         // 0 top-down, 1 bottom-up
    int32_t done;
    int32_t append;      // top-down level appends to the queue (small frontier)
    int32_t queue_ok;    // the current queue holds the current frontier
    int32_t nf[3];       // frontier sizes by slot
    int32_t big[3];      // deferred long rows by slot
    unsigned dmax[3];
    int32_t by_net;      // the network chose the current level's direction
    unsigned long long mf[3];
    unsigned long long d2[3];        // sum of squared out-degrees by slot
    unsigned long long examined;
    unsigned long long ex_prev;      // examined at the previous decision
    unsigned long long m_r;          // entries out of reached vertices (source included)
    long long reached;               // vertices reached (source excluded)
    int32_t pull_levels;
    int32_t levels;
    int32_t qcount;      // queue compaction cursor (zero at every level start)
    int32_t pad2;
    unsigned long long t_prev;       // global timer at the previous decision
    unsigned long long t_comp;       // global timer after this level's compaction
    unsigned long long bar_limit_ns; // grid-barrier wait limit (set by the host before the launch)
    unsigned bar_extra;              // arrivals beyond the grid every barrier waits for (0; tests: 1)
    unsigned pad3;
};

namespace {

struct PAcc {
    unsigned long long mf = 0, ex = 0, d2 = 0;
    unsigned int dm = 0, nf = 0;
};

// Block totals, one atomic per counter per block.  Contains __syncthreads.
__device__ __forceinline__ void p_flush(PAcc a, BfsRunState* st, int slot, bool count_nf) {
    __shared__ unsigned long long s_mf[32], s_ex[32], s_d2[32];
    __shared__ unsigned s_dm[32], s_nf[32];
    a.mf = warp_sum(a.mf);
    a.ex = warp_sum(a.ex);
    a.d2 = warp_sum(a.d2);
    a.nf = warp_sum(a.nf);
    a.dm = warp_max(a.dm);
    if (lane_id() == 0) {
        s_mf[threadIdx.x >> 5] = a.mf;
        s_ex[threadIdx.x >> 5] = a.ex;
        s_d2[threadIdx.x >> 5] = a.d2;
        s_dm[threadIdx.x >> 5] = a.dm;
        s_nf[threadIdx.x >> 5] = a.nf;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long mf = 0, ex = 0, d2 = 0;
        unsigned dm = 0, nf = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            mf += s_mf[i];
            ex += s_ex[i];
            d2 += s_d2[i];
            nf += s_nf[i];
            dm = s_dm[i] > dm ? s_dm[i] : dm;
        }
        if (mf) atomicAdd(&st->mf[slot], mf);
        if (ex) atomicAdd(&st->examined, ex);
        if (d2) atomicAdd(&st->d2[slot], d2);
        if (dm) atomicMax(&st->dmax[slot], dm);
        if (count_nf && nf) atomicAdd(&st->nf[slot], (int32_t)nf);
    }
    __syncthreads();
}

// Claim v for level `next_depth`.  filter: read the visited word before
// the atomic (saves atomics on large frontiers, where most targets are
// already visited); small frontiers skip it, since the read is one more
// dependent round trip per level.  v's row bounds are read before the
// claim so that they arrive while the atomic is in flight.
__device__ __forceinline__ void p_visit(int32_t v, uint32_t* visited, uint32_t* f_next, int32_t* depth,
                                        int32_t next_depth, int32_t* q_next, int32_t* tail, bool append,
                                        const int32_t* __restrict__ rowptr, PAcc& acc, bool filter = true) {
    const uint32_t bit = 1u << (v & 31);
    uint32_t* wp = visited + (v >> 5);
    if (filter && (*wp & bit)) return;
    const int32_t rb = rowptr[v], re = rowptr[v + 1];
    if (atomicOr(wp, bit) & bit) return;
    depth[v] = next_depth;
    atomicOr(f_next + (v >> 5), bit);
    if (append) q_next[warp_append_active(tail)] = v;
    else acc.nf += 1;
    const unsigned dv = (unsigned)(re - rb);
    acc.mf += dv;
    acc.d2 += (unsigned long long)dv * dv;
    acc.dm = dv > acc.dm ? dv : acc.dm;
}

// The release word of the traversal's grid barriers carries, above the
// 16-bit epoch, the next level's state (payload bits below), so that a
// waiting block learns it from the load that ends its wait instead of
// reading the run state after it: one dependent round trip less per level.
constexpr unsigned long long kPlNf = 0x7fffffffull;  // next frontier size
constexpr unsigned long long kPlDone = 1ull << 32;
constexpr unsigned long long kPlDir = 1ull << 33;      // bottom-up
constexpr unsigned long long kPlAppend = 1ull << 34;   // top-down level appends to the queue
constexpr unsigned long long kPlQueueOk = 1ull << 35;  // the queue holds the frontier
constexpr unsigned long long kPlBig = 1ull << 36;      // long rows deferred: no decision yet

__device__ __forceinline__ unsigned long long p_payload(int32_t nf, bool done, int dir, bool append, bool queue_ok) {
    return ((unsigned long long)nf & kPlNf) | (done ? kPlDone : 0ull) | (dir ? kPlDir : 0ull) |
           (append ? kPlAppend : 0ull) | (queue_ok ? kPlQueueOk : 0ull);
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Grid barrier of the traversal (the ordering of grid_sync_block_leader):
// every thread of the last block to arrive runs leader() (which may contain
// __syncthreads) and leaves the payload in *s_pl; the other blocks get it
// there from the release word.  Bounded: a wait over bar_limit_ns raises
// the status and returns false.
template <class F>
__device__ __forceinline__ bool p_sync(BfsRunState* st, const F& leader, unsigned long long* s_pl) {
    __shared__ int s_ok4, s_last4;
    __shared__ unsigned s_ep4;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned nblocks = gridDim.x + st->bar_extra;
        const unsigned old = atom_add_acq_rel_u32(&st->bar_count, 1u);
        s_ep4 = (old / nblocks + 1u) & 0xffffu;
        s_last4 = (old % nblocks == nblocks - 1u) ? 1 : 0;
        s_ok4 = 1;
    }
    __syncthreads();
    if (s_last4) {
        leader();
        __syncthreads();
        if (threadIdx.x == 0) st_release_u64(&st->bar_release, (*s_pl << 16) | s_ep4);
    } else if (threadIdx.x == 0) {
        const unsigned ep = s_ep4;
        const uint64_t limit = st->bar_limit_ns;
        unsigned spins = 0;
        uint64_t t0 = 0;
        while (true) {
            const unsigned long long v = ld_acquire_u64(&st->bar_release);
            if ((int16_t)(uint16_t)((unsigned)v - ep) >= 0) {
                *s_pl = v >> 16;
                break;
            }
            if ((++spins & 127u) == 0) {
                if (*(volatile int32_t*)&st->status != 0) {
                    s_ok4 = 0;
                    break;
                }
                const uint64_t t = global_timer_ns();
                if (t0 == 0) t0 = t;
                else if (t - t0 > limit) {
                    atomicExch(&st->status, (int32_t)kDevBarrierTimeout);
                    s_ok4 = 0;
                    break;
                }
            }
        }
    }
    __syncthreads();
    return s_ok4 != 0;
}

// Output format of a top-down level: fmt 1 queue, 2 bitmap only, 0 by the
// frontier's out-entries.
__device__ __forceinline__ int32_t p_append(int nd, int fmt, unsigned long long mf) {
    return (nd == 0 && (fmt == 1 || (fmt == 0 && mf < (unsigned long long)kAppendMaxEdges))) ? 1 : 0;
}

}  // namespace

// The learned policy's part of a level decision, kept out of line so that
// its registers do not weigh on the traversal loops of the kernel below.
__device__ __noinline__ float level_margin(int dir, int32_t n, int64_t m, int32_t n_f, unsigned long long m_f,
                                           double m_u, float alpha, float beta, float gamma) {
    return rule_margin(dir, (double)n, (double)m, (double)n_f, (double)m_f, m_u, alpha, beta, gamma);
}

// Every thread of the deciding block calls this; the network runs only
// inside the rule's band and leaves its logits in `logit`.
__device__ __noinline__ void level_eval(const float* pol, const float* feat, float* h1, float* h2, float* logit,
                                        float margin, float band) {
    if (margin < band) policy_eval_block(pol, feat, h1, h2, logit);
}

__global__ void __launch_bounds__(512, 2) bfs_persistent_kernel(
    int32_t n, int32_t n_active, const int32_t* __restrict__ out_rp, const int32_t* __restrict__ out_col,
    const int32_t* __restrict__ in_rp, const int32_t* __restrict__ in_col, int32_t src, int32_t max_depth,
    int32_t* depth, uint32_t* visited, uint32_t* f0, uint32_t* f1, uint32_t* f2, int32_t* qa, int32_t* qb, int32_t* qc,
    int32_t* big, int policy, float alpha, float beta, float gamma, float band, int64_t m_total,
    const int8_t* __restrict__ schedule,
    int32_t schedule_len, const int32_t* __restrict__ perm, int32_t* depth_out, BfsRunState* st,
    const float* __restrict__ pol, float* trace, int32_t trace_cap) {
    const int lane = lane_id();
    const int64_t gtid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t gsize = (int64_t)gridDim.x * blockDim.x;
    const int64_t warp = gtid >> 5;
    const int64_t nwarps = gsize >> 5;
    const int64_t words = ((int64_t)n + 31) / 32;
    const int64_t words_active = ((int64_t)n_active + 31) / 32;

    // ---- init
    for (int64_t v = gtid; v < n; v += gsize) depth[v] = (v == src) ? 0 : kInfDepth;
    for (int64_t w = gtid; w < words; w += gsize) {
        const uint32_t bit = (w == (src >> 5)) ? (1u << (src & 31)) : 0u;
        visited[w] = bit;
        f0[w] = bit;
        f1[w] = 0u;
        f2[w] = 0u;
    }
    // The network (parameters + normalisation, 25 KB) is read from global
    // memory by whichever block decides a level inside the rule's band; it
    // stays in L2, and no block pays to stage it in shared memory.
    const bool net = pol != nullptr;
    const bool can_pull = in_rp != nullptr;
    // The first level's state, worked out by every block (s_pl: the state
    // payload each barrier hands on; see p_sync).
    __shared__ unsigned long long s_pl;
    if (threadIdx.x == 0) {
        const unsigned ds = (unsigned)(out_rp[src + 1] - out_rp[src]);
        int d0 = 0, f0req = 0;
        if (policy == GHB_POLICY_SCHEDULE && schedule && schedule_len > 0) {
            d0 = can_pull ? (schedule[0] & 1) : 0;
            f0req = (schedule[0] >> 1) & 3;
        }
        const int32_t app0 = p_append(d0, f0req, ds);
        s_pl = p_payload(1, max_depth <= 0, d0, app0 != 0, true);
        if (blockIdx.x == 0) {
            qa[0] = src;
            st->nf[0] = 1;
            st->mf[0] = ds;
            st->d2[0] = (unsigned long long)ds * ds;
            st->dmax[0] = ds;
            st->m_r = ds;
            st->append = app0;
            st->queue_ok = 1;
            st->level = 0;
            st->dir = d0;
            st->done = max_depth <= 0 ? 1 : 0;
            st->t_prev = global_timer_ns();
            if (trace && trace_cap > 0)
                bfs_features(trace, (double)n, (double)m_total, 1.0, (double)ds, (double)(m_total - (int64_t)ds), 0,
                             (double)ds * ds, (double)ds, 0, 1.0, (double)n - 1.0);
        }
    }
    if (!p_sync(st, [] {}, &s_pl)) return;

    __shared__ float s_feat[kPolIn], s_h1[kPolH], s_h2[kPolH], s_logit[kPolOut];
    __shared__ int32_t s_dec[2];
    __shared__ float s_margin;
    __shared__ int32_t s_flag;

    volatile BfsRunState* vs = st;
    // One iteration per level in every block; the level's state arrived
    // with the previous barrier's release (s_pl).
    // Frontier L - 1's size and whether that level ran top-down (its
    // vertices are then listed in queue (L + 2) % 3); level 0 has none.
    int32_t last_nf = 0;
    bool last_top = true;
    for (int32_t L = 0;; ++L) {
        const unsigned long long pl = s_pl;
        if (pl & kPlDone) break;
        const int dir = (pl & kPlDir) ? 1 : 0;
        const int slot = L % 3, nslot = (L + 1) % 3, cslot = (L + 2) % 3;
        const bool append = (pl & kPlAppend) != 0;
        const int32_t n_f = (int32_t)(pl & kPlNf);
        const bool queue_ok = (pl & kPlQueueOk) != 0;
        // (selects, not an indexed array: an array would live in local memory)
        uint32_t* f_cur = slot == 0 ? f0 : (slot == 1 ? f1 : f2);
        uint32_t* f_next = nslot == 0 ? f0 : (nslot == 1 ? f1 : f2);
        uint32_t* f_clear = cslot == 0 ? f0 : (cslot == 1 ? f1 : f2);
        // Queues triple-buffered like the bitmaps: level L reads queue L % 3,
        // appends to (L + 1) % 3, and queue (L + 2) % 3 still lists frontier
        // L - 1, whose bitmap (f_clear) is cleared through it when that level
        // ran top-down and its frontier was small.
        int32_t* q_cur = slot == 0 ? qa : (slot == 1 ? qb : qc);
        int32_t* q_next = nslot == 0 ? qa : (nslot == 1 ? qb : qc);
        const int32_t* q_clear = cslot == 0 ? qa : (cslot == 1 ? qb : qc);
        const int32_t clear_nf = last_nf;
        const bool clear_sparse = last_top && (int64_t)clear_nf * 4 < words;
        last_nf = n_f;
        last_top = dir == 0;
        auto clear_frontier_bitmap = [&]() {
            if (clear_sparse) {
                for (int64_t i = gtid; i < clear_nf; i += gsize) f_clear[__ldcg(q_clear + i) >> 5] = 0u;
            } else {
                for (int64_t w = gtid; w < words; w += gsize) f_clear[w] = 0u;
            }
        };
        const int32_t next_depth = L + 1;
        PAcc acc;
        // Level decision, run by every thread of the last block to reach the
        // level's final barrier (all counters are settled then).  Thread 0
        // does the bookkeeping and the fixed rules; the block evaluates the
        // network when the learned policy is on.
        auto decide = [&]() {
            int32_t nf_next = 0;
            unsigned long long mf_next = 0;
            if (threadIdx.x == 0) {
                volatile BfsRunState* vd = st;
                nf_next = vd->nf[nslot];
                mf_next = vd->mf[nslot];
                const unsigned long long m_r_prev = vd->m_r;
                const unsigned long long ex_now = vd->examined;
                const long long reached_prev = vd->reached;
                const uint64_t now = global_timer_ns();
                const uint64_t tp = vd->t_prev;
                const float ms = (float)((double)(now - tp) * 1e-6);
                if (trace && L < trace_cap) {
                    float* row = trace + (size_t)L * GHB_TRACE_COLS;
                    const double unvisited = (double)n - 1.0 - (double)reached_prev;
                    const double ex = (double)(ex_now - vd->ex_prev);
                    row[12] = (float)dir;
                    row[13] = ms;
                    row[14] = -1.f;
                    row[15] = -1.f;
                    row[16] = (float)ex;
                    row[17] = (float)nf_next;
                    row[18] = (float)unvisited;
                    row[19] = (float)(4.0 * (dir ? unvisited : (double)n_f) + 4.0 * ex + 4.0 * (double)nf_next);
                    row[20] = dir == 0 ? (append ? 0.f : 1.f) : -1.f;
                    row[21] = (dir == 0 && !queue_ok) ? (float)((double)(vd->t_comp - tp) * 1e-6) : -1.f;
                    row[22] = (float)vd->by_net;
                    row[23] = -1.f;
                }
                st->ex_prev = ex_now;
                st->t_prev = now;
                st->m_r = m_r_prev + mf_next;
                st->reached = reached_prev + nf_next;
                st->levels = L + 1;
                if (dir == 1) st->pull_levels = vd->pull_levels + 1;
                int nd = dir, fmt = 0;
                const double m_u = (double)(m_total - (long long)(m_r_prev + mf_next));
                if (policy == GHB_POLICY_PUSH || !can_pull) {
                    nd = 0;
                } else if (policy == GHB_POLICY_PULL) {
                    nd = 1;
                } else if (policy == GHB_POLICY_SCHEDULE) {
                    if (schedule && L + 1 < schedule_len) {
                        nd = schedule[L + 1] & 1;
                        fmt = (schedule[L + 1] >> 1) & 3;
                    }
                } else {
                    if (dir == 0 && (double)mf_next > m_u / alpha && (double)mf_next > (double)m_total / gamma) nd = 1;
                    else if (dir == 1 && (double)nf_next < (double)n / beta) nd = 0;
                    if (net) s_margin = level_margin(dir, n, m_total, nf_next, mf_next, m_u, alpha, beta, gamma);
                }
                // Features only for the network or a trace: they sit on the
                // level's critical path while the grid waits.
                if (net || trace)
                    bfs_features(s_feat, (double)n, (double)m_total, (double)nf_next, (double)mf_next, m_u, L + 1,
                                 (double)vd->d2[nslot], (double)vd->dmax[nslot], dir, (double)n_f,
                                 (double)n - 1.0 - (double)(reached_prev + nf_next));
                if (trace && L + 1 < trace_cap)
                    for (int k = 0; k < kPolIn; ++k) trace[(size_t)(L + 1) * GHB_TRACE_COLS + k] = s_feat[k];
                s_dec[0] = nd;
                s_dec[1] = fmt;
            }
            if (net) {
                __syncthreads();
                // Levels outside the rule's uncertain band keep the rule's
                // choices: no network evaluation on them (it would sit on
                // the level's critical path while the grid waits).
                level_eval(pol, s_feat, s_h1, s_h2, s_logit, s_margin, band);
            }
            if (threadIdx.x == 0) {
                int nd = s_dec[0], fmt = s_dec[1];
                int by_net = 0;
                if (net && s_margin < band) {
                    nd = (can_pull && s_logit[kHeadDir + 1] > s_logit[kHeadDir]) ? 1 : 0;
                    fmt = s_logit[kHeadFmt + 1] > s_logit[kHeadFmt] ? 2 : 1;
                    by_net = 1;
                }
                st->by_net = by_net;
                st->dir = nd;
                // The next queue holds the next frontier only if this level
                // was top-down and appended.
                st->append = p_append(nd, fmt, mf_next);
                st->queue_ok = (dir == 0 && append) ? 1 : 0;
                st->qcount = 0;
                st->level = L + 1;
                const bool done = nf_next == 0 || L + 1 >= max_depth;
                st->done = done ? 1 : 0;
                s_pl = p_payload(nf_next, done, nd, p_append(nd, fmt, mf_next) != 0, dir == 0 && append);
                st->nf[cslot] = 0;
                st->mf[cslot] = 0;
                st->d2[cslot] = 0;
                st->dmax[cslot] = 0;
                st->big[cslot] = 0;
            }
        };

        if (dir == 0) {
            if (!queue_ok) {
                // Queue from the frontier bitmap (after a bottom-up level).
                for (int64_t w0 = warp * 32; w0 < words_active; w0 += nwarps * 32) {
                    const int64_t w = w0 + lane;
                    uint32_t bits = w < words_active ? f_cur[w] : 0u;
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
                    if (lane == 0) base = atomicAdd(&st->qcount, total);
                    base = __shfl_sync(0xffffffffu, base, 0);
                    int32_t pos = base + incl - c;
                    while (bits) {
                        const int b = __ffs(bits) - 1;
                        bits &= bits - 1;
                        q_cur[pos++] = (int32_t)(w * 32 + b);
                    }
                }
                if (!p_sync(st, [&]() {
                        if (threadIdx.x == 0) st->t_comp = global_timer_ns();
                    }, &s_pl))
                    return;
            }
            // Short and medium rows; rows of >= kBigList entries deferred.
            // A warp takes vpw frontier vertices (one per lane): 32 on large
            // frontiers; on small ones fewer, so that the frontier's entries
            // spread over every warp of the grid instead of queueing behind
            // each other in a few warps (each pass of a warp over its
            // entries is a chain of dependent loads and atomics).
            int32_t vpw = 32;
            if ((int64_t)n_f < nwarps * 16) {
                vpw = 1;
                while (vpw < 32 && (int64_t)vpw * nwarps < n_f) vpw <<= 1;
            }
            const bool filter = vpw == 32;
            for (int64_t base = warp * vpw; base < n_f; base += nwarps * vpw) {
                const int64_t i = base + lane;
                int32_t b = 0, e = 0;
                if (lane < vpw && i < n_f) {
                    const int32_t u = q_cur[i];
                    b = out_rp[u];
                    e = out_rp[u + 1];
                    if (e - b >= kBigList) {
                        big[warp_append_active(&st->big[slot])] = u;
                        e = b;
                    }
                }
                acc.ex += (unsigned long long)(e - b);
                unsigned med = __ballot_sync(0xffffffffu, e - b >= 32);
                while (med) {
                    const int leader = __ffs(med) - 1;
                    med &= med - 1;
                    const int32_t lb = __shfl_sync(0xffffffffu, b, leader);
                    const int32_t le = __shfl_sync(0xffffffffu, e, leader);
                    for (int32_t j = lb + lane; j < le; j += 32)
                        p_visit(out_col[j], visited, f_next, depth, next_depth, q_next, &st->nf[nslot], append,
                                out_rp, acc, filter);
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
                    const int32_t k = k0 + lane;
                    int owner = 0;
#pragma unroll
                    for (int sft = 16; sft >= 1; sft >>= 1) {
                        const int cand = owner + sft;
                        const int32_t ev = __shfl_sync(0xffffffffu, excl, cand);
                        if (ev <= k) owner = cand;
                    }
                    const int32_t ob = __shfl_sync(0xffffffffu, b, owner);
                    const int32_t oe = __shfl_sync(0xffffffffu, excl, owner);
                    if (k < total)
                        p_visit(out_col[ob + (k - oe)], visited, f_next, depth, next_depth, q_next, &st->nf[nslot],
                                append, out_rp, acc, filter);
                }
            }
            clear_frontier_bitmap();
            p_flush(acc, st, nslot, !append);
            acc = PAcc();
            // Decide now unless long rows were deferred (then after them).
            if (!p_sync(st, [&]() {
                    if (threadIdx.x == 0) s_flag = ((volatile BfsRunState*)st)->big[slot] == 0 ? 1 : 0;
                    __syncthreads();
                    if (s_flag) decide();
                    else if (threadIdx.x == 0) s_pl |= kPlBig;
                }, &s_pl))
                return;
            __shared__ int32_t s_nbig;
            const bool big_pending = (s_pl & kPlBig) != 0;
            if (big_pending && threadIdx.x == 0) s_nbig = vs->big[slot];
            __syncthreads();
            const int32_t nbig = big_pending ? s_nbig : 0;
            if (nbig > 0) {
                if (nbig <= kBigChunkRows) {
                    // Deferred rows cut into kBigChunk-entry chunks shared by
                    // every warp of the grid: each block builds the chunk
                    // prefix of the (few) rows in shared memory, a warp takes
                    // chunks round robin and finds the row by binary search.
                    __shared__ int32_t s_cpre[kBigChunkRows + 1];  // indices 0..nbig <= 2047
                    __shared__ int32_t s_wsum[16];
                    const int t = threadIdx.x;
                    int32_t cnt4[4];
                    int32_t tsum = 0;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int32_t r = 4 * t + q;
                        int32_t c = 0;
                        if (r < nbig) {
                            const int32_t u = big[r];
                            c = (out_rp[u + 1] - out_rp[u] + kBigChunk - 1) / kBigChunk;
                        }
                        cnt4[q] = c;
                        tsum += c;
                    }
                    int32_t incl = tsum;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int32_t x = __shfl_up_sync(0xffffffffu, incl, o);
                        if (lane >= o) incl += x;
                    }
                    if (lane == 31) s_wsum[t >> 5] = incl;
                    __syncthreads();
                    int32_t wbase = 0;
                    for (int i = 0; i < (t >> 5); ++i) wbase += s_wsum[i];
                    int32_t run = wbase + incl - tsum;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int32_t r = 4 * t + q;
                        if (r <= nbig) s_cpre[r] = run;
                        run += cnt4[q];
                    }
                    __syncthreads();
                    const int32_t nchunks = s_cpre[nbig];
                    for (int64_t ch = warp; ch < nchunks; ch += nwarps) {
                        int32_t lo = 0, hi = nbig - 1;
                        while (lo < hi) {
                            const int32_t mid = (lo + hi + 1) >> 1;
                            if (s_cpre[mid] <= ch) lo = mid;
                            else hi = mid - 1;
                        }
                        const int32_t u = big[lo];
                        const int32_t rb = out_rp[u] + (int32_t)(ch - s_cpre[lo]) * kBigChunk;
                        const int32_t re = min(out_rp[u + 1], rb + kBigChunk);
                        for (int32_t j = rb + lane; j < re; j += 32)
                            p_visit(out_col[j], visited, f_next, depth, next_depth, q_next, &st->nf[nslot], append,
                                    out_rp, acc);
                        if (lane == 0) acc.ex += (unsigned long long)(re - rb);
                    }
                } else {
                    // Many deferred rows: one block per row (round robin),
                    // except rows of kHugeList or more, which every thread of
                    // the grid strides.
                    for (int32_t r = blockIdx.x; r < nbig; r += gridDim.x) {
                        const int32_t u = big[r];
                        const int32_t rb = out_rp[u], re = out_rp[u + 1];
                        if (re - rb >= kHugeList) continue;
                        for (int32_t j = rb + threadIdx.x; j < re; j += blockDim.x)
                            p_visit(out_col[j], visited, f_next, depth, next_depth, q_next, &st->nf[nslot], append,
                                    out_rp, acc);
                        if (threadIdx.x == 0) acc.ex += (unsigned long long)(re - rb);
                    }
                    for (int32_t r = 0; r < nbig; ++r) {
                        const int32_t u = big[r];
                        const int32_t rb = out_rp[u], re = out_rp[u + 1];
                        if (re - rb < kHugeList) continue;
                        for (int64_t j = rb + gtid; j < re; j += gsize)
                            p_visit(out_col[j], visited, f_next, depth, next_depth, q_next, &st->nf[nslot], append,
                                    out_rp, acc);
                        if (gtid == 0) acc.ex += (unsigned long long)(re - rb);
                    }
                }
                p_flush(acc, st, nslot, !append);
                if (!p_sync(st, decide, &s_pl)) return;
            }
        } else {
            // Bottom-up over the active vertices: a warp owns a bitmap word.
            for (int64_t w = warp; w < words_active; w += nwarps) {
                const uint32_t vis = visited[w];
                if (vis == 0xffffffffu) continue;
                const int64_t v = w * 32 + lane;
                const bool todo = v < n_active && !((vis >> lane) & 1u);
                bool found = false;
                int32_t j = 0, e = 0;
                if (todo) {
                    j = in_rp[v];
                    e = in_rp[v + 1];
                    const int32_t b = j;
                    const int32_t lim = min(e, b + 32);
                    while (j < lim && !found) {
                        int32_t u[4];
#pragma unroll
                        for (int k = 0; k < 4; ++k) u[k] = (j + k < lim) ? in_col[j + k] : -1;
                        bool h[4];
#pragma unroll
                        for (int k = 0; k < 4; ++k) h[k] = u[k] >= 0 && ((f_cur[u[k] >> 5] >> (u[k] & 31)) & 1u);
                        const int hit = h[0] ? 0 : h[1] ? 1 : h[2] ? 2 : h[3] ? 3 : -1;
                        if (hit >= 0) {
                            found = true;
                            j += hit + 1;
                        } else {
                            j = min(j + 4, lim);
                        }
                    }
                    acc.ex += (unsigned long long)(j - b);
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
                        acc.ex += (unsigned long long)scanned;
                    }
                    rest &= rest - 1;
                }
                const unsigned fm = __ballot_sync(0xffffffffu, found);
                if (fm) {
                    if (lane == 0) {
                        visited[w] = vis | fm;
                        f_next[w] = fm;
                    }
                    if (found) {
                        depth[v] = next_depth;
                        const unsigned dv = (unsigned)(out_rp[v + 1] - out_rp[v]);
                        acc.mf += dv;
                        acc.d2 += (unsigned long long)dv * dv;
                        acc.dm = dv > acc.dm ? dv : acc.dm;
                        acc.nf += 1;
                    }
                }
            }
            clear_frontier_bitmap();
            p_flush(acc, st, nslot, true);
            if (!p_sync(st, decide, &s_pl)) return;
        }

    }

    // ---- results in the caller's ids
    if (perm) {
        for (int64_t v = gtid; v < n; v += gsize) depth_out[v] = depth[perm[v]];
    }
}

}  // namespace ghb

namespace ghb {

bool bfs_persistent_available(ghb_workspace* ws, int* blocks) {
    static int cached[64] = {0};
    static bool known[64] = {false};
    const int dev = ws->device;
    if (dev < 0 || dev >= 64) return false;
    if (!known[dev]) {
        int coop = 0, per_sm = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        if (coop && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bfs_persistent_kernel, 512, 0) ==
                        cudaSuccess)
            cached[dev] = std::min(per_sm, 2);
        known[dev] = true;
    }
    // Blocks per SM: the workspace's bfs_blocks_per_sm, at most what fits.
    *blocks = std::min(cached[dev], (int)ws->tune.bfs_blocks_per_sm) * ws->num_sms;
    return *blocks > 0;
}

// One cooperative launch for the whole traversal.  depth: per-vertex output
// in the graph's ids; with perm, depth_out[v] = depth[perm[v]] as well.
int bfs_persistent_run(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* out_rp, const int32_t* out_col,
                       const int32_t* in_rp, const int32_t* in_col, int32_t src, int32_t max_depth, int32_t* depth,
                       const int32_t* perm, int32_t* depth_out, const ghb_bfs_options* opt,
                       ghb_traversal_stats* stats) {
    int blocks = 0;
    if (!bfs_persistent_available(ws, &blocks)) {
        set_error("cooperative launch unavailable");
        return GHB_ERR_UNSUPPORTED;
    }
    cudaStream_t st = ws->stream;
    const int64_t words = ((int64_t)n + 31) / 32;
    Carver sizing(nullptr);
    const bool want_trace = opt && opt->record_trace && opt->trace && opt->trace_cap > 0;
    const int32_t tcap = want_trace ? std::min<int32_t>(opt->trace_cap, 1 << 16) : 0;
    auto carve = [&](Carver& c, uint32_t** vis, uint32_t** f0, uint32_t** f1, uint32_t** f2, int32_t** qa,
                     int32_t** qb, int32_t** qc, int32_t** big, BfsRunState** rs, int8_t** sched, float** tr) {
        *vis = c.take<uint32_t>(words);
        *f0 = c.take<uint32_t>(words);
        *f1 = c.take<uint32_t>(words);
        *f2 = c.take<uint32_t>(words);
        *qa = c.take<int32_t>(n);
        *qb = c.take<int32_t>(n);
        *qc = c.take<int32_t>(n);
        *big = c.take<int32_t>(n);
        *rs = c.take<BfsRunState>(1);
        *sched = c.take<int8_t>(4096);
        *tr = c.take<float>((size_t)(tcap > 0 ? tcap : 1) * GHB_TRACE_COLS);
    };
    uint32_t *vis, *f0, *f1, *f2;
    int32_t *qa, *qb, *qc, *big;
    BfsRunState* rs;
    int8_t* sched;
    float* tr;
    carve(sizing, &vis, &f0, &f1, &f2, &qa, &qb, &qc, &big, &rs, &sched, &tr);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &vis, &f0, &f1, &f2, &qa, &qb, &qc, &big, &rs, &sched, &tr);

    int policy = opt ? opt->policy : GHB_POLICY_HEURISTIC;
    float alpha = (opt && opt->alpha > 0) ? opt->alpha : 256.0f;
    float beta = (opt && opt->beta > 0) ? opt->beta : 24.0f;
    float gamma = (opt && opt->gamma > 0) ? opt->gamma : 1024.0f;
    int32_t sched_len = 0;
    if (policy == GHB_POLICY_SCHEDULE && opt && opt->schedule && opt->schedule_len > 0) {
        sched_len = std::min<int32_t>(opt->schedule_len, 4096);
        GHB_CUDA_TRY(cudaMemcpyAsync(sched, opt->schedule, sched_len, cudaMemcpyHostToDevice, st));
    }
    // The learned policy runs in the kernel when a network is installed;
    // otherwise GHB_POLICY_LEARNED falls back to the heuristic.
    const float* pol = nullptr;
    if (policy == GHB_POLICY_LEARNED) {
        pol = policy_device_params();
        if (!pol) policy = GHB_POLICY_HEURISTIC;
    }
    int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned);
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, out_rp + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaMemsetAsync(rs, 0, sizeof(BfsRunState), st));
    {
        // Barrier limit and test knob (pageable source: staged by the call).
        const unsigned long long bar[2] = {(unsigned long long)ws->tune.barrier_limit_us * 1000ull,
                                           (unsigned long long)ws->tune.barrier_extra};
        GHB_CUDA_TRY(cudaMemcpyAsync(&rs->bar_limit_ns, bar, sizeof(bar), cudaMemcpyHostToDevice, st));
    }
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t m_total = hp[0];
    if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
    GHB_TRY(launch_coop(ws, bfs_persistent_kernel, dim3(blocks), dim3(512), 0, n,
                        n_active, out_rp, out_col, in_rp, in_col, src, max_depth, depth, vis, f0, f1, f2, qa, qb, qc, big,
                        policy, alpha, beta, gamma, (float)ws->tune.pol_band, m_total,
                        (const int8_t*)(sched_len ? sched : nullptr), sched_len,
                        perm,
                        depth_out, rs, pol, tcap > 0 ? tr : (float*)nullptr, tcap));
    if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_stop, st));
    GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, rs, sizeof(BfsRunState), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const BfsRunState* h = reinterpret_cast<const BfsRunState*>(ws->host_pinned);
    if (h->status != kDevOk) {
        set_error("BFS: grid barrier timed out");
        return GHB_ERR_TIMEOUT;
    }
    const int32_t levels = h->levels;
    const int32_t pull_levels = h->pull_levels;
    const int64_t reached = 1 + h->reached;
    const int64_t m_r = (int64_t)h->m_r;
    const int64_t examined = (int64_t)h->examined;
    if (tcap > 0) {
        const int32_t rows = std::min(levels, tcap);
        if (rows > 0) {
            GHB_CUDA_TRY(cudaMemcpyAsync(opt->trace, tr, sizeof(float) * rows * GHB_TRACE_COLS, cudaMemcpyDeviceToHost,
                                         st));
            GHB_CUDA_TRY(cudaStreamSynchronize(st));
        }
    }
    if (stats) {
        float ms = 0.f;
        GHB_CUDA_TRY(cudaEventElapsedTime(&ms, ws->ev_start, ws->ev_stop));
        stats->levels = levels;
        stats->pull_levels = pull_levels;
        stats->reached = reached;
        stats->edges_reached = m_r;
        stats->edges_examined = examined;
        stats->device_ms = ms;
    }
    return GHB_OK;
}

}  // namespace ghb
