// Whole single-source shortest-path traversal in one cooperative launch.
//
// The host-driven delta-stepping (sssp.cu) pays a host round trip and
// several launches per relaxation round, like the reference's
// frontier loop (GPU_SSSP_csr.cuh:286-307, a device-to-host copy of the
// queue length per iteration).  Here every round runs inside one launch and
// the grid meets at a bounded barrier between passes; the last block to
// arrive decides the next pass:
//
//   LIGHT  relax the light range (entries with w < delta of the weight-sorted
//          rows; the whole row when there is no split) of every near-queue
//          vertex.  An improvement below the bucket's end queues the vertex
//          for the next LIGHT pass, one at or above it goes to the far list.
//          Each queued vertex also joins R, the bucket's settled set.
//   HEAVY  relax the heavy range (w >= delta) of every vertex of R once.
//   CHUNK  after a LIGHT or HEAVY pass that met rows of more than kSpDirect
//          entries: those rows, cut into kSpChunk-entry chunks, a chunk per
//          warp, in the same round (same stamps, same next queue).
//   SPLIT  move the far list's entries below the next bucket's end into the
//          near queue; drop entries already settled; keep the rest.
//
// The next bucket's end follows the smallest pending far distance
// (kept in shared memory per block, one global atomic per block and pass),
// so empty buckets cost nothing.
//
// Results are the least fixpoint of d[v] = min_u fl(d[u] + w): any
// relaxation order reaches it bit for bit (see sssp.cu), so they equal the
// CPU Dijkstra's (CPU_shortest_paths.hpp:19-64).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "graph.cuh"

namespace ghb {

// Rows of up to kSpDirect entries are relaxed where the queue hands them to a
// warp; longer ones are cut into kSpChunk-entry chunks that a CHUNK pass, in
// the same round, spreads over every warp (a warp walking a few 1,024-entry
// rows while the rest of the grid waits at the barrier was the bottleneck).
constexpr int32_t kSpDirect = 64;
constexpr int32_t kSpChunk = 256;
constexpr int kSsspThreads = 512;
constexpr unsigned long long kSsspTimeBudgetNs = 120ull * 1000000000ull;  // two minutes

enum SsspMode : int32_t { kLight = 0, kHeavy = 1, kSplit = 2, kDone = 3, kChunk = 4 };

struct SsspRunState {
    unsigned bar_count;  // barrier arrivals (own cache line)
    unsigned pad_a[31];
    unsigned bar_release;  // barrier epochs (own cache line)
    unsigned pad_b[31];
    int32_t status;
    int32_t mode;         // SsspMode of the current pass
    int32_t round;        // stamp of the near queue being filled
    int32_t phase;        // stamp of the far list being filled
    int32_t epoch;        // stamp of R (bumped after every HEAVY pass)
    int32_t nq;           // items of the current queue (near queue, or R in HEAVY)
    int32_t nc;           // chunk items of the current (CHUNK) pass
    int32_t qsel;         // near queue buffer read by the current pass
    int32_t chunk_of;     // the pass (LIGHT or HEAVY) whose rows a CHUNK pass finishes
    int32_t fsel;         // far buffer filled by relaxations
    int32_t q_tail;       // appends to the next near queue
    int32_t c_tail;       // chunks appended by the current pass
    int32_t r_tail;       // appends to R
    int32_t far_tail;     // entries of the far list being filled
    int32_t kept_tail;    // entries kept by a SPLIT pass
    int32_t pad0;
    double thr;           // end of the current bucket
    double new_thr;       // end of the next bucket (SPLIT)
    double delta;
    unsigned long long fmin;  // smallest pending far distance (bits; an upper bound on stale entries)
    unsigned long long examined;
    long long passes, light_passes, heavy_passes, splits, chunk_passes;
    long long pass_budget;            // passes allowed (set by the host)
    unsigned long long t_start;       // global timer at the start
    unsigned long long bar_limit_ns;
    unsigned bar_extra;
    unsigned pad1;
    // Bucket width: the light/heavy split stays at delta; the width of the
    // buckets may move within [width_min, width_max] from one bucket to the
    // next (equal to delta when the width does not adapt).
    double width, width_min, width_max;
    long long lp_mark;              // LIGHT passes before the current bucket
    unsigned long long ex_mark;     // entries examined before the current bucket
    unsigned long long adapt_work;  // a bucket examining fewer entries is small
};

namespace {

__device__ __forceinline__ double sp_dist(const unsigned long long* d, int32_t v) {
    return __longlong_as_double((long long)__ldcg(d + v));
}

struct SpCtx {
    const int32_t* __restrict__ rp;
    const int32_t* __restrict__ le;  // light ends (nullptr: no light/heavy split)
    const int32_t* __restrict__ col;
    const double* __restrict__ wt;
    unsigned long long* dist;
    int32_t* near_stamp;
    int32_t* far_stamp;
    int32_t* r_stamp;
    int32_t* R;
    int32_t* q_next;
    int32_t* far_cur;
    int4* chunks;
    SsspRunState* st;
    double thr;
    int32_t round, phase, epoch;
};

// Entries a lane relaxes per step: their column, weight and distance loads
// are all issued before any compare, so a lane keeps kSpBatch gathers in
// flight instead of one dependent chain.
constexpr int kSpBatch = 4;

// The compare-and-update part of relaxing an entry u -> v, nd = d[u] + w,
// cur = the distance of v read before.
__device__ __forceinline__ void sp_update(const SpCtx& c, int32_t v, double nd, double cur,
                                          unsigned long long* s_fmin) {
    if (nd < cur) {
        const unsigned long long nb = (unsigned long long)__double_as_longlong(nd);
        const unsigned long long old = atomicMin(c.dist + v, nb);
        if (nb < old) {
            if (nd < c.thr) {
                if (atomicExch(c.near_stamp + v, c.round) != c.round) c.q_next[warp_append_active(&c.st->q_tail)] = v;
            } else {
                if (atomicExch(c.far_stamp + v, c.phase) != c.phase)
                    c.far_cur[warp_append_active(&c.st->far_tail)] = v;
                atomicMin(s_fmin, nb);
            }
        }
    }
}

// Relax entries j[q] (those with ok[q]) of rows whose source distances are
// du[q].
__device__ __forceinline__ void sp_relax_batch(const SpCtx& c, const double* du, const int32_t* j, const bool* ok,
                                               unsigned long long& exam, unsigned long long* s_fmin) {
    int32_t v[kSpBatch];
    double w[kSpBatch], cur[kSpBatch];
#pragma unroll
    for (int q = 0; q < kSpBatch; ++q) {
        v[q] = ok[q] ? c.col[j[q]] : 0;
        w[q] = ok[q] ? c.wt[j[q]] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < kSpBatch; ++q) cur[q] = ok[q] ? sp_dist(c.dist, v[q]) : 0.0;
#pragma unroll
    for (int q = 0; q < kSpBatch; ++q)
        if (ok[q]) {
            ++exam;
            sp_update(c, v[q], du[q] + w[q], cur[q], s_fmin);
        }
}

// Relax [jb, je) of one row (distance du) with the whole warp.
__device__ __forceinline__ void sp_warp_range(const SpCtx& c, double du, int32_t jb, int32_t je,
                                              unsigned long long& exam, unsigned long long* s_fmin) {
    const int lane = lane_id();
    for (int32_t j0 = jb + lane; j0 < je; j0 += 32 * kSpBatch) {
        int32_t jj[kSpBatch];
        bool ok[kSpBatch];
        double dd[kSpBatch];
#pragma unroll
        for (int q = 0; q < kSpBatch; ++q) {
            jj[q] = j0 + 32 * q;
            ok[q] = jj[q] < je;
            dd[q] = du;
        }
        sp_relax_batch(c, dd, jj, ok, exam, s_fmin);
    }
}

// Relax [b, e) of the rows held by the warp's lanes (u < 0: none).  Rows
// longer than kSpDirect are appended, whole, to the chunk list of the CHUNK
// pass that follows.
__device__ __forceinline__ void sp_rows(const SpCtx& c, int32_t u, int32_t b, int32_t e, double du,
                                        unsigned long long& exam, unsigned long long* s_fmin) {
    const int lane = lane_id();
    if (e - b > kSpDirect) {
        const int32_t nch = (e - b + kSpChunk - 1) / kSpChunk;
        const int32_t pos = atomicAdd(&c.st->c_tail, nch);
        for (int32_t k = 0; k < nch; ++k) {
            const int32_t cb = b + k * kSpChunk;
            c.chunks[pos + k] = make_int4(u, cb, min(e, cb + kSpChunk), 0);
        }
        e = b;
    }
    // Rows of 32 entries or more: the whole warp, one row at a time.
    unsigned med = __ballot_sync(0xffffffffu, e - b >= 32);
    while (med) {
        const int leader = __ffs(med) - 1;
        med &= med - 1;
        const int32_t lb = __shfl_sync(0xffffffffu, b, leader);
        const int32_t lend = __shfl_sync(0xffffffffu, e, leader);
        const double ld = __shfl_sync(0xffffffffu, du, leader);
        sp_warp_range(c, ld, lb, lend, exam, s_fmin);
    }
    if (e - b >= 32) e = b;
    // Shorter rows: gathered warp-wide over a scan of their lengths.
    const int32_t d = e - b;
    int32_t incl = d;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += x;
    }
    const int32_t excl = incl - d;
    const int32_t total = __shfl_sync(0xffffffffu, incl, 31);
    for (int32_t k0 = 0; k0 < total; k0 += 32 * kSpBatch) {
        int32_t jj[kSpBatch];
        bool ok[kSpBatch];
        double dd[kSpBatch];
#pragma unroll
        for (int q = 0; q < kSpBatch; ++q) {
            const int32_t k = k0 + 32 * q + lane;
            int owner = 0;
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1) {
                const int cand = owner + s;
                const int32_t ev = __shfl_sync(0xffffffffu, excl, cand);
                if (ev <= k) owner = cand;
            }
            const int32_t ob = __shfl_sync(0xffffffffu, b, owner);
            const int32_t oe = __shfl_sync(0xffffffffu, excl, owner);
            dd[q] = __shfl_sync(0xffffffffu, du, owner);
            ok[q] = k < total;
            jj[q] = ob + (k - oe);
        }
        sp_relax_batch(c, dd, jj, ok, exam, s_fmin);
    }
}

__device__ __forceinline__ bool sp_barrier(SsspRunState* st) {
    return grid_sync_leader(&st->bar_count, &st->bar_release, &st->status, NoLeader(), st->bar_limit_ns,
                            st->bar_extra);
}
template <class F>
__device__ __forceinline__ bool sp_barrier(SsspRunState* st, const F& leader) {
    return grid_sync_leader(&st->bar_count, &st->bar_release, &st->status, leader, st->bar_limit_ns,
                            st->bar_extra);
}

// Bucket-width adaptation: more LIGHT passes than this in a bucket halve
// the next bucket's width.
constexpr long long kSpAdaptLight = 4;

// End of the bucket that holds distance mn, on the grid thr + k * delta.
__device__ __forceinline__ double sp_next_thr(double thr, double delta, double mn) {
    double nthr = thr + delta;
    if (mn >= nthr) nthr = thr + delta * floor((mn - thr) / delta + 1.0);
    if (!(nthr > mn)) nthr = mn + delta;                // guards rounding
    if (!(nthr > mn)) nthr = nextafter(mn, INFINITY);  // delta below mn's ulp
    return nthr;
}

}  // namespace

__global__ void __launch_bounds__(kSsspThreads, 2) sssp_persistent_kernel(
    int32_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ le, const int32_t* __restrict__ col,
    const double* __restrict__ wt, int32_t src, double inf, double* dist_d, int32_t* qa, int32_t* qb, int4* chunks,
    int32_t* fa, int32_t* fb, int32_t* near_stamp, int32_t* far_stamp, int32_t* r_stamp, int32_t* R,
    SsspRunState* st, const int32_t* __restrict__ perm, double* out) {
    unsigned long long* dist = reinterpret_cast<unsigned long long*>(dist_d);
    const int64_t gtid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t gsize = (int64_t)gridDim.x * blockDim.x;
    const int64_t warp = gtid >> 5;
    const int64_t nwarps = gsize >> 5;
    const int lane = lane_id();
    const bool split = le != nullptr;

    // ---- init
    const unsigned long long ib = (unsigned long long)__double_as_longlong(inf);
    for (int64_t v = gtid; v < n; v += gsize) {
        dist[v] = (v == src) ? 0ull : ib;
        near_stamp[v] = -1;
        far_stamp[v] = -1;
        if (split) r_stamp[v] = -1;
    }
    if (gtid == 0) {
        qa[0] = src;
        st->nq = 1;
        st->mode = kLight;
        st->round = 1;
        st->fmin = ~0ull;
        st->t_start = global_timer_ns();
    }
    if (!sp_barrier(st)) return;

    __shared__ unsigned long long s_fmin, s_exam;
    __shared__ int32_t s_state[9];
    __shared__ double s_thr, s_new_thr;
    volatile SsspRunState* vs = st;
    while (true) {
        if (threadIdx.x == 0) {
            s_state[0] = vs->mode;
            s_state[1] = vs->nq;
            s_state[2] = vs->nc;
            s_state[3] = vs->qsel;
            s_state[4] = vs->chunk_of;
            s_state[5] = vs->fsel;
            s_state[6] = vs->round;
            s_state[7] = vs->phase;
            s_state[8] = vs->epoch;
            s_thr = vs->thr;
            s_new_thr = vs->new_thr;
            s_fmin = ~0ull;
            s_exam = 0;
        }
        __syncthreads();
        const int32_t mode = s_state[0];
        if (mode == kDone) break;
        const int32_t nq = s_state[1], nc = s_state[2];
        const int32_t qsel = s_state[3], fsel = s_state[5];
        SpCtx c;
        c.rp = rp;
        c.le = le;
        c.col = col;
        c.wt = wt;
        c.dist = dist;
        c.near_stamp = near_stamp;
        c.far_stamp = far_stamp;
        c.r_stamp = r_stamp;
        c.R = R;
        c.q_next = qsel ? qa : qb;
        c.far_cur = fsel ? fb : fa;
        c.chunks = chunks;
        c.st = st;
        c.thr = s_thr;
        c.round = s_state[6];
        c.phase = s_state[7];
        c.epoch = s_state[8];
        unsigned long long exam = 0;

        if (mode == kChunk) {
            // The long rows of the pass just finished, a chunk per warp.
            for (int64_t i = warp; i < nc; i += nwarps) {
                const int4 ch = __ldcg(chunks + i);
                const double du = sp_dist(dist, ch.x);
                sp_warp_range(c, du, ch.y, ch.z, exam, &s_fmin);
            }
        } else if (mode == kLight || mode == kHeavy) {
            const int32_t* q = mode == kHeavy ? R : (qsel ? qb : qa);
            // Queue rows, 32 per warp.
            for (int64_t base = warp * 32; base < nq; base += nwarps * 32) {
                const int64_t i = base + lane;
                int32_t u = -1, b = 0, e = 0;
                double du = 0.0;
                if (i < nq) {
                    u = q[i];
                    du = sp_dist(dist, u);
                    if (mode == kLight) {
                        b = rp[u];
                        e = split ? le[u] : rp[u + 1];
                        if (split && atomicExch(r_stamp + u, c.epoch) != c.epoch)
                            R[warp_append_active(&st->r_tail)] = u;
                    } else {
                        b = le[u];
                        e = rp[u + 1];
                    }
                }
                sp_rows(c, u, b, e, du, exam, &s_fmin);
            }
        } else {  // kSplit
            const int32_t* far = fsel ? fb : fa;
            int32_t* kept = fsel ? fa : fb;
            const double old_thr = s_thr, nthr = s_new_thr;
            const int32_t next_phase = c.phase;  // already advanced by the leader
            for (int64_t i = gtid; i < nq; i += gsize) {
                const int32_t v = far[i];
                const double d = sp_dist(dist, v);
                if (d < old_thr) continue;  // settled in an earlier bucket
                if (d < nthr) {
                    if (atomicExch(near_stamp + v, c.round) != c.round) c.q_next[warp_append_active(&st->q_tail)] = v;
                } else {
                    if (atomicExch(far_stamp + v, next_phase) != next_phase)
                        kept[warp_append_active(&st->kept_tail)] = v;
                    atomicMin(&s_fmin, (unsigned long long)__double_as_longlong(d));
                }
            }
        }
        // Block totals, then the barrier whose last arrival decides.
        exam = warp_sum(exam);
        if (lane == 0 && exam) atomicAdd(&s_exam, exam);
        __syncthreads();
        if (threadIdx.x == 0) {
            if (s_exam) atomicAdd(&st->examined, s_exam);
            if (s_fmin != ~0ull) atomicMin(&st->fmin, s_fmin);
        }
        const bool ok = sp_barrier(st, [&]() {
            SsspRunState* s = st;
            volatile SsspRunState* v = st;
            const int32_t md0 = v->mode;
            s->passes = v->passes + 1;
            if ((md0 == kLight || md0 == kHeavy) && v->c_tail > 0) {
                // Long rows were cut into chunks: a CHUNK pass finishes them
                // in the same round (same stamps, same next queue).
                s->nc = v->c_tail;
                s->c_tail = 0;
                s->chunk_of = md0;
                s->mode = kChunk;
                return;
            }
            if (md0 == kChunk) s->chunk_passes = v->chunk_passes + 1;
            const int32_t md = md0 == kChunk ? v->chunk_of : md0;
            const int32_t nq_next = v->q_tail;
            s->q_tail = 0;
            s->c_tail = 0;
            s->qsel = v->qsel ^ 1;
            s->nq = nq_next;
            s->nc = 0;
            if (md == kSplit) {
                s->far_tail = v->kept_tail;
                s->kept_tail = 0;
                s->fsel = v->fsel ^ 1;
                s->thr = v->new_thr;
                s->splits = v->splits + 1;
            } else if (md == kHeavy) {
                s->r_tail = 0;
                s->epoch = v->epoch + 1;
                s->heavy_passes = v->heavy_passes + 1;
            } else {
                s->light_passes = v->light_passes + 1;
            }
            int32_t next = kDone;
            if (nq_next > 0) {
                next = kLight;
            } else if (md == kLight && v->r_tail > 0) {
                next = kHeavy;
                s->nq = v->r_tail;
            } else if (v->far_tail > 0) {
                // Next bucket: the one holding the smallest pending far
                // distance (its recorded minimum can be low when an entry
                // settled later; a SPLIT that queues nothing then repeats
                // with the exact minimum of the entries it kept).
                const unsigned long long fb_ = v->fmin;
                const double thr = v->thr;
                // The next bucket's width: halved after a bucket that took
                // more than kSpAdaptLight LIGHT passes (its vertices were
                // relaxed again and again), doubled after one that took at
                // most two and examined little (passes with too little work
                // for the grid).  Exact distances do not depend on it: the
                // passes form a label-correcting loop in which a HEAVY pass
                // that lowers a distance inside the bucket sends it back to
                // a LIGHT pass, and R is refilled after every HEAVY pass.
                double width = v->width;
                const long long lp = v->light_passes - v->lp_mark;
                const unsigned long long ex = v->examined - v->ex_mark;
                if (lp > kSpAdaptLight) width = fmax(width * 0.5, v->width_min);
                else if (lp <= 2 && ex < v->adapt_work) width = fmin(width * 2.0, v->width_max);
                s->width = width;
                s->lp_mark = v->light_passes;
                s->ex_mark = v->examined;
                const double mn = fb_ == ~0ull ? thr : __longlong_as_double((long long)fb_);
                s->new_thr = sp_next_thr(thr, width, mn);
                s->fmin = ~0ull;
                s->nq = v->far_tail;
                s->phase = v->phase + 1;
                next = kSplit;
            }
            s->round = v->round + 1;
            // Budgets: a correct run needs far fewer passes and far less
            // time; past either, stop with an error status.
            if (next != kDone &&
                (v->passes > v->pass_budget || global_timer_ns() - v->t_start > kSsspTimeBudgetNs)) {
                s->status = kDevOverflow;
                next = kDone;
            }
            s->mode = next;
        });
        if (!ok) return;
    }

    // ---- results in the caller's ids
    if (perm) {
        for (int64_t v = gtid; v < n; v += gsize) out[v] = sp_dist(dist, perm[v]);
    }
}

// ------------------------------------------------------------------- host
namespace {

__global__ void sp_light_end_kernel(int32_t n, const int32_t* __restrict__ rp, const double* __restrict__ sw_w,
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

__global__ void sp_reached_kernel(int32_t n, const int32_t* __restrict__ rp, const double* __restrict__ dist,
                                  double inf, unsigned long long* out) {
    unsigned long long e = 0, r = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
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

}  // namespace

bool sssp_persistent_available(ghb_workspace* ws, int* blocks) {
    static int cached[64] = {0};
    static bool known[64] = {false};
    const int dev = ws->device;
    if (dev < 0 || dev >= 64) return false;
    if (!known[dev]) {
        int coop = 0, per_sm = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        if (coop && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sssp_persistent_kernel, kSsspThreads, 0) ==
                        cudaSuccess)
            cached[dev] = std::min(per_sm, 2) * ws->num_sms;
        known[dev] = true;
    }
    *blocks = cached[dev];
    return cached[dev] > 0;
}

// Light ends of a resident graph's weight-sorted rows for width delta,
// cached on the handle until a call asks for another width.
int graph_light_ends(ghb_workspace* ws, ghb_graph* g, double delta, const int32_t** le) {
    if (!g->sw_le) {
        GHB_CUDA_TRY(cudaMalloc(&g->sw_le, sizeof(int32_t) * (size_t)g->n));
        g->device_bytes += 4 * (int64_t)g->n;
        g->sw_le_delta = -1.0;
    }
    if (g->sw_le_delta != delta) {
        GHB_TRY(launch(ws, sp_light_end_kernel, dim3(grid_for(g->n, 256, ws->num_sms * 8)), dim3(256), 0, g->n,
                       (const int32_t*)g->rowptr, (const double*)g->sw_w, delta, g->sw_le));
        g->sw_le_delta = delta;
    }
    *le = g->sw_le;
    return GHB_OK;
}

// One cooperative launch for the whole traversal.  rp/col/wt: the rows to
// relax (a resident graph's weight-sorted copy when le is given, whose
// light ranges [rp[u], le[u]) hold the entries below delta).  dist: per
// vertex in the graph's ids; with perm, out[v] = dist[perm[v]] as well.
int sssp_persistent_run(ghb_workspace* ws, int32_t n, const int32_t* rp, const int32_t* le, const int32_t* col,
                        const double* wt, int32_t src, double inf, double delta, double* dist, const int32_t* perm,
                        double* out, ghb_traversal_stats* stats) {
    int blocks = 0;
    if (!sssp_persistent_available(ws, &blocks)) {
        set_error("cooperative launch unavailable");
        return GHB_ERR_UNSUPPORTED;
    }
    cudaStream_t st = ws->stream;
    int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned);
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, rp + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t m = hp[0];
    // Chunks of one pass: rows over kSpDirect entries, ceil(len / kSpChunk)
    // each, so fewer than m / kSpChunk + m / kSpDirect.
    const int64_t chunk_cap = m / 32 + 64;
    auto carve = [&](Carver& c, int32_t** qa, int32_t** qb, int4** ch, int32_t** fa, int32_t** fb,
                     int32_t** ns, int32_t** fs, int32_t** rs, int32_t** R, SsspRunState** rs_state) {
        *qa = c.take<int32_t>(n);
        *qb = c.take<int32_t>(n);
        *ch = c.take<int4>(chunk_cap);
        *fa = c.take<int32_t>(n);
        *fb = c.take<int32_t>(n);
        *ns = c.take<int32_t>(n);
        *fs = c.take<int32_t>(n);
        *rs = c.take<int32_t>(le ? n : 1);
        *R = c.take<int32_t>(le ? n : 1);
        *rs_state = c.take<SsspRunState>(1);
    };
    int32_t *qa, *qb, *fa, *fb, *ns, *fs, *rs, *R;
    int4* ch;
    SsspRunState* rstate;
    Carver sizing(nullptr);
    carve(sizing, &qa, &qb, &ch, &fa, &fb, &ns, &fs, &rs, &R, &rstate);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &qa, &qb, &ch, &fa, &fb, &ns, &fs, &rs, &R, &rstate);

    GHB_CUDA_TRY(cudaMemsetAsync(rstate, 0, sizeof(SsspRunState), st));
    {
        // thr, delta, then the barrier limit and test knob (pageable
        // sources: the copies stage them before returning).
        const double td[2] = {delta, delta};
        GHB_CUDA_TRY(cudaMemcpyAsync(&rstate->thr, td, sizeof(double), cudaMemcpyHostToDevice, st));
        GHB_CUDA_TRY(cudaMemcpyAsync(&rstate->delta, td + 1, sizeof(double), cudaMemcpyHostToDevice, st));
        const unsigned long long bar[2] = {(unsigned long long)ws->tune.barrier_limit_us * 1000ull,
                                           (unsigned long long)ws->tune.barrier_extra};
        GHB_CUDA_TRY(cudaMemcpyAsync(&rstate->bar_limit_ns, bar, sizeof(bar), cudaMemcpyHostToDevice, st));
        // Every productive pass lowers some distance: 64 passes per vertex
        // bound any correct run, as in the host-driven loop.
        const long long budget = 64ll * n + 1024;
        GHB_CUDA_TRY(cudaMemcpyAsync(&rstate->pass_budget, &budget, sizeof(budget), cudaMemcpyHostToDevice, st));
        // Bucket widths: delta, or from delta / 64 to delta * 64 when they
        // adapt; a bucket is small below eight entries per thread.
        const bool adapt = ws->tune.sssp_adapt != 0;
        const double wd[3] = {delta, adapt ? delta / 64.0 : delta, adapt ? delta * 64.0 : delta};
        GHB_CUDA_TRY(cudaMemcpyAsync(&rstate->width, wd, sizeof(wd), cudaMemcpyHostToDevice, st));
        const unsigned long long work = 8ull * (unsigned long long)blocks * kSsspThreads;
        GHB_CUDA_TRY(cudaMemcpyAsync(&rstate->adapt_work, &work, sizeof(work), cudaMemcpyHostToDevice, st));
    }
    if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
    GHB_TRY(launch_coop(ws, sssp_persistent_kernel, dim3(blocks), dim3(kSsspThreads), 0, n, rp, le, col, wt, src, inf,
                        dist, qa, qb, ch, fa, fb, ns, fs, rs, R, rstate, perm, out));
    if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_stop, st));
    GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, rstate, sizeof(SsspRunState), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    SsspRunState h;
    std::memcpy(&h, ws->host_pinned, sizeof(h));
    if (h.status == kDevOverflow) {
        set_error("SSSP: pass or time budget exhausted");
        return GHB_ERR_LIMIT;
    }
    if (h.status != kDevOk) {
        set_error("SSSP: grid barrier timed out");
        return GHB_ERR_TIMEOUT;
    }
    if (stats) {
        unsigned long long* acc = reinterpret_cast<unsigned long long*>(ws->dev_small);
        GHB_CUDA_TRY(cudaMemsetAsync(acc, 0, 2 * sizeof(unsigned long long), st));
        GHB_TRY(launch(ws, sp_reached_kernel, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0, n, rp,
                       (const double*)dist, inf, acc));
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, acc, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                     st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        float ms = 0.f;
        GHB_CUDA_TRY(cudaEventElapsedTime(&ms, ws->ev_start, ws->ev_stop));
        const unsigned long long* ha = reinterpret_cast<const unsigned long long*>(ws->host_pinned);
        stats->levels = (int32_t)(h.light_passes + h.heavy_passes + h.chunk_passes);
        stats->pull_levels = (int32_t)h.splits;
        stats->edges_reached = (int64_t)ha[0];
        stats->reached = (int64_t)ha[1];
        stats->edges_examined = (int64_t)h.examined;
        stats->device_ms = ms;
    }
    return GHB_OK;
}

}  // namespace ghb
