// Multi-source SSSP: up to 256 sources in one bucketed traversal (no
// counterpart in the reference, which runs one source per call,
// GPU_SSSP_csr.cuh:253-327).  Results equal n_src single-source runs bit for
// bit: every source's distances are the least fixpoint of
// d[v] = min_u fl(d[u] + w(u, v)), which any relaxation order reaches.
//
// Layout: dist is vertex-major, dist[v * KS + s] (KS = the pass's source
// count rounded up to 32), so one warp reads or relaxes 32 sources of a
// vertex with one 256-byte access.  act[v] holds W = ceil(KS / 64) words of
// "source s must relax v's edges in this round" bits.
//
// All sources move through the same buckets [lo, lo + delta):
//   scan   a warp per vertex reads its KS distances and sets the act bits of
//          those in [lo, hi) (the bucket's start set), queueing the vertex;
//          it also keeps the smallest distance at or above hi (to skip empty
//          buckets);
//   round  every queued vertex relaxes its out-edges for its active sources:
//          a warp per vertex (rows up to kMsspWarpRow entries) or per
//          256-entry chunk of a longer row (chunk table built per round);
//          lanes run over the sources when at least 4 are active (all 32
//          lanes of the warp relax one edge for 32 sources), over the edges
//          otherwise.  An improved distance below hi activates the target
//          for the next round; one at or above hi waits for its bucket's
//          scan.  Rounds repeat until no vertex is queued, then the next
//          bucket is scanned.
// Output: dist_out[s * n + v] in the caller's ids (perm maps them), with
// `inf` for unreached vertices.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "graph.cuh"
#include "scan.cuh"

namespace ghb {
namespace {

constexpr int32_t kMsspWarpRow = 1024;
constexpr int32_t kMsspChunk = 256;
constexpr unsigned long long kInfBits = 0x7ff0000000000000ull;  // +infinity

struct MsspCounters {
    int32_t queued;       // vertices queued for the next round
    int32_t big;          // rows of the current round handed to the chunk kernel
    unsigned long long pmin;     // smallest pending distance (bits) at or above hi
    unsigned long long examined; // entries relaxed
};

// Each phase is a __device__ body (grid-stride) with a thin kernel around
// it: the host-driven pass launches the kernels, the whole-pass cooperative
// kernel (mssp_pass_kernel) calls the bodies between its grid barriers.
__device__ __forceinline__ void mssp_fill_body(unsigned long long* d, int64_t count, unsigned long long v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = v;
}
__global__ void mssp_fill_kernel(unsigned long long* d, int64_t count, unsigned long long v) {
    mssp_fill_body(d, count, v);
}

__global__ void mssp_seed_kernel(const int32_t* __restrict__ srcs, int32_t k, int32_t ks, unsigned long long* d) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < k) d[(int64_t)srcs[s] * ks + s] = 0ull;  // +0.0
}

// Bucket start: act bits of the distances in [lo, hi), queue, pending min.
__device__ __forceinline__ void mssp_scan_body(int32_t n_scan, int32_t ks, int32_t words, double lo, double hi,
                                               const unsigned long long* d, unsigned long long* act, int32_t* queue,
                                               MsspCounters* cnt) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    double pmin = INFINITY;
    for (int64_t v = warp; v < n_scan; v += nwarps) {
        bool any = false;
        for (int w = 0; w < words; ++w) {
            unsigned long long word = 0;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int s = w * 64 + h * 32 + lane;
                double x = INFINITY;
                if (s < ks) x = __longlong_as_double((long long)__ldcg(d + v * ks + s));
                const bool in = x >= lo && x < hi;
                if (x >= hi && x < pmin) pmin = x;
                word |= (unsigned long long)__ballot_sync(0xffffffffu, in) << (32 * h);
            }
            if (lane == 0) act[v * words + w] = word;
            any |= word != 0;
        }
        if (any && lane == 0) queue[atomicAdd(&cnt->queued, 1)] = (int32_t)v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pmin = fmin(pmin, __shfl_xor_sync(0xffffffffu, pmin, o));
    if (lane == 0 && pmin < INFINITY)
        atomicMin(&cnt->pmin, (unsigned long long)__double_as_longlong(pmin));
}
__global__ void __launch_bounds__(256) mssp_scan_kernel(int32_t n_scan, int32_t ks, int32_t words, double lo,
                                                        double hi, const unsigned long long* d,
                                                        unsigned long long* act, int32_t* queue,
                                                        MsspCounters* cnt) {
    mssp_scan_body(n_scan, ks, words, lo, hi, d, act, queue, cnt);
}

// Relax entries [eb, ee) of v's row for v's active sources.
__device__ __forceinline__ void mssp_relax_range(int32_t v, int32_t eb, int32_t ee, int32_t ks, int32_t words,
                                                 double hi, const int32_t* __restrict__ col,
                                                 const double* __restrict__ wt, unsigned long long* d,
                                                 const unsigned long long* act_cur,
                                                 unsigned long long* act_next, int32_t* inq_next,
                                                 int32_t* queue_next, MsspCounters* cnt,
                                                 unsigned long long& examined) {
    const int lane = lane_id();
    int nact = 0;
    for (int w = 0; w < words; ++w) nact += __popcll(__ldcg(act_cur + (int64_t)v * words + w));
    auto relax_one = [&](int32_t u, int s, double nd) {
        unsigned long long* p = d + (int64_t)u * ks + s;
        const unsigned long long nb = (unsigned long long)__double_as_longlong(nd);
        if (nb < __ldcg(p)) {
            const unsigned long long old = atomicMin(p, nb);
            if (nb < old && nd < hi) {
                atomicOr(act_next + (int64_t)u * words + (s >> 6), 1ull << (s & 63));
                if (atomicExch(inq_next + u, 1) == 0) queue_next[warp_append_active(&cnt->queued)] = u;
            }
        }
    };
    if (nact >= 4) {
        // Lanes over sources: lane handles s = lane + 32 t, t < ks / 32; the
        // row's entries are read once and relaxed for every group.
        const int groups = ks >> 5;
        double dv[8];
        bool a[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int s = lane + 32 * t;
            a[t] = t < groups && ((__ldcg(act_cur + (int64_t)v * words + (s >> 6)) >> (s & 63)) & 1ull);
            dv[t] = a[t] ? __longlong_as_double((long long)__ldcg(d + (int64_t)v * ks + s)) : 0.0;
        }
        for (int32_t j = eb; j < ee; ++j) {
            const int32_t u = col[j];
            const double w = wt[j];
#pragma unroll
            for (int t = 0; t < 8; ++t)
                if (a[t]) relax_one(u, lane + 32 * t, dv[t] + w);
        }
        if (lane == 0) examined += (unsigned long long)(ee - eb) * (unsigned long long)nact;
    } else {
        // Lanes over entries, the few active sources one after another.
        for (int w = 0; w < words; ++w) {
            unsigned long long bits = __ldcg(act_cur + (int64_t)v * words + w);
            while (bits) {
                const int s = w * 64 + __ffsll((long long)bits) - 1;
                bits &= bits - 1;
                const double dv = __longlong_as_double((long long)__ldcg(d + (int64_t)v * ks + s));
                for (int32_t j = eb + lane; j < ee; j += 32) relax_one(col[j], s, dv + wt[j]);
                if (lane == 0) examined += (unsigned long long)(ee - eb);
            }
        }
    }
}

// A warp per queued vertex; rows longer than kMsspWarpRow go to `big`.
__global__ void __launch_bounds__(256) mssp_relax_kernel(int32_t q, const int32_t* __restrict__ queue,
                                                         const int32_t* __restrict__ rp,
                                                         const int32_t* __restrict__ col,
                                                         const double* __restrict__ wt, int32_t ks, int32_t words,
                                                         double hi, unsigned long long* d,
                                                         const unsigned long long* __restrict__ act_cur,
                                                         unsigned long long* act_next, int32_t* inq_next,
                                                         int32_t* queue_next, int32_t* big, MsspCounters* cnt,
                                                         MsspCounters* cnt_cur) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long examined = 0;
    for (int64_t i = warp; i < q; i += nwarps) {
        const int32_t v = queue[i];
        const int32_t eb = rp[v], ee = rp[v + 1];
        if (ee - eb > kMsspWarpRow) {
            if (lane_id() == 0) big[atomicAdd(&cnt_cur->big, 1)] = v;
            continue;
        }
        mssp_relax_range(v, eb, ee, ks, words, hi, col, wt, d, act_cur, act_next, inq_next, queue_next, cnt,
                         examined);
    }
    if (lane_id() == 0 && examined) atomicAdd(&cnt->examined, examined);
}

// Chunk counts of the long rows.
__global__ void mssp_big_chunks_kernel(const int32_t* __restrict__ big, const MsspCounters* cnt_cur,
                                       const int32_t* __restrict__ rp, int32_t* nch) {
    const int32_t nb = cnt_cur->big;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nb; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = big[i];
        nch[i] = (rp[v + 1] - rp[v] + kMsspChunk - 1) / kMsspChunk;
    }
}

// A warp per 256-entry chunk of the long rows (row by binary search).
__global__ void __launch_bounds__(256) mssp_relax_big_kernel(const int32_t* __restrict__ big,
                                                             const int32_t* __restrict__ cpre,
                                                             const MsspCounters* cnt_cur,
                                                             const int32_t* __restrict__ rp,
                                                             const int32_t* __restrict__ col,
                                                             const double* __restrict__ wt, int32_t ks,
                                                             int32_t words, double hi, unsigned long long* d,
                                                             const unsigned long long* __restrict__ act_cur,
                                                             unsigned long long* act_next, int32_t* inq_next,
                                                             int32_t* queue_next, MsspCounters* cnt) {
    const int32_t nb = cnt_cur->big;
    if (nb == 0) return;
    const int32_t total = cpre[nb];
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long examined = 0;
    for (int64_t c = warp; c < total; c += nwarps) {
        int32_t lo = 0, hi_i = nb - 1;
        while (lo < hi_i) {
            const int32_t mid = (lo + hi_i + 1) >> 1;
            if (cpre[mid] <= c) lo = mid;
            else hi_i = mid - 1;
        }
        const int32_t v = big[lo];
        const int32_t eb = rp[v] + (int32_t)(c - cpre[lo]) * kMsspChunk;
        const int32_t ee = min(rp[v + 1], eb + kMsspChunk);
        mssp_relax_range(v, eb, ee, ks, words, hi, col, wt, d, act_cur, act_next, inq_next, queue_next, cnt,
                         examined);
    }
    if (lane_id() == 0 && examined) atomicAdd(&cnt->examined, examined);
}

// After a round: the processed vertices' act words and queue flags are cleared.
__global__ void mssp_clear_kernel(int32_t q, const int32_t* __restrict__ queue, int32_t words,
                                  unsigned long long* act, int32_t* inq) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < q; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = queue[i];
        for (int w = 0; w < words; ++w) act[(int64_t)v * words + w] = 0ull;
        inq[v] = 0;
    }
}

// ---------------------------------------------------------------------------
// The whole pass in one cooperative launch: set-up, every bucket scan and
// relaxation round (long rows as 256-entry chunks in a CHUNK phase of the
// same round, then the clear of the processed vertices' act words), the
// output, separated by the bounded grid barrier; the last block to arrive
// decides the next phase (the host-driven pass's rules: rounds until the
// queue is empty, then the next bucket, empty buckets skipped through the
// smallest pending distance).  No host round trip inside a pass.

constexpr int kMsspThreads = 256;
enum MsspPhase : int32_t { kMpScan = 0, kMpRelax = 1, kMpChunks = 2, kMpClear = 3, kMpDone = 4 };

struct MsspRunState {
    unsigned bar_count;  // barrier arrivals (own cache line)
    unsigned pad_a[31];
    unsigned bar_release;  // barrier epochs (own cache line)
    unsigned pad_b[31];
    int32_t status;
    int32_t phase;     // MsspPhase of the next phase
    int32_t sel;       // which (act, inq, queue) set is current (0: a)
    int32_t q;         // vertices queued for the current round
    int32_t nchunks;   // long-row chunks of the current round
    int32_t c_tail;    // chunks appended by the relax phase
    int32_t pad0, pad1;
    double lo;         // current bucket [lo, lo + delta)
    double delta;
    long long rounds, budget;
    unsigned long long examined;
};

__device__ __forceinline__ double mp_pmin(const MsspCounters* c) {
    const unsigned long long b = *(volatile const unsigned long long*)&c->pmin;
    return b == kInfBits ? INFINITY : __longlong_as_double((long long)b);
}

// Eight blocks per SM, every thread slot of the SM (32 registers, a
// 148-byte spill): 256 sources on RMAT-22 in 1.08 s, against 1.30-1.34 s at
// six blocks per SM (40 registers) and 1.66 s at four (64 registers).  The
// pass waits on its gathers and atomics, so resident warps pay for the
// spill.
__global__ void __launch_bounds__(kMsspThreads, 8) mssp_pass_kernel(
    int32_t n, int32_t n_active, int32_t k, int32_t ks, int32_t words, const int32_t* __restrict__ rp,
    const int32_t* __restrict__ col, const double* __restrict__ wt, const int32_t* srcs, const int32_t* __restrict__ perm,
    double inf, double* dist_out, unsigned long long* d, unsigned long long* act_a, unsigned long long* act_b,
    int32_t* inq_a, int32_t* inq_b, int32_t* q_a, int32_t* q_b, int4* chunks, MsspCounters* cnt, MsspRunState* st,
    unsigned long long bar_limit_ns, unsigned bar_extra) {
    const int64_t gtid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t gsize = (int64_t)gridDim.x * blockDim.x;
    const int64_t warp = gtid >> 5;
    const int64_t nwarps = gsize >> 5;
    const int lane = lane_id();
    auto barrier = [&]() {
        return grid_sync_leader(&st->bar_count, &st->bar_release, &st->status, NoLeader(), bar_limit_ns, bar_extra);
    };
    // ---- set-up: distances +inf, act / inq words zero, the sources at 0
    mssp_fill_body(d, (int64_t)n * ks, kInfBits);
    for (int64_t i = gtid; i < (int64_t)n * words; i += gsize) {
        act_a[i] = 0ull;
        act_b[i] = 0ull;
    }
    for (int64_t i = gtid; i < n; i += gsize) {
        inq_a[i] = 0;
        inq_b[i] = 0;
    }
    if (gtid == 0) {
        cnt->queued = 0;
        cnt->big = 0;
        cnt->pmin = kInfBits;
        cnt->examined = 0;
    }
    if (!barrier()) return;
    if (blockIdx.x == 0 && (int)threadIdx.x < k) d[(int64_t)srcs[threadIdx.x] * ks + threadIdx.x] = 0ull;
    if (!barrier()) return;

    __shared__ int32_t s_st[4];
    __shared__ double s_lo;
    while (true) {
        if (threadIdx.x == 0) {
            volatile MsspRunState* v = st;
            s_st[0] = v->phase;
            s_st[1] = v->sel;
            s_st[2] = v->q;
            s_st[3] = v->nchunks;
            s_lo = v->lo;
        }
        __syncthreads();
        const int32_t phase = s_st[0];
        if (phase == kMpDone) break;
        const int32_t sel = s_st[1], q = s_st[2], nch = s_st[3];
        unsigned long long* act_cur = sel ? act_b : act_a;
        unsigned long long* act_next = sel ? act_a : act_b;
        int32_t* inq_cur = sel ? inq_b : inq_a;
        int32_t* inq_next = sel ? inq_a : inq_b;
        int32_t* q_cur = sel ? q_b : q_a;
        int32_t* q_next = sel ? q_a : q_b;
        MsspCounters* cn = cnt;  // the round being filled
        const double lo = s_lo, hi = lo + st->delta;
        unsigned long long examined = 0;
        if (phase == kMpScan) {
            mssp_scan_body(n_active, ks, words, lo, hi, d, act_cur, q_cur, cn);
        } else if (phase == kMpRelax) {
            for (int64_t i = warp; i < q; i += nwarps) {
                const int32_t v = __ldcg(q_cur + i);
                const int32_t eb = rp[v], ee = rp[v + 1];
                if (ee - eb > kMsspWarpRow) {
                    const int32_t nc = (ee - eb + kMsspChunk - 1) / kMsspChunk;
                    int32_t pos = 0;
                    if (lane == 0) pos = atomicAdd(&st->c_tail, nc);
                    pos = __shfl_sync(0xffffffffu, pos, 0);
                    for (int32_t c = lane; c < nc; c += 32)
                        chunks[pos + c] = make_int4(v, eb + c * kMsspChunk, min(ee, eb + (c + 1) * kMsspChunk), 0);
                    continue;
                }
                mssp_relax_range(v, eb, ee, ks, words, hi, col, wt, d, act_cur, act_next, inq_next, q_next, cn,
                                 examined);
            }
        } else if (phase == kMpChunks) {
            for (int64_t i = warp; i < nch; i += nwarps) {
                const int4 ch = __ldcg(chunks + i);
                mssp_relax_range(ch.x, ch.y, ch.z, ks, words, hi, col, wt, d, act_cur, act_next, inq_next, q_next,
                                 cn, examined);
            }
        } else {  // kMpClear: the processed vertices' act words and queue flags
            for (int64_t i = gtid; i < q; i += gsize) {
                const int32_t v = __ldcg(q_cur + i);
                for (int w = 0; w < words; ++w) act_cur[(int64_t)v * words + w] = 0ull;
                inq_cur[v] = 0;
            }
        }
        if (lane == 0 && examined) atomicAdd(&cn->examined, examined);
        const bool ok = grid_sync_leader(
            &st->bar_count, &st->bar_release, &st->status,
            [&]() {
                MsspRunState* s = st;
                volatile MsspRunState* v = st;
                volatile MsspCounters* c = cnt;
                int32_t next = kMpDone;
                if (phase == kMpRelax && v->c_tail > 0) {
                    s->nchunks = v->c_tail;
                    s->c_tail = 0;
                    next = kMpChunks;
                } else if (phase == kMpRelax || phase == kMpChunks) {
                    next = kMpClear;
                } else {
                    // After a scan or a clear: the queue just filled decides.
                    int32_t queued;
                    if (phase == kMpClear) {
                        s->examined = v->examined + c->examined;
                        queued = c->queued;  // the next round's queue (q_next)
                        s->sel = v->sel ^ 1;
                    } else {
                        queued = c->queued;  // the bucket's start set (q_cur)
                    }
                    const double pmin = mp_pmin(cnt);
                    c->queued = 0;
                    c->examined = 0;
                    c->pmin = kInfBits;
                    if (queued > 0) {
                        s->q = queued;
                        s->rounds = v->rounds + 1;
                        next = kMpRelax;
                        if (v->rounds + 1 > v->budget) {
                            s->status = kDevOverflow;
                            next = kMpDone;
                        }
                    } else if (phase == kMpClear) {
                        s->lo = v->lo + v->delta;  // next bucket
                        next = kMpScan;
                    } else {
                        // An empty bucket: jump to the one holding the
                        // smallest pending distance, or stop.
                        if (pmin < INFINITY) {
                            const double dl = v->delta;
                            double nlo = floor(pmin / dl) * dl;
                            if (nlo > pmin || nlo + dl <= pmin) nlo = pmin;  // rounding: the bucket must hold pmin
                            s->lo = nlo;
                            next = kMpScan;
                        }
                    }
                }
                s->phase = next;
            },
            bar_limit_ns, bar_extra);
        if (!ok) return;
    }
    // ---- output in the caller's ids
    for (int64_t v = gtid; v < n; v += gsize) {
        const int64_t p = perm ? perm[v] : v;
        for (int s = 0; s < k; ++s) {
            const unsigned long long b = __ldcg(d + p * ks + s);
            dist_out[(int64_t)s * n + v] = b == kInfBits ? inf : __longlong_as_double((long long)b);
        }
    }
}

// dist_out[s * n + v] = dist[perm[v] * ks + s] (inf where unreached).
__global__ void __launch_bounds__(256) mssp_out_kernel(int32_t n, int32_t k, int32_t ks,
                                                       const int32_t* __restrict__ perm,
                                                       const unsigned long long* __restrict__ d, double inf,
                                                       double* out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = perm ? perm[v] : v;
        for (int s = 0; s < k; ++s) {
            const unsigned long long b = d[p * ks + s];
            out[(int64_t)s * n + v] = b == kInfBits ? inf : __longlong_as_double((long long)b);
        }
    }
}

}  // namespace

// Bucket width of a pass: the caller's, else mean weight x 32 / mean degree
// (the single-source rule) times 4 (a pass has 256 sources' work per bucket,
// so fewer, fuller buckets pay).
int sssp_pick_delta(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const double* w, double* delta);

static int mssp_pass_blocks(ghb_workspace* ws) {
    static int cached[64] = {0};
    const int dev = ws->device;
    if (dev < 0 || dev >= 64) return 0;
    if (!cached[dev]) {
        int coop = 0, per_sm = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        if (coop && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mssp_pass_kernel, kMsspThreads, 0) ==
                        cudaSuccess)
            cached[dev] = std::max(0, std::min(per_sm, 8)) * ws->num_sms;
        if (!cached[dev]) cached[dev] = -1;
    }
    return cached[dev] > 0 ? cached[dev] : 0;
}

// One pass of k <= 256 sources as one cooperative launch (graph ids on the
// device in srcs_dev); the same results and the same bucket / round rules
// as mssssp_pass below.
int mssssp_pass_one_launch(ghb_workspace* ws, int32_t n, int32_t n_active, int64_t m, const int32_t* rp,
                           const int32_t* col, const double* wt, const int32_t* srcs_dev, int32_t k, double delta,
                           double inf, const int32_t* perm, double* dist_out, int64_t* rounds_out,
                           int64_t* examined_out) {
    GHB_REQUIRE(k >= 1 && k <= 256, "multi-source SSSP pass of 1..256 sources");
    GHB_REQUIRE(delta > 0 && std::isfinite(delta), "bucket width must be positive");
    const int blocks = mssp_pass_blocks(ws);
    if (blocks <= 0) {
        set_error("cooperative launch unavailable");
        return GHB_ERR_UNSUPPORTED;
    }
    cudaStream_t st = ws->stream;
    const int32_t ks = (k + 31) & ~31;
    const int32_t words = (ks + 63) / 64;
    // Chunks of one round: rows over kMsspWarpRow entries, ceil(len / 256) each.
    const int64_t chunk_cap = m / kMsspChunk + m / kMsspWarpRow + 64;
    auto carve = [&](Carver& c, unsigned long long** d, unsigned long long** aa, unsigned long long** ab,
                     int32_t** ia, int32_t** ib, int32_t** qa, int32_t** qb, int4** ch, MsspCounters** cnt,
                     MsspRunState** rs) {
        *d = c.take<unsigned long long>((size_t)n * ks);
        *aa = c.take<unsigned long long>((size_t)n * words);
        *ab = c.take<unsigned long long>((size_t)n * words);
        *ia = c.take<int32_t>(n);
        *ib = c.take<int32_t>(n);
        *qa = c.take<int32_t>(n);
        *qb = c.take<int32_t>(n);
        *ch = c.take<int4>(chunk_cap);
        *cnt = c.take<MsspCounters>(1);
        *rs = c.take<MsspRunState>(1);
    };
    unsigned long long *d, *act_a, *act_b;
    int32_t *inq_a, *inq_b, *q_a, *q_b;
    int4* ch;
    MsspCounters* cnt;
    MsspRunState* rs;
    Carver sizing(nullptr);
    carve(sizing, &d, &act_a, &act_b, &inq_a, &inq_b, &q_a, &q_b, &ch, &cnt, &rs);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &d, &act_a, &act_b, &inq_a, &inq_b, &q_a, &q_b, &ch, &cnt, &rs);
    GHB_CUDA_TRY(cudaMemsetAsync(rs, 0, sizeof(MsspRunState), st));
    {
        // Bucket width and round budget (pageable sources: staged by the copies).
        const double dl = delta;
        const long long budget = 64ll * n + 4096;
        GHB_CUDA_TRY(cudaMemcpyAsync(&rs->delta, &dl, sizeof(dl), cudaMemcpyHostToDevice, st));
        GHB_CUDA_TRY(cudaMemcpyAsync(&rs->budget, &budget, sizeof(budget), cudaMemcpyHostToDevice, st));
    }
    GHB_TRY(launch_coop(ws, mssp_pass_kernel, dim3(blocks), dim3(kMsspThreads), (size_t)0, n, n_active, k, ks, words,
                        rp, col, wt, srcs_dev, perm, inf, dist_out, d, act_a, act_b, inq_a, inq_b, q_a, q_b, ch, cnt,
                        rs, (unsigned long long)ws->tune.barrier_limit_us * 1000ull,
                        (unsigned)ws->tune.barrier_extra));
    GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, rs, sizeof(MsspRunState), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    MsspRunState h;
    std::memcpy(&h, ws->host_pinned, sizeof(h));
    if (h.status == kDevOverflow) {
        set_error("multi-source SSSP round budget exceeded");
        return GHB_ERR_LIMIT;
    }
    if (h.status != kDevOk) {
        set_error("multi-source SSSP: grid barrier timed out");
        return GHB_ERR_TIMEOUT;
    }
    if (rounds_out) *rounds_out += h.rounds;
    if (examined_out) *examined_out += (int64_t)h.examined;
    return GHB_OK;
}

// One pass of k <= 256 sources.  n_active: vertices [n_active, n) have no
// entries.  perm (may be NULL) maps output ids to graph ids.
int mssssp_pass(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* rp, const int32_t* col,
                const double* wt, const int32_t* srcs_dev, int32_t k, double delta, double inf,
                const int32_t* perm, double* dist_out, int64_t* rounds_out, int64_t* examined_out) {
    GHB_REQUIRE(k >= 1 && k <= 256, "multi-source SSSP pass of 1..256 sources");
    GHB_REQUIRE(delta > 0 && std::isfinite(delta), "bucket width must be positive");
    cudaStream_t st = ws->stream;
    const int32_t ks = (k + 31) & ~31;
    const int32_t words = (ks + 63) / 64;
    Carver sizing(nullptr);
    auto carve = [&](Carver& c, unsigned long long** d, unsigned long long** aa, unsigned long long** ab,
                     int32_t** ia, int32_t** ib, int32_t** qa, int32_t** qb, int32_t** big, int32_t** nch,
                     int32_t** cpre, int64_t** bs, MsspCounters** cnt) {
        *d = c.take<unsigned long long>((size_t)n * ks);
        *aa = c.take<unsigned long long>((size_t)n * words);
        *ab = c.take<unsigned long long>((size_t)n * words);
        *ia = c.take<int32_t>(n);
        *ib = c.take<int32_t>(n);
        *qa = c.take<int32_t>(n);
        *qb = c.take<int32_t>(n);
        *big = c.take<int32_t>(n);
        *nch = c.take<int32_t>((size_t)n + 1);
        *cpre = c.take<int32_t>((size_t)n + 1);
        *bs = c.take<int64_t>(scan_scratch_words(n));
        *cnt = c.take<MsspCounters>(2);
    };
    unsigned long long *d, *act_a, *act_b;
    int32_t *inq_a, *inq_b, *q_a, *q_b, *big, *nch, *cpre;
    int64_t* bs;
    MsspCounters* cnt;
    carve(sizing, &d, &act_a, &act_b, &inq_a, &inq_b, &q_a, &q_b, &big, &nch, &cpre, &bs, &cnt);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &d, &act_a, &act_b, &inq_a, &inq_b, &q_a, &q_b, &big, &nch, &cpre, &bs, &cnt);

    const unsigned g = ws->num_sms * 8;
    GHB_TRY(launch(ws, mssp_fill_kernel, dim3(grid_for((int64_t)n * ks, 256, g)), dim3(256), 0, d, (int64_t)n * ks,
                   kInfBits));
    GHB_CUDA_TRY(cudaMemsetAsync(act_a, 0, sizeof(unsigned long long) * (size_t)n * words, st));
    GHB_CUDA_TRY(cudaMemsetAsync(act_b, 0, sizeof(unsigned long long) * (size_t)n * words, st));
    GHB_CUDA_TRY(cudaMemsetAsync(inq_a, 0, sizeof(int32_t) * (size_t)n, st));
    GHB_CUDA_TRY(cudaMemsetAsync(inq_b, 0, sizeof(int32_t) * (size_t)n, st));
    GHB_TRY(launch(ws, mssp_seed_kernel, dim3((k + 255) / 256), dim3(256), 0, srcs_dev, k, ks, d));

    MsspCounters* cn = cnt;      // counters of the round being filled
    MsspCounters* cc = cnt + 1;  // counters of the round being processed (big-row count)
    const MsspCounters* hc = reinterpret_cast<const MsspCounters*>(ws->host_pinned);
    auto read_counters = [&]() -> int {
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, cn, sizeof(MsspCounters), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        return GHB_OK;
    };
    auto reset = [&](MsspCounters* p) -> int {
        const MsspCounters z{0, 0, kInfBits, 0ull};
        std::memcpy(reinterpret_cast<char*>(ws->host_pinned) + 512, &z, sizeof(z));
        GHB_CUDA_TRY(cudaMemcpyAsync(p, reinterpret_cast<char*>(ws->host_pinned) + 512, sizeof(z),
                                     cudaMemcpyHostToDevice, st));
        return GHB_OK;
    };
    // Scan for the bucket [lo, lo + delta) into (act_a, q_a).
    auto scan_bucket = [&](double lo, int32_t* q_count, double* pmin) -> int {
        GHB_TRY(reset(cn));
        GHB_TRY(launch(ws, mssp_scan_kernel, dim3(grid_for((int64_t)n_active * 32, 256, g)), dim3(256), 0, n_active,
                       ks, words, lo, lo + delta, (const unsigned long long*)d, act_a, q_a, cn));
        GHB_TRY(read_counters());
        *q_count = hc->queued;
        unsigned long long pb = hc->pmin;
        std::memcpy(pmin, &pb, sizeof(double));
        return GHB_OK;
    };

    int64_t rounds = 0, examined = 0;
    const int64_t round_budget = 64ll * n + 4096;
    double lo = 0.0;
    int32_t q = 0;
    double pmin = INFINITY;
    GHB_TRY(scan_bucket(lo, &q, &pmin));
    while (true) {
        while (q > 0) {
            GHB_REQUIRE(++rounds <= round_budget, "multi-source SSSP round budget exceeded");
            GHB_TRY(reset(cn));
            GHB_TRY(reset(cc));
            const double hi = lo + delta;
            GHB_TRY(launch(ws, mssp_relax_kernel, dim3(grid_for((int64_t)q * 32, 256, g)), dim3(256), 0, q,
                           (const int32_t*)q_a, rp, col, wt, ks, words, hi, d, (const unsigned long long*)act_a,
                           act_b, inq_b, q_b, big, cn, cc));
            GHB_TRY(launch(ws, mssp_big_chunks_kernel, dim3(grid_for(q, 256, g)), dim3(256), 0, (const int32_t*)big,
                           (const MsspCounters*)cc, rp, nch));
            // Exclusive prefix of the big rows' chunk counts (at most q rows).
            GHB_TRY(scan_exclusive_i32(ws, nch, cpre, q, bs));
            GHB_TRY(launch(ws, mssp_relax_big_kernel, dim3(g), dim3(256), 0, (const int32_t*)big, (const int32_t*)cpre,
                           (const MsspCounters*)cc, rp, col, wt, ks, words, hi, d, (const unsigned long long*)act_a,
                           act_b, inq_b, q_b, cn));
            GHB_TRY(launch(ws, mssp_clear_kernel, dim3(grid_for(q, 256, g)), dim3(256), 0, q, (const int32_t*)q_a,
                           words, act_a, inq_a));
            GHB_TRY(read_counters());
            examined += (int64_t)hc->examined;
            q = hc->queued;
            std::swap(act_a, act_b);
            std::swap(inq_a, inq_b);
            std::swap(q_a, q_b);
        }
        // Next bucket; skip empty ones through the smallest pending distance.
        lo += delta;
        GHB_TRY(scan_bucket(lo, &q, &pmin));
        if (q == 0) {
            if (!(pmin < INFINITY)) break;
            lo = std::floor(pmin / delta) * delta;
            if (lo > pmin || lo + delta <= pmin) lo = pmin;  // rounding: the bucket must hold pmin
            GHB_TRY(scan_bucket(lo, &q, &pmin));
            GHB_REQUIRE(q > 0, "multi-source SSSP: pending distance not found by its bucket");
        }
    }
    GHB_TRY(launch(ws, mssp_out_kernel, dim3(grid_for(n, 256, g)), dim3(256), 0, n, k, ks, perm,
                   (const unsigned long long*)d, inf, dist_out));
    if (rounds_out) *rounds_out += rounds;
    if (examined_out) *examined_out += examined;
    return GHB_OK;
}

int mssssp_run(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* rp, const int32_t* col,
               const double* wt, const int32_t* srcs_host, int32_t n_src, double delta, double inf,
               const int32_t* perm, double* dist, ghb_traversal_stats* stats) {
    cudaStream_t st = ws->stream;
    if (!(delta > 0)) {
        GHB_TRY(sssp_pick_delta(ws, n, rp, wt, &delta));
        delta = std::ldexp(delta, ws->tune.mssp_width_log2);
    }
    GHB_TRY(ws_reserve_stage(ws, sizeof(int32_t) * 256));
    int32_t* sdev = static_cast<int32_t*>(ws->stage);
    if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
    int64_t rounds = 0, examined = 0;
    int64_t m = 0;
    const bool one_launch = ws->tune.mssp_persistent && mssp_pass_blocks(ws) > 0;
    if (one_launch) {
        int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned);
        GHB_CUDA_TRY(cudaMemcpyAsync(hp, rp + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        m = hp[0];
    }
    for (int32_t s0 = 0; s0 < n_src; s0 += 256) {
        const int32_t k = std::min<int32_t>(256, n_src - s0);
        GHB_CUDA_TRY(cudaMemcpyAsync(sdev, srcs_host + s0, sizeof(int32_t) * k, cudaMemcpyHostToDevice, st));
        if (one_launch)
            GHB_TRY(mssssp_pass_one_launch(ws, n, n_active, m, rp, col, wt, sdev, k, delta, inf, perm,
                                           dist + (int64_t)s0 * n, &rounds, &examined));
        else
            GHB_TRY(mssssp_pass(ws, n, n_active, rp, col, wt, sdev, k, delta, inf, perm, dist + (int64_t)s0 * n,
                                &rounds, &examined));
    }
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    if (stats) {
        GHB_CUDA_TRY(cudaEventRecord(ws->ev_stop, st));
        GHB_CUDA_TRY(cudaEventSynchronize(ws->ev_stop));
        float ms = 0.f;
        GHB_CUDA_TRY(cudaEventElapsedTime(&ms, ws->ev_start, ws->ev_stop));
        stats->levels = (int32_t)std::min<int64_t>(rounds, INT32_MAX);
        stats->pull_levels = 0;
        stats->reached = -1;
        stats->edges_reached = -1;
        stats->edges_examined = examined;
        stats->device_ms = ms;
    }
    return GHB_OK;
}

}  // namespace ghb
