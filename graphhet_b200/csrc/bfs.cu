// Single-source BFS: direction-optimising (top-down push over a vertex queue,
// bottom-up pull over a frontier bitmap), replacing the reference's
// expand/contract queue BFS (GPU_BFS_csr.cuh:15-327) and its push/pull
// variant (GPU_BFS_pre_csr.cuh:18-124).  Output semantics follow the CPU
// oracle (CPU_BFS.hpp:10-41): depth[v] = hop distance from src, INT32_MAX when
// unreached or deeper than max_depth.
//
// Layout in HBM: depth int32[n] (the output, written once per vertex); a
// visited bitmap and two frontier bitmaps of ceil(n/32) words (L2 resident:
// 2 MiB each at n = 2^24); two int32[n] vertex queues.
#include <cmath>
#include <vector>

#include "bfs_kernels.cuh"
#include "common.cuh"
#include "policy.cuh"

namespace ghb {

bool bfs_persistent_available(ghb_workspace* ws, int* blocks);

// The whole traversal runs in one cooperative launch (the learned policy's
// network included) unless the caller asks for per-level push/pull timings
// (oracle_timing), or the device cannot launch cooperatively.
bool bfs_use_persistent(ghb_workspace* ws, const ghb_bfs_options* opt) {
    int blocks = 0;
    if (!bfs_persistent_available(ws, &blocks)) return false;
    if (!opt) return true;
    if (opt->oracle_timing) return false;
    if (opt->record_trace && opt->trace_cap < 0) return false;
    return opt->policy == GHB_POLICY_HEURISTIC || opt->policy == GHB_POLICY_PUSH || opt->policy == GHB_POLICY_PULL ||
           opt->policy == GHB_POLICY_SCHEDULE || opt->policy == GHB_POLICY_LEARNED;
}

// n_active: vertices [n_active, n) have no entries at all (a relabelled
// graph puts them last); bottom-up levels skip them.
int bfs_run(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* out_rowptr, const int32_t* out_col,
            const int32_t* in_rowptr, const int32_t* in_col, int32_t src, int32_t max_depth,
            int32_t* depth, const ghb_bfs_options* opt, ghb_traversal_stats* stats) {
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(n_active >= 0 && n_active <= n, "n_active outside [0, n]");
    GHB_REQUIRE(out_rowptr && depth, "NULL graph or output");
    GHB_REQUIRE(src >= 0 && src < n, "source outside [0, n)");
    GHB_REQUIRE(max_depth >= 0, "max_depth < 0");
    ghb_bfs_options defaults = {};
    if (!opt) opt = &defaults;
    const bool can_pull = in_rowptr != nullptr && in_col != nullptr;
    int policy = opt->policy;
    if ((policy == GHB_POLICY_PULL || policy == GHB_POLICY_SCHEDULE || policy == GHB_POLICY_LEARNED ||
         policy == GHB_POLICY_HEURISTIC) && !can_pull)
        policy = GHB_POLICY_PUSH;
    GHB_REQUIRE(!(opt->record_trace && (!opt->trace || opt->trace_cap <= 0)), "trace buffer missing");
    // Beamer's rule with thresholds measured on B200 (a top-down level costs
    // ~0.13 ms per million frontier entries, a bottom-up level ~0.03-0.2 ms
    // on an RMAT scale-24 graph): switch to bottom-up once the frontier's
    // out-entries exceed 1/256 of the unexplored ones, back to top-down when
    // the frontier is under 1/24 of the vertices.
    const float alpha = opt->alpha > 0 ? opt->alpha : 256.0f;
    const float beta = opt->beta > 0 ? opt->beta : 24.0f;
    // A frontier with fewer than m / gamma out-entries never goes bottom-up:
    // a bottom-up level scans every unvisited vertex, which a thin frontier
    // (a grid's late levels, whose ratio to the unexplored entries is large
    // only because little is left) never repays.
    const float gamma = opt->gamma > 0 ? opt->gamma : 1024.0f;
    static_assert(sizeof(BfsPersistState) <= 16 * sizeof(unsigned long long), "persist state slot");

    const int64_t words = ((int64_t)n + 31) / 32;
    Carver sizing(nullptr);
    BfsBuffers::carve(sizing, n, words);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    BfsBuffers B = BfsBuffers::carve(c, n, words);

    cudaStream_t st = ws->stream;
    // m (total CSR entries) and deg(src) from rowptr.
    int32_t* hp32 = reinterpret_cast<int32_t*>(ws->host_pinned);
    GHB_CUDA_TRY(cudaMemcpyAsync(hp32, out_rowptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaMemcpyAsync(hp32 + 1, out_rowptr + src, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_TRY(launch(ws, bfs_init_kernel, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0, n,
                   words, src, depth, B.visited, B.front_a, B.queue_a));
    if (stats || opt->record_trace) GHB_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t m_total = hp32[0];
    const int64_t deg_src = (int64_t)hp32[2] - hp32[1];

    int64_t n_f = 1, m_f = deg_src, m_r = deg_src, examined = 0, reached = 1;
    double deg2_f = (double)deg_src * deg_src, degmax_f = (double)deg_src;
    int level = 0, pull_levels = 0, dir = 0 /* 0 push, 1 pull */, prev_dir = 0;
    double nf_prev = 1.0;  // frontier size of the previous level (growth feature)
    int32_t *q_cur = B.queue_a, *q_next = B.queue_b;
    uint32_t *f_cur = B.front_a, *f_next = B.front_b;
    const int threads = 256;
    const unsigned gmax = ws->num_sms * 8;
    const int64_t words_active = ((int64_t)n_active + 31) / 32;
    bool queue_valid = true;   // q_cur holds the frontier (false after a bottom-up level)
    bool bitmap_valid = true;  // f_cur holds the frontier (false after a persistent run)
    int coop_blocks = 0;       // co-resident 1024-thread blocks for the persistent kernel
    {
        int coop = 0, per_sm = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ws->device);
        if (coop && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bfs_push_persistent_kernel, 1024, 0) ==
                        cudaSuccess &&
            per_sm >= 1)
            coop_blocks = ws->num_sms;
    }
    auto ensure_queue = [&]() -> int {
        if (queue_valid) return GHB_OK;
        GHB_CUDA_TRY(cudaMemsetAsync(&B.counters->big_tail, 0, sizeof(int32_t), st));
        GHB_TRY(launch(ws, bfs_queue_from_bitmap_kernel, dim3(grid_for(words * 32, threads, gmax)),
                       dim3(threads), 0, words, (const uint32_t*)f_cur, out_rowptr, q_cur,
                       &B.counters->big_tail, (BfsCounters*)nullptr));
        queue_valid = true;
        return GHB_OK;
    };

    while (n_f > 0 && level < max_depth) {
        // ---- direction for this level; fmt_req: output of a top-down level
        // (0 by frontier size, 1 queue, 2 bitmap only)
        const int64_t m_u = m_total - m_r;
        int fmt_req = 0;
        bool by_net = false;
        if (policy == GHB_POLICY_PUSH) {
            dir = 0;
        } else if (policy == GHB_POLICY_PULL) {
            dir = level == 0 ? 0 : 1;
        } else if (policy == GHB_POLICY_SCHEDULE) {
            const bool has = opt->schedule && level < opt->schedule_len;
            dir = has ? (opt->schedule[level] & 1) : dir;
            fmt_req = has ? ((opt->schedule[level] >> 1) & 3) : 0;
        } else {
            const int prev_dir_rule = dir;
            int heur = dir;
            if (dir == 0 && (double)m_f > (double)m_u / alpha && (double)m_f > (double)m_total / gamma) heur = 1;
            else if (dir == 1 && (double)n_f < (double)n / beta) heur = 0;
            dir = heur;
            if (policy == GHB_POLICY_LEARNED) {
                float feat[GHB_TRACE_FEATURES];
                bfs_features(feat, n, m_total, n_f, m_f, m_u, level, deg2_f, degmax_f, prev_dir, nf_prev,
                             (double)(n - reached));
                int d = 0, f = 0;
                // The network's choices only inside the rule's uncertain band
                // (rule_margin); the rule's outside it.
                if (policy_pick_level(feat, &d, &f) &&
                    rule_margin(prev_dir_rule, n, m_total, n_f, m_f, m_u, alpha, beta, gamma) <
                        (float)ws->tune.pol_band) {
                    dir = d;
                    fmt_req = f ? 2 : 1;
                    by_net = true;
                }
            }
        }
        float row[GHB_TRACE_COLS];
        if (opt->record_trace && level < opt->trace_cap) {
            bfs_features(row, n, m_total, n_f, m_f, m_u, level, deg2_f, degmax_f, prev_dir, nf_prev,
                         (double)(n - reached));
            for (int k = GHB_TRACE_FEATURES; k < GHB_TRACE_COLS; ++k) row[k] = -1.f;
        }

        float t_push = -1.f, t_pull = -1.f;
        if (dir == 0 || (opt->oracle_timing && can_pull && opt->record_trace)) GHB_TRY(ensure_queue());
        // Runs of small top-down levels: one cooperative launch, no host
        // round trip per level (high-diameter graphs, BFS tails).
        const bool persist_policy = policy == GHB_POLICY_HEURISTIC || policy == GHB_POLICY_PUSH;
        if (dir == 0 && persist_policy && coop_blocks > 0 && !opt->record_trace && m_f < kPersistMaxEdges &&
            degmax_f < (double)kBigList && queue_valid) {
            BfsPersistState* ps = B.persist;
            GHB_CUDA_TRY(cudaMemsetAsync(ps, 0, sizeof(BfsPersistState), st));
            const int32_t nf32 = (int32_t)n_f;
            GHB_CUDA_TRY(cudaMemcpyAsync(&ps->tail[0], &nf32, sizeof(int32_t), cudaMemcpyHostToDevice, st));
            GHB_TRY(launch_coop(ws, bfs_push_persistent_kernel, dim3(coop_blocks), dim3(1024), 0,
                                (const int32_t*)out_rowptr, (const int32_t*)out_col, q_cur, q_next, B.visited, depth,
                                (int32_t)level, (int32_t)max_depth, (int64_t)kPersistMaxEdges, (int64_t)m_total,
                                (int64_t)m_r, policy == GHB_POLICY_PUSH || !can_pull ? 0.f : alpha, ps));
            GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, ps, sizeof(BfsPersistState), cudaMemcpyDeviceToHost, st));
            GHB_CUDA_TRY(cudaStreamSynchronize(st));
            const BfsPersistState* hs = reinterpret_cast<const BfsPersistState*>(ws->host_pinned);
            if (hs->status != kDevOk) {
                set_error("BFS persistent kernel: grid barrier timed out");
                return GHB_ERR_TIMEOUT;
            }
            const int L = hs->levels_done;
            n_f = hs->tail[L % 3];
            m_f = (int64_t)hs->mf[L % 3];
            deg2_f = 0.0;
            degmax_f = (double)hs->dmax[L % 3];
            nf_prev = (double)hs->tail[(L + 2) % 3];
            examined += (int64_t)hs->examined;
            m_r += (int64_t)hs->m_r;
            reached += (int64_t)hs->reached;
            if (L & 1) std::swap(q_cur, q_next);
            level += L;
            prev_dir = 0;
            dir = 0;
            bitmap_valid = false;
            continue;
        }
        if (dir == 1 && !bitmap_valid) {
            GHB_CUDA_TRY(cudaMemsetAsync(f_cur, 0, words * sizeof(uint32_t), st));
            GHB_TRY(launch(ws, bfs_bitmap_from_queue_kernel, dim3(grid_for(n_f, 256, gmax)), dim3(256), 0,
                           (const int32_t*)q_cur, (int32_t)n_f, f_cur));
            bitmap_valid = true;
        }
        if (opt->oracle_timing && can_pull && opt->record_trace) {
            // Time both directions on a snapshot; the state after a level does
            // not depend on the direction, so the run continues unchanged.
            GHB_TRY(bfs_time_both(ws, B, n, words, out_rowptr, out_col, in_rowptr, in_col, q_cur, n_f, m_f,
                                  f_cur, level, depth, &t_push, &t_pull));
        }

        GHB_CUDA_TRY(cudaMemsetAsync(B.counters, 0, sizeof(BfsCounters), st));
        GHB_CUDA_TRY(cudaMemsetAsync(f_next, 0, words * sizeof(uint32_t), st));
        if (opt->record_trace) GHB_CUDA_TRY(cudaEventRecord(ws->ev_a, st));
        const bool append = fmt_req == 1 || (fmt_req == 0 && m_f < kAppendMaxEdges);
        if (dir == 0) {
            GHB_TRY(bfs_push_level(ws, B, n, out_rowptr, out_col, q_cur, n_f, level + 1, depth,
                                   append ? q_next : (int32_t*)nullptr, f_next));
            if (!append)
                GHB_TRY(launch(ws, bfs_queue_from_bitmap_kernel, dim3(grid_for(words * 32, threads, gmax)),
                               dim3(threads), 0, words, (const uint32_t*)f_next, out_rowptr, q_next,
                               &B.counters->tail, B.counters));
        } else {
            GHB_TRY(launch(ws, bfs_pull_kernel, dim3(grid_for(words_active * 32, threads, gmax)),
                           dim3(threads), 0, n_active, words_active, in_rowptr, in_col, out_rowptr,
                           (const uint32_t*)f_cur, B.visited, f_next, depth, level + 1, q_next,
                           B.counters));
            pull_levels++;
        }
        if (opt->record_trace) GHB_CUDA_TRY(cudaEventRecord(ws->ev_b, st));
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, B.counters, sizeof(BfsCounters),
                                     cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        const BfsCounters* hc = reinterpret_cast<const BfsCounters*>(ws->host_pinned);
        float ms = 0.f;
        if (opt->record_trace) GHB_CUDA_TRY(cudaEventElapsedTime(&ms, ws->ev_a, ws->ev_b));
        if (opt->record_trace && level < opt->trace_cap) {
            row[12] = (float)dir;
            row[13] = ms;
            row[14] = t_push;
            row[15] = t_pull;
            const double unvisited = (double)(n - reached);
            row[16] = (float)hc->examined;
            row[17] = (float)hc->tail;
            row[18] = (float)unvisited;
            // Pull reads the rowptr of every unvisited vertex; push reads the
            // rowptr of every frontier vertex.  Both read 4 B per entry
            // examined and write 4 B of depth per vertex reached.
            row[19] = (float)(4.0 * (dir ? unvisited : (double)n_f) + 4.0 * (double)hc->examined +
                              4.0 * (double)hc->tail);
            row[20] = dir == 0 ? (append ? 0.f : 1.f) : -1.f;
            row[22] = by_net ? 1.f : 0.f;
            for (int k = 0; k < GHB_TRACE_COLS; ++k) opt->trace[(size_t)level * GHB_TRACE_COLS + k] = row[k];
        }
        prev_dir = dir;
        nf_prev = (double)n_f;
        n_f = hc->tail;
        m_f = (int64_t)hc->m_f;
        deg2_f = (double)hc->deg2;
        degmax_f = (double)hc->degmax;
        examined += (int64_t)hc->examined;
        m_r += m_f;
        reached += n_f;
        std::swap(q_cur, q_next);
        std::swap(f_cur, f_next);
        queue_valid = (dir == 0);
        bitmap_valid = true;
        ++level;
    }
    if (stats) {
        GHB_CUDA_TRY(cudaEventRecord(ws->ev_stop, st));
        GHB_CUDA_TRY(cudaEventSynchronize(ws->ev_stop));
        float ms = 0.f;
        GHB_CUDA_TRY(cudaEventElapsedTime(&ms, ws->ev_start, ws->ev_stop));
        stats->levels = level;
        stats->pull_levels = pull_levels;
        stats->reached = reached;
        stats->edges_reached = m_r;
        stats->edges_examined = examined;
        stats->device_ms = ms;
    }
    return GHB_OK;
}

}  // namespace ghb

using namespace ghb;

extern "C" {

int ghb_bfs(ghb_workspace* ws, int32_t n, const int32_t* out_rowptr, const int32_t* out_col,
            const int32_t* in_rowptr, const int32_t* in_col, int32_t src, int32_t max_depth,
            int32_t* depth, const ghb_bfs_options* options, ghb_traversal_stats* stats) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    if (bfs_use_persistent(ws, options)) {
        GHB_REQUIRE(n >= 1, "n must be >= 1");
        GHB_REQUIRE(out_rowptr && depth, "NULL graph or output");
        GHB_REQUIRE(src >= 0 && src < n, "source outside [0, n)");
        GHB_REQUIRE(max_depth >= 0, "max_depth < 0");
        const bool can_pull = in_rowptr != nullptr && in_col != nullptr;
        return bfs_persistent_run(ws, n, n, out_rowptr, out_col, can_pull ? in_rowptr : nullptr,
                                  can_pull ? in_col : nullptr, src, max_depth, depth, nullptr, nullptr, options, stats);
    }
    return bfs_run(ws, n, n, out_rowptr, out_col, in_rowptr, in_col, src, max_depth, depth, options,
                   stats);
}

int ghb_bfs_pred(ghb_workspace* ws, int32_t n, const int32_t* out_rowptr, const int32_t* out_col,
                 const int32_t* in_rowptr, const int32_t* in_col, int32_t src, int32_t max_depth,
                 int32_t* depth, int32_t* pred, const ghb_bfs_options* options,
                 ghb_traversal_stats* stats) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(pred != nullptr, "NULL pred");
    GHB_TRY(bfs_run(ws, n, n, out_rowptr, out_col, in_rowptr, in_col, src, max_depth, depth, options,
                    stats));
    const unsigned gmax = ws->num_sms * 8;
    if (in_rowptr && in_col) {
        // Smallest-id parent: first entry of the (sorted) in-row one level up.
        return launch(ws, bfs_pred_pull_kernel, dim3(grid_for((int64_t)n * 32, 256, gmax)), dim3(256),
                      0, n, in_rowptr, in_col, (const int32_t*)depth, src, pred);
    }
    GHB_TRY(launch(ws, fill_i32_kernel, dim3(grid_for(n, 256, gmax)), dim3(256), 0, pred, (int64_t)n,
                   (int32_t)0x7fffffff));
    GHB_TRY(launch(ws, bfs_pred_push_kernel, dim3(grid_for((int64_t)n * 32, 256, gmax)), dim3(256), 0,
                   n, out_rowptr, out_col, (const int32_t*)depth, pred));
    return launch(ws, bfs_pred_finish_kernel, dim3(grid_for(n, 256, gmax)), dim3(256), 0, n, src, pred);
}

}  // extern "C"
