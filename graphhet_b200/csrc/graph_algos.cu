// Algorithms on a resident (degree-relabelled) graph handle: run on the
// relabelled CSR, then map results back to the caller's vertex ids.  Outputs
// are the same as the raw-CSR entry points' (include/ghb.h).
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "bfs_kernels.cuh"
#include "graph.cuh"

namespace ghb {

int bfs_run(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* out_rowptr, const int32_t* out_col,
            const int32_t* in_rowptr, const int32_t* in_col, int32_t src, int32_t max_depth, int32_t* depth,
            const ghb_bfs_options* opt, ghb_traversal_stats* stats);
int sssp_run(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, const double* w, int32_t src,
             double inf, double* dist_out, const ghb_sssp_options* opt, ghb_traversal_stats* stats);
int sssp_pred_run(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, const double* w,
                  const int32_t* in_rp, const int32_t* in_col, const double* in_w, int32_t src, double inf,
                  const double* dist, int32_t* pred);
int sssp_delta_run(ghb_workspace* ws, ghb_graph* g, int32_t src, double inf, double delta, double* dist_out,
                   ghb_traversal_stats* stats);
int sssp_choose_delta(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const double* w, int32_t src,
                      const ghb_sssp_options* opt, double* delta);

// Resident SSSP: delta-stepping with the light/heavy split when the rows fit
// the weight-sorted copy's key (n <= 2^25), else the near/far form.
static int graph_sssp_dispatch(ghb_workspace* ws, const ghb_graph* g, int32_t src_new, double inf, double* dnew,
                               const ghb_sssp_options* options, ghb_traversal_stats* stats) {
    if (g->m > 0 && g->n <= (1 << 25)) {
        double delta = 0.0;
        GHB_TRY(sssp_choose_delta(ws, g->n, g->rowptr, g->w, src_new, options, &delta));
        return sssp_delta_run(ws, const_cast<ghb_graph*>(g), src_new, inf, delta, dnew, stats);
    }
    return sssp_run(ws, g->n, g->rowptr, g->col, g->w, src_new, inf, dnew, options, stats);
}
int wcc_run(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, int32_t* label);
int wcc_afforest_run(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* rowptr, const int32_t* col,
                     int32_t* label);
int mssssp_run(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* rp, const int32_t* col,
               const double* wt, const int32_t* srcs_host, int32_t n_src, double delta, double inf,
               const int32_t* perm, double* dist, ghb_traversal_stats* stats);
int cdlp_run(ghb_workspace* ws, int32_t n, const int32_t* rp, const int32_t* col, int32_t iterations,
             int32_t* labels, const int32_t* init_labels, bool first_min);
int tc_run(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, int64_t* counts64,
           int32_t* counts32, int64_t* total);
int tc_run_cached(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, int64_t* counts64,
                  int32_t* counts32, int64_t* total, std::atomic<int32_t>* flags_cache);
int pagerank_run(ghb_workspace* ws, int32_t n, const int32_t* in_rp, const int32_t* in_col, const int32_t* out_rp,
                 const ghb_pr_options* o, double* rank, int32_t* iters_run);
int msbfs_batch(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* out_rp, const int32_t* out_col,
                const int32_t* in_rp, const int32_t* in_col, const int32_t* srcs_dev, int32_t k,
                const int32_t* perm, int32_t* depth, int64_t* levels_out, int64_t* examined_out);
size_t msbfs_persistent_bytes(int32_t n, int64_t m, int32_t n_src);
int msbfs_persistent_steered(ghb_workspace* ws, int32_t n, int32_t n_active, int64_t m, const int32_t* out_rp,
                             const int32_t* out_col, const int32_t* in_rp, const int32_t* in_col,
                             const int32_t* srcs, int32_t n_src, const int32_t* perm, int32_t* depth,
                             int64_t* levels_out, int64_t* examined_out, const int8_t* schedule,
                             int32_t schedule_len, float* trace, int32_t trace_cap);
bool msbfs_persistent_available(ghb_workspace* ws, int32_t n_src);
int msbfs_persistent(ghb_workspace* ws, int32_t n, int32_t n_active, int64_t m, const int32_t* out_rp,
                     const int32_t* out_col, const int32_t* in_rp, const int32_t* in_col, const int32_t* srcs,
                     int32_t n_src, const int32_t* perm, int32_t* depth, bool finish, int64_t* levels_out,
                     int64_t* examined_out);

namespace {

__global__ void fill_kernel(int32_t* p, int64_t n, int32_t v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

// Smallest caller id in each component: cmin[root] = min iperm over members.
// Most vertices of a power-law graph share one root, the component of new id
// 0 (the top hub): its members are reduced in registers and each warp issues
// one atomic, instead of one same-address atomic per member (those serialise
// at one L2 slice). Other roots take a plain atomic per member.
__global__ void comp_min_kernel(int32_t n, const int32_t* __restrict__ label_new, const int32_t* __restrict__ iperm,
                                int32_t* cmin) {
    const int32_t hot = n > 0 ? label_new[0] : 0;
    int32_t hot_min = INT_MAX;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t l = label_new[v];
        const int32_t id = iperm[v];
        if (l == hot)
            hot_min = min(hot_min, id);
        else
            atomicMin(cmin + l, id);
    }
    hot_min = __reduce_min_sync(0xffffffffu, hot_min);
    if ((threadIdx.x & 31) == 0 && hot_min != INT_MAX) atomicMin(cmin + hot, hot_min);
}

__global__ void comp_map_kernel(int32_t n, const int32_t* __restrict__ perm, const int32_t* __restrict__ label_new,
                                const int32_t* __restrict__ cmin, int32_t* out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        out[v] = cmin[label_new[perm[v]]];
}

// pred_new holds new ids: map the row and the value.
__global__ void pred_map_kernel(int32_t n, const int32_t* __restrict__ perm, const int32_t* __restrict__ iperm,
                                const int32_t* __restrict__ pred_new, int32_t* out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t p = pred_new[perm[v]];
        out[v] = p < 0 ? p : iperm[p];
    }
}

__global__ void tc_map_kernel(int32_t n, const int32_t* __restrict__ perm, const int64_t* __restrict__ c_new,
                              int64_t* c64, int32_t* c32) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = c_new[perm[v]];
        if (c64) c64[v] = c;
        if (c32) c32[v] = (int32_t)(uint32_t)(uint64_t)c;
    }
}

}  // namespace
}  // namespace ghb

using namespace ghb;

#define GRAPH_PRELUDE()                              \
    ws = ws_resolve(ws);                             \
    GHB_REQUIRE(ws, "no workspace");                 \
    GHB_REQUIRE(g, "NULL graph");                    \
    int _cur = 0;                                    \
    GHB_CUDA_TRY(cudaGetDevice(&_cur));              \
    GHB_REQUIRE(_cur == g->device, "graph lives on another device")

extern "C" {

int ghb_graph_bfs(ghb_workspace* ws, const ghb_graph* g, int32_t src, int32_t max_depth, int32_t* depth,
                  const ghb_bfs_options* options, ghb_traversal_stats* stats) {
    GRAPH_PRELUDE();
    GHB_REQUIRE(depth, "NULL depth");
    GHB_REQUIRE(src >= 0 && src < g->n, "source outside [0, n)");
    GHB_TRY(ws_reserve_stage(ws, sizeof(int32_t) * (size_t)g->n));
    int32_t* dnew = static_cast<int32_t*>(ws->stage);
    if (bfs_use_persistent(ws, options))
        return bfs_persistent_run(ws, g->n, g->n_active, g->rowptr, g->col, g->in_rowptr, g->in_col,
                                  g->perm_host[src], max_depth, dnew, g->perm, depth, options, stats);
    GHB_TRY(bfs_run(ws, g->n, g->n_active, g->rowptr, g->col, g->in_rowptr, g->in_col, g->perm_host[src], max_depth,
                    dnew, options, stats));
    return map_back_i32(ws, g, dnew, depth);
}

int ghb_graph_bfs_pred(ghb_workspace* ws, const ghb_graph* g, int32_t src, int32_t max_depth, int32_t* depth,
                       int32_t* pred, const ghb_bfs_options* options, ghb_traversal_stats* stats) {
    GRAPH_PRELUDE();
    GHB_REQUIRE(depth && pred, "NULL output");
    GHB_REQUIRE(src >= 0 && src < g->n, "source outside [0, n)");
    GHB_TRY(ws_reserve_stage(ws, 2 * sizeof(int32_t) * (size_t)g->n + 256));
    int32_t* dnew = static_cast<int32_t*>(ws->stage);
    int32_t* pnew = dnew + (((size_t)g->n + 63) & ~(size_t)63);
    GHB_TRY(ghb_bfs_pred(ws, g->n, g->rowptr, g->col, g->in_rowptr, g->in_col, g->perm_host[src], max_depth, dnew,
                         pnew, options, stats));
    GHB_TRY(map_back_i32(ws, g, dnew, depth));
    return launch(ws, pred_map_kernel, dim3(grid_for(g->n, 256, ws->num_sms * 8)), dim3(256), 0, g->n,
                  (const int32_t*)g->perm, (const int32_t*)g->iperm, (const int32_t*)pnew, pred);
}

int ghb_graph_msbfs(ghb_workspace* ws, const ghb_graph* g, const int32_t* srcs, int32_t n_src, int32_t* depth,
                    ghb_traversal_stats* stats) {
    GRAPH_PRELUDE();
    GHB_REQUIRE(srcs && depth && n_src >= 0, "bad arguments");
    cudaStream_t st = ws->stream;
    std::vector<int32_t> hs(n_src > 0 ? n_src : 1);
    if (n_src > 0) {
        GHB_CUDA_TRY(cudaMemcpyAsync(hs.data(), srcs, sizeof(int32_t) * n_src, cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
    }
    for (int32_t i = 0; i < n_src; ++i) {
        GHB_REQUIRE(hs[i] >= 0 && hs[i] < g->n, "source outside [0, n)");
        hs[i] = g->perm_host[hs[i]];
    }
    if (n_src > 0 && msbfs_persistent_available(ws, n_src)) {
        // One cooperative launch per pass; the kernel maps the caller's
        // sources and writes depths in the caller's ids through perm.
        int64_t levels = 0, examined = 0;
        GHB_TRY(ws_reserve(ws, msbfs_persistent_bytes(g->n, g->m, n_src)));
        if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
        GHB_TRY(msbfs_persistent(ws, g->n, g->n_active, g->m, g->rowptr, g->col, g->in_rowptr, g->in_col, srcs, n_src,
                                 (const int32_t*)g->perm, depth, true, &levels, &examined));
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
    // Sources in the graph's ids; depths go straight to the caller's rows.
    GHB_TRY(ws_reserve_stage(ws, sizeof(int32_t) * kMsPass));
    int32_t* snew = static_cast<int32_t*>(ws->stage);
    if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
    int64_t levels = 0, examined = 0;
    for (int32_t s0 = 0; s0 < n_src; s0 += kMsPass) {
        const int32_t k = std::min<int32_t>(kMsPass, n_src - s0);
        GHB_CUDA_TRY(cudaMemcpyAsync(snew, hs.data() + s0, sizeof(int32_t) * k, cudaMemcpyHostToDevice, st));
        GHB_TRY(msbfs_batch(ws, g->n, g->n_active, g->rowptr, g->col, g->in_rowptr, g->in_col, snew, k,
                            (const int32_t*)g->perm, depth + (int64_t)s0 * g->n, &levels, &examined));
    }
    GHB_CUDA_TRY(cudaStreamSynchronize(st));  // hs (host) is read by the copies above
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

int ghb_graph_msbfs_ex(ghb_workspace* ws, const ghb_graph* g, const int32_t* srcs, int32_t n_src, int32_t* depth,
                       const ghb_msbfs_options* options, ghb_traversal_stats* stats) {
    GRAPH_PRELUDE();
    GHB_REQUIRE(srcs && depth && n_src >= 1, "bad arguments");
    GHB_REQUIRE(!options || options->schedule_len >= 0, "schedule_len < 0");
    GHB_REQUIRE(!options || !options->trace || options->trace_cap >= 0, "trace_cap < 0");
    if (!msbfs_persistent_available(ws, n_src)) {
        set_error("whole-pass multi-source BFS unavailable (no cooperative launch, or ms_persistent = 0)");
        return GHB_ERR_UNSUPPORTED;
    }
    cudaStream_t st = ws->stream;
    std::vector<int32_t> hs(n_src);
    GHB_CUDA_TRY(cudaMemcpyAsync(hs.data(), srcs, sizeof(int32_t) * n_src, cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    for (int32_t i = 0; i < n_src; ++i) GHB_REQUIRE(hs[i] >= 0 && hs[i] < g->n, "source outside [0, n)");
    int64_t levels = 0, examined = 0;
    GHB_TRY(ws_reserve(ws, msbfs_persistent_bytes(g->n, g->m, n_src)));
    if (stats) GHB_CUDA_TRY(cudaEventRecord(ws->ev_start, st));
    GHB_TRY(msbfs_persistent_steered(ws, g->n, g->n_active, g->m, g->rowptr, g->col, g->in_rowptr, g->in_col, srcs,
                                     n_src, (const int32_t*)g->perm, depth, &levels, &examined,
                                     options ? options->schedule : nullptr, options ? options->schedule_len : 0,
                                     options ? options->trace : nullptr, options ? options->trace_cap : 0));
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

int ghb_graph_msbfs_reserve(ghb_workspace* ws, const ghb_graph* g, int32_t n_src) {
    GRAPH_PRELUDE();
    GHB_REQUIRE(n_src >= 1, "n_src must be >= 1");
    if (!msbfs_persistent_available(ws, n_src)) {
        set_error("whole-pass multi-source BFS unavailable (no cooperative launch, or ms_persistent = 0)");
        return GHB_ERR_UNSUPPORTED;
    }
    return ws_reserve(ws, msbfs_persistent_bytes(g->n, g->m, n_src));
}

int ghb_graph_msbfs_launch(ghb_workspace* ws, const ghb_graph* g, const int32_t* srcs, int32_t n_src,
                           int32_t* depth) {
    GRAPH_PRELUDE();
    GHB_REQUIRE(srcs && depth && n_src >= 1, "bad arguments");
    if (!msbfs_persistent_available(ws, n_src)) {
        set_error("whole-pass multi-source BFS unavailable (no cooperative launch, or ms_persistent = 0)");
        return GHB_ERR_UNSUPPORTED;
    }
    return msbfs_persistent(ws, g->n, g->n_active, g->m, g->rowptr, g->col, g->in_rowptr, g->in_col, srcs, n_src,
                            (const int32_t*)g->perm, depth, false, nullptr, nullptr);
}

int ghb_graph_mssssp(ghb_workspace* ws, const ghb_graph* g, const int32_t* srcs, int32_t n_src, double inf,
                     double* dist, ghb_traversal_stats* stats) {
    GRAPH_PRELUDE();
    GHB_REQUIRE(srcs && dist && n_src >= 0, "bad arguments");
    GHB_REQUIRE(g->weighted || g->m == 0, "graph has no weights");
    GHB_REQUIRE(inf >= 0, "inf must be >= 0");
    cudaStream_t st = ws->stream;
    std::vector<int32_t> hs(n_src > 0 ? n_src : 1);
    if (n_src > 0) {
        GHB_CUDA_TRY(cudaMemcpyAsync(hs.data(), srcs, sizeof(int32_t) * n_src, cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
    }
    for (int32_t i = 0; i < n_src; ++i) {
        GHB_REQUIRE(hs[i] >= 0 && hs[i] < g->n, "source outside [0, n)");
        hs[i] = g->perm_host[hs[i]];
    }
    if (n_src == 0) return GHB_OK;
    return mssssp_run(ws, g->n, g->n_active, g->rowptr, g->col, g->w, hs.data(), n_src, 0.0, inf,
                      (const int32_t*)g->perm, dist, stats);
}

int ghb_graph_sssp(ghb_workspace* ws, const ghb_graph* g, int32_t src, double inf, double* dist,
                   const ghb_sssp_options* options, ghb_traversal_stats* stats) {
    GRAPH_PRELUDE();
    GHB_REQUIRE(dist, "NULL dist");
    GHB_REQUIRE(g->weighted || g->m == 0, "graph has no weights");
    GHB_REQUIRE(src >= 0 && src < g->n, "source outside [0, n)");
    GHB_TRY(ws_reserve_stage(ws, sizeof(double) * (size_t)g->n));
    double* dnew = static_cast<double*>(ws->stage);
    GHB_TRY(graph_sssp_dispatch(ws, g, g->perm_host[src], inf, dnew, options, stats));
    return map_back_f64(ws, g, dnew, dist);
}

int ghb_graph_sssp_pred(ghb_workspace* ws, const ghb_graph* g, int32_t src, double inf, double* dist, int32_t* pred,
                        const ghb_sssp_options* options, ghb_traversal_stats* stats) {
    GRAPH_PRELUDE();
    GHB_REQUIRE(dist && pred, "NULL output");
    GHB_REQUIRE(g->weighted || g->m == 0, "graph has no weights");
    GHB_REQUIRE(src >= 0 && src < g->n, "source outside [0, n)");
    GHB_TRY(ws_reserve_stage(ws, (sizeof(double) + sizeof(int32_t)) * (size_t)g->n + 512));
    double* dnew = static_cast<double*>(ws->stage);
    int32_t* pnew = reinterpret_cast<int32_t*>(dnew + (((size_t)g->n + 63) & ~(size_t)63));
    GHB_TRY(graph_sssp_dispatch(ws, g, g->perm_host[src], inf, dnew, options, stats));
    GHB_TRY(sssp_pred_run(ws, g->n, g->rowptr, g->col, g->w, g->in_rowptr, g->in_col, g->in_w, g->perm_host[src], inf,
                          dnew, pnew));
    GHB_TRY(map_back_f64(ws, g, dnew, dist));
    return launch(ws, pred_map_kernel, dim3(grid_for(g->n, 256, ws->num_sms * 8)), dim3(256), 0, g->n,
                  (const int32_t*)g->perm, (const int32_t*)g->iperm, (const int32_t*)pnew, pred);
}

int ghb_graph_wcc(ghb_workspace* ws, const ghb_graph* g, int32_t* label) {
    GRAPH_PRELUDE();
    GHB_REQUIRE(label, "NULL label");
    GHB_TRY(ws_reserve_stage(ws, 2 * sizeof(int32_t) * (size_t)g->n + 256));
    int32_t* lnew = static_cast<int32_t*>(ws->stage);
    int32_t* cmin = lnew + (((size_t)g->n + 63) & ~(size_t)63);
    // Afforest over the relabelled graph's all-CSR (symmetric: in then out
    // neighbours; the CSR itself when undirected).
    GHB_TRY(wcc_afforest_run(ws, g->n, g->n_active, g->all_rowptr, g->all_col, lnew));
    const unsigned gr = grid_for(g->n, 256, ws->num_sms * 8);
    GHB_TRY(launch(ws, fill_kernel, dim3(gr), dim3(256), 0, cmin, (int64_t)g->n, (int32_t)0x7fffffff));
    GHB_TRY(launch(ws, comp_min_kernel, dim3(gr), dim3(256), 0, g->n, (const int32_t*)lnew, (const int32_t*)g->iperm,
                   cmin));
    return launch(ws, comp_map_kernel, dim3(gr), dim3(256), 0, g->n, (const int32_t*)g->perm, (const int32_t*)lnew,
                  (const int32_t*)cmin, label);
}

int ghb_graph_pagerank(ghb_workspace* ws, const ghb_graph* g, const ghb_pr_options* options, double* rank,
                       int32_t* iterations_run) {
    GRAPH_PRELUDE();
    GHB_REQUIRE(rank && options, "NULL argument");
    GHB_REQUIRE(options->iterations >= 0, "iterations < 0");
    GHB_REQUIRE(options->precision == GHB_PR_FP64 || options->precision == GHB_PR_FP32_KAHAN, "bad precision");
    GHB_TRY(ws_reserve_stage(ws, sizeof(double) * (size_t)g->n));
    double* rnew = static_cast<double*>(ws->stage);
    GHB_TRY(pagerank_run(ws, g->n, g->in_rowptr, g->in_col, g->rowptr, options, rnew, iterations_run));
    return map_back_f64(ws, g, rnew, rank);
}

int ghb_graph_cdlp(ghb_workspace* ws, const ghb_graph* g, int32_t iterations, int32_t* labels) {
    GRAPH_PRELUDE();
    GHB_REQUIRE(labels && iterations >= 0, "bad arguments");
    GHB_TRY(ws_reserve_stage(ws, sizeof(int32_t) * (size_t)g->n));
    int32_t* lnew = static_cast<int32_t*>(ws->stage);
    // Label values stay caller ids (iperm), so the smallest-label tie-break is
    // the caller's.
    // Undirected without repeated entries: iperm is a permutation, so the
    // first iteration is a row minimum.
    GHB_TRY(cdlp_run(ws, g->n, g->all_rowptr, g->all_col, iterations, lnew, g->iperm, !g->directed && !g->repeats));
    return map_back_i32(ws, g, lnew, labels);
}

int ghb_graph_tc(ghb_workspace* ws, const ghb_graph* g, int64_t* counts64, int32_t* counts32, int64_t* total) {
    GRAPH_PRELUDE();
    GHB_TRY(ws_reserve_stage(ws, sizeof(int64_t) * (size_t)g->n));
    int64_t* cnew = static_cast<int64_t*>(ws->stage);
    GHB_TRY(tc_run_cached(ws, g->n, g->rowptr, g->col, cnew, nullptr, total, &g->tc_flags));
    return launch(ws, tc_map_kernel, dim3(grid_for(g->n, 256, ws->num_sms * 8)), dim3(256), 0, g->n,
                  (const int32_t*)g->perm, (const int64_t*)cnew, counts64, counts32);
}

}  // extern "C"
