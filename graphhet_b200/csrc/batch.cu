// Many independent graphs in one call; the multi-source SSSP entry point
// (its engine is mssssp.cu).
//
// Batched graphs are packed back to back: graph g owns global vertices
// [vbase[g], vbase[g+1]) and entries [ebase[g], ebase[g+1]) (int64 bases, so
// a batch may hold more than 2^31 entries); its rowptr (n_g + 1 int32 LOCAL
// offsets) starts at index vbase[g] + g and its col holds LOCAL ids.
//
// WCC of a batch is WCC of the disjoint union: one load-balanced union-find
// pass over all graphs' entries (each warp finds its rows' graph by binary
// search over vbase) and one compress pass, then labels are made local again.
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace ghb {

int wcc_run(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, int32_t* label);
size_t tc_oriented_bytes(int32_t n, int64_t m);
int tc_oriented_core(ghb_workspace* ws, int32_t n, int64_t m, const int32_t* rowptr, const int32_t* col, void* base,
                     unsigned long long* cnt, int64_t* counts64);
int tc_run(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, int64_t* counts64,
           int32_t* counts32, int64_t* total);
int mssssp_run(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* rp, const int32_t* col,
               const double* wt, const int32_t* srcs_host, int32_t n_src, double delta, double inf,
               const int32_t* perm, double* dist, ghb_traversal_stats* stats);

namespace {

__device__ __forceinline__ int32_t graph_of(const int64_t* __restrict__ vbase, int32_t ng, int64_t u) {
    int32_t lo = 0, hi = ng - 1;
    while (lo < hi) {
        const int32_t mid = (lo + hi + 1) >> 1;
        if (vbase[mid] <= u) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int32_t bw_find(int32_t* parent, int32_t x) {
    int32_t p = __ldcg(parent + x);
    if (p == x) return x;
    int32_t prev = x, next;
    while (p > (next = __ldcg(parent + p))) {
        parent[prev] = next;
        prev = p;
        p = next;
    }
    return p;
}

__device__ __forceinline__ void bw_unite(int32_t* parent, int32_t u, int32_t v) {
    int32_t ru = bw_find(parent, u), rv = bw_find(parent, v);
    while (ru != rv) {
        if (ru < rv) {
            const int32_t t = ru;
            ru = rv;
            rv = t;
        }
        const int32_t old = atomicCAS(parent + ru, ru, rv);
        if (old == ru) break;
        ru = bw_find(parent, old);
        rv = bw_find(parent, rv);
    }
}

__global__ void bw_iota(int32_t* p, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = (int32_t)i;
}

// Warp per row: all of the row's entries, 32 at a time.
__global__ void __launch_bounds__(256) bw_link_kernel(int32_t ng, const int64_t* __restrict__ vbase,
                                                      const int64_t* __restrict__ ebase,
                                                      const int32_t* __restrict__ rowptr,
                                                      const int32_t* __restrict__ col, int64_t total_v,
                                                      int32_t* parent) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = warp; u < total_v; u += nwarps) {
        const int32_t g = graph_of(vbase, ng, u);
        const int64_t ri = u + g;
        const int64_t eb = ebase[g];
        const int64_t b = eb + rowptr[ri], e = eb + rowptr[ri + 1];
        const int64_t vb = vbase[g];
        for (int64_t j = b + lane; j < e; j += 32) {
            const int32_t v = (int32_t)(vb + col[j]);
            if (v != (int32_t)u) bw_unite(parent, (int32_t)u, v);
        }
    }
}

__global__ void bw_compress_local(int32_t ng, const int64_t* __restrict__ vbase, int64_t total_v, int32_t* parent,
                                  int32_t* label) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < total_v;
         v += (int64_t)gridDim.x * blockDim.x) {
        int32_t p = __ldcg(parent + v), q;
        while (p != (q = __ldcg(parent + p))) p = q;
        const int32_t g = graph_of(vbase, ng, v);
        label[v] = (int32_t)(p - vbase[g]);
    }
}

// Disjoint-union form: a warp per row of the union CSR (global ids).
__global__ void __launch_bounds__(256) uw_link_kernel(int32_t n, const int32_t* __restrict__ rowptr,
                                                      const int32_t* __restrict__ col, int32_t* parent) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = warp; u < n; u += nwarps) {
        const int32_t b = rowptr[u], e = rowptr[u + 1];
        for (int32_t j = b + lane; j < e; j += 32) {
            const int32_t v = col[j];
            if (v > (int32_t)u) bw_unite(parent, (int32_t)u, v);  // symmetric: each edge once
        }
    }
}

// Triangles per graph: block per graph over its vertex range (fixed order).
__global__ void __launch_bounds__(256) union_graph_totals_kernel(int32_t ng, const int64_t* __restrict__ vbase,
                                                                 const unsigned long long* __restrict__ cnt,
                                                                 int64_t* tri) {
    __shared__ unsigned long long red[8];
    for (int32_t g = blockIdx.x; g < ng; g += gridDim.x) {
        unsigned long long s = 0;
        for (int64_t v = vbase[g] + threadIdx.x; v < vbase[g + 1]; v += blockDim.x) s += cnt[v];
        s = warp_sum(s);
        if (lane_id() == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long t = 0;
            for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
            tri[g] = (int64_t)(t / 3);
        }
        __syncthreads();
    }
}

size_t union_bytes(int32_t n, int64_t m) {
    Carver c(nullptr);
    c.take<int32_t>(n);                       // union-find forest
    c.take<unsigned long long>((size_t)n + 1);  // triangles per vertex (+ total)
    c.take<unsigned char>(tc_oriented_bytes(n, m));
    return c.off;
}

}  // namespace
}  // namespace ghb

using namespace ghb;

extern "C" {

int ghb_batch_wcc(ghb_workspace* ws, int32_t n_graphs, const int64_t* vbase, const int64_t* ebase,
                  const int32_t* rowptr, const int32_t* col, int32_t* label) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n_graphs >= 1, "n_graphs must be >= 1");
    GHB_REQUIRE(vbase && ebase && rowptr && label, "NULL argument");
    const int64_t total_v = vbase[n_graphs] - vbase[0];
    GHB_REQUIRE(vbase[0] == 0 && ebase[0] == 0, "bases must start at 0");
    GHB_REQUIRE(total_v >= 1 && total_v < (1ll << 31), "vertex total out of int32 range");
    for (int32_t g = 0; g < n_graphs; ++g)
        GHB_REQUIRE(vbase[g + 1] >= vbase[g] && ebase[g + 1] >= ebase[g], "bases must be non-decreasing");
    cudaStream_t st = ws->stream;
    Carver sizing(nullptr);
    sizing.take<int64_t>(n_graphs + 1);
    sizing.take<int64_t>(n_graphs + 1);
    sizing.take<int32_t>(total_v);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    int64_t* dvb = c.take<int64_t>(n_graphs + 1);
    int64_t* deb = c.take<int64_t>(n_graphs + 1);
    int32_t* parent = c.take<int32_t>(total_v);
    GHB_CUDA_TRY(cudaMemcpyAsync(dvb, vbase, sizeof(int64_t) * (n_graphs + 1), cudaMemcpyHostToDevice, st));
    GHB_CUDA_TRY(cudaMemcpyAsync(deb, ebase, sizeof(int64_t) * (n_graphs + 1), cudaMemcpyHostToDevice, st));
    const unsigned g = ws->num_sms * 8;
    GHB_TRY(launch(ws, bw_iota, dim3(grid_for(total_v, 256, g)), dim3(256), 0, parent, total_v));
    GHB_TRY(launch(ws, bw_link_kernel, dim3(grid_for(total_v * 32, 256, g)), dim3(256), 0, n_graphs,
                   (const int64_t*)dvb, (const int64_t*)deb, rowptr, col, total_v, parent));
    GHB_TRY(launch(ws, bw_compress_local, dim3(grid_for(total_v, 256, g)), dim3(256), 0, n_graphs,
                   (const int64_t*)dvb, total_v, parent, label));
    // The caller's vbase/ebase are host arrays: wait before returning so the
    // copies above are done with them.
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    return GHB_OK;
}

int ghb_batch_tc(ghb_workspace* ws, int32_t n_graphs, const int64_t* vbase, const int64_t* ebase,
                 const int32_t* rowptr, const int32_t* col, int64_t* counts64, int64_t* totals) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n_graphs >= 1, "n_graphs must be >= 1");
    GHB_REQUIRE(vbase && ebase && rowptr, "NULL argument");
    for (int32_t g = 0; g < n_graphs; ++g) {
        const int64_t ng = vbase[g + 1] - vbase[g];
        GHB_REQUIRE(ng >= 0 && ng < (1ll << 31), "graph size out of range");
        if (ng == 0) {
            if (totals) totals[g] = 0;
            continue;
        }
        int64_t t = 0;
        GHB_TRY(tc_run(ws, (int32_t)ng, rowptr + vbase[g] + g, col ? col + ebase[g] : nullptr,
                       counts64 ? counts64 + vbase[g] : nullptr, nullptr, &t));
        if (totals) totals[g] = t;
    }
    return GHB_OK;
}

int ghb_union_reserve(ghb_workspace* ws, int32_t n_total, int64_t m) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n_total >= 1 && m >= 0 && m < (1ll << 31), "sizes out of range");
    return ws_reserve(ws, union_bytes(n_total, m));
}

int ghb_union_wcc_tc(ghb_workspace* ws, int32_t n_graphs, const int64_t* vbase, int32_t n_total, int64_t m,
                     const int32_t* rowptr, const int32_t* col, int32_t* label, int64_t* counts64,
                     int64_t* triangles) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n_graphs >= 1 && n_total >= 1 && m >= 0 && m < (1ll << 31), "sizes out of range");
    GHB_REQUIRE(vbase && rowptr && (m == 0 || col), "NULL argument");
    GHB_REQUIRE(label || counts64 || triangles, "no output requested");
    const size_t need = union_bytes(n_total, m);
    GHB_REQUIRE(ws->scratch_cap >= need, "workspace scratch too small: call ghb_union_reserve first");
    Carver c(ws->scratch);
    int32_t* parent = c.take<int32_t>(n_total);
    unsigned long long* cnt = c.take<unsigned long long>((size_t)n_total + 1);
    void* tcbase = c.take<unsigned char>(tc_oriented_bytes(n_total, m));
    const unsigned g = ws->num_sms * 8;
    if (label) {
        GHB_TRY(launch(ws, bw_iota, dim3(grid_for(n_total, 256, g)), dim3(256), 0, parent, (int64_t)n_total));
        GHB_TRY(launch(ws, uw_link_kernel, dim3(grid_for((int64_t)n_total * 32, 256, g)), dim3(256), 0, n_total,
                       rowptr, col, parent));
        GHB_TRY(launch(ws, bw_compress_local, dim3(grid_for(n_total, 256, g)), dim3(256), 0, n_graphs, vbase,
                       (int64_t)n_total, parent, label));
    }
    if (counts64 || triangles) {
        GHB_TRY(tc_oriented_core(ws, n_total, m, rowptr, col, tcbase, cnt, counts64));
        if (triangles)
            GHB_TRY(launch(ws, union_graph_totals_kernel, dim3(std::min<int32_t>(n_graphs, ws->num_sms * 8)),
                           dim3(256), 0, n_graphs, vbase, (const unsigned long long*)cnt, triangles));
    }
    return GHB_OK;
}

int ghb_mssssp(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, const double* w,
               const int32_t* srcs, int32_t n_src, double inf, double* dist, ghb_traversal_stats* stats) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n >= 1 && n_src >= 0, "bad sizes");
    GHB_REQUIRE(rowptr && col && w && dist && srcs, "NULL argument");
    GHB_REQUIRE(inf >= 0, "inf must be >= 0");
    cudaStream_t st = ws->stream;
    std::vector<int32_t> hs(n_src > 0 ? n_src : 1);
    if (n_src > 0) {
        GHB_CUDA_TRY(cudaMemcpyAsync(hs.data(), srcs, sizeof(int32_t) * n_src, cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
    }
    for (int32_t i = 0; i < n_src; ++i) GHB_REQUIRE(hs[i] >= 0 && hs[i] < n, "source outside [0, n)");
    if (n_src == 0) return GHB_OK;
    return mssssp_run(ws, n, n, rowptr, col, w, hs.data(), n_src, 0.0, inf, nullptr, dist, stats);
}

}  // extern "C"
