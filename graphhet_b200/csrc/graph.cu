// Resident graph handle: the caller's CSR relabelled by degree on the GPU.
//
// New ids rank vertices by total degree, descending (ties by old id), so
//  * hubs have the smallest ids: sorted rows list them first, a bottom-up BFS
//    step meets a frontier hub on its first probe, and gathers of hub values
//    (PageRank contributions, BFS frontier words) hit a few cache lines;
//  * vertices with no entries form the tail [n_active, n): traversal and
//    label kernels skip it;
//  * "v < u" orients every undirected edge from the lower- to the higher-
//    degree end, so triangle counting reads an oriented row as the prefix of
//    the sorted row that precedes u (no copy).
// The relabelling is a one-time step per graph (like the reference's toCSR,
// GPU_csr.hpp:282-339); results are mapped back to the caller's ids.
#include <cub/device/device_radix_sort.cuh>

#include <vector>

#include "common.cuh"
#include "graph.cuh"

namespace ghb {
namespace {

__device__ __forceinline__ uint64_t degree_key(uint32_t d, int64_t v) {
    return ((uint64_t)(0xFFFFFFFFu - d) << 32) | (uint64_t)(uint32_t)v;
}

// Degree keys (descending degree, then id).  When rowptr (and the in-CSR's)
// start on 16-byte boundaries a thread takes four vertices with one 16-byte
// load of rowptr[4q..4q+3] plus rowptr[4q+4].
__global__ void degree_key_kernel(int32_t n, const int32_t* __restrict__ out_rp, const int32_t* __restrict__ in_rp,
                                  uint64_t* keys) {
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const bool vec = ((uintptr_t)out_rp & 15) == 0 && (!in_rp || ((uintptr_t)in_rp & 15) == 0);
    int64_t v0 = 0;
    if (vec) {
        const int64_t quads = n / 4;
        for (int64_t q = tid; q < quads; q += stride) {
            const int4 a = reinterpret_cast<const int4*>(out_rp)[q];
            const int32_t nx = out_rp[4 * q + 4];
            uint32_t d0 = a.y - a.x, d1 = a.z - a.y, d2 = a.w - a.z, d3 = nx - a.w;
            if (in_rp) {
                const int4 b = reinterpret_cast<const int4*>(in_rp)[q];
                const int32_t ny = in_rp[4 * q + 4];
                d0 += b.y - b.x;
                d1 += b.z - b.y;
                d2 += b.w - b.z;
                d3 += ny - b.w;
            }
            keys[4 * q] = degree_key(d0, 4 * q);
            keys[4 * q + 1] = degree_key(d1, 4 * q + 1);
            keys[4 * q + 2] = degree_key(d2, 4 * q + 2);
            keys[4 * q + 3] = degree_key(d3, 4 * q + 3);
        }
        v0 = quads * 4;
    }
    for (int64_t v = v0 + tid; v < n; v += stride) {
        uint32_t d = (uint32_t)(out_rp[v + 1] - out_rp[v]);
        if (in_rp) d += (uint32_t)(in_rp[v + 1] - in_rp[v]);
        keys[v] = degree_key(d, v);
    }
}

__global__ void perm_from_keys_kernel(int32_t n, const uint64_t* __restrict__ keys, int32_t* perm, int32_t* iperm,
                                      int32_t* n_active) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        const int32_t old = (int32_t)(uint32_t)k;
        iperm[i] = old;
        perm[old] = (int32_t)i;
        const bool zero = (uint32_t)(k >> 32) == 0xFFFFFFFFu;
        const bool prev_nonzero = i == 0 || (uint32_t)(keys[i - 1] >> 32) != 0xFFFFFFFFu;
        if (zero && prev_nonzero) *n_active = (int32_t)i;
    }
}

// One key per entry: (new row << bits) | new col, value = entry index.  A
// warp per row; rows of 64 or more entries read col with 16-byte loads (four
// entries a lane) between a scalar head up to the first 4-aligned entry and
// a scalar tail, when col starts on a 16-byte boundary.
__global__ void relabel_keys_kernel(int32_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                                    const int32_t* __restrict__ perm, int bits, uint64_t* keys, uint32_t* vals) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const bool vec = ((uintptr_t)col & 15) == 0;
    for (int64_t u = warp; u < n; u += nwarps) {
        const uint64_t nu = (uint64_t)(uint32_t)perm[u] << bits;
        const int32_t b = rp[u], e = rp[u + 1];
        int32_t j0 = b, j1 = b;  // [j0, j1): the 4-aligned body
        if (vec && e - b >= 64) {
            j0 = (b + 3) & ~3;
            j1 = e & ~3;
        }
        for (int32_t j = j0 + 4 * lane; j < j1; j += 128) {
            const int4 c = *reinterpret_cast<const int4*>(col + j);
            keys[j] = nu | (uint64_t)(uint32_t)perm[c.x];
            keys[j + 1] = nu | (uint64_t)(uint32_t)perm[c.y];
            keys[j + 2] = nu | (uint64_t)(uint32_t)perm[c.z];
            keys[j + 3] = nu | (uint64_t)(uint32_t)perm[c.w];
            if (vals) *reinterpret_cast<uint4*>(vals + j) = make_uint4(j, j + 1, j + 2, j + 3);
        }
        // Head [b, j0) and tail [j1, e) (the whole row when no body).
        const int32_t head = j0 - b;
        const int32_t rest = head + (e - j1);
        for (int32_t t = lane; t < rest; t += 32) {
            const int32_t j = t < head ? b + t : j1 + (t - head);
            keys[j] = nu | (uint64_t)(uint32_t)perm[col[j]];
            if (vals) vals[j] = (uint32_t)j;
        }
    }
}

__global__ void relabel_out_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals, int64_t m,
                                   int bits, const double* __restrict__ w, int32_t* col, double* w_out) {
    const uint64_t mask = (1ull << bits) - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        col[i] = (int32_t)(keys[i] & mask);
        if (w_out) w_out[i] = w[vals[i]];
    }
}

__global__ void rowptr_from_keys_kernel(const uint64_t* __restrict__ keys, int64_t m, int bits, int32_t n,
                                        int32_t* __restrict__ rowptr) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p <= m; p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t prev = (p == 0) ? -1 : (int64_t)(keys[p - 1] >> bits);
        const int64_t cur = (p == m) ? (int64_t)n : (int64_t)(keys[p] >> bits);
        for (int64_t r = prev + 1; r <= cur; ++r) rowptr[r] = (int32_t)p;
    }
}

__global__ void outdeg_kernel(int32_t n, const int32_t* __restrict__ rp, int32_t* outdeg) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        outdeg[v] = rp[v + 1] - rp[v];
}

template <class T>
__global__ void map_back_kernel(int32_t n, const int32_t* __restrict__ perm, const T* __restrict__ src, T* dst) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        dst[v] = src[perm[v]];
}

int bits_for_n(int32_t n) {
    int bits = 1;
    while (bits < 31 && (1ll << bits) < (int64_t)n) ++bits;
    return bits;
}

template <class T>
int dalloc(T** p, size_t count, int64_t* total) {
    GHB_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * (count ? count : 1)));
    *total += (int64_t)(sizeof(T) * (count ? count : 1));
    return GHB_OK;
}

// Relabel one CSR (rows and columns through perm), rows sorted, weights
// carried along.
// Sets *flag when a sorted row holds an entry twice (warp per row).
__global__ void repeat_check_kernel(int32_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                                    int32_t* flag) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = warp; v < n; v += nwarps) {
        const int32_t b = rp[v], e = rp[v + 1];
        for (int32_t j = b + 1 + lane_id(); j < e; j += 32)
            if (col[j] == col[j - 1]) *flag = 1;
    }
}

int relabel_csr(ghb_workspace* ws, int32_t n, int64_t m, const int32_t* rp, const int32_t* col, const double* w,
                const int32_t* perm, int32_t* rp_out, int32_t* col_out, double* w_out) {
    if (m == 0) {
        GHB_CUDA_TRY(cudaMemsetAsync(rp_out, 0, sizeof(int32_t) * ((size_t)n + 1), ws->stream));
        return GHB_OK;
    }
    const int bits = bits_for_n(n);
    const bool want_vals = w != nullptr && w_out != nullptr;
    size_t sort_tmp = 0;
    {
        cub::DoubleBuffer<uint64_t> dk(nullptr, nullptr);
        cub::DoubleBuffer<uint32_t> dv(nullptr, nullptr);
        if (want_vals) cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, dk, dv, m, 0, 2 * bits);
        else cub::DeviceRadixSort::SortKeys(nullptr, sort_tmp, dk, m, 0, 2 * bits);
    }
    auto carve = [&](Carver& c, uint64_t** k0, uint64_t** k1, uint32_t** v0, uint32_t** v1, void** tmp) {
        *k0 = c.take<uint64_t>(m);
        *k1 = c.take<uint64_t>(m);
        *v0 = want_vals ? c.take<uint32_t>(m) : nullptr;
        *v1 = want_vals ? c.take<uint32_t>(m) : nullptr;
        *tmp = c.take<char>(sort_tmp);
    };
    uint64_t *k0, *k1;
    uint32_t *v0, *v1;
    void* tmp;
    Carver sizing(nullptr);
    carve(sizing, &k0, &k1, &v0, &v1, &tmp);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &k0, &k1, &v0, &v1, &tmp);
    const unsigned g = ws->num_sms * 8;
    GHB_TRY(launch(ws, relabel_keys_kernel, dim3(g), dim3(256), 0, n, rp, col, perm, bits, k0, v0));
    cub::DoubleBuffer<uint64_t> dk(k0, k1);
    cub::DoubleBuffer<uint32_t> dv(v0, v1);
    size_t tb = sort_tmp;
    if (want_vals) GHB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, dk, dv, m, 0, 2 * bits, ws->stream));
    else GHB_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp, tb, dk, m, 0, 2 * bits, ws->stream));
    ws->launches++;
    GHB_TRY(launch(ws, relabel_out_kernel, dim3(g), dim3(256), 0, (const uint64_t*)dk.Current(),
                   (const uint32_t*)(want_vals ? dv.Current() : nullptr), m, bits, w, col_out,
                   want_vals ? w_out : (double*)nullptr));
    GHB_TRY(launch(ws, rowptr_from_keys_kernel, dim3(grid_for(m + 1, 256, g)), dim3(256), 0,
                   (const uint64_t*)dk.Current(), m, bits, n, rp_out));
    return GHB_OK;
}

}  // namespace

int map_back_i32(ghb_workspace* ws, const ghb_graph* g, const int32_t* src_new, int32_t* dst_old) {
    return launch(ws, map_back_kernel<int32_t>, dim3(grid_for(g->n, 256, ws->num_sms * 8)), dim3(256), 0, g->n,
                  (const int32_t*)g->perm, src_new, dst_old);
}
int map_back_f64(ghb_workspace* ws, const ghb_graph* g, const double* src_new, double* dst_old) {
    return launch(ws, map_back_kernel<double>, dim3(grid_for(g->n, 256, ws->num_sms * 8)), dim3(256), 0, g->n,
                  (const int32_t*)g->perm, src_new, dst_old);
}
int map_back_i64(ghb_workspace* ws, const ghb_graph* g, const int64_t* src_new, int64_t* dst_old) {
    return launch(ws, map_back_kernel<int64_t>, dim3(grid_for(g->n, 256, ws->num_sms * 8)), dim3(256), 0, g->n,
                  (const int32_t*)g->perm, src_new, dst_old);
}

}  // namespace ghb

using namespace ghb;

extern "C" {

int ghb_graph_destroy(ghb_graph* g) {
    if (!g) return GHB_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(g->device);
    cudaFree(g->perm);
    cudaFree(g->iperm);
    cudaFree(g->rowptr);
    cudaFree(g->col);
    cudaFree(g->w);
    cudaFree(g->outdeg);
    cudaFree(g->sw_col);
    cudaFree(g->sw_w);
    cudaFree(g->sw_le);
    if (g->directed) {
        cudaFree(g->in_rowptr);
        cudaFree(g->in_col);
        cudaFree(g->in_w);
        cudaFree(g->all_rowptr);
        cudaFree(g->all_col);
    }
    cudaSetDevice(cur);
    delete g;
    return GHB_OK;
}

int ghb_graph_create(ghb_workspace* ws, int32_t n, const int32_t* out_rowptr, const int32_t* out_col,
                     const double* out_w, const int32_t* in_rowptr, const int32_t* in_col, const double* in_w,
                     ghb_graph** out) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(out, "NULL out");
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(out_rowptr, "NULL out_rowptr");
    *out = nullptr;
    cudaStream_t st = ws->stream;
    const bool directed = in_rowptr != nullptr && in_rowptr != out_rowptr;
    int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned);
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, out_rowptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    if (directed) GHB_CUDA_TRY(cudaMemcpyAsync(hp + 1, in_rowptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    ghb_graph* g = new ghb_graph();
    g->n = n;
    g->m = hp[0];
    g->m_in = directed ? hp[1] : hp[0];
    g->directed = directed;
    g->weighted = out_w != nullptr;
    GHB_CUDA_TRY(cudaGetDevice(&g->device));
    GHB_CUDA_TRY(cudaEventRecord(ws->ev_a, st));
    auto fail = [&](int s) {
        ghb_graph_destroy(g);
        return s;
    };
    int s = GHB_OK;
#define GG_TRY(x)                 \
    do {                          \
        s = (x);                  \
        if (s != GHB_OK) return fail(s); \
    } while (0)
    GG_TRY(dalloc(&g->perm, n, &g->device_bytes));
    GG_TRY(dalloc(&g->iperm, n, &g->device_bytes));
    GG_TRY(dalloc(&g->rowptr, (size_t)n + 1, &g->device_bytes));
    GG_TRY(dalloc(&g->col, (size_t)g->m, &g->device_bytes));
    if (g->weighted) GG_TRY(dalloc(&g->w, (size_t)g->m, &g->device_bytes));
    GG_TRY(dalloc(&g->outdeg, n, &g->device_bytes));
    if (directed) {
        GG_TRY(dalloc(&g->in_rowptr, (size_t)n + 1, &g->device_bytes));
        GG_TRY(dalloc(&g->in_col, (size_t)g->m_in, &g->device_bytes));
        if (in_w) GG_TRY(dalloc(&g->in_w, (size_t)g->m_in, &g->device_bytes));
    } else {
        g->in_rowptr = g->rowptr;
        g->in_col = g->col;
        g->in_w = g->w;
        g->all_rowptr = g->rowptr;
        g->all_col = g->col;
    }
    // 1. degree ranking -> perm / iperm / n_active
    {
        size_t sort_tmp = 0;
        cub::DoubleBuffer<uint64_t> dk0(nullptr, nullptr);
        cub::DeviceRadixSort::SortKeys(nullptr, sort_tmp, dk0, (int64_t)n, 0, 64);
        Carver sizing(nullptr);
        sizing.take<uint64_t>(n);
        sizing.take<uint64_t>(n);
        sizing.take<int32_t>(8);
        sizing.take<char>(sort_tmp);
        GG_TRY(ws_reserve(ws, sizing.off));
        Carver c(ws->scratch);
        uint64_t* k0 = c.take<uint64_t>(n);
        uint64_t* k1 = c.take<uint64_t>(n);
        int32_t* nact = c.take<int32_t>(8);
        void* tmp = c.take<char>(sort_tmp);
        const unsigned gr = grid_for(n, 256, ws->num_sms * 8);
        GG_TRY(launch(ws, degree_key_kernel, dim3(gr), dim3(256), 0, n, out_rowptr,
                      directed ? in_rowptr : (const int32_t*)nullptr, k0));
        cub::DoubleBuffer<uint64_t> dk(k0, k1);
        size_t tb = sort_tmp;
        cudaError_t e = cub::DeviceRadixSort::SortKeys(tmp, tb, dk, (int64_t)n, 0, 64, st);
        if (e != cudaSuccess) {
            set_error(std::string("degree sort: ") + cudaGetErrorString(e));
            return fail(GHB_ERR_CUDA);
        }
        ws->launches++;
        int32_t nn = n;
        e = cudaMemcpyAsync(nact, &nn, sizeof(int32_t), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return fail(GHB_ERR_CUDA);
        GG_TRY(launch(ws, perm_from_keys_kernel, dim3(gr), dim3(256), 0, n, (const uint64_t*)dk.Current(), g->perm,
                      g->iperm, nact));
        e = cudaMemcpyAsync(hp, nact, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(GHB_ERR_CUDA);
        g->n_active = hp[0];
    }
    // 2. relabelled CSRs
    GG_TRY(relabel_csr(ws, n, g->m, out_rowptr, out_col, out_w, g->perm, g->rowptr, g->col, g->w));
    if (directed) GG_TRY(relabel_csr(ws, n, g->m_in, in_rowptr, in_col, in_w, g->perm, g->in_rowptr, g->in_col, g->in_w));
    GG_TRY(launch(ws, outdeg_kernel, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0, n,
                  (const int32_t*)g->rowptr, g->outdeg));
    {
        int32_t* flag = reinterpret_cast<int32_t*>(ws->dev_small);
        GG_TRY(cudaMemsetAsync(flag, 0, sizeof(int32_t), st) == cudaSuccess ? GHB_OK : GHB_ERR_CUDA);
        GG_TRY(launch(ws, repeat_check_kernel, dim3(grid_for((int64_t)n * 32, 256, ws->num_sms * 8)), dim3(256), 0, n,
                      (const int32_t*)g->rowptr, (const int32_t*)g->col, flag));
        GG_TRY(cudaMemcpyAsync(hp + 2, flag, sizeof(int32_t), cudaMemcpyDeviceToHost, st) == cudaSuccess ? GHB_OK
                                                                                                      : GHB_ERR_CUDA);
        GG_TRY(cudaStreamSynchronize(st) == cudaSuccess ? GHB_OK : GHB_ERR_CUDA);
        g->repeats = hp[2] != 0;
    }
    if (directed) {
        GG_TRY(dalloc(&g->all_rowptr, (size_t)n + 1, &g->device_bytes));
        GG_TRY(dalloc(&g->all_col, (size_t)(g->m + g->m_in), &g->device_bytes));
        GG_TRY(ghb_csr_merge_in_out(ws, n, g->in_rowptr, g->in_col, g->rowptr, g->col, g->all_rowptr, g->all_col));
    }
    g->perm_host.resize(n);
    GG_TRY(cudaMemcpyAsync(g->perm_host.data(), g->perm, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st) == cudaSuccess
               ? GHB_OK
               : GHB_ERR_CUDA);
#undef GG_TRY
    GHB_CUDA_TRY(cudaEventRecord(ws->ev_b, st));
    GHB_CUDA_TRY(cudaEventSynchronize(ws->ev_b));
    cudaEventElapsedTime(&g->build_ms, ws->ev_a, ws->ev_b);
    *out = g;
    return GHB_OK;
}

int ghb_graph_info(const ghb_graph* g, int64_t* m, int32_t* n_active, int64_t* device_bytes, float* build_ms) {
    GHB_REQUIRE(g, "NULL graph");
    if (m) *m = g->m;
    if (n_active) *n_active = g->n_active;
    if (device_bytes) *device_bytes = g->device_bytes;
    if (build_ms) *build_ms = g->build_ms;
    return GHB_OK;
}

int ghb_graph_perm(const ghb_graph* g, const int32_t** perm, const int32_t** iperm) {
    GHB_REQUIRE(g, "NULL graph");
    if (perm) *perm = g->perm;
    if (iperm) *iperm = g->iperm;
    return GHB_OK;
}

}  // extern "C"
