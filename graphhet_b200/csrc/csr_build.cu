// CSR builder: edge list -> (rowptr, col, w) with rows sorted by neighbour id,
// duplicates merged and, on request, self-loops dropped and both directions
// added.  This replaces toCSR's host flattening (GPU_csr.hpp:282-339) for
// edge-list inputs; the resulting layout is the reference's CSR layout.
//
// Method: pack each entry as key = (row << bits) | col, radix-sort the keys
// (CUB DeviceRadixSort, once per graph, not on any timed traversal path),
// keep the last entry of every equal-key run, and derive rowptr from the run
// boundaries without atomics.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "ghb_gen.h"

namespace ghb {
namespace {

__global__ void make_keys_kernel(const int32_t* __restrict__ src, const int32_t* __restrict__ dst,
                                 int64_t n_edges, int32_t n, int bits, int flags,
                                 uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                 int32_t* __restrict__ bad) {
    const bool sym = flags & GHB_BUILD_SYMMETRIZE;
    const bool drop = flags & GHB_BUILD_DROP_SELF_LOOPS;
    const bool tr = flags & GHB_BUILD_TRANSPOSE;
    const uint64_t sentinel = 1ull << (2 * bits);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_edges;
         i += (int64_t)gridDim.x * blockDim.x) {
        int32_t u = src[i], v = dst[i];
        bool ok = u >= 0 && u < n && v >= 0 && v < n;
        if (!ok) atomicExch(bad, 1);
        if (tr) {
            int32_t t = u;
            u = v;
            v = t;
        }
        uint64_t k = (ok && !(drop && u == v)) ? (((uint64_t)u << bits) | (uint64_t)v) : sentinel;
        if (sym) {
            uint64_t km = (ok && !(drop && u == v)) ? (((uint64_t)v << bits) | (uint64_t)u) : sentinel;
            keys[2 * i] = k;
            keys[2 * i + 1] = km;
            if (vals) {
                vals[2 * i] = (uint32_t)i;
                vals[2 * i + 1] = (uint32_t)i;
            }
        } else {
            keys[i] = k;
            if (vals) vals[i] = (uint32_t)i;
        }
    }
}

// keep[i] = 1 when entry i is the last of its equal-key run and not a sentinel.
__global__ void mark_last_kernel(const uint64_t* __restrict__ keys, int64_t count, uint64_t sentinel,
                                 int32_t* __restrict__ keep) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t k = keys[i];
        bool last = (i + 1 == count) || keys[i + 1] != k;
        keep[i] = (last && k != sentinel) ? 1 : 0;
    }
}

__global__ void compact_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                               const int32_t* __restrict__ keep, const int32_t* __restrict__ pos,
                               int64_t count, int bits, const double* __restrict__ w_in,
                               int weight_mode, uint64_t wstream, int transposed,
                               uint64_t* __restrict__ out_keys, int32_t* __restrict__ col,
                               double* __restrict__ w) {
    const uint64_t mask = (1ull << bits) - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (!keep[i]) continue;
        uint64_t k = keys[i];
        int32_t p = pos[i];
        uint32_t r = (uint32_t)(k >> bits), c = (uint32_t)(k & mask);
        out_keys[p] = k;
        col[p] = (int32_t)c;
        if (w) {
            if (w_in) {
                w[p] = w_in[vals[i]];
            } else {
                uint32_t a = transposed ? c : r, b = transposed ? r : c;
                w[p] = ghb_pair_weight(wstream, a, b, weight_mode);
            }
        }
    }
}

// rowptr from sorted row ids: rowptr[r] = number of entries with row < r.
__global__ void rowptr_from_sorted_kernel(const uint64_t* __restrict__ keys, int64_t m, int bits,
                                          int32_t n, int32_t* __restrict__ rowptr) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p <= m;
         p += (int64_t)gridDim.x * blockDim.x) {
        // Boundary between entry p-1 and entry p: rows (prev, cur] start at p.
        int64_t prev = (p == 0) ? -1 : (int64_t)(keys[p - 1] >> bits);
        int64_t cur = (p == m) ? (int64_t)n : (int64_t)(keys[p] >> bits);
        for (int64_t r = prev + 1; r <= cur; ++r) rowptr[r] = (int32_t)p;
    }
}

__global__ void transpose_keys_kernel(const int32_t* __restrict__ rowptr,
                                      const int32_t* __restrict__ col, int32_t n, int bits,
                                      uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    // One warp per row.
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = warp; u < n; u += nwarps) {
        int32_t b = rowptr[u], e = rowptr[u + 1];
        for (int32_t i = b + lane_id(); i < e; i += 32) {
            keys[i] = ((uint64_t)(uint32_t)col[i] << bits) | (uint64_t)u;
            if (vals) vals[i] = (uint32_t)i;
        }
    }
}

__global__ void transpose_out_kernel(const uint64_t* __restrict__ keys,
                                     const uint32_t* __restrict__ vals, int64_t m, int bits,
                                     const double* __restrict__ w, int32_t* __restrict__ t_col,
                                     double* __restrict__ t_w) {
    const uint64_t mask = (1ull << bits) - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        t_col[i] = (int32_t)(keys[i] & mask);
        if (t_w) t_w[i] = w[vals[i]];
    }
}

__global__ void merge_rowptr_kernel(const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                                    int32_t n, int32_t* __restrict__ out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v <= n;
         v += (int64_t)gridDim.x * blockDim.x)
        out[v] = a[v] + b[v];
}

__global__ void merge_rows_kernel(const int32_t* __restrict__ in_rp, const int32_t* __restrict__ in_col,
                                  const int32_t* __restrict__ out_rp,
                                  const int32_t* __restrict__ out_col, int32_t n,
                                  const int32_t* __restrict__ all_rp, int32_t* __restrict__ all_col) {
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = warp; v < n; v += nwarps) {
        int32_t dst = all_rp[v];
        int32_t ib = in_rp[v], ie = in_rp[v + 1];
        for (int32_t i = ib + lane_id(); i < ie; i += 32) all_col[dst + (i - ib)] = in_col[i];
        dst += ie - ib;
        int32_t ob = out_rp[v], oe = out_rp[v + 1];
        for (int32_t i = ob + lane_id(); i < oe; i += 32) all_col[dst + (i - ob)] = out_col[i];
    }
}

int bits_for(int32_t n) {
    int bits = 1;
    while (bits < 31 && (1ll << bits) < (int64_t)n) ++bits;
    return bits;
}

}  // namespace
}  // namespace ghb

using namespace ghb;

extern "C" {

int ghb_csr_build(ghb_workspace* ws, int32_t n, const int32_t* src, const int32_t* dst,
                  const double* w_in, int64_t n_edges, int32_t flags, int32_t weight_mode,
                  uint64_t weight_seed, int32_t* rowptr, int32_t* col, double* w, int64_t* m_out) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(n_edges >= 0 && n_edges < (1ll << 32), "n_edges out of range");
    GHB_REQUIRE(rowptr && m_out, "NULL rowptr / m_out");
    GHB_REQUIRE(n_edges == 0 || (src && dst && col), "NULL edge arrays");
    GHB_REQUIRE(weight_mode >= 0 && weight_mode <= 2, "bad weight_mode");
    const bool sym = flags & GHB_BUILD_SYMMETRIZE;
    const int64_t count = sym ? 2 * n_edges : n_edges;
    GHB_REQUIRE(count < (1ll << 31), "too many entries for int32 offsets");
    const int bits = bits_for(n);
    const int end_bit = 2 * bits + 1;  // + sentinel bit
    const uint64_t sentinel = 1ull << (2 * bits);
    const bool want_vals = (w_in != nullptr) && (w != nullptr);

    // Scratch: keys x2, vals x2, keep, pos, compacted keys, CUB temp.
    size_t sort_tmp = 0, scan_tmp = 0;
    {
        cub::DoubleBuffer<uint64_t> dk(nullptr, nullptr);
        cub::DoubleBuffer<uint32_t> dv(nullptr, nullptr);
        if (want_vals)
            cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, dk, dv, (int64_t)count, 0, end_bit);
        else
            cub::DeviceRadixSort::SortKeys(nullptr, sort_tmp, dk, (int64_t)count, 0, end_bit);
        cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, (int32_t*)nullptr, (int32_t*)nullptr,
                                      (int64_t)count);
    }
    auto carve = [&](Carver& c, uint64_t** k0, uint64_t** k1, uint32_t** v0, uint32_t** v1,
                     int32_t** keep, int32_t** pos, void** tmp, int32_t** bad) {
        *k0 = c.take<uint64_t>(count + 1);
        *k1 = c.take<uint64_t>(count + 1);
        *v0 = want_vals ? c.take<uint32_t>(count + 1) : nullptr;
        *v1 = want_vals ? c.take<uint32_t>(count + 1) : nullptr;
        *keep = c.take<int32_t>(count + 1);
        *pos = c.take<int32_t>(count + 1);
        *tmp = c.take<char>(sort_tmp > scan_tmp ? sort_tmp : scan_tmp);
        *bad = c.take<int32_t>(4);
    };
    uint64_t *k0, *k1;
    uint32_t *v0, *v1;
    int32_t *keep, *pos, *bad;
    void* tmp;
    Carver sizing(nullptr);
    carve(sizing, &k0, &k1, &v0, &v1, &keep, &pos, &tmp, &bad);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &k0, &k1, &v0, &v1, &keep, &pos, &tmp, &bad);

    GHB_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int32_t), ws->stream));
    const unsigned g = ws->num_sms * 8;
    if (n_edges > 0) {
        GHB_TRY(launch(ws, make_keys_kernel, dim3(g), dim3(256), 0, src, dst, n_edges, n, bits,
                       (int)flags, k0, v0, bad));
        cub::DoubleBuffer<uint64_t> dk(k0, k1);
        cub::DoubleBuffer<uint32_t> dv(v0, v1);
        size_t tb = sort_tmp;
        if (want_vals)
            GHB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, dk, dv, (int64_t)count, 0, end_bit,
                                                         ws->stream));
        else
            GHB_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp, tb, dk, (int64_t)count, 0, end_bit,
                                                        ws->stream));
        ws->launches++;
        uint64_t* keys = dk.Current();
        uint32_t* vals = want_vals ? dv.Current() : nullptr;
        uint64_t* other = dk.Alternate();
        GHB_TRY(launch(ws, mark_last_kernel, dim3(g), dim3(256), 0, (const uint64_t*)keys, count,
                       sentinel, keep));
        size_t sb = scan_tmp;
        GHB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, sb, keep, pos, (int64_t)count, ws->stream));
        ws->launches++;
        // m = pos[count-1] + keep[count-1]
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, pos + count - 1, sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, ws->stream));
        GHB_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<int32_t*>(ws->host_pinned) + 1, keep + count - 1,
                                     sizeof(int32_t), cudaMemcpyDeviceToHost, ws->stream));
        GHB_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<int32_t*>(ws->host_pinned) + 2, bad,
                                     sizeof(int32_t), cudaMemcpyDeviceToHost, ws->stream));
        GHB_CUDA_TRY(cudaStreamSynchronize(ws->stream));
        const int32_t* hp = reinterpret_cast<const int32_t*>(ws->host_pinned);
        if (hp[2]) {
            set_error("invalid argument: edge endpoint outside [0, n)");
            return GHB_ERR_INVALID_ARGUMENT;
        }
        const int64_t m = (int64_t)hp[0] + hp[1];
        GHB_TRY(launch(ws, compact_kernel, dim3(g), dim3(256), 0, (const uint64_t*)keys,
                       (const uint32_t*)vals, (const int32_t*)keep, (const int32_t*)pos, count,
                       bits, w_in, (int)(w_in ? 0 : weight_mode),
                       ghb_stream(weight_seed, GHB_PURPOSE_WEIGHT),
                       (int)((flags & GHB_BUILD_TRANSPOSE) != 0), other, col,
                       (weight_mode != 0 || w_in) ? w : (double*)nullptr));
        GHB_TRY(launch(ws, rowptr_from_sorted_kernel, dim3(grid_for(m + 1, 256, g)), dim3(256), 0,
                       (const uint64_t*)other, m, bits, n, rowptr));
        *m_out = m;
    } else {
        GHB_CUDA_TRY(cudaMemsetAsync(rowptr, 0, sizeof(int32_t) * ((size_t)n + 1), ws->stream));
        *m_out = 0;
    }
    return GHB_OK;
}

int ghb_csr_transpose(ghb_workspace* ws, int32_t n, int64_t m, const int32_t* rowptr,
                      const int32_t* col, const double* w, int32_t* t_rowptr, int32_t* t_col,
                      double* t_w) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n >= 1 && m >= 0 && m < (1ll << 31), "bad sizes");
    GHB_REQUIRE(rowptr && t_rowptr, "NULL rowptr");
    if (m == 0) {
        GHB_CUDA_TRY(cudaMemsetAsync(t_rowptr, 0, sizeof(int32_t) * ((size_t)n + 1), ws->stream));
        return GHB_OK;
    }
    GHB_REQUIRE(col && t_col, "NULL col");
    const int bits = bits_for(n);
    const bool want_vals = (w != nullptr && t_w != nullptr);
    size_t sort_tmp = 0;
    {
        cub::DoubleBuffer<uint64_t> dk(nullptr, nullptr);
        cub::DoubleBuffer<uint32_t> dv(nullptr, nullptr);
        if (want_vals)
            cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, dk, dv, m, 0, 2 * bits);
        else
            cub::DeviceRadixSort::SortKeys(nullptr, sort_tmp, dk, m, 0, 2 * bits);
    }
    Carver sizing(nullptr);
    sizing.take<uint64_t>(m);
    sizing.take<uint64_t>(m);
    if (want_vals) {
        sizing.take<uint32_t>(m);
        sizing.take<uint32_t>(m);
    }
    sizing.take<char>(sort_tmp);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    uint64_t* k0 = c.take<uint64_t>(m);
    uint64_t* k1 = c.take<uint64_t>(m);
    uint32_t* v0 = want_vals ? c.take<uint32_t>(m) : nullptr;
    uint32_t* v1 = want_vals ? c.take<uint32_t>(m) : nullptr;
    void* tmp = c.take<char>(sort_tmp);
    const unsigned g = ws->num_sms * 8;
    GHB_TRY(launch(ws, transpose_keys_kernel, dim3(g), dim3(256), 0, rowptr, col, n, bits, k0, v0));
    cub::DoubleBuffer<uint64_t> dk(k0, k1);
    cub::DoubleBuffer<uint32_t> dv(v0, v1);
    size_t tb = sort_tmp;
    if (want_vals)
        GHB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, dk, dv, m, 0, 2 * bits, ws->stream));
    else
        GHB_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp, tb, dk, m, 0, 2 * bits, ws->stream));
    ws->launches++;
    GHB_TRY(launch(ws, transpose_out_kernel, dim3(g), dim3(256), 0, (const uint64_t*)dk.Current(),
                   (const uint32_t*)(want_vals ? dv.Current() : nullptr), m, bits, w, t_col,
                   want_vals ? t_w : (double*)nullptr));
    GHB_TRY(launch(ws, rowptr_from_sorted_kernel, dim3(grid_for(m + 1, 256, g)), dim3(256), 0,
                   (const uint64_t*)dk.Current(), m, bits, n, t_rowptr));
    return GHB_OK;
}

int ghb_csr_merge_in_out(ghb_workspace* ws, int32_t n, const int32_t* in_rowptr,
                         const int32_t* in_col, const int32_t* out_rowptr, const int32_t* out_col,
                         int32_t* all_rowptr, int32_t* all_col) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(in_rowptr && out_rowptr && all_rowptr, "NULL rowptr");
    const unsigned g = ws->num_sms * 8;
    GHB_TRY(launch(ws, merge_rowptr_kernel, dim3(grid_for(n + 1, 256, g)), dim3(256), 0, in_rowptr,
                   out_rowptr, n, all_rowptr));
    GHB_TRY(launch(ws, merge_rows_kernel, dim3(g), dim3(256), 0, in_rowptr, in_col, out_rowptr,
                   out_col, n, (const int32_t*)all_rowptr, all_col));
    return GHB_OK;
}

}  // extern "C"
