// Community detection by synchronous label propagation (replaces
// GPU_CDLP_csr.cuh:28-210, which gathers every row's labels into an E-length
// array and segment-sorts all E keys each iteration).  Semantics of the CPU
// path (CPU_Community_Detection.hpp:12-64): the new label of v is the most
// frequent label among its row's entries, the smallest such label on ties; a
// vertex with an empty row keeps its label.  Labels start as vertex ids.
//
// Rows are classed by length once per call and each class has its own
// kernel, so no row pays for another's size:
//   0        keep the label
//   1..32    W lanes per row (W = 2..32): bitonic sort of the W labels in
//            registers through shuffles, run lengths by ballot
//   33..256  one warp per row, open-addressing (label -> count) table of 512
//            slots in shared memory
//   257..4096 one block per row, 8192-slot shared-memory table
//   > 4096   one block per row, table in global scratch sized to the row
// Every table ends with a max-reduction over (count, -label), which yields
// the most frequent label with the smallest-label tie-break.
#include <vector>

#include "common.cuh"
#include "edge_walk.cuh"

namespace ghb {
namespace {

constexpr int kCdlpClasses = 9;  // 0:empty 1..5: W=2,4,8,16,32  6:warp 7:block 8:global
constexpr int32_t kEmpty = -1;
constexpr int32_t kWarpSlots = 512;
constexpr int32_t kBlockSlots = 8192;
constexpr int kCdlpThreads = 256;

__device__ __forceinline__ int cdlp_class(int32_t d) {
    if (d == 0) return 0;
    if (d <= 2) return 1;
    if (d <= 4) return 2;
    if (d <= 8) return 3;
    if (d <= 16) return 4;
    if (d <= 32) return 5;
    if (d <= 256) return 6;
    if (d <= 4096) return 7;
    return 8;
}

__device__ __forceinline__ uint32_t hash_label(int32_t x) {
    uint32_t h = (uint32_t)x * 0x9E3779B1u;
    return h ^ (h >> 16);
}

// Packs (count, label) so that a larger key = more frequent, then smaller label.
__device__ __forceinline__ unsigned long long pack_best(uint32_t count, int32_t label) {
    return ((unsigned long long)count << 32) | (unsigned long long)(0x7FFFFFFFu - (uint32_t)label);
}
__device__ __forceinline__ int32_t unpack_label(unsigned long long k) {
    return (int32_t)(0x7FFFFFFFu - (uint32_t)(k & 0xFFFFFFFFull));
}

// Insert label x (valid lanes) into an open-addressing table of `slots`
// (power of two) entries, K = labels, C = counts.  Lanes of the warp holding
// the same label are merged first (one atomic per distinct label per warp),
// which matters once labels converge and a hub's row repeats a few labels.
// Every lane of the warp must call it.
__device__ __forceinline__ void table_insert_merged(int32_t* K, int32_t* C, uint32_t slots, int32_t x, bool valid) {
    const unsigned act = __ballot_sync(0xffffffffu, valid);
    if (!valid) return;
    const unsigned same = __match_any_sync(act, x);
    if (lane_id() != __ffs(same) - 1) return;
    uint32_t h = hash_label(x) & (slots - 1);
    while (true) {
        const int32_t k = atomicCAS(&K[h], kEmpty, x);
        if (k == kEmpty || k == x) {
            atomicAdd(&C[h], __popc(same));
            return;
        }
        h = (h + 1) & (slots - 1);
    }
}

// First iteration over labels that are all distinct, on rows without
// repeated entries: every count is 1, so the new label is the smallest
// neighbour label.  Lanes that share a row merge their minimum first.
struct MinLabelVisitor {
    const int32_t* lab;
    int32_t* out;
    __device__ bool want_row(int32_t) const { return true; }
    __device__ void operator()(int32_t u, int32_t v, int32_t) const {
        const int32_t x = lab[v];
        const unsigned same = __match_any_sync(__activemask(), u);
        const int32_t m = __reduce_min_sync(same, x);
        if (lane_id() == __ffs(same) - 1) atomicMin(out + u, m);
    }
    __device__ void finish() const {}
};

__global__ void cdlp_fill_max_kernel(int32_t* p, int32_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = 0x7FFFFFFF;
}

__global__ void cdlp_count_classes_kernel(int32_t n, const int32_t* __restrict__ rp, int32_t* counts) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = rp[v + 1] - rp[v];
        const int c = cdlp_class(d);
        const unsigned same = __match_any_sync(__activemask(), c);
        const int leader = __ffs(same) - 1;
        if (lane_id() == leader) atomicAdd(&counts[c], __popc(same));
        if (c == 8) atomicAdd(&counts[14], d);
    }
}

__global__ void cdlp_fill_classes_kernel(int32_t n, const int32_t* __restrict__ rp, int32_t* cursor,
                                         int32_t* rows) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int c = cdlp_class(rp[v + 1] - rp[v]);
        const unsigned active = __activemask();
        const unsigned same = __match_any_sync(active, c);
        const int leader = __ffs(same) - 1;
        int32_t base = 0;
        if (lane_id() == leader) base = atomicAdd(&cursor[c], __popc(same));
        base = __shfl_sync(same, base, leader);
        rows[base + __popc(same & ((1u << lane_id()) - 1u))] = (int32_t)v;
    }
}

__global__ void cdlp_iota_kernel(int32_t* p, int32_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = (int32_t)i;
}

__global__ void cdlp_copy_kernel(const int32_t* __restrict__ rows, int32_t count,
                                 const int32_t* __restrict__ lab, int32_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = rows[i];
        out[v] = lab[v];
    }
}

// W lanes per row, rows of 1..W entries.
template <int W>
__global__ void __launch_bounds__(kCdlpThreads) cdlp_small_kernel(
    const int32_t* __restrict__ rows, int32_t count, const int32_t* __restrict__ rp,
    const int32_t* __restrict__ col, const int32_t* __restrict__ lab, int32_t* __restrict__ out) {
    const int lane = lane_id();
    const int li = lane & (W - 1);
    const int64_t group = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / W;
    const int64_t ngroups = ((int64_t)gridDim.x * blockDim.x) / W;
    const int64_t rounds = ((int64_t)count + ngroups - 1) / ngroups;
    const unsigned gmask = (W == 32) ? 0xffffffffu : (((1u << W) - 1u) << (lane & ~(W - 1)));
    for (int64_t r = 0; r < rounds; ++r) {
        const int64_t i = group + r * ngroups;
        int32_t v = -1, b = 0, d = 0;
        if (i < count) {
            v = rows[i];
            b = rp[v];
            d = rp[v + 1] - b;
        }
        int32_t x = 0x7FFFFFFF;
        if (li < d) x = lab[col[b + li]];
        // Bitonic sort, ascending, within each W-lane group.
#pragma unroll
        for (int k = 2; k <= W; k <<= 1) {
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
                const int32_t y = __shfl_xor_sync(0xffffffffu, x, j);
                const bool up = (li & k) == 0;
                const bool lower = (li & j) == 0;
                x = (lower == up) ? min(x, y) : max(x, y);
            }
        }
        // Run starts inside the group, then run length = next start - start.
        const int32_t prev = __shfl_up_sync(0xffffffffu, x, 1);
        const bool valid = li < d;
        const bool start = valid && (li == 0 || prev != x);
        const unsigned starts = __ballot_sync(0xffffffffu, start) & gmask;
        unsigned long long best = 0;
        if (start) {
            const unsigned above = starts & ~((2u << lane) - 1u);
            const int next_li = above ? ((__ffs(above) - 1) & (W - 1)) : d;
            best = pack_best((uint32_t)(next_li - li), x);
        }
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) {
            const unsigned long long y = __shfl_xor_sync(0xffffffffu, best, o);
            best = y > best ? y : best;
        }
        if (li == 0 && i < count) out[v] = unpack_label(best);
    }
}

// One warp per row of 33..256 entries, 512-slot table per warp in shared memory.
__global__ void __launch_bounds__(kCdlpThreads) cdlp_warp_kernel(
    const int32_t* __restrict__ rows, int32_t count, const int32_t* __restrict__ rp,
    const int32_t* __restrict__ col, const int32_t* __restrict__ lab, int32_t* __restrict__ out) {
    __shared__ int32_t keys[kCdlpThreads / 32][kWarpSlots];
    __shared__ int32_t cnts[kCdlpThreads / 32][kWarpSlots];
    const int lane = lane_id();
    const int wib = threadIdx.x >> 5;
    int32_t* K = keys[wib];
    int32_t* C = cnts[wib];
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < count; i += nwarps) {
        const int32_t v = rows[i];
        const int32_t b = rp[v], e = rp[v + 1];
        for (int s = lane; s < kWarpSlots; s += 32) {
            K[s] = kEmpty;
            C[s] = 0;
        }
        __syncwarp();
        for (int32_t j0 = b; j0 < e; j0 += 32) {
            const int32_t j = j0 + lane;
            table_insert_merged(K, C, kWarpSlots, j < e ? lab[col[j]] : 0, j < e);
        }
        __syncwarp();
        unsigned long long best = 0;
        for (int s = lane; s < kWarpSlots; s += 32) {
            const int32_t k = K[s];
            if (k != kEmpty) {
                const unsigned long long key = pack_best((uint32_t)C[s], k);
                best = key > best ? key : best;
            }
        }
        best = warp_max(best);
        if (lane == 0) out[v] = unpack_label(best);
        __syncwarp();
    }
}

__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long x, unsigned long long* red) {
    x = warp_max(x);
    if (lane_id() == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned long long y = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0ull;
        y = warp_max(y);
        if (threadIdx.x == 0) red[0] = y;
    }
    __syncthreads();
    const unsigned long long r = red[0];
    __syncthreads();
    return r;
}

// One block per row of 257..4096 entries; 8192-slot table in dynamic smem.
__global__ void __launch_bounds__(kCdlpThreads) cdlp_block_kernel(
    const int32_t* __restrict__ rows, int32_t count, const int32_t* __restrict__ rp,
    const int32_t* __restrict__ col, const int32_t* __restrict__ lab, int32_t* __restrict__ out) {
    extern __shared__ int32_t smem[];
    __shared__ unsigned long long red[32];
    int32_t* K = smem;
    int32_t* C = smem + kBlockSlots;
    for (int64_t i = blockIdx.x; i < count; i += gridDim.x) {
        const int32_t v = rows[i];
        const int32_t b = rp[v], e = rp[v + 1];
        // Table of the next power of two >= 2 x the row (at most kBlockSlots).
        uint32_t cap = 512;
        while (cap < 2u * (uint32_t)(e - b) && cap < (uint32_t)kBlockSlots) cap <<= 1;
        for (uint32_t s = threadIdx.x; s < cap; s += blockDim.x) {
            K[s] = kEmpty;
            C[s] = 0;
        }
        __syncthreads();
        for (int32_t j0 = b; j0 < e; j0 += blockDim.x) {
            const int32_t j = j0 + threadIdx.x;
            table_insert_merged(K, C, cap, j < e ? lab[col[j]] : 0, j < e);
        }
        __syncthreads();
        unsigned long long best = 0;
        for (uint32_t s = threadIdx.x; s < cap; s += blockDim.x) {
            const int32_t k = K[s];
            if (k != kEmpty) {
                const unsigned long long key = pack_best((uint32_t)C[s], k);
                best = key > best ? key : best;
            }
        }
        best = block_max_u64(best, red);
        if (threadIdx.x == 0) out[v] = unpack_label(best);
    }
}

// One block per row of > 4096 entries (many blocks, round robin); each row
// owns a table in global scratch at tab_off[i] (the next power of two >= 2 x
// the row), left empty after use, so only the first call clears the pool.
__global__ void __launch_bounds__(kCdlpThreads) cdlp_global_kernel(
    const int32_t* __restrict__ rows, int32_t count, const int32_t* __restrict__ rp,
    const int32_t* __restrict__ col, const int32_t* __restrict__ lab, int32_t* __restrict__ out,
    int32_t* pool, const int64_t* __restrict__ tab_off) {
    __shared__ unsigned long long red[32];
    for (int64_t i = blockIdx.x; i < count; i += gridDim.x) {
        const int32_t v = rows[i];
        const int32_t b = rp[v], e = rp[v + 1];
        const uint32_t cap = (uint32_t)((tab_off[i + 1] - tab_off[i]) / 2);
        int32_t* K = pool + tab_off[i];
        int32_t* C = K + cap;
        for (int32_t j0 = b; j0 < e; j0 += blockDim.x) {
            const int32_t j = j0 + threadIdx.x;
            table_insert_merged(K, C, cap, j < e ? lab[col[j]] : 0, j < e);
        }
        __syncthreads();
        unsigned long long best = 0;
        for (uint32_t s = threadIdx.x; s < cap; s += blockDim.x) {
            const int32_t k = __ldcg(&K[s]);
            if (k != kEmpty) {
                const unsigned long long key = pack_best((uint32_t)__ldcg(&C[s]), k);
                best = key > best ? key : best;
                K[s] = kEmpty;  // leave the table empty for the next iteration
                C[s] = 0;
            }
        }
        best = block_max_u64(best, red);
        if (threadIdx.x == 0) out[v] = unpack_label(best);
    }
}

// Block per row: keys kEmpty, counts 0.
__global__ void cdlp_pool_clear_kernel(int32_t* pool, const int64_t* __restrict__ tab_off, int32_t count) {
    for (int64_t i = blockIdx.x; i < count; i += gridDim.x) {
        const int64_t b = tab_off[i], half = (tab_off[i + 1] - b) / 2;
        for (int64_t s = threadIdx.x; s < half; s += blockDim.x) {
            pool[b + s] = kEmpty;
            pool[b + half + s] = 0;
        }
    }
}

// Table sizes of the global-class rows: 2 x (next power of two >= 2 d) ints each.
__global__ void cdlp_table_sizes_kernel(const int32_t* __restrict__ rows, int32_t count,
                                        const int32_t* __restrict__ rp, int64_t* sizes) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = rows[i];
        int64_t cap = 1;
        while (cap < 2 * (int64_t)(rp[v + 1] - rp[v])) cap <<= 1;
        sizes[i] = 2 * cap;
    }
}

}  // namespace

// init_labels (device, may be NULL = vertex ids): starting label values.
// first_min: the rows repeat no entry and the starting labels are distinct,
// so the first iteration is a minimum over each row's labels.
int cdlp_run(ghb_workspace* ws, int32_t n, const int32_t* rp, const int32_t* col, int32_t iterations,
             int32_t* labels, const int32_t* init_labels, bool first_min) {
    cudaStream_t st = ws->stream;
    const unsigned grid_global = ws->num_sms * 8;
    int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned);

    // Pass 1: class sizes.
    Carver pre(nullptr);
    pre.take<int32_t>(16);
    GHB_TRY(ws_reserve(ws, pre.off + (size_t)n * 4 * 3 + 4096));
    int32_t* counts = reinterpret_cast<int32_t*>(ws->scratch);
    GHB_CUDA_TRY(cudaMemsetAsync(counts, 0, 16 * sizeof(int32_t), st));
    GHB_TRY(launch(ws, cdlp_count_classes_kernel, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0, n,
                   rp, counts));
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, counts, 16 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    int32_t cls[kCdlpClasses], off[kCdlpClasses + 1];
    off[0] = 0;
    for (int k = 0; k < kCdlpClasses; ++k) {
        cls[k] = hp[k];
        off[k + 1] = off[k] + cls[k];
    }
    // Global-class tables: 2 x (next power of two >= 2 d) ints per row, so
    // fewer than 8 ints per entry of those rows.
    const int64_t pool_bound = cls[8] > 0 ? 8 * (int64_t)hp[14] + 16 : 1;
    Carver sizing(nullptr);
    sizing.take<int32_t>(16);
    sizing.take<int32_t>(16);
    sizing.take<int32_t>(n);
    sizing.take<int32_t>(n);
    sizing.take<int32_t>(pool_bound);
    sizing.take<int64_t>((size_t)cls[8] + 1);
    WalkBuffers::carve(sizing, n);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    counts = c.take<int32_t>(16);
    int32_t* cursor = c.take<int32_t>(16);
    int32_t* rows = c.take<int32_t>(n);
    int32_t* other = c.take<int32_t>(n);
    int32_t* pool = c.take<int32_t>(pool_bound);
    int64_t* tab_off = c.take<int64_t>((size_t)cls[8] + 1);
    WalkBuffers wb = WalkBuffers::carve(c, n);

    for (int k = 0; k < kCdlpClasses; ++k) hp[k] = off[k];
    GHB_CUDA_TRY(cudaMemcpyAsync(cursor, hp, kCdlpClasses * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    GHB_TRY(launch(ws, cdlp_fill_classes_kernel, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0, n, rp,
                   cursor, rows));
    if (cls[8] > 0) {
        // Table offsets on the host (a few thousand rows), then an empty pool.
        GHB_TRY(launch(ws, cdlp_table_sizes_kernel, dim3(grid_for(cls[8], 256, ws->num_sms)), dim3(256), 0,
                       (const int32_t*)(rows + off[8]), cls[8], rp, tab_off));
        std::vector<int64_t> sz((size_t)cls[8] + 1);
        GHB_CUDA_TRY(cudaMemcpyAsync(sz.data(), tab_off, sizeof(int64_t) * cls[8], cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        int64_t acc = 0;
        for (int32_t i = 0; i < cls[8]; ++i) {
            const int64_t x = sz[i];
            sz[i] = acc;
            acc += x;
        }
        sz[cls[8]] = acc;
        GHB_REQUIRE(acc <= pool_bound, "CDLP table pool bound");
        GHB_CUDA_TRY(cudaMemcpyAsync(tab_off, sz.data(), sizeof(int64_t) * (cls[8] + 1), cudaMemcpyHostToDevice, st));
        // Empty = kEmpty keys (0xffffffff) and zero counts; the offsets are
        // even, so keys and counts are the two halves of each row's table.
        GHB_TRY(launch(ws, cdlp_pool_clear_kernel, dim3(grid_for(cls[8], 1, grid_global)), dim3(256), 0, pool,
                       (const int64_t*)tab_off, cls[8]));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));  // sz is read by the copy above
    }
    if (init_labels)
        GHB_CUDA_TRY(cudaMemcpyAsync(labels, init_labels, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
    else
        GHB_TRY(launch(ws, cdlp_iota_kernel, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0, labels, n));

    GHB_CUDA_TRY(cudaFuncSetAttribute(cdlp_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(2 * kBlockSlots * sizeof(int32_t))));
    int32_t* cur = labels;
    int32_t* nxt = other;
    const unsigned g = ws->num_sms * 8;
    for (int it = 0; it < iterations; ++it) {
        const int32_t* R = rows;
        if (it == 0 && first_min) {
            GHB_TRY(launch(ws, cdlp_fill_max_kernel, dim3(grid_for(n, 256, g)), dim3(256), 0, nxt, n));
            GHB_TRY(walk(ws, rp, col, (const int32_t*)nullptr, (const int32_t*)nullptr, (int64_t)n, (int64_t)n, wb,
                         MinLabelVisitor{(const int32_t*)cur, nxt}));
            if (cls[0]) GHB_TRY(launch(ws, cdlp_copy_kernel, dim3(grid_for(cls[0], 256, g)), dim3(256), 0, R + off[0], cls[0], (const int32_t*)cur, nxt));
            std::swap(cur, nxt);
            continue;
        }
        if (cls[0]) GHB_TRY(launch(ws, cdlp_copy_kernel, dim3(grid_for(cls[0], 256, g)), dim3(256), 0, R + off[0], cls[0], (const int32_t*)cur, nxt));
        if (cls[1]) GHB_TRY(launch(ws, cdlp_small_kernel<2>, dim3(grid_for((int64_t)cls[1] * 2, kCdlpThreads, g)), dim3(kCdlpThreads), 0, R + off[1], cls[1], rp, col, (const int32_t*)cur, nxt));
        if (cls[2]) GHB_TRY(launch(ws, cdlp_small_kernel<4>, dim3(grid_for((int64_t)cls[2] * 4, kCdlpThreads, g)), dim3(kCdlpThreads), 0, R + off[2], cls[2], rp, col, (const int32_t*)cur, nxt));
        if (cls[3]) GHB_TRY(launch(ws, cdlp_small_kernel<8>, dim3(grid_for((int64_t)cls[3] * 8, kCdlpThreads, g)), dim3(kCdlpThreads), 0, R + off[3], cls[3], rp, col, (const int32_t*)cur, nxt));
        if (cls[4]) GHB_TRY(launch(ws, cdlp_small_kernel<16>, dim3(grid_for((int64_t)cls[4] * 16, kCdlpThreads, g)), dim3(kCdlpThreads), 0, R + off[4], cls[4], rp, col, (const int32_t*)cur, nxt));
        if (cls[5]) GHB_TRY(launch(ws, cdlp_small_kernel<32>, dim3(grid_for((int64_t)cls[5] * 32, kCdlpThreads, g)), dim3(kCdlpThreads), 0, R + off[5], cls[5], rp, col, (const int32_t*)cur, nxt));
        if (cls[6]) GHB_TRY(launch(ws, cdlp_warp_kernel, dim3(grid_for((int64_t)cls[6] * 32, kCdlpThreads, g)), dim3(kCdlpThreads), 0, R + off[6], cls[6], rp, col, (const int32_t*)cur, nxt));
        if (cls[7]) GHB_TRY(launch(ws, cdlp_block_kernel, dim3(grid_for(cls[7], 1, ws->num_sms * 2)), dim3(kCdlpThreads), (size_t)(2 * kBlockSlots * sizeof(int32_t)), R + off[7], cls[7], rp, col, (const int32_t*)cur, nxt));
        if (cls[8]) GHB_TRY(launch(ws, cdlp_global_kernel, dim3(grid_for(cls[8], 1, grid_global)), dim3(kCdlpThreads), 0, R + off[8], cls[8], rp, col, (const int32_t*)cur, nxt, pool, (const int64_t*)tab_off));
        std::swap(cur, nxt);
    }
    if (cur != labels)
        GHB_CUDA_TRY(cudaMemcpyAsync(labels, cur, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
    return GHB_OK;
}

}  // namespace ghb

using namespace ghb;

extern "C" int ghb_cdlp(ghb_workspace* ws, int32_t n, const int32_t* all_rowptr, const int32_t* all_col,
                        int32_t iterations, int32_t* labels) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(all_rowptr && labels, "NULL argument");
    GHB_REQUIRE(iterations >= 0, "iterations < 0");
    return cdlp_run(ws, n, all_rowptr, all_col, iterations, labels, nullptr, false);
}
