// Load-balanced iteration over the CSR entries of a set of rows.
//
// A warp takes 32 rows.  Rows of 32 .. kWalkBig-1 entries are walked by the
// whole warp, one row at a time (each step reads 32 consecutive entries).
// Shorter rows are gathered warp-wide over an exclusive scan of their
// lengths, so a step again reads 32 consecutive entries of the packed rows.
// Rows of kWalkBig or more entries are deferred to a list and walked
// entry-parallel by the whole grid (walk_big_kernel), so one hub row never
// serialises a warp.
//
// The visitor F is a small struct copied into each thread: operator()(u, v, j)
// is called for entry j (u -> v), finish() once per thread at the end.
#pragma once

#include "common.cuh"

namespace ghb {

constexpr int32_t kWalkBig = 4096;

// Row u spans entries [rb[u], re[u]) (a CSR passes rb = rowptr,
// re = rowptr + 1; other views select part of every row).
template <class F>
__device__ __forceinline__ void walk_rows(const int32_t* __restrict__ rb, const int32_t* __restrict__ re,
                                          const int32_t* __restrict__ col,
                                          const int32_t* __restrict__ queue, int64_t count,
                                          int32_t* big, int32_t* big_tail, F& f) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * 32; base < count; base += nwarps * 32) {
        const int64_t i = base + lane;
        int32_t u = -1, b = 0, e = 0;
        if (i < count) {
            u = queue ? queue[i] : (int32_t)i;
            if (f.want_row(u)) {
                b = rb[u];
                e = re[u];
                if (big && e - b >= kWalkBig) {
                    int32_t pos = warp_append_active(big_tail);
                    big[pos] = u;
                    e = b;
                }
            }
        }
        unsigned med = __ballot_sync(0xffffffffu, e - b >= 32);
        while (med) {
            const int leader = __ffs(med) - 1;
            const int32_t lu = __shfl_sync(0xffffffffu, u, leader);
            const int32_t lb = __shfl_sync(0xffffffffu, b, leader);
            const int32_t le = __shfl_sync(0xffffffffu, e, leader);
            for (int32_t j = lb + lane; j < le; j += 32) f(lu, col[j], j);
            med &= med - 1;
        }
        if (e - b >= 32) e = b;
        const int32_t d = e - b;
        int32_t incl = d;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int32_t x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += x;
        }
        const int32_t excl = incl - d;
        const int32_t total = __shfl_sync(0xffffffffu, incl, 31);
        for (int32_t k0 = 0; k0 < total; k0 += 32) {
            const int32_t k = k0 + lane;
            int owner = 0;
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1) {
                const int cand = owner + s;
                const int32_t ev = __shfl_sync(0xffffffffu, excl, cand);
                if (ev <= k) owner = cand;
            }
            const int32_t ou = __shfl_sync(0xffffffffu, u, owner);
            const int32_t ob = __shfl_sync(0xffffffffu, b, owner);
            const int32_t oe = __shfl_sync(0xffffffffu, excl, owner);
            if (k < total) {
                const int32_t j = ob + (k - oe);
                f(ou, col[j], j);
            }
        }
    }
}

template <class F>
__global__ void __launch_bounds__(256) walk_kernel(const int32_t* __restrict__ rb, const int32_t* __restrict__ re,
                                                   const int32_t* __restrict__ col,
                                                   const int32_t* __restrict__ queue,
                                                   const int32_t* count_dev, int64_t count_host,
                                                   int32_t* big, int32_t* big_tail, F f) {
    const int64_t count = count_dev ? (int64_t)*count_dev : count_host;
    walk_rows(rb, re, col, queue, count, big, big_tail, f);
    f.finish();
}

// Exclusive prefix of the deferred rows' lengths; prefix[count] = total.
__global__ void __launch_bounds__(1024) walk_big_scan_kernel(const int32_t* __restrict__ rb,
                                                             const int32_t* __restrict__ re,
                                                             const int32_t* __restrict__ big,
                                                             const int32_t* big_tail,
                                                             int64_t* prefix);

template <class F>
__global__ void __launch_bounds__(256) walk_big_kernel(const int32_t* __restrict__ rb,
                                                       const int32_t* __restrict__ col,
                                                       const int32_t* __restrict__ big,
                                                       const int32_t* big_tail,
                                                       const int64_t* __restrict__ prefix, F f) {
    const int32_t count = *big_tail;
    if (count > 0) {
        const int64_t total = prefix[count];
        const int lane = lane_id();
        const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
        const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
        // 128-entry chunks cross at most one row boundary (rows >= kWalkBig).
        for (int64_t c0 = warp * 128; c0 < total; c0 += nwarps * 128) {
            int32_t lo = 0, hi = count - 1;
            while (lo < hi) {
                const int32_t mid = (lo + hi + 1) >> 1;
                if (prefix[mid] <= c0) lo = mid;
                else hi = mid - 1;
            }
            const int64_t start0 = prefix[lo];
            const int64_t start1 = prefix[lo + 1];
            const int32_t u0 = big[lo];
            const int32_t b0 = rb[u0];
            int32_t u1 = u0, b1 = 0;
            if (start1 < c0 + 128 && lo + 1 < count) {
                u1 = big[lo + 1];
                b1 = rb[u1];
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int64_t p = c0 + lane + 32 * k;
                if (p < total) {
                    const bool first = p < start1;
                    const int32_t j = first ? b0 + (int32_t)(p - start0) : b1 + (int32_t)(p - start1);
                    f(first ? u0 : u1, col[j], j);
                }
            }
        }
    }
    f.finish();
}

// Scratch for one walk: deferred-row list, its count and prefix.
struct WalkBuffers {
    int32_t* big;
    int32_t* big_tail;
    int64_t* prefix;
    static WalkBuffers carve(Carver& c, int64_t rows) {
        WalkBuffers w;
        w.big = c.take<int32_t>(rows > 0 ? rows : 1);
        w.big_tail = c.take<int32_t>(8);
        w.prefix = c.take<int64_t>((rows > 0 ? rows : 1) + 1);
        return w;
    }
};

// Walk every entry [rb[u], re[u]) of the given rows (queue == nullptr: rows
// [0, count)).  count_dev, when set, is read on the device instead of
// count_host.
template <class F>
int walk_range(ghb_workspace* ws, const int32_t* rb, const int32_t* re, const int32_t* col, const int32_t* queue,
               const int32_t* count_dev, int64_t count_host, int64_t grid_rows, const WalkBuffers& wb, const F& f) {
    const unsigned gmax = ws->num_sms * 8;
    GHB_CUDA_TRY(cudaMemsetAsync(wb.big_tail, 0, sizeof(int32_t), ws->stream));
    GHB_TRY(launch(ws, walk_kernel<F>, dim3(grid_for(grid_rows * 32, 256, gmax)), dim3(256), 0,
                   rb, re, col, queue, count_dev, count_host, wb.big, wb.big_tail, f));
    GHB_TRY(launch(ws, walk_big_scan_kernel, dim3(1), dim3(1024), 0, rb, re,
                   (const int32_t*)wb.big, (const int32_t*)wb.big_tail, wb.prefix));
    GHB_TRY(launch(ws, walk_big_kernel<F>, dim3(gmax), dim3(256), 0, rb, col,
                   (const int32_t*)wb.big, (const int32_t*)wb.big_tail,
                   (const int64_t*)wb.prefix, f));
    return GHB_OK;
}

// Walk every entry of the given rows of a CSR.
template <class F>
int walk(ghb_workspace* ws, const int32_t* rowptr, const int32_t* col, const int32_t* queue,
         const int32_t* count_dev, int64_t count_host, int64_t grid_rows, const WalkBuffers& wb,
         const F& f) {
    return walk_range(ws, rowptr, rowptr + 1, col, queue, count_dev, count_host, grid_rows, wb, f);
}

}  // namespace ghb
