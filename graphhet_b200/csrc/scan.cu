#include "scan.cuh"

namespace ghb {
namespace {

__device__ __forceinline__ int64_t block_inclusive_scan(int64_t x, int64_t* warp_buf, int64_t* total) {
    const int lane = lane_id(), wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_buf[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int64_t t = (lane < (int)(blockDim.x >> 5)) ? warp_buf[lane] : 0;
        int64_t ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += y;
        }
        warp_buf[lane] = ti - t;
        if (lane == 31) *total = ti;
    }
    __syncthreads();
    const int64_t r = x + warp_buf[wid];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const int32_t* __restrict__ in, int64_t count,
                                                                    int64_t* block_sums) {
    __shared__ int64_t wb[32];
    __shared__ int64_t tot;
    const int64_t base = blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int64_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < count) s += in[base + k];
    block_inclusive_scan(s, wb, &tot);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) scan_blocks_kernel(int64_t* block_sums, int64_t nblocks) {
    __shared__ int64_t wb[32];
    __shared__ int64_t tot;
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t b0 = 0; b0 < nblocks; b0 += blockDim.x) {
        const int64_t i = b0 + threadIdx.x;
        const int64_t x = i < nblocks ? block_sums[i] : 0;
        const int64_t incl = block_inclusive_scan(x, wb, &tot);
        const int64_t c = carry;
        if (i < nblocks) block_sums[i] = c + incl - x;
        __syncthreads();
        if (threadIdx.x == 0) carry = c + tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) block_sums[nblocks] = carry;
}

__global__ void __launch_bounds__(kScanThreads) scan_down_kernel(const int32_t* __restrict__ in, int64_t count,
                                                                  const int64_t* __restrict__ block_sums,
                                                                  int32_t* __restrict__ out, int64_t nblocks) {
    __shared__ int64_t wb[32];
    __shared__ int64_t tot;
    const int64_t base = blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems];
    int64_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < count) ? in[base + k] : 0;
        s += v[k];
    }
    const int64_t incl = block_inclusive_scan(s, wb, &tot);
    int64_t run = block_sums[blockIdx.x] + incl - s;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < count) out[base + k] = (int32_t)run;
        run += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[count] = (int32_t)block_sums[nblocks];
}

}  // namespace

int scan_exclusive_i32(ghb_workspace* ws, const int32_t* in, int32_t* out, int64_t count,
                       int64_t* block_sums) {
    const int64_t nblocks = (count + kScanTile - 1) / kScanTile;
    if (count == 0) {
        GHB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int32_t), ws->stream));
        return GHB_OK;
    }
    GHB_TRY(launch(ws, scan_reduce_kernel, dim3((unsigned)nblocks), dim3(kScanThreads), 0, in, count, block_sums));
    GHB_TRY(launch(ws, scan_blocks_kernel, dim3(1), dim3(1024), 0, block_sums, nblocks));
    GHB_TRY(launch(ws, scan_down_kernel, dim3((unsigned)nblocks), dim3(kScanThreads), 0, in, count,
                   (const int64_t*)block_sums, out, nblocks));
    return GHB_OK;
}

}  // namespace ghb
