// Shared kernel of the load-balanced row walker (edge_walk.cuh).
#include "edge_walk.cuh"

namespace ghb {

__global__ void __launch_bounds__(1024) walk_big_scan_kernel(const int32_t* __restrict__ rb,
                                                             const int32_t* __restrict__ re,
                                                             const int32_t* __restrict__ big,
                                                             const int32_t* big_tail,
                                                             int64_t* prefix) {
    __shared__ int64_t warp_tot[32];
    __shared__ int64_t carry;
    const int32_t count = *big_tail;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int32_t base = 0; base < count; base += blockDim.x) {
        const int32_t i = base + threadIdx.x;
        int64_t d = 0;
        if (i < count) {
            const int32_t u = big[i];
            d = re[u] - rb[u];
        }
        int64_t incl = d;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane_id() >= o) incl += x;
        }
        if (lane_id() == 31) warp_tot[threadIdx.x >> 5] = incl;
        __syncthreads();
        if (threadIdx.x < 32) {
            const int64_t t = (threadIdx.x < (blockDim.x >> 5)) ? warp_tot[threadIdx.x] : 0;
            int64_t ti = t;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t x = __shfl_up_sync(0xffffffffu, ti, o);
                if (lane_id() >= o) ti += x;
            }
            warp_tot[threadIdx.x] = ti - t;
        }
        __syncthreads();
        const int64_t c0 = carry;
        const int64_t mine = c0 + warp_tot[threadIdx.x >> 5] + incl;
        if (i < count) prefix[i] = mine - d;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = mine;
        __syncthreads();
    }
    if (threadIdx.x == 0) prefix[count] = carry;
}

}  // namespace ghb
