// Seeded synthetic graph generators (RMAT, 2-D grid, Erdos-Renyi).  The edge
// lists are pure functions of (seed, edge number) defined in ghb_gen.h, so a
// CPU restatement reproduces them exactly.
#include "common.cuh"
#include "ghb_gen.h"

namespace ghb {
namespace {

__global__ void rmat_kernel(int scale, int64_t n_edges, uint64_t stream, ghb_rmat_thresholds t,
                            int permute, ghb_perm perm, int32_t* __restrict__ src,
                            int32_t* __restrict__ dst) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_edges;
         e += (int64_t)gridDim.x * blockDim.x) {
        uint32_t u, v;
        ghb_rmat_edge(stream, t, scale, (uint64_t)e, &u, &v);
        if (permute) {
            u = ghb_perm_apply(&perm, u);
            v = ghb_perm_apply(&perm, v);
        }
        src[e] = (int32_t)u;
        dst[e] = (int32_t)v;
    }
}

__global__ void grid_kernel(int32_t rows, int32_t cols, int32_t* __restrict__ src,
                            int32_t* __restrict__ dst) {
    // Edges 0 .. rows*(cols-1)-1 go right, the rest go down.
    int64_t right = (int64_t)rows * (cols - 1);
    int64_t down = (int64_t)(rows - 1) * cols;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < right + down;
         e += (int64_t)gridDim.x * blockDim.x) {
        int64_t u, v;
        if (e < right) {
            int64_t r = e / (cols - 1), c = e % (cols - 1);
            u = r * cols + c;
            v = u + 1;
        } else {
            int64_t k = e - right;
            u = k;
            v = k + cols;
        }
        src[e] = (int32_t)u;
        dst[e] = (int32_t)v;
    }
}

__global__ void er_kernel(uint32_t n, int64_t n_edges, uint64_t stream, int32_t* __restrict__ src,
                          int32_t* __restrict__ dst) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_edges;
         e += (int64_t)gridDim.x * blockDim.x) {
        uint32_t u, v;
        ghb_er_edge(stream, n, (uint64_t)e, &u, &v);
        src[e] = (int32_t)u;
        dst[e] = (int32_t)v;
    }
}

// Chung-Lu power-law graph: both endpoints drawn with probability
// proportional to (i+1)^-theta, theta = 1/(gamma-1), through the inverse of
// the continuous cumulative weight, then scattered by the seed's permutation.
__global__ void powerlaw_kernel(int scale, int64_t n_edges, double theta, uint64_t stream, ghb_perm perm,
                                int32_t* __restrict__ src, int32_t* __restrict__ dst) {
    const double n = (double)(1u << scale);
    const double q = 1.0 - theta;
    const double span = pow(n + 1.0, q) - 1.0;
    const uint32_t last = (1u << scale) - 1u;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_edges;
         e += (int64_t)gridDim.x * blockDim.x) {
        uint32_t id[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const double u = (double)(ghb_draw(stream, 2 * (uint64_t)e + k) >> 11) * 0x1.0p-53;
            const double x = pow(1.0 + u * span, 1.0 / q) - 1.0;
            uint32_t i = x <= 0.0 ? 0u : (x >= (double)last ? last : (uint32_t)x);
            id[k] = ghb_perm_apply(&perm, i);
        }
        src[e] = (int32_t)id[0];
        dst[e] = (int32_t)id[1];
    }
}

__global__ void keep_not_dangling_kernel(int64_t n_edges, const int32_t* __restrict__ src, uint64_t dstream,
                                         uint32_t threshold, uint8_t* __restrict__ keep) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_edges;
         e += (int64_t)gridDim.x * blockDim.x)
        keep[e] = ghb_is_dangling(dstream, (uint32_t)src[e], threshold) ? 0 : 1;
}

}  // namespace
}  // namespace ghb

using namespace ghb;

extern "C" {

int ghb_gen_rmat(ghb_workspace* ws, int32_t scale, int64_t n_edges, uint64_t seed, double a,
                 double b, double c, int32_t permute, int32_t* src, int32_t* dst) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(scale >= 0 && scale <= 30, "scale must be in [0, 30]");
    GHB_REQUIRE(n_edges >= 0, "n_edges < 0");
    GHB_REQUIRE(n_edges == 0 || (src && dst), "NULL output");
    GHB_REQUIRE(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0, "bad RMAT probabilities");
    ghb_rmat_thresholds t = ghb_rmat_make_thresholds(a, b, c);
    ghb_perm perm = ghb_perm_make(seed, scale);
    uint64_t stream = ghb_stream(seed, GHB_PURPOSE_RMAT);
    unsigned g = grid_for(n_edges, 256, ws->num_sms * 16);
    return launch(ws, rmat_kernel, dim3(g), dim3(256), 0, (int)scale, n_edges, stream, t,
                  (int)permute, perm, src, dst);
}

int ghb_gen_grid(ghb_workspace* ws, int32_t rows, int32_t cols, int32_t* src, int32_t* dst) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(rows >= 1 && cols >= 1, "rows and cols must be >= 1");
    GHB_REQUIRE((int64_t)rows * cols < (1ll << 31), "grid too large for int32 ids");
    int64_t ne = (int64_t)rows * (cols - 1) + (int64_t)(rows - 1) * cols;
    if (ne == 0) return GHB_OK;
    GHB_REQUIRE(src && dst, "NULL output");
    unsigned g = grid_for(ne, 256, ws->num_sms * 16);
    return launch(ws, grid_kernel, dim3(g), dim3(256), 0, rows, cols, src, dst);
}

int ghb_gen_er(ghb_workspace* ws, int32_t n, int64_t n_edges, uint64_t seed, int32_t* src,
               int32_t* dst) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(n_edges >= 0, "n_edges < 0");
    if (n_edges == 0) return GHB_OK;
    GHB_REQUIRE(src && dst, "NULL output");
    unsigned g = grid_for(n_edges, 256, ws->num_sms * 16);
    return launch(ws, er_kernel, dim3(g), dim3(256), 0, (uint32_t)n, n_edges,
                  ghb_stream(seed, GHB_PURPOSE_ER), src, dst);
}

int ghb_gen_dangling_keep(ghb_workspace* ws, int64_t n_edges, const int32_t* src, uint64_t seed, double fraction,
                          uint8_t* keep) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n_edges >= 0, "n_edges < 0");
    GHB_REQUIRE(fraction >= 0.0 && fraction <= 1.0, "fraction outside [0, 1]");
    if (n_edges == 0) return GHB_OK;
    GHB_REQUIRE(src && keep, "NULL argument");
    const uint32_t threshold = fraction >= 1.0 ? 0xffffffffu : (uint32_t)(fraction * 4294967296.0);
    return launch(ws, keep_not_dangling_kernel, dim3(grid_for(n_edges, 256, ws->num_sms * 16)), dim3(256), 0,
                  n_edges, src, ghb_stream(seed, GHB_PURPOSE_DANGLING), threshold, keep);
}

int ghb_gen_powerlaw(ghb_workspace* ws, int32_t scale, int64_t n_edges, double exponent, uint64_t seed,
                     int32_t* src, int32_t* dst) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(scale >= 1 && scale <= 30, "scale must be in [1, 30]");
    GHB_REQUIRE(n_edges >= 0, "n_edges < 0");
    GHB_REQUIRE(exponent > 2.0 && exponent < 10.0, "exponent must be in (2, 10)");
    if (n_edges == 0) return GHB_OK;
    GHB_REQUIRE(src && dst, "NULL output");
    unsigned g = grid_for(n_edges, 256, ws->num_sms * 16);
    return launch(ws, powerlaw_kernel, dim3(g), dim3(256), 0, (int)scale, n_edges, 1.0 / (exponent - 1.0),
                  ghb_stream(seed, GHB_PURPOSE_POWERLAW), ghb_perm_make(seed, scale), src, dst);
}

}  // extern "C"
