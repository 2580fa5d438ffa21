// Weakly connected components by lock-free union-find: every CSR entry
// (u, v) links the larger of the two roots under the smaller one with one
// atomicCAS, and a final pass points every vertex at its root.  Because a
// root is only ever linked under a smaller id, each component's root is its
// smallest vertex id, which is the label the reference produces
// (GPU_WCC_csr.cuh:40-81 hooks larger onto smaller the same way;
// CPU_connected_components.hpp:29-44 converges to the same labelling).
// The reference's two sampling rounds + full_link + compress become one
// load-balanced pass over all entries (edge_walk.cuh) + one compress pass.
//
// The label array is the union-find forest (int32[n], L2 resident at
// n = 2^24); parent reads bypass L1 (ld.cg) so updates from other SMs are
// seen without going through stale lines.
#include "common.cuh"
#include "edge_walk.cuh"

namespace ghb {
namespace {

__device__ __forceinline__ int32_t wcc_find(int32_t* parent, int32_t x) {
    int32_t p = __ldcg(parent + x);
    if (p == x) return x;
    int32_t prev = x, next;
    while (p > (next = __ldcg(parent + p))) {
        parent[prev] = next;  // prev is not a root: point it at an ancestor
        prev = p;
        p = next;
    }
    return p;
}

__device__ __forceinline__ void wcc_unite(int32_t* parent, int32_t u, int32_t v) {
    int32_t ru = wcc_find(parent, u), rv = wcc_find(parent, v);
    while (ru != rv) {
        if (ru < rv) {
            const int32_t t = ru;
            ru = rv;
            rv = t;
        }
        const int32_t old = atomicCAS(parent + ru, ru, rv);
        if (old == ru) break;
        ru = wcc_find(parent, old);
        rv = wcc_find(parent, rv);
    }
}

struct UniteVisitor {
    int32_t* parent;
    __device__ bool want_row(int32_t) const { return true; }
    __device__ void operator()(int32_t u, int32_t v, int32_t) const {
        if (u != v) wcc_unite(parent, u, v);
    }
    __device__ void finish() const {}
};

__global__ void iota_kernel(int32_t* p, int32_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = (int32_t)i;
}

__global__ void wcc_compress_kernel(int32_t* parent, int32_t n) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        int32_t p = __ldcg(parent + v);
        int32_t q;
        while (p != (q = __ldcg(parent + p))) p = q;
        parent[v] = p;
    }
}

}  // namespace

int wcc_run(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, int32_t* label) {
    Carver sizing(nullptr);
    WalkBuffers::carve(sizing, n);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    WalkBuffers wb = WalkBuffers::carve(c, n);
    const unsigned g = grid_for(n, 256, ws->num_sms * 8);
    GHB_TRY(launch(ws, iota_kernel, dim3(g), dim3(256), 0, label, n));
    UniteVisitor f{label};
    GHB_TRY(walk(ws, rowptr, col, (const int32_t*)nullptr, (const int32_t*)nullptr, (int64_t)n,
                 (int64_t)n, wb, f));
    return launch(ws, wcc_compress_kernel, dim3(g), dim3(256), 0, label, n);
}

}  // namespace ghb

using namespace ghb;

extern "C" int ghb_wcc(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col,
                       int32_t* label) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(rowptr && label, "NULL argument");
    return wcc_run(ws, n, rowptr, col, label);
}

