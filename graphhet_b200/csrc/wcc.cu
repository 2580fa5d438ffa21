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
#include <mutex>
#include <string>

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

// Points every vertex at its root, halving the paths it walks on the way
// (a pointer may only move to an ancestor), so that walkers of one chain
// shorten it for each other.
__global__ void wcc_compress_halving_kernel(int32_t* parent, int32_t n) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x)
        parent[v] = wcc_find(parent, (int32_t)v);
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

// Afforest (Sutton, Ben-Nun and Barak, IPDPS 2018), for symmetric CSRs:
// a sampled forest first, compressed, then the largest component is found
// from a sample of labels, and only vertices outside it link their entries.
// Skipping a giant-component vertex's entries is safe because each such
// entry (u, v) with v outside the giant component is also entry (v, u) of
// v's row, which is processed.
//
// The sampled forest here is a hook, not a union: every vertex points at
// the first of its first kAffSample neighbours whose degree is strictly
// higher than its own (on a degree-relabelled graph that neighbour has a
// smaller id, and the first entries of a row are its hubs), or at itself.
// Pointers only go to smaller ids, so the result is a forest whose trees
// are connected sets, and a path in it climbs strictly in degree, so its
// trees stay shallow (a grid, where all degrees are equal, hooks almost
// nothing and is linked in full below).  A sampled entry that the hook did
// not join is joined later, because the rows outside the giant component
// are linked in full.  One write per vertex instead of two unions: on RMAT
// scale 24 the sampling went from 0.50 ms to a streaming pass, and WCC from
// 0.94-1.64 ms (the unions' contention varied from run to run) to 0.71 ms.
constexpr int32_t kAffSample = 2;
constexpr int kAffProbe = 1024;

__global__ void aff_hook_kernel(int32_t n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                int32_t* parent) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = rowptr[v], e0 = rowptr[v + 1];
        const int32_t e = min(e0, b + kAffSample), dv = e0 - b;
        int32_t p = (int32_t)v;
        for (int32_t j = b; j < e && p == (int32_t)v; ++j) {
            const int32_t c = col[j];
            if (c < (int32_t)v && rowptr[c + 1] - rowptr[c] > dv) p = c;
        }
        parent[v] = p;
    }
}

// The most frequent label among kAffProbe hashed vertices of [0, n_active)
// (ties: the smaller label), by a bitonic sort in shared memory.
__global__ void __launch_bounds__(kAffProbe) aff_giant_kernel(int32_t n_active, const int32_t* __restrict__ parent,
                                                              int32_t* giant) {
    __shared__ int32_t s[kAffProbe];
    const int t = threadIdx.x;
    const uint64_t h = (uint64_t)(t + 1) * 0x9E3779B97F4A7C15ull;
    s[t] = n_active > 0 ? __ldcg(parent + (int64_t)((h >> 33) % (uint64_t)n_active)) : 0;
    __syncthreads();
    for (int size = 2; size <= kAffProbe; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const int o = t ^ stride;
            if (o > t) {
                const bool up = (t & size) == 0;
                const int32_t a = s[t], b = s[o];
                if ((a > b) == up) {
                    s[t] = b;
                    s[o] = a;
                }
            }
            __syncthreads();
        }
    if (t == 0) {
        int32_t bl = s[0], bc = 0, cl = s[0], cc = 0;
        for (int i = 0; i < kAffProbe; ++i) {
            if (s[i] == cl) ++cc;
            else {
                cl = s[i];
                cc = 1;
            }
            if (cc > bc) {
                bc = cc;
                bl = cl;
            }
        }
        *giant = bl;
    }
}

struct UniteRestVisitor {
    int32_t* parent;
    const int32_t* giant;  // written by aff_giant_kernel before the walk
    __device__ bool want_row(int32_t u) const { return __ldcg(parent + u) != __ldg(giant); }
    __device__ void operator()(int32_t u, int32_t v, int32_t) const {
        if (u != v) wcc_unite(parent, u, v);
    }
    __device__ void finish() const {}
};

}  // namespace

// Symmetric CSR (every entry (u, v) also present as (v, u)) only.
int wcc_afforest_run(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* rowptr, const int32_t* col,
                     int32_t* label) {
    Carver sizing(nullptr);
    WalkBuffers::carve(sizing, n);
    sizing.take<int32_t>(8);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    WalkBuffers wb = WalkBuffers::carve(c, n);
    int32_t* giant = c.take<int32_t>(8);
    const unsigned g = grid_for(n, 256, ws->num_sms * 8);
    GHB_TRY(launch(ws, aff_hook_kernel, dim3(g), dim3(256), 0, n, rowptr, col, label));
    GHB_TRY(launch(ws, wcc_compress_halving_kernel, dim3(g), dim3(256), 0, label, n));
    GHB_TRY(launch(ws, aff_giant_kernel, dim3(1), dim3(kAffProbe), 0, n_active, (const int32_t*)label, giant));
    // The giant label is read on the device by the visitor (no round trip).
    GHB_TRY(walk(ws, rowptr, col, (const int32_t*)nullptr, (const int32_t*)nullptr, (int64_t)n, (int64_t)n, wb,
                 UniteRestVisitor{label, (const int32_t*)giant}));
    return launch(ws, wcc_compress_kernel, dim3(g), dim3(256), 0, label, n);
}

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

// ---------------------------------------------------------------------------
// WCC that allocates nothing.
//
// Some callers of this library must not allocate device memory while it
// runs: an application that owns the GPU's memory through its own pool
// allocator (the library loaded as a plugin inside a database or a serving
// process, where a cudaMalloc behind the pool's back can fail or fragment
// it), and latency-critical callers for which cudaMalloc / cudaFree would
// synchronise the device.  Such a caller cannot create a ghb_workspace
// either, since a workspace allocates its scratch and pinned counters.
//
// ghb_wcc_noalloc takes a stream instead of a workspace.  Its only scratch
// is the row walker's deferred long-row list, kept in the fixed file-scope
// device array below, which every GPU that loads libghb.so holds until the
// process exits.  Limit: at most kNoAllocMaxEntries CSR entries, which bounds
// the rows of kWalkBig or more entries by the list's capacity.
namespace ghb {
namespace {

constexpr int64_t kNoAllocMaxEntries = 1ll << 28;                  // 268,435,456 entries
constexpr int64_t kNoAllocBigRows = kNoAllocMaxEntries / kWalkBig;  // 65,536 long rows
constexpr size_t kNoAllocScratchBytes = 800 * 1024;

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {};

}  // namespace
}  // namespace ghb

// Device-side scratch of ghb_wcc_noalloc.  In host code this name is only a
// host-side stand-in for the symbol, not a device address: the device
// address is looked up per device with cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_wcc_noalloc_scratch[ghb::kNoAllocScratchBytes];

namespace ghb {

// Device address of the scratch array on the current device, looked up once
// per device (with that device current) and cached for the process's life.
// A cudaDeviceReset would leave the cached address stale; the header says
// that a reset device must not be used with this entry point again.
static int noalloc_scratch_address(void** out) {
    int dev = 0;
    GHB_CUDA_TRY(cudaGetDevice(&dev));
    GHB_REQUIRE(dev >= 0 && dev < 64, "device index outside [0, 64)");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        GHB_CUDA_TRY(cudaGetSymbolAddress(&p, g_wcc_noalloc_scratch));
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return GHB_OK;
}

}  // namespace ghb

extern "C" int ghb_wcc_noalloc(int32_t n, const int32_t* rowptr, const int32_t* col, int32_t* label,
                               void* stream) {
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(rowptr && label, "NULL argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Entry count, for the size limit (one small read-back on `stream`).
    int32_t m = 0;
    GHB_CUDA_TRY(cudaMemcpyAsync(&m, rowptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    if (m < 0 || (int64_t)m > kNoAllocMaxEntries) {
        set_error("invalid argument: ghb_wcc_noalloc handles at most 268435456 CSR entries (its scratch is a "
                  "fixed 800 KiB device array); this graph has " + std::to_string(m) + ", use ghb_wcc");
        return GHB_ERR_INVALID_ARGUMENT;
    }
    void* base = nullptr;
    GHB_TRY(noalloc_scratch_address(&base));
    Carver c(base);
    WalkBuffers wb = WalkBuffers::carve(c, kNoAllocBigRows);
    if (c.off > kNoAllocScratchBytes) {
        set_error("internal: ghb_wcc_noalloc scratch layout exceeds its array");
        return GHB_ERR_UNSUPPORTED;
    }
    // A stack workspace carries only the stream and SM count to the launch
    // helpers; it owns no memory.
    ghb_workspace tmp;
    tmp.stream = st;
    int dev = 0;
    GHB_CUDA_TRY(cudaGetDevice(&dev));
    GHB_CUDA_TRY(cudaDeviceGetAttribute(&tmp.num_sms, cudaDevAttrMultiProcessorCount, dev));
    const unsigned g = grid_for(n, 256, tmp.num_sms * 8);
    GHB_TRY(launch(&tmp, iota_kernel, dim3(g), dim3(256), 0, label, n));
    // walk() zeroes the list's counter first: the array keeps the previous
    // call's contents.
    GHB_TRY(walk(&tmp, rowptr, col, (const int32_t*)nullptr, (const int32_t*)nullptr, (int64_t)n, (int64_t)n, wb,
                 UniteVisitor{label}));
    return launch(&tmp, wcc_compress_kernel, dim3(g), dim3(256), 0, label, n);
}
