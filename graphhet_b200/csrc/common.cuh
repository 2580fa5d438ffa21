// Shared host/device plumbing for libghb: workspace, error reporting, kernel
// launch accounting, scratch carving and the bounded grid barrier used by the
// persistent traversal kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstddef>
#include <string>

#include "ghb.h"

namespace ghb {

// ------------------------------------------------------------------ errors
void set_error(const std::string& msg);
void clear_error();

#define GHB_CUDA_TRY(expr)                                                         \
    do {                                                                           \
        cudaError_t _e = (expr);                                                   \
        if (_e != cudaSuccess) {                                                   \
            ::ghb::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e) +  \
                             " (" __FILE__ ":" + std::to_string(__LINE__) + ")");   \
            return _e == cudaErrorMemoryAllocation ? GHB_ERR_OUT_OF_MEMORY          \
                                                   : GHB_ERR_CUDA;                  \
        }                                                                          \
    } while (0)

#define GHB_TRY(expr)                \
    do {                             \
        int _s = (expr);             \
        if (_s != GHB_OK) return _s; \
    } while (0)

#define GHB_REQUIRE(cond, msg)                                              \
    do {                                                                    \
        if (!(cond)) {                                                      \
            ::ghb::set_error(std::string("invalid argument: ") + (msg));    \
            return GHB_ERR_INVALID_ARGUMENT;                                \
        }                                                                   \
    } while (0)

// -------------------------------------------------------------- constants
constexpr int kWarp = 32;
constexpr int32_t kInfDepth = 0x7fffffff;
// Sources per multi-source BFS pass (4 uint64 words of source bits per vertex).
constexpr int32_t kMsPass = 256;

// Device status word written by kernels whose waits gave up or whose budgets
// ran out; read back by the host after the launch.
enum DeviceStatus : int32_t {
    kDevOk = 0,
    kDevBarrierTimeout = 1,
    kDevOverflow = 2,
};

// Launch shapes and thresholds, per workspace.  The defaults are the
// autotuner's choices on B200 (graphhet_b200/autotune.py on RMAT scale 24
// for PageRank, scales 22 and 24 for the multi-source BFS); ghb_tune_set
// changes them for other graphs.
struct Tuning {
    int32_t pr_cache_kb = 144;     // PageRank hub cache: shared memory per block (KB)
    int32_t pr_threads = 1024;     // threads of the persistent PageRank blocks
    int32_t pr_blocks_per_sm = 1;  // persistent PageRank blocks per SM
    int32_t pr_short = 64;         // rows up to this many entries: one thread per row
    int32_t pr_chunk = 1024;       // longer rows: chunks of this many entries, warp per chunk
    int32_t ms_warp_rest = 512;    // multi-source pull: longer rest of a row -> a block
    int32_t ms_pull_div = 16;      // multi-source: pull when frontier entries > m / ms_pull_div
    int32_t pol_band = 1;          // learned policy: the network picks a level's direction and format only
                                   // where the direction rule's test is within 2^pol_band of its threshold
    int32_t barrier_limit_us = 2000000;  // persistent kernels: a grid-barrier wait gives up after this long
    int32_t barrier_extra = 0;     // test knob: barriers wait for this many arrivals beyond the grid, so
                                   // every wait runs out and the timeout path is exercised (0 or 1)
    int32_t sssp_persistent = 1;   // SSSP: 1 = one cooperative launch per traversal, 0 = host-driven rounds
    int32_t sssp_adapt = 0;        // one-launch SSSP: 1 = bucket widths adapt from bucket to bucket
    int32_t tc_hash = 1;           // TC: 1 = shared-memory hash probes per oriented row, 0 = galloping merges
    int32_t tc_block_row = 8192;   // TC hash path: longest oriented row a block hashes; longer rows gallop
    int32_t ms_persistent = 1;     // multi-source BFS: 1 = one cooperative launch per pass, 0 = host-driven levels
    int32_t ms_learned = 0;        // multi-source BFS pass: 1 = the installed direction model decides each level
    int32_t bfs_blocks_per_sm = 2; // whole-traversal BFS: 512-thread blocks per SM (1 or 2)
    int32_t pr_gathers = 4;        // PageRank long rows: contribution gathers in flight per lane (4 or 8)
    int32_t mssp_persistent = 1;   // multi-source SSSP: 1 = one cooperative launch per pass, 0 = host-driven
    int32_t tc_slice_blocks = 16;  // triangle counting: blocks per SM of the 2,048-slot slice kernel
    int32_t tc_trim_min = 0;       // triangle counting: lists N+(b) over this many entries are range-trimmed
    int32_t mssp_width_log2 = 2;   // multi-source SSSP bucket width: the single-source rule's times 2^k
};

}  // namespace ghb

// --------------------------------------------------------------- workspace
struct ghb_workspace {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    void* scratch = nullptr;  // cached device scratch (grown on demand)
    size_t scratch_cap = 0;
    void* stage = nullptr;    // results in relabelled ids before mapping back
    size_t stage_cap = 0;
    int64_t* host_pinned = nullptr;  // pinned host mirror for small readbacks
    int64_t* dev_small = nullptr;    // small device block (counters, status)
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;
    int64_t launches = 0;
    ghb::Tuning tune;
    // Many-source BFS into host memory (bfs_host.cu): device depth and byte
    // buffers, pinned byte buffers, a copy stream and its events.
    void* pipe_dev = nullptr;
    size_t pipe_dev_cap = 0;
    void* pipe_host = nullptr;
    size_t pipe_host_cap = 0;
    cudaStream_t pipe_stream = nullptr;
    cudaEvent_t pipe_ev[4] = {nullptr, nullptr, nullptr, nullptr};
};

namespace ghb {

constexpr int kHostPinnedWords = 1024;
constexpr int kDevSmallWords = 1024;

// Ensure at least `bytes` of scratch; the previous contents are not kept.
int ws_reserve(ghb_workspace* ws, size_t bytes);
// Ensure at least `bytes` of the staging area (kept apart from scratch, so an
// algorithm can write its relabelled result there while using scratch).
int ws_reserve_stage(ghb_workspace* ws, size_t bytes);
// Resolve NULL to the default workspace.
ghb_workspace* ws_resolve(ghb_workspace* ws);
// Copy `words` int64 counters from dev_small to host_pinned and wait.
int ws_read_small(ghb_workspace* ws, int words);

// Bump allocator over a scratch block.  Run it once with base == nullptr to
// size the block, reserve, then run it again on the real base.
struct Carver {
    char* base;
    size_t off = 0;
    explicit Carver(void* b) : base(static_cast<char*>(b)) {}
    template <class T>
    T* take(size_t count) {
        off = (off + 255) & ~size_t(255);
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += count * sizeof(T);
        return p;
    }
};

// Launch with accounting and an immediate launch-error check.
template <class Kernel, class... Args>
int launch(ghb_workspace* ws, Kernel kernel, dim3 grid, dim3 block, size_t smem, Args... args) {
    if (grid.x == 0 || grid.y == 0 || grid.z == 0) return GHB_OK;
    kernel<<<grid, block, smem, ws->stream>>>(args...);
    ws->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("kernel launch: ") + cudaGetErrorString(e));
        return GHB_ERR_CUDA;
    }
    return GHB_OK;
}

// Cooperative launch (all blocks co-resident) for kernels that use grid_barrier.
template <class... Args>
int launch_coop(ghb_workspace* ws, void (*kernel)(Args...), dim3 grid, dim3 block, size_t smem,
                Args... args) {
    void* ptrs[] = {static_cast<void*>(&args)...};
    cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), grid, block,
                                                ptrs, smem, ws->stream);
    ws->launches++;
    if (e != cudaSuccess) {
        set_error(std::string("cooperative launch: ") + cudaGetErrorString(e));
        return GHB_ERR_CUDA;
    }
    return GHB_OK;
}

inline unsigned grid_for(int64_t items, int threads, int64_t cap = 1 << 30) {
    int64_t g = (items + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return static_cast<unsigned>(g);
}

// ---------------------------------------------------------- device helpers
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// L2 cache policies (createpolicy) for loads that stream once (evict_first)
// and for gathered data that should stay resident (evict_last).
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ int ld_stream(const int* p, uint64_t pol) {
    int v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;"
                 : "=r"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ int4 ld_stream4(const int4* p, uint64_t pol) {
    int4 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.b32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_keep_f32(const float* p, uint64_t pol) {
    float v;
    asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double ld_keep_f64(const double* p, uint64_t pol) {
    double v;
    asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}

// Grid-wide barrier for cooperatively launched kernels.  The wait is bounded
// (limit_ns of wall time); on expiry it raises *status and returns false, and
// the caller must leave the kernel.  count/gen live in device memory and start
// at zero.
__device__ __forceinline__ bool grid_barrier(unsigned* count, unsigned* gen, int32_t* status,
                                             uint64_t limit_ns = 2000000000ull) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
        unsigned g = ld_acquire_u32(gen);
        __threadfence();
        unsigned arrived = atomicAdd(count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(count, 0u);
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            uint64_t t0 = global_timer_ns();
            unsigned spins = 0;
            while (ld_acquire_u32(gen) == g) {
                if (*(volatile int32_t*)status != 0) { ok = 0; break; }
                if ((++spins & 63u) == 0 && global_timer_ns() - t0 > limit_ns) {
                    atomicExch(status, (int32_t)kDevBarrierTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(20);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Grid barrier with leader work, for cooperatively launched kernels.
// *count (arrivals) and *release (epochs) must sit on different cache lines
// and start at zero.  A block's thread 0 adds one arrival; the last block to
// arrive runs leader() (every other block is waiting and has published its
// writes), then publishes the epoch on *release, for which the others wait.
// Bounded like grid_barrier: a wait that exceeds limit_ns raises *status and
// returns false, and the caller must leave the kernel.
//
// Ordering without full fences: the arrival is an acquire-release add at gpu
// scope (it publishes the block's writes, which __syncthreads orders before
// it, and the last arrival acquires every earlier one through the chain of
// adds), the epoch is a release store, the waiters' loads are acquire loads,
// and __syncthreads carries each side to the rest of its block.  (A grid
// barrier with fence.sc before and after each step measured 3.1 us on a
// B200, 2.4 us this way.)
struct NoLeader {
    __device__ void operator()() const {}
};

__device__ __forceinline__ unsigned atom_add_acq_rel_u32(unsigned* p, unsigned v) {
    unsigned r;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(r) : "l"(p), "r"(v) : "memory");
    return r;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Thread 0's bounded wait for the epoch; false when it gave up.
__device__ __forceinline__ bool grid_wait_epoch(const unsigned* release, unsigned epoch, int32_t* status,
                                                uint64_t limit_ns) {
    unsigned spins = 0;
    uint64_t t0 = 0;
    while ((int)(ld_acquire_u32(release) - epoch) < 0) {
        if ((++spins & 127u) == 0) {
            if (*(volatile int32_t*)status != 0) return false;
            const uint64_t t = global_timer_ns();
            if (t0 == 0) t0 = t;
            else if (t - t0 > limit_ns) {
                atomicExch(status, (int32_t)kDevBarrierTimeout);
                return false;
            }
        }
    }
    return true;
}

// `extra` (normally 0) adds arrivals that never come: the tests use it to
// make every wait run out.
template <class Leader>
__device__ __forceinline__ bool grid_sync_leader(unsigned* count, unsigned* release, int32_t* status,
                                                 const Leader& leader, uint64_t limit_ns = 2000000000ull,
                                                 unsigned extra = 0) {
    __shared__ int s_ok2;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z + extra;
        const unsigned old = atom_add_acq_rel_u32(count, 1u);
        const unsigned epoch = old / nblocks + 1u;
        if (old % nblocks == nblocks - 1u) {
            leader();
            st_release_u32(release, epoch);
        } else {
            ok = grid_wait_epoch(release, epoch, status, limit_ns) ? 1 : 0;
        }
        s_ok2 = ok;
    }
    __syncthreads();
    return s_ok2 != 0;
}

// As grid_sync_leader, but every thread of the last block to arrive runs
// leader() (which may contain __syncthreads) before the release, so a
// decision can use the whole block (the policy network's layers).
template <class Leader>
__device__ __forceinline__ bool grid_sync_block_leader(unsigned* count, unsigned* release, int32_t* status,
                                                       const Leader& leader, uint64_t limit_ns = 2000000000ull,
                                                       unsigned extra = 0) {
    __shared__ int s_ok3, s_last3;
    __shared__ unsigned s_epoch3;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z + extra;
        const unsigned old = atom_add_acq_rel_u32(count, 1u);
        s_epoch3 = old / nblocks + 1u;
        s_last3 = (old % nblocks == nblocks - 1u) ? 1 : 0;
        s_ok3 = 1;
    }
    __syncthreads();
    if (s_last3) {
        leader();
        __syncthreads();
        if (threadIdx.x == 0) st_release_u32(release, s_epoch3);
    } else if (threadIdx.x == 0) {
        s_ok3 = grid_wait_epoch(release, s_epoch3, status, limit_ns) ? 1 : 0;
    }
    __syncthreads();
    return s_ok3 != 0;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <class T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T x = __shfl_xor_sync(0xffffffffu, v, o);
        v = x > v ? x : v;
    }
    return v;
}

// Warp-aggregated append: each lane with `want` gets a distinct slot of
// *tail.  Returns the slot (undefined for lanes without `want`).
__device__ __forceinline__ int32_t warp_append(int32_t* tail, bool want) {
    unsigned mask = __ballot_sync(0xffffffffu, want);
    if (mask == 0) return -1;
    int leader = __ffs(mask) - 1;
    int32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(tail, __popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + __popc(mask & ((1u << lane_id()) - 1u));
}

// Active-lane variant (only the lanes in `active` participate).
__device__ __forceinline__ int32_t warp_append_active(int32_t* tail) {
    unsigned active = __activemask();
    int leader = __ffs(active) - 1;
    int32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(tail, __popc(active));
    base = __shfl_sync(active, base, leader);
    return base + __popc(active & ((1u << lane_id()) - 1u));
}

}  // namespace ghb
