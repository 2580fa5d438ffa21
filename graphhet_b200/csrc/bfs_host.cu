// Many BFS on a resident graph straight into the caller's host array.
//
// The reference returns each BFS to the host as a vector<int> (Cuda_BFS,
// GPU_BFS_csr.cuh:13, 320-327: one cudaMemcpy of n ints per call).  Here a
// batch of sources is pipelined over three resources at once:
//   GPU         traversal of source i (one cooperative launch), then a pack
//               of its depths to one byte each when the traversal ran fewer
//               than 255 levels (255 = unreached);
//   copy engine the bytes of source i - 1 over PCIe (a quarter of the int32
//               depths' bytes);
//   host        threads widening source i - 2's bytes into the caller's
//               int32 array (255 -> INT32_MAX).
// A traversal of 255 levels or more is copied as int32 depths instead.
// The caller's array ends up exactly as k calls of ghb_graph_bfs followed by
// k device-to-host copies would leave it.
#include <immintrin.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"
#include "graph.cuh"

namespace ghb {
namespace {

constexpr int32_t kByteUnreached = 255;

// bytes[v] = depth[v] if it is below 255, else 255; four per thread (both
// buffers padded to a multiple of 16 entries).
__global__ void depth_pack_kernel(int64_t n4, const int4* __restrict__ depth, uchar4* __restrict__ bytes) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
        const int4 d = depth[i];
        auto b = [](int32_t x) -> unsigned char {
            return (x >= 0 && x < kByteUnreached) ? (unsigned char)x : (unsigned char)kByteUnreached;
        };
        bytes[i] = make_uchar4(b(d.x), b(d.y), b(d.z), b(d.w));
    }
}

// dst[i] = src[i], 255 -> INT32_MAX.  With AVX2: eight at a time, written
// with streaming stores (the caller's array is not read back here, so its
// lines need not be fetched before they are overwritten: half the host
// memory traffic of plain stores).
__attribute__((target("avx2"))) void widen_avx2(int32_t* dst, const uint8_t* src, int64_t n) {
    int64_t i = 0;
    for (; i < n && (reinterpret_cast<uintptr_t>(dst + i) & 31u); ++i)
        dst[i] = src[i] == kByteUnreached ? kInfDepth : src[i];
    const __m256i k255 = _mm256_set1_epi32(kByteUnreached), kinf = _mm256_set1_epi32(kInfDepth);
    for (; i + 8 <= n; i += 8) {
        __m256i v = _mm256_cvtepu8_epi32(_mm_loadl_epi64(reinterpret_cast<const __m128i*>(src + i)));
        v = _mm256_blendv_epi8(v, kinf, _mm256_cmpeq_epi32(v, k255));
        _mm256_stream_si256(reinterpret_cast<__m256i*>(dst + i), v);
    }
    for (; i < n; ++i) dst[i] = src[i] == kByteUnreached ? kInfDepth : src[i];
    _mm_sfence();
}

void widen_scalar(int32_t* dst, const uint8_t* src, int64_t n) {
    for (int64_t i = 0; i < n; ++i) dst[i] = src[i] == kByteUnreached ? kInfDepth : src[i];
}

// Host threads that widen byte depths into int32 slices of the caller's
// array.  Work is queued per pipeline slot; wait(slot) returns when every
// slice queued for that slot is done.
class WidenPool {
  public:
    explicit WidenPool(int threads) {
        for (int t = 0; t < threads; ++t) workers_.emplace_back([this] { run(); });
    }
    ~WidenPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& w : workers_) w.join();
    }
    void submit(int32_t* dst, const uint8_t* src, int64_t n, int slot) {
        const int parts = (int)workers_.size();
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (int p = 0; p < parts; ++p) {
                const int64_t lo = n * p / parts, hi = n * (p + 1) / parts;
                if (hi > lo) {
                    tasks_.push_back(Task{dst + lo, src + lo, hi - lo, slot});
                    ++pending_[slot];
                }
            }
        }
        cv_.notify_all();
    }
    void wait(int slot) {
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return pending_[slot] == 0; });
    }

  private:
    struct Task {
        int32_t* dst;
        const uint8_t* src;
        int64_t n;
        int slot;
    };
    void run() {
        std::unique_lock<std::mutex> lk(mu_);
        while (true) {
            cv_.wait(lk, [&] { return stop_ || head_ < tasks_.size(); });
            if (head_ >= tasks_.size()) return;  // stop_ and nothing queued
            const Task t = tasks_[head_++];
            lk.unlock();
            if (avx2_) widen_avx2(t.dst, t.src, t.n);
            else widen_scalar(t.dst, t.src, t.n);
            lk.lock();
            if (--pending_[t.slot] == 0) done_.notify_all();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    std::vector<Task> tasks_;
    size_t head_ = 0;
    int pending_[2] = {0, 0};
    bool stop_ = false;
    const bool avx2_ = __builtin_cpu_supports("avx2");
};

}  // namespace

// Device and pinned buffers, the copy stream and its events, kept on the
// workspace between calls.
int ws_pipe_reserve(ghb_workspace* ws, size_t dev_bytes, size_t host_bytes) {
    if (dev_bytes > ws->pipe_dev_cap) {
        if (ws->pipe_dev) {
            GHB_CUDA_TRY(cudaStreamSynchronize(ws->stream));
            GHB_CUDA_TRY(cudaFree(ws->pipe_dev));
            ws->pipe_dev = nullptr;
            ws->pipe_dev_cap = 0;
        }
        GHB_CUDA_TRY(cudaMalloc(&ws->pipe_dev, dev_bytes));
        ws->pipe_dev_cap = dev_bytes;
    }
    if (host_bytes > ws->pipe_host_cap) {
        if (ws->pipe_host) {
            GHB_CUDA_TRY(cudaFreeHost(ws->pipe_host));
            ws->pipe_host = nullptr;
            ws->pipe_host_cap = 0;
        }
        GHB_CUDA_TRY(cudaMallocHost(&ws->pipe_host, host_bytes));
        ws->pipe_host_cap = host_bytes;
    }
    if (!ws->pipe_stream) GHB_CUDA_TRY(cudaStreamCreateWithFlags(&ws->pipe_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 4; ++i)
        if (!ws->pipe_ev[i]) GHB_CUDA_TRY(cudaEventCreateWithFlags(&ws->pipe_ev[i], cudaEventDisableTiming));
    return GHB_OK;
}

}  // namespace ghb

using namespace ghb;

extern "C" int ghb_graph_bfs_many_host(ghb_workspace* ws, const ghb_graph* g, const int32_t* srcs, int32_t n_src,
                                       int32_t max_depth, int32_t* depth_host, int32_t host_threads,
                                       const ghb_bfs_options* options, ghb_traversal_stats* stats) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(g, "NULL graph");
    GHB_REQUIRE(n_src >= 0, "n_src < 0");
    GHB_REQUIRE(n_src == 0 || (srcs && depth_host), "NULL argument");
    GHB_REQUIRE(host_threads >= 0 && host_threads <= 256, "host_threads outside [0, 256]");
    for (int32_t i = 0; i < n_src; ++i) GHB_REQUIRE(srcs[i] >= 0 && srcs[i] < g->n, "source outside [0, n)");
    const auto t0 = std::chrono::steady_clock::now();
    if (stats) *stats = ghb_traversal_stats{};
    if (n_src == 0) return GHB_OK;
    const int64_t n = g->n;
    const int64_t n16 = (n + 15) & ~(int64_t)15;
    GHB_TRY(ws_pipe_reserve(ws, 2 * (size_t)n16 * (sizeof(int32_t) + 1), 2 * (size_t)n16));
    int32_t* d32[2] = {static_cast<int32_t*>(ws->pipe_dev), static_cast<int32_t*>(ws->pipe_dev) + n16};
    uint8_t* d8[2] = {reinterpret_cast<uint8_t*>(d32[1] + n16), reinterpret_cast<uint8_t*>(d32[1] + n16) + n16};
    uint8_t* h8[2] = {static_cast<uint8_t*>(ws->pipe_host), static_cast<uint8_t*>(ws->pipe_host) + n16};
    cudaEvent_t* ev_packed = ws->pipe_ev;      // [2]
    cudaEvent_t* ev_copied = ws->pipe_ev + 2;  // [2]
    int threads = host_threads;
    // Default: half the host's threads, at most 8 (on a 16-thread host, 8
    // widened RMAT-24 depths at 634 GTEPS end to end, 16 at 503, 32 at 444:
    // the widening is bound by host memory writes, and more threads only
    // contend with the calling thread and the driver's).
    if (threads == 0) threads = (int)std::min<unsigned>(8u, std::max(1u, std::thread::hardware_concurrency() / 2));
    int rc = GHB_OK;
    bool bytes_of[2] = {false, false};
    {
        WidenPool pool(threads);
        // Widening of source j once its byte copy has landed.
        auto widen = [&](int32_t j) -> int {
            const int s = j & 1;
            GHB_CUDA_TRY(cudaEventSynchronize(ev_copied[s]));
            pool.submit(depth_host + (int64_t)j * n, h8[s], n, s);
            return GHB_OK;
        };
        for (int32_t i = 0; i < n_src && rc == GHB_OK; ++i) {
            const int s = i & 1;
            ghb_traversal_stats st{};
            // d32[s] and d8[s] are free: source i - 2's pack ran earlier on
            // this stream and its copy was waited for before its widening
            // was queued.
            rc = ghb_graph_bfs(ws, g, srcs[i], max_depth, d32[s], options, &st);
            if (rc != GHB_OK) break;
            if (stats) {
                stats->levels = std::max(stats->levels, st.levels);
                stats->pull_levels += st.pull_levels;
                stats->reached += st.reached;
                stats->edges_reached += st.edges_reached;
                stats->edges_examined += st.edges_examined;
            }
            bytes_of[s] = st.levels < kByteUnreached;
            if (bytes_of[s]) {
                rc = launch(ws, depth_pack_kernel, dim3(grid_for(n16 / 4, 256, ws->num_sms * 8)), dim3(256), 0,
                            n16 / 4, reinterpret_cast<const int4*>(d32[s]), reinterpret_cast<uchar4*>(d8[s]));
                if (rc != GHB_OK) break;
                cudaError_t e = cudaEventRecord(ev_packed[s], ws->stream);
                // h8[s] may still be read by the widening of source i - 2.
                pool.wait(s);
                if (e == cudaSuccess) e = cudaStreamWaitEvent(ws->pipe_stream, ev_packed[s], 0);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(h8[s], d8[s], (size_t)n, cudaMemcpyDeviceToHost, ws->pipe_stream);
                if (e == cudaSuccess) e = cudaEventRecord(ev_copied[s], ws->pipe_stream);
                if (e != cudaSuccess) {
                    set_error(std::string("BFS host pipeline: ") + cudaGetErrorString(e));
                    rc = GHB_ERR_CUDA;
                    break;
                }
            } else {
                // 255 levels or more: the int32 depths themselves.
                cudaError_t e = cudaMemcpyAsync(depth_host + (int64_t)i * n, d32[s], sizeof(int32_t) * (size_t)n,
                                                cudaMemcpyDeviceToHost, ws->stream);
                if (e == cudaSuccess) e = cudaStreamSynchronize(ws->stream);
                if (e != cudaSuccess) {
                    set_error(std::string("BFS host pipeline: ") + cudaGetErrorString(e));
                    rc = GHB_ERR_CUDA;
                    break;
                }
            }
            if (i >= 1 && bytes_of[(i - 1) & 1]) rc = widen(i - 1);
        }
        if (rc == GHB_OK && bytes_of[(n_src - 1) & 1]) rc = widen(n_src - 1);
        if (rc != GHB_OK) cudaStreamSynchronize(ws->pipe_stream);  // no copy may outlive the call
        pool.wait(0);
        pool.wait(1);
    }
    if (rc != GHB_OK) return rc;
    if (stats)
        stats->device_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return GHB_OK;
}
