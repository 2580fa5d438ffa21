// Workspace lifecycle, error reporting and status strings of the C ABI.
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"

namespace ghb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }

ghb_workspace* ws_resolve(ghb_workspace* ws) { return ws ? ws : ghb_default_workspace(); }

int ws_reserve(ghb_workspace* ws, size_t bytes) {
    if (bytes <= ws->scratch_cap) return GHB_OK;
    if (ws->scratch) {
        GHB_CUDA_TRY(cudaStreamSynchronize(ws->stream));
        GHB_CUDA_TRY(cudaFree(ws->scratch));
        ws->scratch = nullptr;
        ws->scratch_cap = 0;
    }
    // Round up to 64 MiB steps so repeated calls of growing size do not
    // reallocate every time.
    size_t cap = (bytes + (64ull << 20) - 1) & ~((64ull << 20) - 1);
    GHB_CUDA_TRY(cudaMalloc(&ws->scratch, cap));
    ws->scratch_cap = cap;
    return GHB_OK;
}

int ws_reserve_stage(ghb_workspace* ws, size_t bytes) {
    if (bytes <= ws->stage_cap) return GHB_OK;
    if (ws->stage) {
        GHB_CUDA_TRY(cudaStreamSynchronize(ws->stream));
        GHB_CUDA_TRY(cudaFree(ws->stage));
        ws->stage = nullptr;
        ws->stage_cap = 0;
    }
    size_t cap = (bytes + (16ull << 20) - 1) & ~((16ull << 20) - 1);
    GHB_CUDA_TRY(cudaMalloc(&ws->stage, cap));
    ws->stage_cap = cap;
    return GHB_OK;
}

int ws_read_small(ghb_workspace* ws, int words) {
    GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, ws->dev_small, sizeof(int64_t) * words,
                                 cudaMemcpyDeviceToHost, ws->stream));
    GHB_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    return GHB_OK;
}

}  // namespace ghb

using namespace ghb;

extern "C" {

const char* ghb_status_string(int status) {
    switch (status) {
        case GHB_OK: return "ok";
        case GHB_ERR_INVALID_ARGUMENT: return "invalid argument";
        case GHB_ERR_CUDA: return "CUDA error";
        case GHB_ERR_OUT_OF_MEMORY: return "out of device memory";
        case GHB_ERR_TIMEOUT: return "device wait timed out";
        case GHB_ERR_LIMIT: return "iteration budget exhausted";
        case GHB_ERR_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

const char* ghb_last_error(void) { return g_last_error.c_str(); }

int ghb_version(void) { return 10000; }

int ghb_workspace_create(ghb_workspace** out) {
    GHB_REQUIRE(out != nullptr, "out is NULL");
    *out = nullptr;
    ghb_workspace* ws = new ghb_workspace();
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ws->num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaMallocHost(&ws->host_pinned, sizeof(int64_t) * kHostPinnedWords);
    if (e == cudaSuccess) e = cudaMalloc(&ws->dev_small, sizeof(int64_t) * kDevSmallWords);
    if (e == cudaSuccess) e = cudaMemset(ws->dev_small, 0, sizeof(int64_t) * kDevSmallWords);
    if (e == cudaSuccess) e = cudaEventCreate(&ws->ev_start);
    if (e == cudaSuccess) e = cudaEventCreate(&ws->ev_stop);
    if (e == cudaSuccess) e = cudaEventCreate(&ws->ev_a);
    if (e == cudaSuccess) e = cudaEventCreate(&ws->ev_b);
    if (e != cudaSuccess) {
        set_error(std::string("workspace create: ") + cudaGetErrorString(e));
        ghb_workspace_destroy(ws);
        return e == cudaErrorMemoryAllocation ? GHB_ERR_OUT_OF_MEMORY : GHB_ERR_CUDA;
    }
    ws->device = dev;
    *out = ws;
    return GHB_OK;
}

int ghb_workspace_destroy(ghb_workspace* ws) {
    if (!ws) return GHB_OK;
    if (ws->stream || ws->scratch) cudaStreamSynchronize(ws->stream);
    if (ws->scratch) cudaFree(ws->scratch);
    if (ws->stage) cudaFree(ws->stage);
    if (ws->host_pinned) cudaFreeHost(ws->host_pinned);
    if (ws->dev_small) cudaFree(ws->dev_small);
    if (ws->ev_start) cudaEventDestroy(ws->ev_start);
    if (ws->ev_stop) cudaEventDestroy(ws->ev_stop);
    if (ws->ev_a) cudaEventDestroy(ws->ev_a);
    if (ws->ev_b) cudaEventDestroy(ws->ev_b);
    if (ws->pipe_stream) cudaStreamSynchronize(ws->pipe_stream);
    if (ws->pipe_dev) cudaFree(ws->pipe_dev);
    if (ws->pipe_host) cudaFreeHost(ws->pipe_host);
    if (ws->pipe_stream) cudaStreamDestroy(ws->pipe_stream);
    for (cudaEvent_t e : ws->pipe_ev)
        if (e) cudaEventDestroy(e);
    delete ws;
    return GHB_OK;
}

namespace {
struct TuneField {
    const char* name;
    int32_t ghb::Tuning::*field;
    int32_t lo, hi;
};
const TuneField kTuneFields[] = {
    {"pr_cache_kb", &ghb::Tuning::pr_cache_kb, 0, 200},
    {"pr_threads", &ghb::Tuning::pr_threads, 128, 1024},
    {"pr_blocks_per_sm", &ghb::Tuning::pr_blocks_per_sm, 1, 8},
    {"pr_short", &ghb::Tuning::pr_short, 4, 256},
    {"pr_chunk", &ghb::Tuning::pr_chunk, 64, 4096},
    {"ms_warp_rest", &ghb::Tuning::ms_warp_rest, 32, 1 << 20},
    {"ms_pull_div", &ghb::Tuning::ms_pull_div, 1, 1024},
    {"pol_band", &ghb::Tuning::pol_band, 0, 64},
    {"barrier_limit_us", &ghb::Tuning::barrier_limit_us, 100, 60000000},
    {"barrier_extra", &ghb::Tuning::barrier_extra, 0, 1},
    {"sssp_persistent", &ghb::Tuning::sssp_persistent, 0, 1},
    {"sssp_adapt", &ghb::Tuning::sssp_adapt, 0, 1},
    {"tc_hash", &ghb::Tuning::tc_hash, 0, 1},
    {"tc_block_row", &ghb::Tuning::tc_block_row, 128, 8192},
    {"ms_persistent", &ghb::Tuning::ms_persistent, 0, 1},
    {"ms_learned", &ghb::Tuning::ms_learned, 0, 1},
    {"bfs_blocks_per_sm", &ghb::Tuning::bfs_blocks_per_sm, 1, 2},
    {"pr_gathers", &ghb::Tuning::pr_gathers, 4, 8},
    {"mssp_persistent", &ghb::Tuning::mssp_persistent, 0, 1},
    {"mssp_width_log2", &ghb::Tuning::mssp_width_log2, -10, 10},
    {"tc_trim_min", &ghb::Tuning::tc_trim_min, 0, 1 << 20},
    {"tc_slice_blocks", &ghb::Tuning::tc_slice_blocks, 1, 16},
};
const TuneField* tune_field(const char* name) {
    if (!name) return nullptr;
    for (const TuneField& f : kTuneFields)
        if (std::strcmp(f.name, name) == 0) return &f;
    return nullptr;
}
}  // namespace

int ghb_tune_set(ghb_workspace* ws, const char* name, int32_t value) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    const TuneField* f = tune_field(name);
    GHB_REQUIRE(f, std::string("unknown tuning parameter: ") + (name ? name : "(null)"));
    GHB_REQUIRE(value >= f->lo && value <= f->hi,
                std::string(f->name) + " outside [" + std::to_string(f->lo) + ", " + std::to_string(f->hi) + "]");
    if (f->field == &ghb::Tuning::pr_threads) GHB_REQUIRE(value % 32 == 0, "pr_threads must be a multiple of 32");
    if (f->field == &ghb::Tuning::pr_gathers) GHB_REQUIRE(value == 4 || value == 8, "pr_gathers must be 4 or 8");
    ws->tune.*(f->field) = value;
    return GHB_OK;
}

int ghb_tune_get(ghb_workspace* ws, const char* name, int32_t* value) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && value, "NULL argument");
    const TuneField* f = tune_field(name);
    GHB_REQUIRE(f, std::string("unknown tuning parameter: ") + (name ? name : "(null)"));
    *value = ws->tune.*(f->field);
    return GHB_OK;
}

int ghb_workspace_set_stream(ghb_workspace* ws, void* stream) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws != nullptr, "no workspace");
    ws->stream = static_cast<cudaStream_t>(stream);
    return GHB_OK;
}

void* ghb_workspace_get_stream(ghb_workspace* ws) {
    ws = ws_resolve(ws);
    return ws ? static_cast<void*>(ws->stream) : nullptr;
}

int ghb_workspace_trim(ghb_workspace* ws) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws != nullptr, "no workspace");
    if (ws->scratch) {
        GHB_CUDA_TRY(cudaStreamSynchronize(ws->stream));
        GHB_CUDA_TRY(cudaFree(ws->scratch));
    }
    ws->scratch = nullptr;
    ws->scratch_cap = 0;
    if (ws->stage) GHB_CUDA_TRY(cudaFree(ws->stage));
    ws->stage = nullptr;
    ws->stage_cap = 0;
    if (ws->pipe_stream) GHB_CUDA_TRY(cudaStreamSynchronize(ws->pipe_stream));
    if (ws->pipe_dev) GHB_CUDA_TRY(cudaFree(ws->pipe_dev));
    ws->pipe_dev = nullptr;
    ws->pipe_dev_cap = 0;
    if (ws->pipe_host) GHB_CUDA_TRY(cudaFreeHost(ws->pipe_host));
    ws->pipe_host = nullptr;
    ws->pipe_host_cap = 0;
    return GHB_OK;
}

int ghb_workspace_counters(ghb_workspace* ws, int64_t* kernel_launches, int64_t* scratch_bytes) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws != nullptr, "no workspace");
    if (kernel_launches) *kernel_launches = ws->launches;
    if (scratch_bytes) *scratch_bytes = static_cast<int64_t>(ws->scratch_cap + ws->stage_cap);
    return GHB_OK;
}

ghb_workspace* ghb_default_workspace(void) {
    // One default workspace per device, created on first use.
    static std::mutex mu;
    static ghb_workspace* per_device[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!per_device[dev]) {
        ghb_workspace* ws = nullptr;
        if (ghb_workspace_create(&ws) != GHB_OK) return nullptr;
        per_device[dev] = ws;
    }
    return per_device[dev];
}

}  // extern "C"
