// Shared helpers of the drop-in algorithm headers (host side only).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include <GPU_csr/GPU_csr.hpp>
#include <ghb.h>

namespace ghb_dropin {

// Device buffer for one call's output, freed at scope exit.
template <typename T>
struct DeviceBuffer {
    T* p = nullptr;
    std::size_t count = 0;
    explicit DeviceBuffer(std::size_t c) : count(c) { p = device_alloc<T>(c ? c : 1, "cudaMalloc(result)"); }
    ~DeviceBuffer() { device_free(p); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    bool to_host(std::vector<T>& out) const {
        out.resize(count);
        if (!count) return true;
        return cuda_ok(cudaMemcpy(out.data(), p, count * sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy(result)");
    }
};

inline ghb_workspace* workspace() {
    ghb_workspace* ws = ghb_default_workspace();
    if (ws) ghb_workspace_set_stream(ws, nullptr);
    return ws;
}

}  // namespace ghb_dropin
