// Shared helpers of the drop-in algorithm headers (host side only).
#pragma once

#include <cuda_runtime.h>

#include <iostream>
#include <string>
#include <utility>
#include <vector>

#include <GPU_csr/GPU_csr.hpp>
#include <ghb.h>

namespace ghb_dropin {

// Device buffer for one call's output, freed at scope exit (the lower-level
// entry points that take raw CSR pointers use it).
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

// Result array of the CSR_graph entry points: one device buffer per element
// type, kept between calls and grown on demand (the reference allocates and
// frees one per call, e.g. GPU_BFS_csr.cuh:266-283).  Single host thread,
// like the reference's API.
template <typename T>
inline T* result_buffer(std::size_t count) {
    static T* p = nullptr;
    static std::size_t cap = 0;
    if (count > cap) {
        device_free(p);
        cap = 0;
        p = device_alloc<T>(count, "cudaMalloc(result)");
        if (p) cap = count;
    }
    return p;
}

template <typename T>
inline bool result_to_host(const T* p, std::size_t count, std::vector<T>& out) {
    out.resize(count);
    if (!count) return true;
    return cuda_ok(cudaMemcpy(out.data(), p, count * sizeof(T), cudaMemcpyDeviceToHost), "cudaMemcpy(result)");
}

template <typename W>
inline ghb_graph* resident(CSR_graph<W>& csr, int vertices) {
    return resident_graph(workspace(), vertices, csr.OUTs_Edges.size(), csr.out_pointer, csr.out_edge,
                          csr.out_edge_weight, csr.in_pointer, csr.in_edge, csr.in_edge_weight);
}

// graph.res_trans_id_val (CPU_adj_list.hpp:208-218) on the host's threads:
// (name, value) for every vertex that exists, in id order.
template <typename W, typename T>
inline std::vector<std::pair<std::string, T>> trans_id_val(graph_structure<W>& graph, const std::vector<T>& res) {
    const int n = (int)res.size();
    const unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    const unsigned parts = n < 65536 ? 1u : nt;
    std::vector<long long> base(parts + 1, 0);
    parallel_rows_parts(n, parts, [&](unsigned t, int b, int e) {
        long long c = 0;
        for (int i = b; i < e; ++i) c += graph.vertex_id_to_str[i].second ? 1 : 0;
        base[t + 1] = c;
    });
    for (unsigned t = 0; t < parts; ++t) base[t + 1] += base[t];
    std::vector<std::pair<std::string, T>> out((std::size_t)base[parts]);
    parallel_rows_parts(n, parts, [&](unsigned t, int b, int e) {
        long long o = base[t];
        for (int i = b; i < e; ++i)
            if (graph.vertex_id_to_str[i].second) {
                out[(std::size_t)o].first = graph.vertex_id_to_str[i].first;
                out[(std::size_t)o].second = res[i];
                ++o;
            }
    });
    return out;
}

// graph.res_trans_id_id (CPU_adj_list.hpp:220-233) on the host's threads:
// (name, name of the label vertex); a label that names no vertex is reported
// on stderr and its pair left out, as there.
template <typename W>
inline std::vector<std::pair<std::string, std::string>> trans_id_id(graph_structure<W>& graph,
                                                                   const std::vector<int>& res) {
    const int n = (int)res.size();
    const unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    const unsigned parts = n < 65536 ? 1u : nt;
    std::vector<long long> base(parts + 1, 0);
    auto keep = [&](int i) { return graph.vertex_id_to_str[i].second && graph.vertex_id_to_str[res[i]].second; };
    parallel_rows_parts(n, parts, [&](unsigned t, int b, int e) {
        long long c = 0;
        for (int i = b; i < e; ++i) c += keep(i) ? 1 : 0;
        base[t + 1] = c;
    });
    for (unsigned t = 0; t < parts; ++t) base[t + 1] += base[t];
    std::vector<std::pair<std::string, std::string>> out((std::size_t)base[parts]);
    parallel_rows_parts(n, parts, [&](unsigned t, int b, int e) {
        long long o = base[t];
        for (int i = b; i < e; ++i)
            if (keep(i)) {
                out[(std::size_t)o].first = graph.vertex_id_to_str[i].first;
                out[(std::size_t)o].second = graph.vertex_id_to_str[res[i]].first;
                ++o;
            }
    });
    for (int i = 0; i < n; ++i)
        if (graph.vertex_id_to_str[i].second && !graph.vertex_id_to_str[res[i]].second)
            std::cerr << "vertex " << graph.vertex_id_to_str[res[i]].first << " not exist!" << std::endl;
    return out;
}

}  // namespace ghb_dropin
