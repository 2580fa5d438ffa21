// GPU_BFS_csr.cuh - drop-in Cuda_BFS / csr_bfs (reference:
// include/GPU_csr/algorithm/GPU_BFS_csr.cuh:13, 258-334) over libghb's
// direction-optimising BFS: Cuda_BFS on the CSR_graph's resident relabelled
// copy (ghb_graph_bfs), csr_bfs on the raw arrays it is given (ghb_bfs).
// Depth of unreached vertices: INT_MAX.
#pragma once

#include <climits>
#include <string>
#include <utility>
#include <vector>

#include <GPU_gpma/GPU_gpma.hpp>
#include <GPU_csr/GPU_csr.hpp>
#include <GPU_csr/algorithm/ghb_dropin_util.hpp>

// keys = out_edge, values = out_edge_weight (unused), row_offsets = out_pointer.
// Only the out-CSR is given here, so every level runs top-down.
inline std::vector<int> csr_bfs(int* keys, double* values, int* row_offsets, int node_size, int edge_size,
                                int start_node, int max_depth) {
    (void)values;
    (void)edge_size;
    using namespace ghb_dropin;
    std::vector<int> result;
    DeviceBuffer<int> depth((std::size_t)node_size);
    if (!ghb_ok(ghb_bfs(workspace(), node_size, row_offsets, keys, nullptr, nullptr, start_node, max_depth, depth.p,
                        nullptr, nullptr),
                "ghb_bfs"))
        return result;
    depth.to_host(result);
    return result;
}

inline std::vector<std::pair<std::string, int>> Cuda_BFS(graph_structure<double>& graph, CSR_graph<double>& csr_graph,
                                                         std::string src_v, int min_depth = 0,
                                                         int max_depth = INT_MAX) {
    (void)min_depth;
    using namespace ghb_dropin;
    const int V = graph.V;
    const int src = graph.vertex_str_to_id[src_v];
    std::vector<int> depth;
    // The CSR_graph's resident relabelled copy (built on its first call; the
    // in-CSR, aliasing the out-CSR when undirected, enables bottom-up levels).
    ghb_graph* g = resident(csr_graph, V);
    // The depths come over as one byte each and are widened on host threads
    // (ghb_graph_bfs_many_host with one source) into a host vector that this
    // thread keeps between calls, so no page of it is first touched per call.
    static thread_local std::vector<int> host_depth;
    host_depth.resize((std::size_t)V);
    if (g && ghb_ok(ghb_graph_bfs_many_host(workspace(), g, &src, 1, max_depth, host_depth.data(), 0, nullptr,
                                            nullptr),
                    "ghb_graph_bfs_many_host"))
        return trans_id_val(graph, host_depth);
    return trans_id_val(graph, depth);
}
