// GPU_TC_csr.cuh - drop-in Cuda_TC / Cuda_TC_PerNode (reference:
// include/GPU_csr/algorithm/GPU_TC_csr.cuh:46-68): Cuda_TC over ghb_graph_tc on
// the CSR_graph's resident relabelled copy, Cuda_TC_PerNode over ghb_tc on
// the raw arrays it is given: the
// reference's per-vertex counts (6 x triangles on a symmetric graph), in its
// wrapping int32.
#pragma once

#include <string>
#include <utility>
#include <vector>

#include <GPU_gpma/GPU_gpma.hpp>
#include <GPU_csr/GPU_csr.hpp>
#include <GPU_csr/algorithm/ghb_dropin_util.hpp>

inline std::vector<int> Cuda_TC_PerNode(int* d_row_offsets, int* d_col_indices, int node_size) {
    using namespace ghb_dropin;
    std::vector<int> counts;
    DeviceBuffer<int> c((std::size_t)node_size);
    if (ghb_ok(ghb_tc(workspace(), node_size, d_row_offsets, d_col_indices, nullptr, c.p, nullptr), "ghb_tc"))
        c.to_host(counts);
    return counts;
}

inline std::vector<std::pair<std::string, int>> Cuda_TC(graph_structure<double>& graph,
                                                        CSR_graph<double>& csr_graph) {
    using namespace ghb_dropin;
    std::vector<int> c;
    ghb_graph* g = resident(csr_graph, graph.V);
    int* counts = result_buffer<int>((std::size_t)graph.V);
    if (g && counts && ghb_ok(ghb_graph_tc(workspace(), g, nullptr, counts, nullptr), "ghb_graph_tc"))
        result_to_host(counts, (std::size_t)graph.V, c);
    return trans_id_val(graph, c);
}
