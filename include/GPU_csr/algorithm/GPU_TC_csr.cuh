// GPU_TC_csr.cuh - drop-in Cuda_TC / Cuda_TC_PerNode (reference:
// include/GPU_csr/algorithm/GPU_TC_csr.cuh:46-68) over ghb_tc: the
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
    std::vector<int> c = Cuda_TC_PerNode(csr_graph.out_pointer, csr_graph.out_edge, graph.V);
    return graph.res_trans_id_val(c);
}
