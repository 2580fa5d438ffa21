// GPU_TC_gpma.cuh - drop-in Cuda_TC (GPMA overload) / Cuda_TC_PerNode
// (reference: include/GPU_gpma/algorithm/GPU_TC_gpma.cuh:67-91) over
// libghb's triangle counting on the GPMA's compact CSR of an undirected
// graph: per vertex, 6 x the triangles through it (int32, as the reference).
#pragma once

#include <string>
#include <utility>
#include <vector>

#include <GPU_gpma/algorithm/ghb_gpma_util.hpp>

inline std::vector<int> Cuda_TC_PerNode(GPMA& gpma_graph, int V) {
    using namespace ghb_gpma_dropin;
    std::vector<int> result;
    CsrView g = csr_of(gpma_graph, false);
    if (!g.valid) return result;
    ghb_dropin::DeviceBuffer<int> counts((std::size_t)g.n);
    if (ok(ghb_tc(workspace(), g.n, g.rowptr, g.col, nullptr, counts.p, nullptr), "ghb_tc")) counts.to_host(result);
    result.resize((std::size_t)V, 0);
    return result;
}

inline std::vector<std::pair<std::string, int>> Cuda_TC(graph_structure<double>& graph, GPMA& gpma_graph) {
    std::vector<int> tc = Cuda_TC_PerNode(gpma_graph, graph.size());
    return graph.res_trans_id_val(tc);
}
