// GPU_WCC_csr.cuh - drop-in Cuda_WCC / WCC_GPU (reference:
// include/GPU_csr/algorithm/GPU_WCC_csr.cuh:83-129) over ghb_graph_wcc: every
// vertex labelled with the smallest vertex id of its weak component.
#pragma once

#include <string>
#include <utility>
#include <vector>

#include <GPU_csr/GPU_csr.hpp>
#include <GPU_csr/algorithm/ghb_dropin_util.hpp>

inline std::vector<int> WCC_GPU(graph_structure<double>& graph, CSR_graph<double>& input_graph) {
    using namespace ghb_dropin;
    const int N = graph.size();
    std::vector<int> result;
    // The CSR_graph's resident copy links over its symmetric in+out rows,
    // which hold every edge of the graph (the reference walks the in-CSR).
    ghb_graph* g = resident(input_graph, N);
    int* label = result_buffer<int>((std::size_t)N);
    if (g && label && ghb_ok(ghb_graph_wcc(workspace(), g, label), "ghb_graph_wcc"))
        result_to_host(label, (std::size_t)N, result);
    return result;
}

inline std::vector<std::pair<std::string, std::string>> Cuda_WCC(graph_structure<double>& graph,
                                                                 CSR_graph<double>& csr_graph) {
    std::vector<int> r = WCC_GPU(graph, csr_graph);
    return ghb_dropin::trans_id_id(graph, r);
}
