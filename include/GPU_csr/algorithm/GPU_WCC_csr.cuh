// GPU_WCC_csr.cuh - drop-in Cuda_WCC / WCC_GPU (reference:
// include/GPU_csr/algorithm/GPU_WCC_csr.cuh:83-129) over ghb_wcc: every
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
    DeviceBuffer<int> label((std::size_t)N);
    // The in-CSR holds every edge once (the reference links over it too).
    if (ghb_ok(ghb_wcc(workspace(), N, input_graph.in_pointer, input_graph.in_edge, label.p), "ghb_wcc"))
        label.to_host(result);
    return result;
}

inline std::vector<std::pair<std::string, std::string>> Cuda_WCC(graph_structure<double>& graph,
                                                                 CSR_graph<double>& csr_graph) {
    std::vector<int> r = WCC_GPU(graph, csr_graph);
    return graph.res_trans_id_id(r);
}
