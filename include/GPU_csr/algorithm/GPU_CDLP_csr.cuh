// GPU_CDLP_csr.cuh - drop-in Cuda_CDLP / CDLP_GPU (reference:
// include/GPU_csr/algorithm/GPU_CDLP_csr.cuh:25-210) over ghb_cdlp: most
// frequent label over the all-CSR row (in then out), smallest on ties; a
// vertex with an empty row keeps its label, as on the CPU path
// (CPU_Community_Detection.hpp:37).
#pragma once

#include <string>
#include <utility>
#include <vector>

#include <GPU_csr/GPU_csr.hpp>
#include <GPU_csr/algorithm/ghb_dropin_util.hpp>

inline void CDLP_GPU(graph_structure<double>& graph, CSR_graph<double>& input_graph, std::vector<std::string>& res,
                     int max_iterations) {
    using namespace ghb_dropin;
    const int N = graph.size();
    res.clear();
    DeviceBuffer<int> labels((std::size_t)N);
    std::vector<int> lab;
    if (!ghb_ok(ghb_cdlp(workspace(), N, input_graph.all_pointer, input_graph.all_edge, max_iterations, labels.p),
                "ghb_cdlp"))
        return;
    labels.to_host(lab);
    res.resize(N);
    for (int i = 0; i < N; ++i) res[i] = graph.vertex_id_to_str[lab[i]].first;
}

inline std::vector<std::pair<std::string, std::string>> Cuda_CDLP(graph_structure<double>& graph,
                                                                  CSR_graph<double>& input_graph, int max_iterations) {
    std::vector<std::string> result;
    CDLP_GPU(graph, input_graph, result, max_iterations);
    std::vector<std::pair<std::string, std::string>> res;
    res.reserve(result.size());
    for (std::size_t i = 0; i < result.size(); ++i) res.emplace_back(graph.vertex_id_to_str[i].first, result[i]);
    return res;
}
