// GPU_CDLP_csr.cuh - drop-in Cuda_CDLP / CDLP_GPU (reference:
// include/GPU_csr/algorithm/GPU_CDLP_csr.cuh:25-210) over ghb_graph_cdlp on
// the CSR_graph's resident relabelled copy: most
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
    std::vector<int> lab;
    ghb_graph* g = resident(input_graph, N);
    int* labels = result_buffer<int>((std::size_t)N);
    if (!g || !labels || !ghb_ok(ghb_graph_cdlp(workspace(), g, max_iterations, labels), "ghb_graph_cdlp")) return;
    result_to_host(labels, (std::size_t)N, lab);
    res.resize(N);
    parallel_rows(N, [&](int b, int e) {
        for (int i = b; i < e; ++i) res[i] = graph.vertex_id_to_str[lab[i]].first;
    });
}

inline std::vector<std::pair<std::string, std::string>> Cuda_CDLP(graph_structure<double>& graph,
                                                                  CSR_graph<double>& input_graph, int max_iterations) {
    std::vector<std::string> result;
    CDLP_GPU(graph, input_graph, result, max_iterations);
    std::vector<std::pair<std::string, std::string>> res(result.size());
    ghb_dropin::parallel_rows((int)result.size(), [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            res[i].first = graph.vertex_id_to_str[i].first;
            res[i].second = std::move(result[i]);
        }
    });
    return res;
}
