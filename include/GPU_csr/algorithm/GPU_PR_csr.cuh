// GPU_PR_csr.cuh - drop-in Cuda_PR / GPU_PR (reference:
// include/GPU_csr/algorithm/GPU_PR_csr.cuh:29-197) over ghb_pagerank (FP64
// pull form, dangling mass spread uniformly).  The ranks are within 1e-6
// relative L1 of the CPU path's FP64 values.
#pragma once

#include <string>
#include <utility>
#include <vector>

#include <GPU_csr/GPU_csr.hpp>
#include <GPU_csr/algorithm/ghb_dropin_util.hpp>

inline void GPU_PR(graph_structure<double>& graph, CSR_graph<double>& csr_graph, std::vector<double>& result,
                   int iterations, double damping) {
    using namespace ghb_dropin;
    const int N = graph.V;
    result.clear();
    DeviceBuffer<double> rank((std::size_t)N);
    ghb_pr_options o{};
    o.iterations = iterations;
    o.damping = damping;
    o.precision = GHB_PR_FP64;
    if (ghb_ok(ghb_pagerank(workspace(), N, csr_graph.in_pointer, csr_graph.in_edge, csr_graph.out_pointer, &o,
                            rank.p, nullptr),
               "ghb_pagerank"))
        rank.to_host(result);
}

inline std::vector<std::pair<std::string, double>> Cuda_PR(graph_structure<double>& graph,
                                                           CSR_graph<double>& csr_graph, int iterations,
                                                           double damping) {
    std::vector<double> result;
    GPU_PR(graph, csr_graph, result, iterations, damping);
    return graph.res_trans_id_val(result);
}
