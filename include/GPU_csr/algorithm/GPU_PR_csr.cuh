// GPU_PR_csr.cuh - drop-in Cuda_PR / GPU_PR (reference:
// include/GPU_csr/algorithm/GPU_PR_csr.cuh:29-197) over ghb_graph_pagerank on
// the CSR_graph's resident relabelled copy (FP64
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
    ghb_pr_options o{};
    o.iterations = iterations;
    o.damping = damping;
    o.precision = GHB_PR_FP64;
    ghb_graph* g = resident(csr_graph, N);
    double* rank = result_buffer<double>((std::size_t)N);
    if (g && rank && ghb_ok(ghb_graph_pagerank(workspace(), g, &o, rank, nullptr), "ghb_graph_pagerank"))
        result_to_host(rank, (std::size_t)N, result);
}

inline std::vector<std::pair<std::string, double>> Cuda_PR(graph_structure<double>& graph,
                                                           CSR_graph<double>& csr_graph, int iterations,
                                                           double damping) {
    std::vector<double> result;
    GPU_PR(graph, csr_graph, result, iterations, damping);
    return ghb_dropin::trans_id_val(graph, result);
}
