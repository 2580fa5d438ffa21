// GPU_PR_gpma.cuh - drop-in Cuda_PR_optimized / gpma_pr (reference:
// include/GPU_gpma/algorithm/GPU_PR_gpma.cuh:160-245) over libghb's FP64
// PageRank: pull over gpma_in's rows, out-degrees from gpma_out's rows (the
// reference takes them from the host graph_structure, which a batch of GPMA
// updates does not change), dangling mass spread uniformly.
#pragma once

#include <string>
#include <utility>
#include <vector>

#include <GPU_gpma/algorithm/ghb_gpma_util.hpp>

inline std::vector<double> gpma_pr(GPMA& gpma_in, GPMA& gpma_out, int iterations, double damping) {
    using namespace ghb_gpma_dropin;
    std::vector<double> result;
    CsrView in = csr_of(gpma_in, false);
    CsrView out = csr_of(gpma_out, false);
    if (!in.valid || !out.valid) return result;
    if (in.n != out.n) {
        std::fprintf(stderr, "gpma_pr: in and out GPMAs differ in size\n");
        return result;
    }
    ghb_dropin::DeviceBuffer<double> rank((std::size_t)in.n);
    ghb_pr_options o{};
    o.iterations = iterations;
    o.damping = damping;
    o.precision = GHB_PR_FP64;
    if (ok(ghb_pagerank(workspace(), in.n, in.rowptr, in.col, out.rowptr, &o, rank.p, nullptr), "ghb_pagerank"))
        rank.to_host(result);
    return result;
}

inline std::vector<std::pair<std::string, double>> Cuda_PR_optimized(graph_structure<double>& graph, GPMA& gpma_in,
                                                                     GPMA& gpma_out, int iterations, double damping) {
    std::vector<double> rank = gpma_pr(gpma_in, gpma_out, iterations, damping);
    return graph.res_trans_id_val(rank);
}
