// GPU_CDLP_gpma.cuh - drop-in Cuda_CDLP_optimized / gpma_cdlp (reference:
// include/GPU_gpma/algorithm/GPU_CDLP_gpma.cuh:245-371) over libghb's CDLP:
// each vertex takes the most frequent label over its gpma_in row then its
// gpma_out row (smallest label on ties); isolated vertices keep their own.
#pragma once

#include <string>
#include <utility>
#include <vector>

#include <GPU_gpma/algorithm/ghb_gpma_util.hpp>

inline void gpma_cdlp(graph_structure<double>& graph, GPMA& gpma_in, GPMA& gpma_out, std::vector<std::string>& res,
                      int max_iterations) {
    using namespace ghb_gpma_dropin;
    res.clear();
    CsrView in = csr_of(gpma_in, false);
    if (!in.valid) return;
    // gpma_in's view stays valid while gpma_out's is made (they are separate
    // graphs, or the same one).
    CsrView out = csr_of(gpma_out, false);
    if (!out.valid || in.n != out.n) return;
    int32_t m_in = 0, m_out = 0;
    cudaMemcpy(&m_in, in.rowptr + in.n, sizeof(int32_t), cudaMemcpyDeviceToHost);
    cudaMemcpy(&m_out, out.rowptr + out.n, sizeof(int32_t), cudaMemcpyDeviceToHost);
    ghb_dropin::DeviceBuffer<int> all_rp((std::size_t)in.n + 1);
    ghb_dropin::DeviceBuffer<int> all_col((std::size_t)m_in + (std::size_t)m_out);
    ghb_dropin::DeviceBuffer<int> labels((std::size_t)in.n);
    if (!ok(ghb_csr_merge_in_out(workspace(), in.n, in.rowptr, in.col, out.rowptr, out.col, all_rp.p, all_col.p),
            "ghb_csr_merge_in_out"))
        return;
    if (!ok(ghb_cdlp(workspace(), in.n, all_rp.p, all_col.p, max_iterations, labels.p), "ghb_cdlp")) return;
    std::vector<int> lab;
    labels.to_host(lab);
    res.resize(lab.size());
    for (std::size_t i = 0; i < lab.size(); ++i) res[i] = graph.vertex_id_to_str[lab[i]].first;
}

inline std::vector<std::pair<std::string, std::string>> Cuda_CDLP_optimized(graph_structure<double>& graph,
                                                                            GPMA& gpma_in, GPMA& gpma_out,
                                                                            int max_iterations) {
    std::vector<std::string> result;
    gpma_cdlp(graph, gpma_in, gpma_out, result, max_iterations);
    std::vector<std::pair<std::string, std::string>> res;
    res.reserve(result.size());
    for (std::size_t i = 0; i < result.size(); ++i) res.emplace_back(graph.vertex_id_to_str[i].first, result[i]);
    return res;
}
