// GPU_SSSP_gpma.cuh - drop-in Cuda_SSSP_optimized / gpma_sssp (reference:
// include/GPU_gpma/algorithm/GPU_SSSP_gpma.cuh:13, 262-339) over libghb's
// delta-stepping SSSP on the GPMA's compact CSR; the GPMA values are the
// weights.  Unreached vertices get max_dis (1e10 by default, as the
// reference's prototype has it).
#pragma once

#include <string>
#include <utility>
#include <vector>

#include <GPU_gpma/algorithm/ghb_gpma_util.hpp>

inline std::vector<double> gpma_sssp(GPMA& gpma, SIZE_TYPE start_node, double INF) {
    using namespace ghb_gpma_dropin;
    std::vector<double> result;
    CsrView g = csr_of(gpma, true);
    if (!g.valid) return result;
    ghb_dropin::DeviceBuffer<double> dist((std::size_t)g.n);
    if (!ok(ghb_sssp(workspace(), g.n, g.rowptr, g.col, g.w, (int32_t)start_node, INF, dist.p, nullptr, nullptr),
            "ghb_sssp"))
        return result;
    dist.to_host(result);
    return result;
}

inline std::vector<std::pair<std::string, double>> Cuda_SSSP_optimized(graph_structure<double>& graph, GPMA& gpma,
                                                                       std::string src_v,
                                                                       double max_dis = 10000000000) {
    const int src = graph.vertex_str_to_id[src_v];
    std::vector<double> dist = gpma_sssp(gpma, (SIZE_TYPE)src, max_dis);
    return graph.res_trans_id_val(dist);
}
