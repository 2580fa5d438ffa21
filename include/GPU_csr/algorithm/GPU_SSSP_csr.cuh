// GPU_SSSP_csr.cuh - drop-in Cuda_SSSP / csr_sssp (reference:
// include/GPU_csr/algorithm/GPU_SSSP_csr.cuh:253-327) over libghb's FP64
// delta-stepping: Cuda_SSSP on the CSR_graph's resident relabelled copy
// (ghb_graph_sssp), csr_sssp on the raw arrays it is given (ghb_sssp).
// Unreached vertices get INF (LDBC passes DBL_MAX).  The distances equal the
// CPU Dijkstra's bit for bit.
#pragma once

#include <string>
#include <utility>
#include <vector>

#include <GPU_gpma/GPU_gpma.hpp>
#include <GPU_csr/GPU_csr.hpp>
#include <GPU_csr/algorithm/ghb_dropin_util.hpp>

inline std::vector<double> csr_sssp(int* keys, double* values, int* row_offsets, SIZE_TYPE node_size,
                                    SIZE_TYPE edge_size, SIZE_TYPE start_node, double INF = 10000000000) {
    (void)edge_size;
    using namespace ghb_dropin;
    std::vector<double> result;
    DeviceBuffer<double> dist((std::size_t)node_size);
    if (!ghb_ok(ghb_sssp(workspace(), (int32_t)node_size, row_offsets, keys, values, (int32_t)start_node, INF, dist.p,
                         nullptr, nullptr),
                "ghb_sssp"))
        return result;
    dist.to_host(result);
    return result;
}

inline std::vector<std::pair<std::string, double>> Cuda_SSSP(graph_structure<double>& graph,
                                                             CSR_graph<double>& csr_graph, std::string src_v,
                                                             double max_dis) {
    using namespace ghb_dropin;
    const int V = (int)csr_graph.OUTs_Neighbor_start_pointers.size() - 1;
    const int src = graph.vertex_str_to_id[src_v];
    std::vector<double> d;
    ghb_graph* g = resident(csr_graph, V);
    double* dist = result_buffer<double>((std::size_t)V);
    if (g && dist &&
        ghb_ok(ghb_graph_sssp(workspace(), g, src, max_dis, dist, nullptr, nullptr), "ghb_graph_sssp"))
        result_to_host(dist, (std::size_t)V, d);
    return trans_id_val(graph, d);
}
