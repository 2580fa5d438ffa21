// GPU_SSSP_pre_csr.cuh - drop-in Cuda_SSSP_pre / csr_sssp_pre (reference:
// include/GPU_csr/algorithm/GPU_SSSP_pre_csr.cuh:256-368) over
// ghb_sssp_pred: FP64 distances plus, per reached vertex, the smallest-id
// predecessor u with dist[u] + w(u, v) == dist[v] exactly (-1 for the source
// and unreached vertices).  The reference's spin-locked relax becomes a
// lock-free pass after the distances are final.
#pragma once

#include <cmath>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include <GPU_gpma/GPU_gpma.hpp>
#include <GPU_csr/GPU_csr.hpp>
#include <GPU_csr/algorithm/GPU_SSSP_csr.cuh>
#include <GPU_csr/algorithm/ghb_dropin_util.hpp>

inline std::vector<double> csr_sssp_pre(int* keys, double* values, int* row_offsets, SIZE_TYPE node_size,
                                        SIZE_TYPE edge_size, SIZE_TYPE start_node, std::vector<int>& pre_v,
                                        double INF = 10000000000) {
    (void)edge_size;
    using namespace ghb_dropin;
    std::vector<double> result;
    DeviceBuffer<double> dist((std::size_t)node_size);
    DeviceBuffer<int> pred((std::size_t)node_size);
    // Only the out-CSR is given: predecessors come from a push pass.
    if (!ghb_ok(ghb_sssp_pred(workspace(), (int32_t)node_size, row_offsets, keys, values, nullptr, nullptr, nullptr,
                              (int32_t)start_node, INF, dist.p, pred.p, nullptr, nullptr),
                "ghb_sssp_pred"))
        return result;
    dist.to_host(result);
    pred.to_host(pre_v);
    return result;
}

inline std::vector<std::pair<std::string, double>> Cuda_SSSP_pre(graph_structure<double>& graph,
                                                                 CSR_graph<double>& csr_graph, std::string src_v,
                                                                 std::vector<int>& pre_v, double max_dis) {
    const int V = (int)csr_graph.OUTs_Neighbor_start_pointers.size() - 1;
    const int E = (int)csr_graph.OUTs_Edges.size();
    const int src = graph.vertex_str_to_id[src_v];
    pre_v.resize(graph.V);
    std::vector<double> d = csr_sssp_pre(csr_graph.out_edge, csr_graph.out_edge_weight, csr_graph.out_pointer,
                                         (SIZE_TYPE)V, (SIZE_TYPE)E, (SIZE_TYPE)src, pre_v, max_dis);
    // Path-sum self-check of the reference (GPU_SSSP_pre_csr.cuh:339-365).
    for (int i = 0; i < (int)d.size(); ++i) {
        int now = i, pre = pre_v[i];
        if (pre == -1) continue;
        double sum = 0;
        while (pre != -1) {
            bool found = false;
            for (const auto& e : graph.OUTs[pre])
                if (e.first == now) {
                    sum += e.second;
                    found = true;
                    break;
                }
            if (!found) {
                std::printf("Not found!\n");
                break;
            }
            now = pre;
            pre = pre_v[pre];
        }
        if (std::fabs(sum - d[i]) > 1e-4)
            std::printf("Error: pre_v is wrong!\nvertex: %d, sum: %.5lf, dis: %.5lf\n", i, sum, d[i]);
    }
    return graph.res_trans_id_val(d);
}
