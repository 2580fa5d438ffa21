// GPU_BFS_pre_csr.cuh - drop-in Cuda_BFS_pre / bfs_pre (reference:
// include/GPU_csr/algorithm/GPU_BFS_pre_csr.cuh:15, 62-155) over
// ghb_bfs_pred: depths plus, for every reached vertex, its smallest-id parent
// one level up (-1 for the source and unreached vertices).
#pragma once

#include <climits>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include <GPU_csr/GPU_csr.hpp>
#include <GPU_csr/algorithm/ghb_dropin_util.hpp>

inline std::vector<int> bfs_pre(int* d_row_offsets_out, int* d_column_indices_out, int* d_row_offsets_in,
                                int* d_column_indices_in, int num_nodes, int start_node, std::vector<int>& pre_v,
                                int max_depth) {
    using namespace ghb_dropin;
    std::vector<int> result;
    DeviceBuffer<int> depth((std::size_t)num_nodes), pred((std::size_t)num_nodes);
    if (!ghb_ok(ghb_bfs_pred(workspace(), num_nodes, d_row_offsets_out, d_column_indices_out, d_row_offsets_in,
                             d_column_indices_in, start_node, max_depth, depth.p, pred.p, nullptr, nullptr),
                "ghb_bfs_pred"))
        return result;
    depth.to_host(result);
    pred.to_host(pre_v);
    return result;
}

inline std::vector<std::pair<std::string, int>> Cuda_BFS_pre(graph_structure<double>& graph,
                                                             CSR_graph<double>& csr_graph, std::string src_v,
                                                             std::vector<int>& pre_v, int min_depth = 0,
                                                             int max_depth = INT_MAX) {
    (void)min_depth;
    const int V = (int)csr_graph.OUTs_Neighbor_start_pointers.size() - 1;
    pre_v.resize(graph.V);
    const int src = graph.vertex_str_to_id[src_v];
    std::vector<int> depth = bfs_pre(csr_graph.out_pointer, csr_graph.out_edge, csr_graph.in_pointer,
                                     csr_graph.in_edge, V, src, pre_v, max_depth);
    // The reference walks every parent chain back to the source and reports
    // a broken link (GPU_BFS_pre_csr.cuh:132-153); kept as a self-check.
    for (int i = 0; i < (int)depth.size(); ++i) {
        int now = i, pre = pre_v[i];
        while (pre != -1) {
            bool found = false;
            for (const auto& e : graph.OUTs[pre])
                if (e.first == now) {
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
    }
    return graph.res_trans_id_val(depth);
}
