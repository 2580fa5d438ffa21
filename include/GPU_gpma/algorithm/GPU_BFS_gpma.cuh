// GPU_BFS_gpma.cuh - drop-in Cuda_BFS_optimized / gpma_bfs (reference:
// include/GPU_gpma/algorithm/GPU_BFS_gpma.cuh:13, 263-339) over libghb's BFS
// on the GPMA's compact CSR.  Depth of unreached vertices: max_depth
// (INT_MAX by default), as the reference's init_label sets it.
#pragma once

#include <climits>
#include <string>
#include <utility>
#include <vector>

#include <GPU_gpma/algorithm/ghb_gpma_util.hpp>

inline std::vector<int> gpma_bfs(GPMA& gpma, SIZE_TYPE start_node, int max_depth) {
    using namespace ghb_gpma_dropin;
    std::vector<int> result;
    CsrView g = csr_of(gpma, false);
    if (!g.valid) return result;
    ghb_dropin::DeviceBuffer<int> depth((std::size_t)g.n);
    if (!ok(ghb_bfs(workspace(), g.n, g.rowptr, g.col, nullptr, nullptr, (int32_t)start_node, max_depth, depth.p,
                    nullptr, nullptr),
            "ghb_bfs"))
        return result;
    depth.to_host(result);
    if (max_depth != INT_MAX)
        for (int& d : result)
            if (d == INT_MAX) d = max_depth;
    return result;
}

inline std::vector<std::pair<std::string, int>> Cuda_BFS_optimized(graph_structure<double>& graph, GPMA& gpma,
                                                                   std::string src_v, int min_depth = 0,
                                                                   int max_depth = INT_MAX) {
    (void)min_depth;
    const int src = graph.vertex_str_to_id[src_v];
    std::vector<int> depth = gpma_bfs(gpma, (SIZE_TYPE)src, max_depth);
    return graph.res_trans_id_val(depth);
}
