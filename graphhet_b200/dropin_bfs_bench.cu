// dropin_bfs_bench - the reference-facing Cuda_BFS (include/GPU_csr/
// algorithm/GPU_BFS_csr.cuh) timed end to end on a seeded RMAT graph, the
// way the reference's LDBC driver times its entry points
// (LDBC_GPU_csr.cu:82-95: one untimed call, then timed calls): graph_structure
// filled from the generator, toCSR, then per source the call that a driver
// makes (name in, vector<pair<name, depth>> out).  Besides the whole call it
// times its parts on the same resident handle: the BFS plus the copy of the
// depth vector to the host (what the call does before naming the results),
// the multi-threaded id -> name conversion the drop-in uses, and the
// reference's own serial res_trans_id_val.  Prints one JSON line.
//
// usage: dropin_bfs_bench scale edge_factor seed src0,src1,...
// Built by `make dropin` (needs the reference's include tree for
// graph_structure); bench.py runs it.
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <sstream>
#include <string>
#include <vector>

#include <GPU_csr/GPU_csr.hpp>
#include <GPU_csr/algorithm/GPU_BFS_csr.cuh>
#include <ghb.h>

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool check(int status, const char* what) {
    if (status != GHB_OK) {
        std::fprintf(stderr, "%s: %s (%s)\n", what, ghb_status_string(status), ghb_last_error());
        return false;
    }
    return true;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s scale edge_factor seed src0,src1,...\n", argv[0]);
        return 2;
    }
    const int scale = std::atoi(argv[1]);
    const long long edge_factor = std::atoll(argv[2]);
    const unsigned long long seed = std::strtoull(argv[3], nullptr, 10);
    std::vector<int> srcs;
    {
        std::stringstream ss(argv[4]);
        std::string tok;
        while (std::getline(ss, tok, ',')) srcs.push_back(std::atoi(tok.c_str()));
    }
    if (scale < 1 || scale > 30 || srcs.empty()) return 2;
    const int n = 1 << scale;
    const long long ne = edge_factor << scale;
    ghb_workspace* ws = ghb_default_workspace();
    if (!ws) return 1;

    // Seeded RMAT (a/b/c = .57/.19/.19, permuted ids), symmetrised, loops
    // dropped, weights from the seed: the benchmark graph.
    const double t_gen = now_s();
    int *src = nullptr, *dst = nullptr, *rp = nullptr, *col = nullptr;
    double* w = nullptr;
    long long m = 0;
    bool ok = cudaMalloc(&src, sizeof(int) * ne) == cudaSuccess && cudaMalloc(&dst, sizeof(int) * ne) == cudaSuccess &&
              cudaMalloc(&rp, sizeof(int) * (n + 1ll)) == cudaSuccess &&
              cudaMalloc(&col, sizeof(int) * 2 * ne) == cudaSuccess &&
              cudaMalloc(&w, sizeof(double) * 2 * ne) == cudaSuccess;
    ok = ok && check(ghb_gen_rmat(ws, scale, ne, seed, 0.57, 0.19, 0.19, 1, src, dst), "ghb_gen_rmat");
    int64_t m64 = 0;
    ok = ok && check(ghb_csr_build(ws, n, src, dst, nullptr, ne, GHB_BUILD_SYMMETRIZE | GHB_BUILD_DROP_SELF_LOOPS, 1,
                                   seed, rp, col, w, &m64),
                     "ghb_csr_build");
    if (!ok) return 1;
    m = m64;
    std::vector<int> h_rp(n + 1ll), h_col(m);
    std::vector<double> h_w(m);
    cudaMemcpy(h_rp.data(), rp, sizeof(int) * (n + 1ll), cudaMemcpyDeviceToHost);
    cudaMemcpy(h_col.data(), col, sizeof(int) * m, cudaMemcpyDeviceToHost);
    cudaMemcpy(h_w.data(), w, sizeof(double) * m, cudaMemcpyDeviceToHost);
    cudaFree(src);
    cudaFree(dst);
    cudaFree(rp);
    cudaFree(col);
    cudaFree(w);

    // The reference's graph_structure, rows in sorted order (what its
    // add_edge inserts produce), vertex names = decimal ids.
    graph_structure<double> graph(n);
    graph.vertex_id_to_str.resize(n);
    ghb_dropin::parallel_rows(n, [&](int b, int e) {
        for (int v = b; v < e; ++v) {
            auto& o = graph.OUTs[v];
            auto& i = graph.INs[v];
            o.reserve(h_rp[v + 1] - h_rp[v]);
            i.reserve(h_rp[v + 1] - h_rp[v]);
            for (int j = h_rp[v]; j < h_rp[v + 1]; ++j) {
                o.emplace_back(h_col[j], h_w[j]);
                i.emplace_back(h_col[j], h_w[j]);
            }
            graph.vertex_id_to_str[v] = std::make_pair(std::to_string(v), true);
        }
    });
    graph.vertex_str_to_id.reserve((std::size_t)n);
    for (int v = 0; v < n; ++v) graph.vertex_str_to_id[graph.vertex_id_to_str[v].first] = v;
    graph.E = m;
    std::vector<int>().swap(h_col);
    std::vector<double>().swap(h_w);
    const double gen_s = now_s() - t_gen;

    const double t_csr = now_s();
    CSR_graph<double> csr;
    csr = toCSR(graph, false);
    const double csr_s = now_s() - t_csr;

    // First call: builds the CSR_graph's resident copy (untimed warm-up in
    // the reference's driver).
    const double t_first = now_s();
    auto first = Cuda_BFS(graph, csr, std::to_string(srcs[0]));
    const double first_s = now_s() - t_first;

    long long edges = 0;
    double t_call = 0, t_core = 0, t_conv = 0, t_conv_ref = 0;
    bool same = first.size() == (std::size_t)n;
    ghb_graph* g = ghb_dropin::resident(csr, n);
    std::vector<int> depth((std::size_t)n);
    for (int s : srcs) {
        // The whole reference-facing call.
        double t0 = now_s();
        auto res = Cuda_BFS(graph, csr, std::to_string(s));
        t_call += now_s() - t0;
        // Its parts: BFS + the depths in a host vector (the call's own
        // route: one-byte copy, widening on host threads) ...
        t0 = now_s();
        ok = check(ghb_graph_bfs_many_host(ws, g, &s, 1, INT_MAX, depth.data(), 0, nullptr, nullptr),
                   "ghb_graph_bfs_many_host");
        t_core += now_s() - t0;
        if (!ok) return 1;
        // ... the drop-in's id -> name conversion, and the reference's.
        t0 = now_s();
        auto conv = ghb_dropin::trans_id_val(graph, depth);
        t_conv += now_s() - t0;
        t0 = now_s();
        auto conv_ref = graph.res_trans_id_val(depth);
        t_conv_ref += now_s() - t0;
        same = same && conv == conv_ref && res == conv_ref;
        for (int v = 0; v < n; ++v)
            if (depth[v] != INT_MAX) edges += h_rp[v + 1] - h_rp[v];
    }
    const double k = (double)srcs.size();
    std::printf("{\"n\": %d, \"m\": %lld, \"sources\": %d, \"gteps_call\": %.4f, \"gteps_bfs_plus_copy\": %.4f, "
                "\"ms_per_call\": %.3f, \"ms_bfs_plus_copy\": %.3f, \"ms_name_conversion\": %.3f, "
                "\"ms_reference_name_conversion\": %.3f, \"first_call_s\": %.3f, \"to_csr_s\": %.3f, "
                "\"graph_structure_s\": %.3f, \"results_identical\": %s}\n",
                n, m, (int)srcs.size(), edges / t_call / 1e9, edges / t_core / 1e9, 1e3 * t_call / k,
                1e3 * t_core / k, 1e3 * t_conv / k, 1e3 * t_conv_ref / k, first_s, csr_s, gen_s,
                same ? "true" : "false");
    return same ? 0 : 3;
}
