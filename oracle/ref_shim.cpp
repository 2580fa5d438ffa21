// ref_shim.cpp - TEST INFRASTRUCTURE ONLY.  Exposes the reference's own CPU
// adjacency-list algorithms (GraphHET include/CPU_adj_list/algorithm/*.hpp,
// compiled from the reference tree by oracle/Makefile) through a C ABI, so
// the tests can pin the oracle restatement and bench.py can time the
// reference's CPU path.  The graph is loaded into the reference's
// graph_structure<double> directly in sorted order (the same rows that
// add_edge's sorted inserts produce, CPU_adj_list.hpp:110-114).
#include <CPU_adj_list/CPU_adj_list.hpp>
#include <CPU_adj_list/algorithm/CPU_BFS.hpp>
#include <CPU_adj_list/algorithm/CPU_BFS_pre.hpp>
#include <CPU_adj_list/algorithm/CPU_Community_Detection.hpp>
#include <CPU_adj_list/algorithm/CPU_PageRank.hpp>
#include <CPU_adj_list/algorithm/CPU_TC.hpp>
#include <CPU_adj_list/algorithm/CPU_connected_components.hpp>
#include <CPU_adj_list/algorithm/CPU_shortest_paths.hpp>
#include <CPU_adj_list/algorithm/CPU_sssp_pre.hpp>

#include <string>
#include <thread>

namespace {
graph_structure<double>* g_graph = nullptr;
}

extern "C" {

void ref_free() {
    delete g_graph;
    g_graph = nullptr;
}

// out-CSR and in-CSR (the same arrays for an undirected graph).  Weights may
// be NULL (then 1.0).  Vertex names are the decimal ids.
int ref_load(int n, const int* out_rp, const int* out_col, const double* out_w, const int* in_rp,
             const int* in_col, const double* in_w) {
    ref_free();
    g_graph = new graph_structure<double>(n);
    g_graph->vertex_id_to_str.resize(n);
    const unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t) {
        pool.emplace_back([=]() {
            for (int v = (int)((long long)n * t / nt); v < (int)((long long)n * (t + 1) / nt); ++v) {
                auto& o = g_graph->OUTs[v];
                o.reserve(out_rp[v + 1] - out_rp[v]);
                for (int j = out_rp[v]; j < out_rp[v + 1]; ++j) o.emplace_back(out_col[j], out_w ? out_w[j] : 1.0);
                auto& i = g_graph->INs[v];
                i.reserve(in_rp[v + 1] - in_rp[v]);
                for (int j = in_rp[v]; j < in_rp[v + 1]; ++j) i.emplace_back(in_col[j], in_w ? in_w[j] : 1.0);
                g_graph->vertex_id_to_str[v] = std::make_pair(std::to_string(v), true);
            }
        });
    }
    for (auto& th : pool) th.join();
    g_graph->E = out_rp[n];
    return 0;
}

int ref_bfs(int src, int max_depth, int* depth) {
    std::vector<int> d = CPU_BFS(g_graph->OUTs, src, 0, max_depth);
    std::copy(d.begin(), d.end(), depth);
    return 0;
}

int ref_bfs_pre(int src, int* depth, int* pre) {
    std::vector<int> p(g_graph->V, -1);
    std::vector<int> d = CPU_BFS(g_graph->OUTs, p, src, 0, INT_MAX);
    std::copy(d.begin(), d.end(), depth);
    std::copy(p.begin(), p.end(), pre);
    return 0;
}

int ref_sssp(int src, double* dist) {
    std::vector<double> d = CPU_shortest_paths(g_graph->OUTs, src);
    std::copy(d.begin(), d.end(), dist);
    return 0;
}

int ref_sssp_pre(int src, double* dist, int* pre) {
    std::vector<int> p(g_graph->V, -1);
    std::vector<double> d = CPU_shortest_paths_pre(g_graph->OUTs, src, p);
    std::copy(d.begin(), d.end(), dist);
    std::copy(p.begin(), p.end(), pre);
    return 0;
}

int ref_wcc(int* comp) {
    std::vector<int> c = CPU_connected_components(g_graph->OUTs, g_graph->INs);
    std::copy(c.begin(), c.end(), comp);
    return 0;
}

int ref_pagerank(double damping, int iterations, double* rank) {
    std::vector<double> r = PageRank(g_graph->INs, g_graph->OUTs, damping, iterations);
    std::copy(r.begin(), r.end(), rank);
    return 0;
}

int ref_cdlp(int iterations, int* labels) {
    std::vector<std::string> l = CDLP(*g_graph, iterations);
    for (size_t i = 0; i < l.size(); ++i) labels[i] = std::stoi(l[i]);
    return 0;
}

int ref_tc(int* counts) {
    std::vector<int> c = Tri_Counting(g_graph->OUTs);
    std::copy(c.begin(), c.end(), counts);
    return 0;
}

// Apply edge updates in order through the reference's own graph_structure
// edits (CPU_adj_list.hpp:110-128): weight 0 -> remove_edge(u, v), any other
// weight -> add_edge(u, v, w), which inserts or overwrites the weight.  These
// are the edits the reference's GPMA drivers mirror on the GPU
// (batch_add_edge / batch_delete_edge, LDBC_GPU_gpma.cu:124-148).
int ref_apply_updates(long long count, const int* src, const int* dst, const double* w) {
    if (!g_graph) return -1;
    for (long long i = 0; i < count; ++i) {
        if (w[i] == 0.0) g_graph->remove_edge(src[i], dst[i]);
        else g_graph->add_edge(src[i], dst[i], w[i]);
    }
    return 0;
}

// Entries of the current out-rows.
long long ref_out_entries() {
    long long m = 0;
    if (g_graph)
        for (const auto& row : g_graph->OUTs) m += (long long)row.size();
    return m;
}

// The current out-rows as a CSR (rp n + 1, col / w ref_out_entries()).
int ref_export_out(int* rp, int* col, double* w) {
    if (!g_graph) return -1;
    long long o = 0;
    const int n = (int)g_graph->OUTs.size();
    for (int v = 0; v < n; ++v) {
        rp[v] = (int)o;
        for (const auto& e : g_graph->OUTs[v]) {
            col[o] = e.first;
            w[o] = e.second;
            ++o;
        }
    }
    rp[n] = (int)o;
    return 0;
}

int ref_hardware_threads() { return (int)std::thread::hardware_concurrency(); }

}  // extern "C"
