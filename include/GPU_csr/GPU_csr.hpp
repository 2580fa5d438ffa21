// GPU_csr.hpp - drop-in CSR_graph / toCSR for GraphHET's GPU CSR path,
// backed by libghb (include/ghb.h).
//
// Same public interface and layout as the reference's
// include/GPU_csr/GPU_csr.hpp:62-118 (class CSR_graph) and :282-339 (toCSR):
// host vectors of row starts / neighbours / weights, device pointers
// in/out/all_pointer, in/out/all_edge, in/out_edge_weight (double) and E_all.
// For an undirected graph (is_directed == false) the in and all arrays alias
// the out arrays, as in the reference (GPU_csr.hpp:133-140).  Copies are deep,
// moves transfer the device buffers.
//
// graph_structure<T> comes from the reference's own header
// <CPU_adj_list/CPU_adj_list.hpp> (the reference include tree must be on
// the include path after this repository's include/).
#pragma once

#include <cuda_runtime.h>
#include <cuda_runtime_api.h>

#include <algorithm>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <thread>
#include <cstddef>
#include <mutex>
#include <utility>
#include <vector>

#include <CPU_adj_list/CPU_adj_list.hpp>
#include <ghb.h>

namespace ghb_dropin {

// The reference prints CUDA failures and carries on (GPU_csr.hpp:21-25);
// the same here.
inline bool cuda_ok(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "CUDA error during %s: %s\n", what, cudaGetErrorString(e));
        return false;
    }
    return true;
}

inline bool ghb_ok(int status, const char* what) {
    if (status != GHB_OK) {
        std::fprintf(stderr, "%s failed: %s (%s)\n", what, ghb_status_string(status), ghb_last_error());
        return false;
    }
    return true;
}

template <typename T>
inline T* device_alloc(std::size_t count, const char* what) {
    if (count == 0) return nullptr;
    void* p = nullptr;
    if (!cuda_ok(cudaMalloc(&p, count * sizeof(T)), what)) return nullptr;
    return static_cast<T*>(p);
}

template <typename T>
inline void device_free(T*& p) {
    if (p) cuda_ok(cudaFree(p), "cudaFree");
    p = nullptr;
}

template <typename T>
inline void upload(T* dst, const std::vector<T>& src, const char* what) {
    if (!src.empty() && dst) cuda_ok(cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice), what);
}

template <typename T>
inline void device_copy(T* dst, const T* src, std::size_t count, const char* what) {
    if (count && dst && src) cuda_ok(cudaMemcpy(dst, src, count * sizeof(T), cudaMemcpyDeviceToDevice), what);
}

// Run f(begin, end) over [0, n) on the host's threads.
template <class F>
inline void parallel_rows(int n, F f) {
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    if (n < 65536) nt = 1;
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t) {
        const int b = (int)((long long)n * t / nt), e = (int)((long long)n * (t + 1) / nt);
        if (nt == 1) {
            f(b, e);
        } else {
            pool.emplace_back([=]() { f(b, e); });
        }
    }
    for (auto& th : pool) th.join();
}

// Run f(part, begin, end) over `parts` equal slices of [0, n), one thread each.
template <class F>
inline void parallel_rows_parts(int n, unsigned parts, F f) {
    if (parts <= 1) {
        f(0u, 0, n);
        return;
    }
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < parts; ++t) {
        const int b = (int)((long long)n * t / parts), e = (int)((long long)n * (t + 1) / parts);
        pool.emplace_back([=]() { f(t, b, e); });
    }
    for (auto& th : pool) th.join();
}

// Resident (degree-relabelled) copies of the CSR_graphs that the drop-in
// algorithms run on (ghb_graph_create), built on a CSR_graph's first
// algorithm call and kept until that CSR_graph releases its arrays, so the
// reference's drivers reach the relabelled kernels without changing a line.
// The reference has no counterpart: its entry points read the CSR arrays
// directly on every call (e.g. GPU_BFS_csr.cuh:258-283).  Keyed on every
// device array and the sizes; the arrays must not be rewritten in place
// while the CSR_graph lives (the reference never does).
struct ResidentEntry {
    const void* key[6];
    int vertices;
    std::size_t entries;
    ghb_graph* graph;
};

inline std::mutex& resident_mutex() {
    static std::mutex m;
    return m;
}

inline std::vector<ResidentEntry>& resident_entries() {
    static std::vector<ResidentEntry> v;
    return v;
}

// Drops (and frees) the resident copies built from the CSR whose out-row
// array is out_pointer.
inline void resident_forget(const void* out_pointer) {
    if (!out_pointer) return;
    std::lock_guard<std::mutex> lock(resident_mutex());
    auto& es = resident_entries();
    for (std::size_t i = 0; i < es.size();) {
        if (es[i].key[0] == out_pointer) {
            ghb_graph_destroy(es[i].graph);
            es.erase(es.begin() + (std::ptrdiff_t)i);
        } else {
            ++i;
        }
    }
}

// The resident copy of a CSR (built on first use; NULL after a failure,
// which is printed).  in_* equal to out_* (or NULL) means undirected.
inline ghb_graph* resident_graph(ghb_workspace* ws, int vertices, std::size_t entries, const int* out_p,
                                 const int* out_e, const double* out_w, const int* in_p, const int* in_e,
                                 const double* in_w) {
    const void* key[6] = {out_p, out_e, out_w, in_p, in_e, in_w};
    std::lock_guard<std::mutex> lock(resident_mutex());
    auto& es = resident_entries();
    for (auto& e : es) {
        bool same = e.vertices == vertices && e.entries == entries;
        for (int k = 0; k < 6 && same; ++k) same = e.key[k] == key[k];
        if (same) return e.graph;
    }
    // A new CSR at an address of an old one: the old copy is stale.
    for (std::size_t i = 0; i < es.size();) {
        if (es[i].key[0] == out_p) {
            ghb_graph_destroy(es[i].graph);
            es.erase(es.begin() + (std::ptrdiff_t)i);
        } else {
            ++i;
        }
    }
    ghb_graph* g = nullptr;
    const bool undirected = in_p == nullptr || in_p == out_p;
    const int status = ghb_graph_create(ws, vertices, out_p, entries ? out_e : nullptr, entries ? out_w : nullptr,
                                        undirected ? nullptr : in_p, undirected ? nullptr : in_e,
                                        undirected ? nullptr : in_w, &g);
    if (!ghb_ok(status, "ghb_graph_create")) return nullptr;
    ResidentEntry e;
    for (int k = 0; k < 6; ++k) e.key[k] = key[k];
    e.vertices = vertices;
    e.entries = entries;
    e.graph = g;
    es.push_back(e);
    return g;
}

}  // namespace ghb_dropin

template <typename weight_type>
class CSR_graph {
public:
    CSR_graph() = default;
    CSR_graph(const CSR_graph& other);
    CSR_graph(CSR_graph&& other) noexcept;
    CSR_graph& operator=(CSR_graph other) noexcept {
        swap(*this, other);
        return *this;
    }
    ~CSR_graph() { release(); }

    template <typename other_weight_type>
    friend CSR_graph<other_weight_type> toCSR(graph_structure<other_weight_type>& graph, bool is_directed);

    friend void swap(CSR_graph& a, CSR_graph& b) noexcept {
        using std::swap;
        swap(a.is_directed, b.is_directed);
        swap(a.INs_Neighbor_start_pointers, b.INs_Neighbor_start_pointers);
        swap(a.OUTs_Neighbor_start_pointers, b.OUTs_Neighbor_start_pointers);
        swap(a.ALL_start_pointers, b.ALL_start_pointers);
        swap(a.INs_Edges, b.INs_Edges);
        swap(a.OUTs_Edges, b.OUTs_Edges);
        swap(a.all_Edges, b.all_Edges);
        swap(a.INs_Edge_weights, b.INs_Edge_weights);
        swap(a.OUTs_Edge_weights, b.OUTs_Edge_weights);
        swap(a.in_pointer, b.in_pointer);
        swap(a.out_pointer, b.out_pointer);
        swap(a.in_edge, b.in_edge);
        swap(a.out_edge, b.out_edge);
        swap(a.all_pointer, b.all_pointer);
        swap(a.all_edge, b.all_edge);
        swap(a.in_edge_weight, b.in_edge_weight);
        swap(a.out_edge_weight, b.out_edge_weight);
        swap(a.E_all, b.E_all);
    }

    bool is_directed = true;
    std::vector<int> INs_Neighbor_start_pointers, OUTs_Neighbor_start_pointers, ALL_start_pointers;
    std::vector<int> INs_Edges, OUTs_Edges, all_Edges;
    std::vector<weight_type> INs_Edge_weights, OUTs_Edge_weights;
    int *in_pointer = nullptr, *out_pointer = nullptr, *in_edge = nullptr, *out_edge = nullptr;
    int *all_pointer = nullptr, *all_edge = nullptr;
    double *in_edge_weight = nullptr, *out_edge_weight = nullptr;
    std::size_t E_all = 0;

private:
    void allocate(int vertices, std::size_t out_e, std::size_t in_e, std::size_t all_e) {
        using namespace ghb_dropin;
        out_pointer = device_alloc<int>((std::size_t)vertices + 1, "cudaMalloc(out_pointer)");
        out_edge = device_alloc<int>(out_e, "cudaMalloc(out_edge)");
        out_edge_weight = device_alloc<double>(out_e, "cudaMalloc(out_edge_weight)");
        if (is_directed) {
            in_pointer = device_alloc<int>((std::size_t)vertices + 1, "cudaMalloc(in_pointer)");
            all_pointer = device_alloc<int>((std::size_t)vertices + 1, "cudaMalloc(all_pointer)");
            in_edge = device_alloc<int>(in_e, "cudaMalloc(in_edge)");
            all_edge = device_alloc<int>(all_e, "cudaMalloc(all_edge)");
            in_edge_weight = device_alloc<double>(in_e, "cudaMalloc(in_edge_weight)");
        } else {
            in_pointer = all_pointer = out_pointer;
            in_edge = all_edge = out_edge;
            in_edge_weight = out_edge_weight;
        }
    }

    void release() {
        using namespace ghb_dropin;
        resident_forget(out_pointer);
        if (is_directed) {
            device_free(in_pointer);
            device_free(in_edge);
            device_free(in_edge_weight);
            device_free(all_pointer);
            device_free(all_edge);
        } else {
            in_pointer = all_pointer = in_edge = all_edge = nullptr;
            in_edge_weight = nullptr;
        }
        device_free(out_pointer);
        device_free(out_edge);
        device_free(out_edge_weight);
    }
};

template <typename weight_type>
CSR_graph<weight_type>::CSR_graph(const CSR_graph& o)
    : is_directed(o.is_directed),
      INs_Neighbor_start_pointers(o.INs_Neighbor_start_pointers),
      OUTs_Neighbor_start_pointers(o.OUTs_Neighbor_start_pointers),
      ALL_start_pointers(o.ALL_start_pointers),
      INs_Edges(o.INs_Edges),
      OUTs_Edges(o.OUTs_Edges),
      all_Edges(o.all_Edges),
      INs_Edge_weights(o.INs_Edge_weights),
      OUTs_Edge_weights(o.OUTs_Edge_weights),
      E_all(o.E_all) {
    using namespace ghb_dropin;
    if (OUTs_Neighbor_start_pointers.empty()) return;
    const int v = (int)OUTs_Neighbor_start_pointers.size() - 1;
    allocate(v, OUTs_Edges.size(), INs_Edges.size(), E_all);
    device_copy(out_pointer, o.out_pointer, (std::size_t)v + 1, "cudaMemcpy(copy out_pointer)");
    device_copy(out_edge, o.out_edge, OUTs_Edges.size(), "cudaMemcpy(copy out_edge)");
    device_copy(out_edge_weight, o.out_edge_weight, OUTs_Edges.size(), "cudaMemcpy(copy out_edge_weight)");
    if (is_directed) {
        device_copy(in_pointer, o.in_pointer, (std::size_t)v + 1, "cudaMemcpy(copy in_pointer)");
        device_copy(all_pointer, o.all_pointer, (std::size_t)v + 1, "cudaMemcpy(copy all_pointer)");
        device_copy(in_edge, o.in_edge, INs_Edges.size(), "cudaMemcpy(copy in_edge)");
        device_copy(all_edge, o.all_edge, all_Edges.size(), "cudaMemcpy(copy all_edge)");
        device_copy(in_edge_weight, o.in_edge_weight, INs_Edges.size(), "cudaMemcpy(copy in_edge_weight)");
    }
}

template <typename weight_type>
CSR_graph<weight_type>::CSR_graph(CSR_graph&& o) noexcept
    : is_directed(o.is_directed),
      INs_Neighbor_start_pointers(std::move(o.INs_Neighbor_start_pointers)),
      OUTs_Neighbor_start_pointers(std::move(o.OUTs_Neighbor_start_pointers)),
      ALL_start_pointers(std::move(o.ALL_start_pointers)),
      INs_Edges(std::move(o.INs_Edges)),
      OUTs_Edges(std::move(o.OUTs_Edges)),
      all_Edges(std::move(o.all_Edges)),
      INs_Edge_weights(std::move(o.INs_Edge_weights)),
      OUTs_Edge_weights(std::move(o.OUTs_Edge_weights)),
      in_pointer(o.in_pointer),
      out_pointer(o.out_pointer),
      in_edge(o.in_edge),
      out_edge(o.out_edge),
      all_pointer(o.all_pointer),
      all_edge(o.all_edge),
      in_edge_weight(o.in_edge_weight),
      out_edge_weight(o.out_edge_weight),
      E_all(o.E_all) {
    o.in_pointer = o.out_pointer = o.in_edge = o.out_edge = o.all_pointer = o.all_edge = nullptr;
    o.in_edge_weight = o.out_edge_weight = nullptr;
    o.E_all = 0;
}

// Flattens graph_structure's sorted rows (OUTs, INs) into the reference's CSR
// layout on the host's threads, then uploads it.  Row v of the all-CSR is
// v's in-row followed by its out-row (directed graphs only).
template <typename weight_type>
CSR_graph<weight_type> toCSR(graph_structure<weight_type>& graph, bool is_directed = true) {
    using namespace ghb_dropin;
    CSR_graph<weight_type> a;
    a.is_directed = is_directed;
    const int V = graph.size();
    auto offsets = [&](const std::vector<std::vector<std::pair<int, weight_type>>>& rows, std::vector<int>& ptr) {
        ptr.assign((std::size_t)V + 1, 0);
        long long acc = 0;
        for (int i = 0; i < V; ++i) {
            ptr[i] = (int)acc;
            acc += (long long)rows[i].size();
        }
        ptr[V] = (int)acc;
    };
    auto fill = [&](const std::vector<std::vector<std::pair<int, weight_type>>>& rows, const std::vector<int>& ptr,
                    std::vector<int>& edges, std::vector<weight_type>& weights) {
        edges.resize((std::size_t)ptr[V]);
        weights.resize((std::size_t)ptr[V]);
        parallel_rows(V, [&](int b, int e) {
            for (int i = b; i < e; ++i) {
                int o = ptr[i];
                for (const auto& x : rows[i]) {
                    edges[o] = x.first;
                    weights[o] = x.second;
                    ++o;
                }
            }
        });
    };
    offsets(graph.OUTs, a.OUTs_Neighbor_start_pointers);
    fill(graph.OUTs, a.OUTs_Neighbor_start_pointers, a.OUTs_Edges, a.OUTs_Edge_weights);
    if (is_directed) {
        offsets(graph.INs, a.INs_Neighbor_start_pointers);
        fill(graph.INs, a.INs_Neighbor_start_pointers, a.INs_Edges, a.INs_Edge_weights);
        a.ALL_start_pointers.assign((std::size_t)V + 1, 0);
        for (int i = 0; i <= V; ++i)
            a.ALL_start_pointers[i] = a.INs_Neighbor_start_pointers[i] + a.OUTs_Neighbor_start_pointers[i];
        a.all_Edges.resize((std::size_t)a.ALL_start_pointers[V]);
        parallel_rows(V, [&](int b, int e) {
            for (int i = b; i < e; ++i) {
                int o = a.ALL_start_pointers[i];
                for (const auto& x : graph.INs[i]) a.all_Edges[o++] = x.first;
                for (const auto& x : graph.OUTs[i]) a.all_Edges[o++] = x.first;
            }
        });
    }
    const std::size_t out_e = a.OUTs_Edges.size(), in_e = a.INs_Edges.size();
    a.E_all = is_directed ? in_e + out_e : out_e;
    a.allocate(V, out_e, in_e, a.E_all);
    upload(a.out_pointer, a.OUTs_Neighbor_start_pointers, "cudaMemcpy(out_pointer)");
    upload(a.out_edge, a.OUTs_Edges, "cudaMemcpy(out_edge)");
    // Device weights are double whatever weight_type is (GPU_csr.hpp:109).
    if (a.out_edge_weight && out_e) {
        std::vector<double> w(a.OUTs_Edge_weights.begin(), a.OUTs_Edge_weights.end());
        upload(a.out_edge_weight, w, "cudaMemcpy(out_edge_weight)");
    }
    if (is_directed) {
        upload(a.in_pointer, a.INs_Neighbor_start_pointers, "cudaMemcpy(in_pointer)");
        upload(a.all_pointer, a.ALL_start_pointers, "cudaMemcpy(all_pointer)");
        upload(a.in_edge, a.INs_Edges, "cudaMemcpy(in_edge)");
        upload(a.all_edge, a.all_Edges, "cudaMemcpy(all_edge)");
        if (a.in_edge_weight && in_e) {
            std::vector<double> w(a.INs_Edge_weights.begin(), a.INs_Edge_weights.end());
            upload(a.in_edge_weight, w, "cudaMemcpy(in_edge_weight)");
        }
    }
    cuda_ok(cudaDeviceSynchronize(), "cudaDeviceSynchronize(toCSR)");
    return a;
}
