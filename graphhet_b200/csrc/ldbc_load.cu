// LDBC text loader straight into the GPU CSR builder (replaces the
// reference's LDBC::load_graph, include/LDBC/ldbc.hpp:181-253, which inserts
// every edge into graph_structure's sorted per-vertex vectors, O(degree) per
// insert, before toCSR flattens them).
//
// Same result as the reference: vertices get ids in the order of their
// first line in the .v file (a repeated name keeps its first id); an edge
// line "a b [w]" adds a, then b, when they were not seen before (ids after
// the .v vertices, in edge-file order); the weight is the third field read
// with strtod, else 1; an undirected graph stores both directions with the
// line's weight; a repeated ordered pair keeps the weight of its last line;
// self-loops are kept (graph_structure keeps them).
//
// Both files are read with one pass of several host threads over disjoint
// line ranges; names become ids through one hash map (filled in file order,
// then read by every thread); the edge list goes to ghb_csr_build on the
// device (sort, deduplication with last-wins weights, symmetrisation) and,
// for a directed graph, ghb_csr_transpose builds the in-CSR.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <string>
#include <string_view>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"

struct ghb_ldbc_graph {
    int32_t n = 0;
    int64_t m = 0;      // out-CSR entries
    int64_t m_in = 0;
    bool directed = false;
    bool weighted = false;
    int32_t *rowptr = nullptr, *col = nullptr, *in_rowptr = nullptr, *in_col = nullptr;
    double *w = nullptr, *in_w = nullptr;
    std::deque<std::string> names;  // id -> name (a deque never moves its strings)
    std::unordered_map<std::string_view, int32_t> ids;  // views into `names`
};

namespace ghb {
namespace {

struct MappedFile {
    const char* data = nullptr;
    size_t size = 0;
    int fd = -1;
    ~MappedFile() {
        if (data && size) munmap(const_cast<char*>(data), size);
        if (fd >= 0) close(fd);
    }
    int open_file(const char* path) {
        fd = ::open(path, O_RDONLY);
        if (fd < 0) {
            set_error(std::string("cannot open ") + path);
            return GHB_ERR_INVALID_ARGUMENT;
        }
        struct stat st;
        if (fstat(fd, &st) != 0) {
            set_error(std::string("cannot stat ") + path);
            return GHB_ERR_INVALID_ARGUMENT;
        }
        size = (size_t)st.st_size;
        if (size == 0) return GHB_OK;
        void* p = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
        if (p == MAP_FAILED) {
            set_error(std::string("cannot map ") + path);
            size = 0;
            return GHB_ERR_INVALID_ARGUMENT;
        }
        data = static_cast<const char*>(p);
        return GHB_OK;
    }
};

// Byte ranges of `parts` chunks that start at line starts.
std::vector<size_t> line_chunks(const char* d, size_t size, int parts) {
    std::vector<size_t> cut{0};
    for (int i = 1; i < parts; ++i) {
        size_t p = size * (size_t)i / (size_t)parts;
        if (p <= cut.back()) continue;
        while (p < size && d[p - 1] != '\n') ++p;
        if (p < size && p > cut.back()) cut.push_back(p);
    }
    cut.push_back(size);
    return cut;
}

// Fields of one line split on single spaces (the reference's parse_string
// with " "); a trailing '\r' is dropped.
inline int split_fields(std::string_view line, std::string_view* f, int maxf) {
    if (!line.empty() && line.back() == '\r') line.remove_suffix(1);
    int k = 0;
    size_t s = 0;
    while (k < maxf) {
        const size_t e = line.find(' ', s);
        if (e == std::string_view::npos) {
            f[k++] = line.substr(s);
            break;
        }
        f[k++] = line.substr(s, e - s);
        s = e + 1;
    }
    return k;
}

template <class F>
void for_lines(const char* d, size_t b, size_t e, F&& f) {
    size_t s = b;
    while (s < e) {
        const char* nl = static_cast<const char*>(std::memchr(d + s, '\n', e - s));
        const size_t t = nl ? (size_t)(nl - d) : e;
        f(std::string_view(d + s, t - s));
        s = t + 1;
    }
}

}  // namespace
}  // namespace ghb

using namespace ghb;

extern "C" {

int ghb_ldbc_free(ghb_ldbc_graph* g) {
    if (!g) return GHB_OK;
    cudaFree(g->rowptr);
    cudaFree(g->col);
    cudaFree(g->w);
    cudaFree(g->in_rowptr);
    cudaFree(g->in_col);
    cudaFree(g->in_w);
    delete g;
    return GHB_OK;
}

int ghb_ldbc_load(ghb_workspace* ws, const char* vertex_path, const char* edge_path, int32_t directed,
                  ghb_ldbc_graph** out) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && vertex_path && edge_path && out, "NULL argument");
    *out = nullptr;
    const int threads = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    auto* g = new ghb_ldbc_graph();
    g->directed = directed != 0;
    auto fail = [&](int s) {
        ghb_ldbc_free(g);
        return s;
    };

    // ---- vertices, in line order
    MappedFile vf;
    int s0 = vf.open_file(vertex_path);
    if (s0 != GHB_OK) return fail(s0);
    {
        std::vector<size_t> cut = line_chunks(vf.data, vf.size, threads);
        std::vector<std::vector<std::string_view>> part(cut.size() - 1);
        std::vector<std::thread> pool;
        for (size_t t = 0; t + 1 < cut.size(); ++t)
            pool.emplace_back([&, t]() {
                for_lines(vf.data, cut[t], cut[t + 1], [&](std::string_view line) {
                    if (!line.empty() && line.back() == '\r') line.remove_suffix(1);
                    part[t].push_back(line);
                });
            });
        for (auto& th : pool) th.join();
        size_t total = 0;
        for (auto& p : part) total += p.size();
        g->ids.reserve(total * 2 + 16);
        for (auto& p : part)
            for (std::string_view nm : p) {
                if (g->ids.find(nm) == g->ids.end()) {
                    g->names.emplace_back(nm);
                    g->ids.emplace(std::string_view(g->names.back()), (int32_t)(g->names.size() - 1));
                }
            }
    }

    // ---- edges: parallel parse and lookup, then names seen first here
    MappedFile ef;
    s0 = ef.open_file(edge_path);
    if (s0 != GHB_OK) return fail(s0);
    std::vector<size_t> cut = line_chunks(ef.data, ef.size, threads);
    const size_t parts = cut.size() - 1;
    struct Part {
        std::vector<int32_t> u, v;
        std::vector<double> w;
        std::vector<std::pair<size_t, std::string_view>> unknown;  // (edge index in part * 2 + end, name)
        bool weighted = false;
    };
    std::vector<Part> pp(parts);
    {
        std::vector<std::thread> pool;
        for (size_t t = 0; t < parts; ++t)
            pool.emplace_back([&, t]() {
                Part& P = pp[t];
                for_lines(ef.data, cut[t], cut[t + 1], [&](std::string_view line) {
                    std::string_view f[3];
                    const int k = split_fields(line, f, 3);
                    if (k < 2) return;  // the reference skips lines of fewer than two fields
                    const size_t idx = P.u.size();
                    int32_t id[2];
                    for (int e = 0; e < 2; ++e) {
                        auto it = g->ids.find(f[e]);
                        if (it == g->ids.end()) {
                            id[e] = -1;
                            P.unknown.emplace_back(idx * 2 + e, f[e]);
                        } else {
                            id[e] = it->second;
                        }
                    }
                    double w = 1.0;
                    if (k > 2) {
                        w = std::strtod(std::string(f[2]).c_str(), nullptr);
                        P.weighted = true;
                    }
                    P.u.push_back(id[0]);
                    P.v.push_back(id[1]);
                    P.w.push_back(w);
                });
            });
        for (auto& th : pool) th.join();
    }
    // Names not in the .v file get ids in edge-file order (a, then b).
    for (Part& P : pp)
        for (auto& [pos, nm] : P.unknown) {
            auto it = g->ids.find(nm);
            int32_t id;
            if (it == g->ids.end()) {
                id = (int32_t)g->names.size();
                g->names.emplace_back(nm);
                g->ids.emplace(std::string_view(g->names.back()), id);
            } else {
                id = it->second;
            }
            (pos & 1 ? P.v : P.u)[pos >> 1] = id;
        }
    if (g->names.size() >= (size_t)INT32_MAX) return fail((set_error("too many vertices for int32 ids"),
                                                           GHB_ERR_INVALID_ARGUMENT));
    g->n = (int32_t)g->names.size();
    int64_t ne = 0;
    for (Part& P : pp) {
        ne += (int64_t)P.u.size();
        g->weighted |= P.weighted;
    }
    if (g->n == 0) return fail((set_error("empty graph"), GHB_ERR_INVALID_ARGUMENT));

    // ---- device CSR
    cudaStream_t st = ws->stream;
    int32_t *du = nullptr, *dv = nullptr;
    double* dw = nullptr;
    const int64_t cap = g->directed ? ne : 2 * ne;
    auto cuda_fail = [&](cudaError_t e) {
        set_error(std::string("LDBC load: ") + cudaGetErrorString(e));
        cudaFree(du);
        cudaFree(dv);
        cudaFree(dw);
        return fail(e == cudaErrorMemoryAllocation ? GHB_ERR_OUT_OF_MEMORY : GHB_ERR_CUDA);
    };
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc(&du, sizeof(int32_t) * std::max<int64_t>(ne, 1));
    if (e == cudaSuccess) e = cudaMalloc(&dv, sizeof(int32_t) * std::max<int64_t>(ne, 1));
    if (e == cudaSuccess) e = cudaMalloc(&dw, sizeof(double) * std::max<int64_t>(ne, 1));
    if (e == cudaSuccess) e = cudaMalloc(&g->rowptr, sizeof(int32_t) * ((size_t)g->n + 1));
    if (e == cudaSuccess) e = cudaMalloc(&g->col, sizeof(int32_t) * std::max<int64_t>(cap, 1));
    if (e == cudaSuccess) e = cudaMalloc(&g->w, sizeof(double) * std::max<int64_t>(cap, 1));
    if (e != cudaSuccess) return cuda_fail(e);
    int64_t off = 0;
    for (Part& P : pp) {
        const size_t k = P.u.size();
        if (k == 0) continue;
        if (e == cudaSuccess) e = cudaMemcpyAsync(du + off, P.u.data(), sizeof(int32_t) * k, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dv + off, P.v.data(), sizeof(int32_t) * k, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dw + off, P.w.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st);
        off += (int64_t)k;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the parts' host vectors are read by the copies
    if (e != cudaSuccess) return cuda_fail(e);
    int64_t m = 0;
    int s = ghb_csr_build(ws, g->n, du, dv, dw, ne, g->directed ? 0 : GHB_BUILD_SYMMETRIZE, 0, 0, g->rowptr, g->col,
                          g->w, &m);
    if (s == GHB_OK && g->directed) {
        e = cudaSuccess;
        if (e == cudaSuccess) e = cudaMalloc(&g->in_rowptr, sizeof(int32_t) * ((size_t)g->n + 1));
        if (e == cudaSuccess) e = cudaMalloc(&g->in_col, sizeof(int32_t) * std::max<int64_t>(m, 1));
        if (e == cudaSuccess) e = cudaMalloc(&g->in_w, sizeof(double) * std::max<int64_t>(m, 1));
        if (e != cudaSuccess) return cuda_fail(e);
        s = ghb_csr_transpose(ws, g->n, m, g->rowptr, g->col, g->w, g->in_rowptr, g->in_col, g->in_w);
    }
    cudaStreamSynchronize(st);
    cudaFree(du);
    cudaFree(dv);
    cudaFree(dw);
    du = dv = nullptr;
    dw = nullptr;
    if (s != GHB_OK) return fail(s);
    g->m = m;
    g->m_in = m;
    *out = g;
    return GHB_OK;
}

int ghb_ldbc_info(const ghb_ldbc_graph* g, int32_t* n, int64_t* m, int32_t* weighted) {
    GHB_REQUIRE(g, "NULL graph");
    if (n) *n = g->n;
    if (m) *m = g->m;
    if (weighted) *weighted = g->weighted ? 1 : 0;
    return GHB_OK;
}

int ghb_ldbc_csr(const ghb_ldbc_graph* g, const int32_t** rowptr, const int32_t** col, const double** w,
                 const int32_t** in_rowptr, const int32_t** in_col, const double** in_w) {
    GHB_REQUIRE(g, "NULL graph");
    if (rowptr) *rowptr = g->rowptr;
    if (col) *col = g->col;
    if (w) *w = g->w;
    if (in_rowptr) *in_rowptr = g->directed ? g->in_rowptr : g->rowptr;
    if (in_col) *in_col = g->directed ? g->in_col : g->col;
    if (in_w) *in_w = g->directed ? g->in_w : g->w;
    return GHB_OK;
}

int ghb_ldbc_copy(ghb_workspace* ws, const ghb_ldbc_graph* g, int32_t* rowptr, int32_t* col, double* w,
                  int32_t* in_rowptr, int32_t* in_col, double* in_w) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && g, "NULL argument");
    cudaStream_t st = ws->stream;
    const size_t n1 = (size_t)g->n + 1, m = (size_t)g->m;
    auto cp = [&](void* d, const void* s, size_t bytes) -> int {
        if (d && bytes) GHB_CUDA_TRY(cudaMemcpyAsync(d, s, bytes, cudaMemcpyDeviceToDevice, st));
        return GHB_OK;
    };
    GHB_TRY(cp(rowptr, g->rowptr, sizeof(int32_t) * n1));
    GHB_TRY(cp(col, g->col, sizeof(int32_t) * m));
    GHB_TRY(cp(w, g->w, sizeof(double) * m));
    if (g->directed) {
        GHB_TRY(cp(in_rowptr, g->in_rowptr, sizeof(int32_t) * n1));
        GHB_TRY(cp(in_col, g->in_col, sizeof(int32_t) * m));
        GHB_TRY(cp(in_w, g->in_w, sizeof(double) * m));
    }
    return GHB_OK;
}

int ghb_ldbc_name(const ghb_ldbc_graph* g, int32_t id, const char** name) {
    GHB_REQUIRE(g && name, "NULL argument");
    GHB_REQUIRE(id >= 0 && id < g->n, "id outside [0, n)");
    *name = g->names[id].c_str();
    return GHB_OK;
}

int ghb_ldbc_id(const ghb_ldbc_graph* g, const char* name, int32_t* id) {
    GHB_REQUIRE(g && name && id, "NULL argument");
    auto it = g->ids.find(std::string_view(name));
    GHB_REQUIRE(it != g->ids.end(), std::string("unknown vertex name: ") + name);
    *id = it->second;
    return GHB_OK;
}

}  // extern "C"
