// A resident graph: the caller's CSR relabelled once by degree, plus the
// permutations to map results back to the caller's vertex ids.
#pragma once

#include <atomic>
#include <vector>

#include "common.cuh"

struct ghb_graph {
    int32_t n = 0;
    int64_t m = 0;           // out-CSR entries
    int64_t m_in = 0;        // in-CSR entries (== m when undirected)
    int32_t n_active = 0;    // vertices with at least one entry: new ids [0, n_active)
    bool directed = false;
    bool weighted = false;
    bool repeats = false;    // some out-row holds an entry twice
    int device = 0;
    // perm[old] = new, iperm[new] = old.  New ids are ranked by total degree,
    // descending, ties by old id.
    int32_t* perm = nullptr;
    int32_t* iperm = nullptr;
    int32_t* rowptr = nullptr;  // out-CSR in new ids, rows sorted
    int32_t* col = nullptr;
    double* w = nullptr;
    int32_t* in_rowptr = nullptr;  // == rowptr when undirected
    int32_t* in_col = nullptr;
    double* in_w = nullptr;
    int32_t* all_rowptr = nullptr;  // CDLP rows (in then out); == rowptr when undirected
    int32_t* all_col = nullptr;
    int32_t* outdeg = nullptr;       // out-degree per new id
    std::vector<int32_t> perm_host;  // host copy of perm (maps sources without a round trip)
    // Rows of the out-CSR sorted by weight instead of by column (built on the
    // first SSSP call; same rowptr), for delta-stepping's light/heavy split.
    int32_t* sw_col = nullptr;
    double* sw_w = nullptr;
    // First entry of each weight-sorted row whose weight is >= sw_le_delta
    // (the light/heavy boundary of the last SSSP width used; built on demand).
    int32_t* sw_le = nullptr;
    double sw_le_delta = -1.0;
    // Triangle counting's input check on this (immutable) graph: -1 until the
    // first TC call, then its flags (0 = symmetric, loop-free, strictly
    // increasing rows: the oriented path).  Atomic (relaxed): two host
    // threads may run TC on one handle; both compute the same flags.
    mutable std::atomic<int32_t> tc_flags{-1};
    int64_t device_bytes = 0;
    float build_ms = 0.f;
};

namespace ghb {

// Result mapping kernels (new-id array -> caller's ids).
int map_back_i32(ghb_workspace* ws, const ghb_graph* g, const int32_t* src_new, int32_t* dst_old);
int map_back_f64(ghb_workspace* ws, const ghb_graph* g, const double* src_new, double* dst_old);
int map_back_i64(ghb_workspace* ws, const ghb_graph* g, const int64_t* src_new, int64_t* dst_old);

}  // namespace ghb
