// Device kernels of the single-source BFS (see bfs.cu for the driver).
#pragma once

#include "common.cuh"

namespace ghb {

// Lists at least this long are expanded edge-parallel across the whole grid
// instead of by one warp (a warp walking a long list is a chain of dependent
// claims, 32 entries per step).
constexpr int32_t kBigList = 256;
// In the persistent kernel, deferred lists at least this long are walked by
// every thread of the grid; shorter deferred lists by one block each.
constexpr int32_t kHugeList = 1 << 16;

struct BfsCounters {
    int32_t tail;       // next-queue length
    int32_t big_tail;   // deferred long lists this level
    unsigned long long m_f;       // sum of out-degrees of newly reached vertices
    unsigned long long examined;  // CSR entries read
    double deg2;                  // sum of squared out-degrees (trace features)
    unsigned int degmax;
    int32_t pad;
    unsigned long long big_edges;  // entries in the deferred long lists
};

struct BfsPersistState;

struct BfsBuffers {
    uint32_t* visited;
    uint32_t* front_a;
    uint32_t* front_b;
    int32_t* queue_a;
    int32_t* queue_b;
    int32_t* big;          // deferred long-list vertices
    int64_t* big_prefix;   // exclusive prefix of their degrees (+ total)
    int32_t* depth_snap;   // snapshots for oracle timing
    uint32_t* visited_snap;
    BfsCounters* counters;
    BfsPersistState* persist;

    static BfsBuffers carve(Carver& c, int32_t n, int64_t words) {
        BfsBuffers b;
        b.visited = c.take<uint32_t>(words);
        b.front_a = c.take<uint32_t>(words);
        b.front_b = c.take<uint32_t>(words);
        b.queue_a = c.take<int32_t>(n);
        b.queue_b = c.take<int32_t>(n);
        b.big = c.take<int32_t>(n);
        b.big_prefix = c.take<int64_t>((size_t)n + 1);
        b.depth_snap = c.take<int32_t>(n);
        b.visited_snap = c.take<uint32_t>(words);
        b.counters = c.take<BfsCounters>(1);
        b.persist = reinterpret_cast<BfsPersistState*>(c.take<unsigned long long>(16));
        return b;
    }
};

__global__ void fill_i32_kernel(int32_t* p, int64_t count, int32_t value);

__global__ void bfs_init_kernel(int32_t n, int64_t words, int32_t src, int32_t* depth,
                                uint32_t* visited, uint32_t* front, int32_t* queue);

__global__ void bfs_pull_kernel(int32_t n, int64_t words, const int32_t* __restrict__ in_rp,
                                const int32_t* __restrict__ in_col,
                                const int32_t* __restrict__ out_rp,
                                const uint32_t* __restrict__ f_cur, uint32_t* visited,
                                uint32_t* f_next, int32_t* depth, int32_t next_depth,
                                int32_t* q_next, BfsCounters* cnt);

__global__ void bfs_queue_from_bitmap_kernel(int64_t words, const uint32_t* __restrict__ f,
                                             const int32_t* __restrict__ rowptr, int32_t* queue, int32_t* tail,
                                             BfsCounters* cnt);

// Top-down levels whose frontier has at least this many out-entries write
// only the frontier bitmap; the queue is compacted from it afterwards.
constexpr int64_t kAppendMaxEdges = 1 << 16;

__global__ void bfs_pred_pull_kernel(int32_t n, const int32_t* __restrict__ in_rp,
                                     const int32_t* __restrict__ in_col,
                                     const int32_t* __restrict__ depth, int32_t src,
                                     int32_t* __restrict__ pred);
__global__ void bfs_pred_push_kernel(int32_t n, const int32_t* __restrict__ out_rp,
                                     const int32_t* __restrict__ out_col,
                                     const int32_t* __restrict__ depth, int32_t* pred);
__global__ void bfs_pred_finish_kernel(int32_t n, int32_t src, int32_t* pred);

// One top-down level: the queue kernel (short and medium lists), then the
// long lists edge-parallel.
int bfs_push_level(ghb_workspace* ws, const BfsBuffers& B, int32_t n, const int32_t* rowptr,
                   const int32_t* col, const int32_t* q_cur, int64_t n_f, int32_t next_depth,
                   int32_t* depth, int32_t* q_next, uint32_t* f_next);

// Oracle timing of both directions for one level (state restored after each).
int bfs_time_both(ghb_workspace* ws, const BfsBuffers& B, int32_t n, int64_t words,
                  const int32_t* out_rowptr, const int32_t* out_col, const int32_t* in_rowptr,
                  const int32_t* in_col, const int32_t* q_cur, int64_t n_f, int64_t m_f, const uint32_t* f_cur,
                  int level, int32_t* depth, float* t_push, float* t_pull);

}  // namespace ghb

namespace ghb {

// State of the persistent top-down kernel (device memory, zeroed before a run).
struct BfsPersistState {
    unsigned bar_count, bar_gen;
    int32_t status;                 // kDevOk or kDevBarrierTimeout
    int32_t levels_done;            // levels expanded in this run
    int32_t tail[3];                // frontier sizes, triple-buffered by level
    int32_t pad;
    unsigned long long mf[3];       // frontier out-entries, triple-buffered
    unsigned int dmax[3];           // largest frontier row, triple-buffered
    unsigned int pad2;
    unsigned long long examined;
    unsigned long long m_r;         // out-entries of all vertices reached in this run
    long long reached;              // vertices reached in this run
};

// Frontiers with fewer out-entries than this run in the persistent kernel.
constexpr int64_t kPersistMaxEdges = 1 << 20;

__global__ void bfs_push_persistent_kernel(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                           int32_t* qa, int32_t* qb, uint32_t* visited, int32_t* depth,
                                           int32_t start_level, int32_t max_depth, int64_t exit_edges,
                                           int64_t m_total, int64_t m_r_start, float alpha, BfsPersistState* ps);

__global__ void bfs_bitmap_from_queue_kernel(const int32_t* __restrict__ q, int32_t count, uint32_t* f);

bool bfs_use_persistent(ghb_workspace* ws, const ghb_bfs_options* opt);
int bfs_persistent_run(ghb_workspace* ws, int32_t n, int32_t n_active, const int32_t* out_rp, const int32_t* out_col,
                       const int32_t* in_rp, const int32_t* in_col, int32_t src, int32_t max_depth, int32_t* depth,
                       const int32_t* perm, int32_t* depth_out, const ghb_bfs_options* opt,
                       ghb_traversal_stats* stats);

}  // namespace ghb
