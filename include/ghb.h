/*
 * ghb.h - C ABI of the B200 (sm_100a) CSR analytics library (libghb.so).
 *
 * Every entry point takes plain device pointers and sizes, runs on the
 * workspace's CUDA stream, and returns a status code (GHB_OK on success).
 * A failed call leaves a message for ghb_last_error() (per host thread).
 *
 * Graph layout (the reference's CSR_graph, include/GPU_csr/GPU_csr.hpp:97-110):
 *   rowptr  int32[n + 1]   offsets into col
 *   col     int32[m]       neighbour ids, sorted ascending inside each row
 *   w       double[m]      edge weights (SSSP only)
 * An undirected graph stores both directions; then the "in" arrays may alias
 * the "out" arrays, exactly as toCSR does for is_directed == false
 * (GPU_csr.hpp:133-140).
 *
 * The header-inline C++ entry points in include/GPU_csr/algorithm/*.cuh
 * (Cuda_BFS, Cuda_SSSP, ...) are the reference-facing API; they call these.
 */
#ifndef GHB_H
#define GHB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
    GHB_OK = 0,
    GHB_ERR_INVALID_ARGUMENT = 1,
    GHB_ERR_CUDA = 2,
    GHB_ERR_OUT_OF_MEMORY = 3,
    GHB_ERR_TIMEOUT = 4,   /* a bounded device-side wait gave up           */
    GHB_ERR_LIMIT = 5,     /* a level / phase / iteration budget ran out     */
    GHB_ERR_UNSUPPORTED = 6
};

const char* ghb_status_string(int status);
/* Detail of the last failure on this host thread ("" if none). */
const char* ghb_last_error(void);
/* Library version, major * 10000 + minor * 100 + patch. */
int ghb_version(void);

/* ------------------------------------------------------------- workspace */
/* A workspace owns a CUDA stream binding, cached scratch memory, pinned host
 * counters and timing events.  Calls on one workspace are serialised on its
 * stream; use one workspace per host thread.  The reference allocates and
 * frees scratch inside every call (e.g. GPU_BFS_csr.cuh:258-283); the
 * workspace keeps it across calls instead. */
typedef struct ghb_workspace ghb_workspace;

int ghb_workspace_create(ghb_workspace** out);
int ghb_workspace_destroy(ghb_workspace* ws);
/* Bind a cudaStream_t (NULL = legacy default stream). */
int ghb_workspace_set_stream(ghb_workspace* ws, void* stream);
void* ghb_workspace_get_stream(ghb_workspace* ws);
/* Free cached scratch. */
int ghb_workspace_trim(ghb_workspace* ws);
/* Launch counter of this library's kernels on this workspace and the scratch
 * bytes currently reserved. */
int ghb_workspace_counters(ghb_workspace* ws, int64_t* kernel_launches, int64_t* scratch_bytes);
/* Process-wide workspace on the current device (used by the C++ wrappers). */
ghb_workspace* ghb_default_workspace(void);
/* Launch shapes and thresholds of this workspace (no counterpart in the
 * reference): "pr_cache_kb" PageRank hub cache in shared memory, "pr_threads"
 * and "pr_blocks_per_sm" its persistent blocks, "pr_short" / "pr_chunk" its
 * row split, "ms_warp_rest" / "ms_pull_div" the multi-source BFS's block-row
 * threshold and direction switch, "pol_band" (0-64) the band, in log2
 * units around the direction rule's threshold, inside which the learned
 * policy's network chooses a BFS level's direction and output format (0:
 * never; 64: always), "barrier_limit_us" (100 - 60,000,000; default
 * 2,000,000) how long a persistent kernel's grid-barrier wait lasts before
 * it gives up and the call returns GHB_ERR_TIMEOUT, "sssp_persistent" (0 or
 * 1; default 1) whether SSSP runs as one cooperative launch per traversal
 * or as host-driven rounds, "tc_hash" (0 or 1; default 1) whether triangle
 * counting probes a shared-memory hash of each oriented row or gallops
 * through sorted rows, "tc_block_row" (128 - 8192; default 8192) the longest
 * oriented row the hash path takes (longer rows gallop), "ms_persistent" (0
 * or 1; default 1) whether a multi-source BFS pass is one cooperative launch
 * or host-driven levels, "bfs_blocks_per_sm" (1 or 2; default 2) the blocks
 * per SM of the whole-traversal BFS launch, "pr_gathers" (4 or 8) the
 * contribution gathers PageRank keeps in flight per lane on long rows,
 * "mssp_persistent" (0 or 1; default 1) whether a multi-source SSSP pass is
 * one cooperative launch or host-driven rounds, "mssp_width_log2" (-10 -
 * 10; default 2) the multi-source bucket width as the single-source weight
 * rule's times 2^k, "tc_trim_min" (0 - 2^20; default 0) the shortest list
 * N+(b) that triangle counting cuts to N+(a)'s id range before probing,
 * "tc_slice_blocks" (1 - 16; default 16) the blocks per SM of the slice
 * kernel for oriented rows of 129 - 1,024 entries, "sssp_adapt" (0 or 1;
 * default 0) whether the one-launch SSSP halves or doubles the bucket width
 * from one bucket to the next (the light/heavy split stays at the width
 * chosen for the call), "ms_learned" (0 or 1; default 0) whether the
 * multi-source pass's directions come from the model installed by
 * ghb_ms_policy_load.
 * Results do not depend on them.  "barrier_extra" (0 or 1) is a test knob:
 * 1 makes every grid barrier of the persistent kernels wait for one arrival
 * more than there are blocks, so every wait runs out after barrier_limit_us
 * and the call returns GHB_ERR_TIMEOUT (the workspace stays usable).
 * Unknown names and values outside the documented ranges are rejected. */
int ghb_tune_set(ghb_workspace* ws, const char* name, int32_t value);
int ghb_tune_get(ghb_workspace* ws, const char* name, int32_t* value);

/* ------------------------------------------------------------ generators */
/* Seeded synthetic inputs (include/ghb_gen.h).  Outputs are device arrays of
 * n_edges entries.  They stand in for the LDBC/Graph500 datasets that the
 * reference loads from text (include/LDBC/ldbc.hpp:181-253). */
int ghb_gen_rmat(ghb_workspace* ws, int32_t scale, int64_t n_edges, uint64_t seed,
                 double a, double b, double c, int32_t permute,
                 int32_t* src, int32_t* dst);
/* rows x cols 4-neighbour grid, one entry per undirected edge (right, down):
 * n_edges = rows*(cols-1) + (rows-1)*cols. */
int ghb_gen_grid(ghb_workspace* ws, int32_t rows, int32_t cols, int32_t* src, int32_t* dst);
int ghb_gen_er(ghb_workspace* ws, int32_t n, int64_t n_edges, uint64_t seed,
               int32_t* src, int32_t* dst);
/* Chung-Lu power-law graph on 2^scale vertices: each endpoint is vertex i
 * with probability proportional to (i+1)^(-1/(exponent-1)) (degree
 * distribution ~ d^-exponent), ids scattered by the seed's permutation.
 * exponent in (2, 10).  Training graphs for the schedule policy. */
int ghb_gen_powerlaw(ghb_workspace* ws, int32_t scale, int64_t n_edges, double exponent,
                     uint64_t seed, int32_t* src, int32_t* dst);
/* keep[e] = 0 when src[e] is one of the seed's dangling vertices (about
 * `fraction` of all ids, ghb_is_dangling), else 1: dropping those edges makes
 * the PageRank precision workload's sinks. */
int ghb_gen_dangling_keep(ghb_workspace* ws, int64_t n_edges, const int32_t* src, uint64_t seed,
                          double fraction, uint8_t* keep);

/* ----------------------------------------------------------- LDBC loader */
/* LDBC .v / .e text files straight into device CSRs (replaces
 * LDBC::load_graph, include/LDBC/ldbc.hpp:181-253, and toCSR's flattening of
 * graph_structure): ids follow first appearance (.v lines, then names first
 * seen in .e, a before b), weights are the third field (else 1), an
 * undirected graph gets both directions, a repeated ordered pair keeps its
 * last line's weight, self-loops are kept.  The handle owns the arrays; a
 * directed graph also gets the in-CSR (undirected: in = out). */
typedef struct ghb_ldbc_graph ghb_ldbc_graph;
int ghb_ldbc_load(ghb_workspace* ws, const char* vertex_path, const char* edge_path,
                  int32_t directed, ghb_ldbc_graph** out);
int ghb_ldbc_info(const ghb_ldbc_graph* g, int32_t* n, int64_t* m, int32_t* weighted);
int ghb_ldbc_csr(const ghb_ldbc_graph* g, const int32_t** rowptr, const int32_t** col,
                 const double** w, const int32_t** in_rowptr, const int32_t** in_col,
                 const double** in_w);
/* Copies the handle's arrays into caller-owned device arrays (any may be
 * NULL; in_* only for a directed graph), on the workspace's stream. */
int ghb_ldbc_copy(ghb_workspace* ws, const ghb_ldbc_graph* g, int32_t* rowptr, int32_t* col,
                  double* w, int32_t* in_rowptr, int32_t* in_col, double* in_w);
/* Vertex name of an id (valid while the handle lives) and the id of a name. */
int ghb_ldbc_name(const ghb_ldbc_graph* g, int32_t id, const char** name);
int ghb_ldbc_id(const ghb_ldbc_graph* g, const char* name, int32_t* id);
int ghb_ldbc_free(ghb_ldbc_graph* g);

/* ----------------------------------------------------------- CSR builder */
/* Build a CSR from an edge list (replaces the host flattening in toCSR,
 * GPU_csr.hpp:282-339, for edge-list inputs).  Flags: */
#define GHB_BUILD_SYMMETRIZE 1      /* add (v,u) for every (u,v)                */
#define GHB_BUILD_DROP_SELF_LOOPS 2 /* drop (u,u)                              */
#define GHB_BUILD_TRANSPOSE 4       /* build the in-CSR (rows = destinations)  */
/* Duplicates are always merged (graph_structure::add_edge keeps one entry per
 * pair, sorted_vector_binary_operations.hpp:89-101).  Weights: if w_in is not
 * NULL the LAST occurrence of a pair wins (add_edge overwrites); otherwise
 * weight_mode / weight_seed generate ghb_pair_weight(); mode 0 writes none.
 * col / w must hold the worst case (n_edges, doubled when symmetrising);
 * *m_out receives the entry count. */
int ghb_csr_build(ghb_workspace* ws, int32_t n, const int32_t* src, const int32_t* dst,
                  const double* w_in, int64_t n_edges, int32_t flags,
                  int32_t weight_mode, uint64_t weight_seed,
                  int32_t* rowptr, int32_t* col, double* w, int64_t* m_out);
/* Transpose an existing CSR (out -> in), weights optional. */
int ghb_csr_transpose(ghb_workspace* ws, int32_t n, int64_t m, const int32_t* rowptr,
                      const int32_t* col, const double* w, int32_t* t_rowptr,
                      int32_t* t_col, double* t_w);
/* all-CSR of a directed graph: row v = in-neighbours of v then out-neighbours
 * of v (toCSR, GPU_csr.hpp:315-330). */
int ghb_csr_merge_in_out(ghb_workspace* ws, int32_t n, const int32_t* in_rowptr,
                         const int32_t* in_col, const int32_t* out_rowptr,
                         const int32_t* out_col, int32_t* all_rowptr, int32_t* all_col);

/* ------------------------------------------------------------------- BFS */
/* Direction policy per level. */
#define GHB_POLICY_HEURISTIC 0 /* Beamer alpha/beta rule + frontier guard     */
#define GHB_POLICY_LEARNED 1   /* the trained MLP (ghb_policy_*); falls back   */
#define GHB_POLICY_PUSH 2      /* top-down every level                        */
#define GHB_POLICY_PULL 3      /* bottom-up every level after the first       */
#define GHB_POLICY_SCHEDULE 4  /* options.schedule[level] (0 push, 1 pull)    */

typedef struct {
    int32_t policy;
    float alpha;             /* switch to pull when m_f > m_u / alpha (0: 256) */
    float beta;              /* back to push when n_f < n / beta (0: 24)      */
    const int8_t* schedule;  /* host array for GHB_POLICY_SCHEDULE: per level
                                bit 0 direction (0 push, 1 pull); bits 1-2 the
                                output of a top-down level: 0 by frontier size,
                                2 queue, 4 bitmap only                        */
    int32_t schedule_len;
    int32_t record_trace;    /* 1: fill trace[] with one row per level         */
    float* trace;            /* host, trace_cap x GHB_TRACE_COLS               */
    int32_t trace_cap;
    int32_t oracle_timing;   /* 1: time push and pull at every level (slow)   */
    float gamma;             /* ... and only when m_f > m / gamma (0: 1024)   */
} ghb_bfs_options;

/* Trace row (one per level): 12 policy features of the level's frontier,
 * then 12 direction used, 13 level time (ms), 14 push time and 15 pull time
 * (ms) when oracle_timing is set (else -1), 16 CSR entries read, 17 vertices
 * reached by the level, 18 vertices unvisited before it, 19 the level's
 * algorithmic bytes (rowptr + col + depth), 20 output format of a top-down
 * level (0 queue, 1 bitmap), 21 time (ms) spent turning the frontier bitmap
 * into a queue at the level's start (-1 none), 22 1 when the learned network
 * chose the level's direction, 23 reserved (-1). */
#define GHB_TRACE_FEATURES 12
#define GHB_TRACE_COLS 24

typedef struct {
    int32_t levels;          /* frontier expansions run                      */
    int32_t pull_levels;     /* of which bottom-up                           */
    int64_t reached;         /* vertices with a finite depth                 */
    int64_t edges_reached;   /* m_r: CSR entries out of reached vertices      */
    int64_t edges_examined;  /* CSR entries the kernels read                 */
    double device_ms;        /* CUDA-event time of the traversal             */
} ghb_traversal_stats;

/* Unweighted depths from src over the out-CSR (Cuda_BFS / csr_bfs,
 * GPU_BFS_csr.cuh:13, 258-327; CPU_BFS.hpp:10-41).  depth[v] = INT32_MAX when
 * v is unreached or deeper than max_depth.  in_rowptr/in_col enable bottom-up
 * levels (pass the out arrays for an undirected graph, NULL to force push). */
int ghb_bfs(ghb_workspace* ws, int32_t n, const int32_t* out_rowptr, const int32_t* out_col,
            const int32_t* in_rowptr, const int32_t* in_col, int32_t src, int32_t max_depth,
            int32_t* depth, const ghb_bfs_options* options, ghb_traversal_stats* stats);

/* BFS with predecessors (Cuda_BFS_pre / bfs_pre, GPU_BFS_pre_csr.cuh:15,
 * 62-124).  pred[v] = an out-neighbour parent at depth[v]-1 (the smallest
 * such id), -1 for the source and for unreached vertices. */
int ghb_bfs_pred(ghb_workspace* ws, int32_t n, const int32_t* out_rowptr,
                 const int32_t* out_col, const int32_t* in_rowptr, const int32_t* in_col,
                 int32_t src, int32_t max_depth, int32_t* depth, int32_t* pred,
                 const ghb_bfs_options* options, ghb_traversal_stats* stats);

/* Many sources at once: one bit per source in 1, 2 or 4 uint64 words per
 * vertex, so one traversal serves up to 256 sources (larger n_src runs in
 * passes of 256).  depth is n_src x n, row s holding the depths from srcs[s]
 * (the values of n_src ghb_bfs calls). */
int ghb_msbfs(ghb_workspace* ws, int32_t n, const int32_t* out_rowptr, const int32_t* out_col,
              const int32_t* in_rowptr, const int32_t* in_col, const int32_t* srcs,
              int32_t n_src, int32_t* depth, ghb_traversal_stats* stats);

/* ------------------------------------------------------------------ SSSP */
typedef struct {
    double delta;            /* bucket width; <= 0 picks one from the weights */
    int32_t policy;          /* GHB_POLICY_HEURISTIC or GHB_POLICY_LEARNED     */
    int32_t record_trace;
    float* trace;
    int32_t trace_cap;
} ghb_sssp_options;

/* FP64 distances from src over the out-CSR (Cuda_SSSP / csr_sssp,
 * GPU_SSSP_csr.cuh:253-327; CPU_shortest_paths.hpp:19-64).  Unreached
 * vertices get `inf` (LDBC passes DBL_MAX).  Weights must be >= 0. */
int ghb_sssp(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col,
             const double* w, int32_t src, double inf, double* dist,
             const ghb_sssp_options* options, ghb_traversal_stats* stats);

/* With predecessors (Cuda_SSSP_pre, GPU_SSSP_pre_csr.cuh:332-368): pred[v] is
 * the smallest-id u with dist[u] + w(u,v) == dist[v] (exact FP64), -1 for the
 * source and for unreached vertices.  in_* is the transposed CSR with its
 * weights (the out-CSR of an undirected graph). */
int ghb_sssp_pred(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col,
                  const double* w, const int32_t* in_rowptr, const int32_t* in_col,
                  const double* in_w, int32_t src, double inf, double* dist, int32_t* pred,
                  const ghb_sssp_options* options, ghb_traversal_stats* stats);

/* Many sources: dist is n_src x n, row s the distances from srcs[s] (the
 * values of n_src ghb_sssp calls).  Up to 256 sources share one bucketed
 * traversal (a vertex's distances for all of them side by side); more run in
 * passes of 256. */
int ghb_mssssp(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col,
               const double* w, const int32_t* srcs, int32_t n_src, double inf, double* dist,
               ghb_traversal_stats* stats);

/* ------------------------------------------------------------------- WCC */
/* Weakly connected components (Cuda_WCC / WCC_GPU, GPU_WCC_csr.cuh:83-129;
 * CPU_connected_components.hpp:12-66).  label[v] = the smallest vertex id in
 * v's component.  Either direction of a directed graph covers every edge. */
int ghb_wcc(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col,
            int32_t* label);

/* The same WCC without any device allocation, for callers that must not
 * allocate while the library runs: an application that owns the GPU's memory
 * through its own pool (the library as a plugin inside a database or a
 * serving process) or a latency-critical caller for which cudaMalloc would
 * synchronise the device.  No counterpart in the reference.  It takes a
 * cudaStream_t instead of a workspace; its scratch is a fixed 800 KiB device
 * array inside libghb.so, held by every GPU that loads the library until the
 * process exits.  Limit: at most 268,435,456 (2^28) CSR entries; larger
 * graphs are rejected with GHB_ERR_INVALID_ARGUMENT.  The first call on a
 * device does a one-time set-up: it looks up the array's device address
 * (cudaGetSymbolAddress) and keeps it for the life of the process; make that
 * first call before any stream capture begins.  A device reset
 * (cudaDeviceReset) is not supported: the kept address would be stale, so do
 * not call this function on a device after resetting it.  Every call shares
 * the array, so calls that overlap on the GPU race: serialise them.  Each
 * call reads rowptr[n] back and synchronises `stream`. */
int ghb_wcc_noalloc(int32_t n, const int32_t* rowptr, const int32_t* col, int32_t* label,
                    void* stream);

/* -------------------------------------------------------------- PageRank */
#define GHB_PR_FP64 0
#define GHB_PR_FP32_KAHAN 1

typedef struct {
    int32_t iterations;      /* maximum iterations                            */
    double damping;
    int32_t precision;       /* GHB_PR_FP64 or GHB_PR_FP32_KAHAN               */
    double tolerance;        /* > 0: stop once the L1 change <= tolerance      */
    double* l1_history;      /* host, optional: L1 change per iteration        */
} ghb_pr_options;

/* LDBC PageRank, pull form (Cuda_PR / GPU_PR, GPU_PR_csr.cuh:34-117, 193-197;
 * CPU_PageRank.hpp:12-56): pr' = (1-d)/N + d*S/N + d*sum_{u in in(v)} pr[u]/out(u),
 * S = sum of the ranks of vertices with no out-edges.  `rank` is FP64 either
 * way; FP32 mode stores ranks and contributions in FP32 with per-row Kahan
 * sums and keeps S and the L1 norm in FP64.  *iterations_run may be NULL. */
int ghb_pagerank(ghb_workspace* ws, int32_t n, const int32_t* in_rowptr, const int32_t* in_col,
                 const int32_t* out_rowptr, const ghb_pr_options* options, double* rank,
                 int32_t* iterations_run);

/* ------------------------------------------------------------------ CDLP */
/* Synchronous label propagation (Cuda_CDLP / CDLP_GPU, GPU_CDLP_csr.cuh:75-210;
 * CPU_Community_Detection.hpp:12-64): new label = the most frequent label
 * among the row's entries, smallest label on ties; a vertex with an empty row
 * keeps its label.  Labels start as vertex ids.  Pass the all-CSR (in then
 * out) of a directed graph, the out-CSR of an undirected one. */
int ghb_cdlp(ghb_workspace* ws, int32_t n, const int32_t* all_rowptr, const int32_t* all_col,
             int32_t iterations, int32_t* labels);

/* -------------------------------------------------------------------- TC */
/* Per-vertex triangle incidences with the reference's counting
 * (Cuda_TC / Cuda_TC_PerNode, GPU_TC_csr.cuh:15-68; CPU_TC.hpp:31-60): for
 * every entry u->v and every w in row(u) and row(v), add 1 to u, v and w.
 * On a symmetric graph without self-loops that is 6 x triangles(x).
 * counts64 (exact) and counts32 (the reference's wrapping int32) may each be
 * NULL; *total receives sum(counts64) / 3 (may be NULL). */
int ghb_tc(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col,
           int64_t* counts64, int32_t* counts32, int64_t* total);

/* ---------------------------------------------------- resident graphs */
/* A graph handle: the caller's CSR (device arrays, only read during the
 * call) relabelled once on the GPU by total degree, descending, so hubs get
 * the smallest ids, sorted rows list hubs first and vertices without entries
 * form a tail the kernels skip.  This is the one-time preparation the
 * reference does in toCSR (GPU_csr.hpp:282-339); every ghb_graph_* call then
 * returns exactly what the raw-CSR entry point of the same name returns, in
 * the caller's vertex ids (BFS/SSSP predecessors: a valid parent, not
 * necessarily the smallest id).  in_* == NULL or == out_*: undirected.  The
 * handle owns its device memory; calls on one handle may share a workspace
 * but must not overlap. */
typedef struct ghb_graph ghb_graph;

int ghb_graph_create(ghb_workspace* ws, int32_t n, const int32_t* out_rowptr,
                     const int32_t* out_col, const double* out_w,
                     const int32_t* in_rowptr, const int32_t* in_col, const double* in_w,
                     ghb_graph** out);
int ghb_graph_destroy(ghb_graph* g);
int ghb_graph_info(const ghb_graph* g, int64_t* m, int32_t* n_active, int64_t* device_bytes,
                   float* build_ms);
/* Device arrays perm[old] = new and iperm[new] = old (owned by the handle). */
int ghb_graph_perm(const ghb_graph* g, const int32_t** perm, const int32_t** iperm);

int ghb_graph_bfs(ghb_workspace* ws, const ghb_graph* g, int32_t src, int32_t max_depth,
                  int32_t* depth, const ghb_bfs_options* options, ghb_traversal_stats* stats);
/* BFS from each of n_src sources into the caller's HOST array depth_host
 * (n_src x n int32, row i for srcs[i], caller's ids; srcs is a host array):
 * the same values as n_src calls of ghb_graph_bfs followed by copies to the
 * host.  No counterpart in the reference, whose Cuda_BFS returns one host
 * vector per call (GPU_BFS_csr.cuh:320-327).  The sources are pipelined:
 * the GPU traverses one while the copy engine brings the previous one's
 * depths over as one byte each (traversals under 255 levels; deeper ones
 * as int32) and host_threads host threads (0: half the host's, at most 8)
 * widen the one before into depth_host, with streaming stores where the
 * host has AVX2.  stats: levels is the maximum, the other counts
 * are sums, device_ms is the call's wall time.  The workspace keeps two
 * device depth buffers, their byte copies and two pinned byte buffers. */
int ghb_graph_bfs_many_host(ghb_workspace* ws, const ghb_graph* g, const int32_t* srcs, int32_t n_src,
                            int32_t max_depth, int32_t* depth_host, int32_t host_threads,
                            const ghb_bfs_options* options, ghb_traversal_stats* stats);
int ghb_graph_bfs_pred(ghb_workspace* ws, const ghb_graph* g, int32_t src, int32_t max_depth,
                       int32_t* depth, int32_t* pred, const ghb_bfs_options* options,
                       ghb_traversal_stats* stats);
int ghb_graph_msbfs(ghb_workspace* ws, const ghb_graph* g, const int32_t* srcs, int32_t n_src,
                    int32_t* depth, ghb_traversal_stats* stats);
/* ghb_graph_msbfs with its levels' directions forced and timed (no
 * counterpart in the reference): schedule (device int8 array, or NULL for
 * the direction rule) gives level L's direction at schedule[L] (0 push, 1
 * pull; levels past schedule_len follow the rule); trace (device float
 * array, or NULL) receives GHB_MS_TRACE_COLS floats per level of the first
 * pass (trace_cap rows at most): direction, level time in ms, frontier
 * vertices and out-entries expanded, vertices and out-entries found.  A
 * level finds the same vertices in either direction, so timing a pass under
 * all-push and all-pull schedules gives each level's cheaper direction.
 * Depths do not depend on the schedule.  Needs the one-launch pass
 * (ms_persistent = 1 and cooperative launch). */
#define GHB_MS_TRACE_COLS 6
typedef struct {
    const int8_t* schedule;
    int32_t schedule_len;
    float* trace;
    int32_t trace_cap;
} ghb_msbfs_options;
int ghb_graph_msbfs_ex(ghb_workspace* ws, const ghb_graph* g, const int32_t* srcs, int32_t n_src,
                       int32_t* depth, const ghb_msbfs_options* options, ghb_traversal_stats* stats);
/* The same multi-source BFS as launches only, for CUDA-graph capture (no
 * counterpart in the reference, which runs one source per call): each pass
 * of up to 256 sources is one cooperative launch that runs every level, its
 * direction choices and the depth output on the device, with no host
 * round trip and no allocation.  Call ghb_graph_msbfs_reserve once (outside
 * any capture) with the largest n_src to size the workspace; a launch whose
 * workspace is too small fails with GHB_ERR_INVALID_ARGUMENT.  Sources are
 * caller ids on the device and are not checked on the host: a source
 * outside [0, n) is skipped and its depth row is all INT32_MAX.  A grid
 * barrier that times out leaves the pass's output incomplete without a
 * status (ghb_graph_msbfs reports it). */
int ghb_graph_msbfs_reserve(ghb_workspace* ws, const ghb_graph* g, int32_t n_src);
int ghb_graph_msbfs_launch(ghb_workspace* ws, const ghb_graph* g, const int32_t* srcs, int32_t n_src,
                           int32_t* depth);
int ghb_graph_mssssp(ghb_workspace* ws, const ghb_graph* g, const int32_t* srcs, int32_t n_src,
                     double inf, double* dist, ghb_traversal_stats* stats);
int ghb_graph_sssp(ghb_workspace* ws, const ghb_graph* g, int32_t src, double inf, double* dist,
                   const ghb_sssp_options* options, ghb_traversal_stats* stats);
int ghb_graph_sssp_pred(ghb_workspace* ws, const ghb_graph* g, int32_t src, double inf,
                        double* dist, int32_t* pred, const ghb_sssp_options* options,
                        ghb_traversal_stats* stats);
int ghb_graph_wcc(ghb_workspace* ws, const ghb_graph* g, int32_t* label);
int ghb_graph_pagerank(ghb_workspace* ws, const ghb_graph* g, const ghb_pr_options* options,
                       double* rank, int32_t* iterations_run);
int ghb_graph_cdlp(ghb_workspace* ws, const ghb_graph* g, int32_t iterations, int32_t* labels);
int ghb_graph_tc(ghb_workspace* ws, const ghb_graph* g, int64_t* counts64, int32_t* counts32,
                 int64_t* total);

/* ------------------------------------------------------ batched graphs */
/* Many independent graphs packed back to back.  vbase / ebase are HOST
 * arrays of n_graphs + 1 int64: graph g owns global vertices
 * [vbase[g], vbase[g+1]) and entries [ebase[g], ebase[g+1]) (a batch may hold
 * more than 2^31 entries); its rowptr (n_g + 1 int32 LOCAL offsets) starts at
 * rowptr[vbase[g] + g]; col holds LOCAL ids.  Outputs are indexed by global
 * vertex and hold local values. */
/* WCC of every graph (label = smallest local id of the component). */
int ghb_batch_wcc(ghb_workspace* ws, int32_t n_graphs, const int64_t* vbase,
                  const int64_t* ebase, const int32_t* rowptr, const int32_t* col,
                  int32_t* label);
/* Triangle counts of every graph: counts64 per vertex (device, may be NULL),
 * totals[g] triangles of graph g (host, may be NULL). */
int ghb_batch_tc(ghb_workspace* ws, int32_t n_graphs, const int64_t* vbase,
                 const int64_t* ebase, const int32_t* rowptr, const int32_t* col,
                 int64_t* counts64, int64_t* totals);

/* Disjoint-union batches: many graphs in one CSR whose graph g owns the
 * global vertices [vbase[g], vbase[g+1]) (vbase: DEVICE int64, n_graphs + 1
 * entries, vbase[0] = 0, vbase[n_graphs] = n_total), every row of it pointing
 * into its own graph, symmetric, sorted, loop- and duplicate-free (what
 * ghb_csr_build with SYMMETRIZE | DROP_SELF_LOOPS writes for an edge list of
 * global ids), m = rowptr[n_total] < 2^31.  No counterpart in the reference
 * (it runs one graph per call).
 * ghb_union_reserve sizes the workspace once; ghb_union_wcc_tc then only
 * launches kernels (no allocation, no host round trip), so a stream capture
 * can record it.  label (local ids: smallest local id of the component),
 * counts64 (the reference's 6x per-vertex triangle count) and triangles
 * (per graph) are device arrays; any may be NULL. */
int ghb_union_reserve(ghb_workspace* ws, int32_t n_total, int64_t m);
int ghb_union_wcc_tc(ghb_workspace* ws, int32_t n_graphs, const int64_t* vbase, int32_t n_total,
                     int64_t m, const int32_t* rowptr, const int32_t* col, int32_t* label,
                     int64_t* counts64, int64_t* triangles);

/* ----------------------------------------------------- dynamic graph */
/* A GPU-resident graph that takes batches of edge updates (the reference's
 * GPMA, include/GPU_gpma/GPU_gpma.hpp).  Update semantics of update_gpma
 * (GPU_gpma.hpp:756-824, handle_del_mod at :166-180): key = (row << 32) |
 * col with row, col < n; value 0 deletes the entry if present (no-op when
 * absent); any other value sets the weight of an existing entry or inserts
 * it.  Repeated keys in one batch: the last occurrence wins.  Rows stay
 * sorted by column.  keys / values are DEVICE arrays.  Analytics read the
 * compact CSR of ghb_gpma_csr (rows sorted, m < 2^31), which is rebuilt on
 * the first call after a change and then cached. */
typedef struct ghb_gpma ghb_gpma;
#define GHB_GPMA_STATS 8 /* batches, inserted, deleted, modified, rows moved,
                            repacks, arena slots used, arena slots */
/* Empty graph over n vertices (init_csr_gpma, GPU_gpma.hpp:911-928). */
int ghb_gpma_create(ghb_workspace* ws, int32_t n, ghb_gpma** out);
int ghb_gpma_destroy(ghb_gpma* g);
/* Deep copy (GPMA's copy assignment, LDBC_GPU_gpma.cu:206). */
int ghb_gpma_clone(ghb_workspace* ws, const ghb_gpma* src, ghb_gpma** out);
/* Remove every edge. */
int ghb_gpma_clear(ghb_workspace* ws, ghb_gpma* g);
/* Replace the contents with a CSR (rowptr[0] = 0, rows strictly increasing,
 * columns in [0, n)); w NULL means weight 1, a weight of 0 is refused
 * (init_gpma_from_csr, GPU_gpma.hpp:851-909). */
int ghb_gpma_load_csr(ghb_workspace* ws, ghb_gpma* g, const int32_t* rowptr, const int32_t* col,
                      const double* w);
/* Apply one batch (update_gpma).  totals (host, may be NULL) receives
 * inserted, deleted, modified, ignored (repeats and deletes of absent keys).
 * A key outside [0, n) x [0, n) fails the whole batch with
 * GHB_ERR_INVALID_ARGUMENT before anything is applied (batches beyond 2^25
 * updates are applied in passes of 2^25, in order: the final graph is the
 * same, totals count each pass's own effects, and a failing pass leaves the
 * earlier passes applied). */
int ghb_gpma_update(ghb_workspace* ws, ghb_gpma* g, const uint64_t* keys, const double* values,
                    int64_t count, int64_t* totals);
/* n, live entries, arena slots, version (bumped by every change). */
int ghb_gpma_info(const ghb_gpma* g, int32_t* n, int64_t* m, int64_t* slots, int64_t* version);
int ghb_gpma_stats(const ghb_gpma* g, int64_t* stats /* GHB_GPMA_STATS */);
/* Device pointers of the compact CSR (valid until the next change or
 * destroy); weights != 0 also materialises w. */
int ghb_gpma_csr(ghb_workspace* ws, ghb_gpma* g, int32_t weights, const int32_t** rowptr,
                 const int32_t** col, const double** w);
/* The compact CSR copied into caller buffers (rowptr n + 1, col / w m; w may
 * be NULL). */
int ghb_gpma_export(ghb_workspace* ws, ghb_gpma* g, int32_t* rowptr, int32_t* col, double* w);
/* Weight of each key, 0 when the entry is absent. */
int ghb_gpma_find(ghb_workspace* ws, const ghb_gpma* g, const uint64_t* keys, int64_t count,
                  double* values);

/* ------------------------------------------------------- schedule policy */
/* The learned schedule policy: an MLP 12 -> 64 -> 64 (ReLU) -> 20 logits in
 * three heads: [0,2) BFS direction (push, pull), [2,4) top-down frontier
 * format (queue, bitmap), [4,20) SSSP bucket width (bin k: 2^(k-6) times the
 * weight-derived base width).  No counterpart in the reference (its direction
 * is fixed per kernel).  Parameters, row-major x @ W, FP32:
 * W1[12][64] b1[64] W2[64][64] b2[64] W3[64][20] b3[20].  norm: mean[12]
 * then 1/std[12], applied to the features first. */
#define GHB_POLICY_PARAMS 6292
#define GHB_POLICY_OUT 20

/* Install a network (host arrays) for GHB_POLICY_LEARNED in every BFS and
 * SSSP call of this process; it is copied to each device on first use.
 * Both NULL: uninstall (GHB_POLICY_LEARNED then runs the heuristic). */
int ghb_policy_load(const float* params, const float* norm);
/* 1 when a network is installed. */
int ghb_policy_loaded(void);
/* Install the multi-source pass's learned direction model (host array of 9
 * floats: a bias, then one weight per level feature; NULL uninstalls).  A
 * workspace with "ms_learned" = 1 then pulls a level when the model's score
 * is positive instead of following the direction rule; depths do not
 * change.  Trained by graphhet_b200/policy.py from levels timed under
 * all-push and all-pull schedules (ghb_graph_msbfs_ex).  No counterpart in
 * the reference. */
int ghb_ms_policy_load(const float* weights, int32_t count);

/* Device arrays: logits[batch][20] = network(x[batch][12]). */
int ghb_mlp_forward(ghb_workspace* ws, const float* params, const float* norm, const float* x,
                    int32_t batch, float* logits);
/* Device arrays: grad[GHB_POLICY_PARAMS] of the sum over the three heads of
 * the weighted mean softmax cross-entropy; y[batch][3] holds the class of
 * each head (-1: no label); sample_weight[batch] (may be NULL: all 1) weighs
 * the rows.  loss (host, may be NULL) gets the loss. */
int ghb_mlp_grad(ghb_workspace* ws, const float* params, const float* norm, const float* x,
                 const int32_t* y, const float* sample_weight, int32_t batch, float* grad,
                 float* loss);
/* `epochs` full-batch Adam steps on device params (in place); loss_history
 * (host, may be NULL) gets the loss before each step. */
int ghb_mlp_train(ghb_workspace* ws, float* params, const float* norm, const float* x,
                  const int32_t* y, const float* sample_weight, int32_t batch, int32_t epochs,
                  float lr, float* loss_history);

#ifdef __cplusplus
}
#endif

#endif /* GHB_H */
