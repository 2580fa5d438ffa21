// Dynamic graph: batches of edge inserts, deletes and weight changes applied
// to a GPU-resident graph, which the CSR analytics then read through a
// compact snapshot.  This is the B200 counterpart of the reference's GPMA+
// (include/GPU_gpma/GPU_gpma.hpp), with the update semantics of update_gpma
// (GPU_gpma.hpp:756-824) and handle_del_mod (GPU_gpma.hpp:166-180):
//   * an update is (key, value) with key = (row << 32) | col;
//   * value 0 (VALUE_NONE, GPU_gpma.hpp:33) deletes the entry if it is there
//     and does nothing otherwise;
//   * any other value sets the weight of an existing entry, or inserts it.
// Repeated keys inside one batch: the last occurrence wins (the reference
// leaves this case to racing writes for a present key and keeps two copies
// of an absent one).
//
// Layout.  The reference keeps one sorted key array with gaps (a packed
// memory array over the whole graph) and rebalances segments level by level
// with a device sync per step.  Here each row owns a slot range of its own in
// one arena: start[v] (int64), deg[v] live entries sorted by column, cap[v]
// slots (deg + 25 % + 4, a multiple of 4).  A batch is sorted once, every
// update is classified by one binary search in its row, rows that change are
// rebuilt into a scratch area by rank arithmetic (each surviving entry and
// each insert knows its output position from prefix counts, no sequential
// merge), and copied back in place, or to fresh slots at the arena's end when
// a row outgrows its slack.  When the arena runs out the graph is repacked
// with fresh slack (the reference's resize_gpma, GPU_gpma.hpp:680-710).
//
// Analytics read a compact CSR snapshot (rowptr/col, optionally weights),
// rebuilt on demand after a change by one scan of deg and one coalesced copy
// of the rows: the same bytes a GPMA kernel would stream over its gaps, but
// afterwards every CSR kernel of the library runs unchanged.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>

#include "common.cuh"
#include "scan.cuh"

struct ghb_gpma {
    int32_t n = 0;
    int64_t m = 0;       // live entries
    int64_t slots = 0;   // arena capacity
    int64_t used = 0;    // arena slots handed out (rows + abandoned ranges)
    int64_t* start = nullptr;
    int32_t* deg = nullptr;
    int32_t* cap = nullptr;
    int32_t* col = nullptr;
    double* val = nullptr;
    // Batch scratch, grown on demand and kept.
    void* bbuf = nullptr;
    size_t bbuf_cap = 0;
    // Compact snapshot.
    int32_t* s_rowptr = nullptr;
    int32_t* s_col = nullptr;
    double* s_val = nullptr;
    int64_t s_col_cap = 0, s_val_cap = 0;
    bool s_ok = false, s_val_ok = false;
    int64_t version = 0;
    int64_t stats[GHB_GPMA_STATS] = {};
    unsigned long long* moved = nullptr;  // device: rows moved to fresh slots
    // The arena a merge rebuild left behind, kept for the next one (the
    // rebuilds of large batches alternate between the two).
    int32_t* spare_col = nullptr;
    double* spare_val = nullptr;
    int64_t spare_slots = 0;
};

namespace ghb {
namespace {

constexpr int kNop = 0, kIns = 1, kDel = 2, kMod = 3;
// Updates applied per pass; larger batches are applied in consecutive passes
// of this size, which keeps "last occurrence wins" and bounds the scratch.
constexpr int64_t kPassUpdates = 1ll << 25;
// Snapshot / repack copies: rows of at least this many entries are cut into
// chunks of this size, one warp per chunk.
constexpr int32_t kCopyChunk = 256;
// Rows of the batch with at most row_warp_max existing entries + updates
// are rebuilt by one warp (a launch argument: kRowWarpSmall for small
// batches, where a long row on one warp would be the critical path,
// kRowWarpLarge otherwise); longer rows by the grid-wide kernels.
constexpr int32_t kRowWarpSmall = 256;
constexpr int32_t kRowWarpLarge = 4096;
// The grid-wide kernels give each warp a chunk of this many entries of a
// long row (one search for the chunk's row, 8 entries per lane).
constexpr int32_t kBigChunk = 256;
// Batches up to this many updates scan their flags in one block.
constexpr int64_t kSmallScan = 32768;
// Live entries are bounded so the snapshot's int32 offsets hold them.
constexpr int64_t kMaxEntries = (1ll << 31) - 1;

__host__ __device__ __forceinline__ int64_t slack_cap(int64_t d) {
    if (d <= 0) return 0;
    int64_t c = (d + (d >> 2) + 4 + 3) & ~int64_t(3);
    return c > 0x7fffffff ? 0x7fffffff : c;
}

int key_bits(int32_t n) {
    int bits = 1;
    while (bits < 31 && (1ll << bits) < (int64_t)n) ++bits;
    return bits;
}

template <class T>
int dev_alloc(T** p, int64_t count) {
    *p = nullptr;
    if (count <= 0) return GHB_OK;
    GHB_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * (size_t)count));
    return GHB_OK;
}

template <class T>
void dev_free(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// ------------------------------------------------------------ batch kernels

__global__ void upd_prep_kernel(const uint64_t* __restrict__ keys, int64_t b, int32_t n,
                                uint32_t* __restrict__ idx, unsigned long long* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        idx[i] = (uint32_t)i;
        if ((k >> 32) >= (uint64_t)n || (k & 0xffffffffull) >= (uint64_t)n) atomicAdd(bad, 1ull);
    }
}

// One thread per sorted update.  Only the last update of an equal-key run
// acts; it binary-searches its row: found -> DEL (value 0) or MOD, absent ->
// INS (value != 0) or nothing.  pos = index of the entry, or of its insertion
// point, inside the row.
__global__ void upd_classify_kernel(const int64_t* __restrict__ start, const int32_t* __restrict__ deg,
                                    const int32_t* __restrict__ col, const uint64_t* __restrict__ skey,
                                    const uint32_t* __restrict__ sidx, const double* __restrict__ values,
                                    int64_t b, int32_t n, int32_t* __restrict__ ins, int32_t* __restrict__ del,
                                    int32_t* __restrict__ head, int32_t* __restrict__ pos,
                                    int8_t* __restrict__ typ, unsigned long long* __restrict__ n_mod) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = skey[i];
        const uint32_t r = (uint32_t)(k >> 32), c = (uint32_t)k;
        head[i] = (i == 0 || (skey[i - 1] >> 32) != (uint64_t)r) ? 1 : 0;
        int t = kNop;
        int32_t p = 0;
        const bool last = (i + 1 == b) || skey[i + 1] != k;
        if (last && r < (uint32_t)n && c < (uint32_t)n) {
            const double v = values[sidx[i]];
            const int32_t* row = col + start[r];
            int32_t lo = 0, hi = deg[r];
            while (lo < hi) {
                const int32_t mid = (lo + hi) >> 1;
                if ((uint32_t)row[mid] < c) lo = mid + 1;
                else hi = mid;
            }
            p = lo;
            const bool found = lo < deg[r] && (uint32_t)row[lo] == c;
            if (found) t = (v == 0.0) ? kDel : kMod;
            else t = (v == 0.0) ? kNop : kIns;
        }
        ins[i] = t == kIns;
        del[i] = t == kDel;
        typ[i] = (int8_t)t;
        pos[i] = p;
        if (t == kMod) atomicAdd(n_mod, 1ull);
    }
}

// Row table: row_id[k], row_first[k] for the k-th distinct row of the batch;
// row_first[K] = b.
__global__ void upd_rows_kernel(const uint64_t* __restrict__ skey, const int32_t* __restrict__ head,
                                const int32_t* __restrict__ headX, int64_t b, int32_t* __restrict__ row_id,
                                int32_t* __restrict__ row_first) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
        if (head[i]) {
            const int32_t k = headX[i];
            row_id[k] = (int32_t)(skey[i] >> 32);
            row_first[k] = (int32_t)i;
        }
        if (i == 0) row_first[headX[b]] = (int32_t)b;
    }
}

// Per distinct row: new degree, existing entries to re-rank, slots to hand
// out when the row no longer fits.  Entries k >= K are zero so the scans can
// run over b + 1 entries without the host knowing K.
__global__ void upd_row_summary_kernel(const int32_t* __restrict__ row_id, const int32_t* __restrict__ row_first,
                                       const int32_t* __restrict__ headX, const int32_t* __restrict__ insX,
                                       const int32_t* __restrict__ delX, const int32_t* __restrict__ deg,
                                       const int32_t* __restrict__ cap, int64_t b, int32_t* __restrict__ scrn,
                                       int32_t* __restrict__ exn, int64_t* __restrict__ reln,
                                       int32_t row_warp_max, unsigned long long* __restrict__ n_long) {
    const int64_t K = headX[b];
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < b; k += (int64_t)gridDim.x * blockDim.x) {
        int32_t s = 0, e = 0;
        int64_t rl = 0;
        if (k < K) {
            const int32_t a = row_first[k], z = row_first[k + 1], r = row_id[k];
            const int32_t ni = insX[z] - insX[a], nd = delX[z] - delX[a];
            if (ni + nd > 0) {
                const int32_t d = deg[r];
                const int32_t d2 = d + ni - nd;
                s = d2;
                e = d;
                if (d2 > cap[r]) rl = slack_cap(d2);
                if ((int64_t)d + (z - a) > row_warp_max) atomicAdd(n_long, 1ull);
            }
        }
        scrn[k] = s;
        exn[k] = e;
        reln[k] = rl;
    }
}

__global__ void upd_totals_kernel(const int32_t* __restrict__ insX, const int32_t* __restrict__ delX,
                                  const int32_t* __restrict__ headX, const int32_t* __restrict__ scrX,
                                  const int32_t* __restrict__ exX, const int64_t* __restrict__ relX, int64_t b,
                                  int64_t* __restrict__ out) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        out[0] = insX[b];
        out[1] = delX[b];
        out[2] = headX[b];
        out[3] = scrX[b];
        out[4] = exX[b];
        out[5] = relX[b];
    }
}

__global__ void upd_modify_kernel(const uint64_t* __restrict__ skey, const uint32_t* __restrict__ sidx,
                                  const double* __restrict__ values, const int8_t* __restrict__ typ,
                                  const int32_t* __restrict__ pos, const int64_t* __restrict__ start, int64_t b,
                                  double* __restrict__ val) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
        if (typ[i] == kMod) val[start[skey[i] >> 32] + pos[i]] = values[sidx[i]];
    }
}

// Index k with X[k] <= t < X[k + 1] over a nondecreasing X[0..len].
template <class T>
__device__ __forceinline__ int64_t seg_of(const T* __restrict__ X, int64_t len, int64_t t) {
    int64_t lo = 0, hi = len + 1;  // first index with X[idx] > t, in (0, len]
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)X[mid] <= t) lo = mid + 1;
        else hi = mid;
    }
    return lo - 1;
}

// Rank of an existing entry (column c at index j of row k) in the rebuilt
// row: j + (inserts before c) - (deletes before c); -1 when it is deleted.
// Updates of row k are skey[a, z), sorted.
__device__ __forceinline__ int32_t old_rank(const uint64_t* __restrict__ skey, const int8_t* __restrict__ typ,
                                            const int32_t* __restrict__ insX, const int32_t* __restrict__ delX,
                                            int32_t a, int32_t z, uint32_t r, int32_t c, int32_t j) {
    const uint64_t key = ((uint64_t)r << 32) | (uint32_t)c;
    int32_t lo = a, hi = z;
    while (lo < hi) {
        const int32_t mid = (lo + hi) >> 1;
        if (skey[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    if (lo < z && skey[lo] == key) {
        int32_t q = lo;
        while (q + 1 < z && skey[q + 1] == key) ++q;
        if (typ[q] == kDel) return -1;
    }
    return j + (insX[lo] - insX[a]) - (delX[lo] - delX[a]);
}

// Rank of insert i (its row's updates start at a): insertion point - deletes
// before it + inserts before it.
__device__ __forceinline__ int32_t new_rank(const int32_t* __restrict__ pos, const int32_t* __restrict__ insX,
                                            const int32_t* __restrict__ delX, int32_t a, int32_t i) {
    return pos[i] + (insX[i] - insX[a]) - (delX[i] - delX[a]);
}

// Rows of the batch with at most kRowWarpMax existing entries + updates, one
// warp each: rank the surviving entries and the inserts into the row's
// scratch range, then (after __syncwarp, which orders the warp's scratch
// writes before its reads) copy the range to the row's slots, in place or
// to fresh ones at base + relX[k], and finish deg / start / cap.  In a merge
// rebuild (dst_start given) the rows go straight to dst_start[r] in the new
// arena (scol / sval), and the row table is finished by the host.  Longer rows
// go to `big` (with the chunk counts of their old and new entries in big_d /
// big_d2, zero past the list) for the grid-wide kernels; big_flag[k] tells
// them apart.
__global__ void upd_rows_warp_kernel(const int32_t* __restrict__ row_id, const int32_t* __restrict__ row_first,
                                     const int32_t* __restrict__ headX, const int32_t* __restrict__ scrX,
                                     const int32_t* __restrict__ exX, const int64_t* __restrict__ relX,
                                     const uint64_t* __restrict__ skey, const uint32_t* __restrict__ sidx,
                                     const double* __restrict__ values, const int8_t* __restrict__ typ,
                                     const int32_t* __restrict__ pos, const int32_t* __restrict__ insX,
                                     const int32_t* __restrict__ delX, int64_t base, int64_t b,
                                     int64_t* __restrict__ start, int32_t* __restrict__ deg,
                                     int32_t* __restrict__ cap, int32_t* __restrict__ col, double* __restrict__ val,
                                     int32_t* __restrict__ scol, double* __restrict__ sval,
                                     int32_t* __restrict__ big, int32_t* __restrict__ big_tail,
                                     int32_t* __restrict__ big_d, int32_t* __restrict__ big_d2,
                                     int8_t* __restrict__ big_flag, int32_t row_warp_max,
                                     const int64_t* __restrict__ dst_start, unsigned long long* __restrict__ moved,
                                     unsigned long long* __restrict__ bad_rank) {
    const int lane = lane_id();
    const int64_t K = headX[b];
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t k = warp; k < K; k += nwarps) {
        const int32_t d = exX[k + 1] - exX[k], d2 = scrX[k + 1] - scrX[k];
        const int32_t a = row_first[k], z = row_first[k + 1];
        const bool changed = d > 0 || d2 > 0;
        const bool is_big = changed && (int64_t)d + (z - a) > row_warp_max;
        if (lane == 0) {
            big_flag[k] = is_big ? 1 : 0;
            if (is_big) {
                const int32_t i = atomicAdd(big_tail, 1);
                big[i] = (int32_t)k;
                big_d[i] = (d + kBigChunk - 1) / kBigChunk;
                big_d2[i] = (d2 + kBigChunk - 1) / kBigChunk;
            }
        }
        if (!changed || is_big) continue;
        const int32_t r = row_id[k];
        const int64_t s = start[r];
        const int64_t o = dst_start ? dst_start[r] : (int64_t)scrX[k];
        unsigned long long bad = 0;
        for (int32_t j = lane; j < d; j += 32) {
            const int32_t c = col[s + j];
            const int32_t rk = old_rank(skey, typ, insX, delX, a, z, (uint32_t)r, c, j);
            if (rk < 0) continue;
            if (rk >= d2) {
                ++bad;
                continue;
            }
            scol[o + rk] = c;
            sval[o + rk] = val[s + j];
        }
        for (int32_t i = a + lane; i < z; i += 32) {
            if (typ[i] != kIns) continue;
            const int32_t rk = new_rank(pos, insX, delX, a, i);
            if (rk < 0 || rk >= d2) {
                ++bad;
                continue;
            }
            scol[o + rk] = (int32_t)(uint32_t)skey[i];
            sval[o + rk] = values[sidx[i]];
        }
        if (bad) atomicAdd(bad_rank, bad);
        if (dst_start) continue;  // merge rebuild: written to its final place
        __syncwarp();
        const int32_t cp = cap[r];
        const int64_t dst = d2 <= cp ? s : base + relX[k];
        for (int32_t j = lane; j < d2; j += 32) {
            col[dst + j] = scol[o + j];
            val[dst + j] = sval[o + j];
        }
        if (lane == 0) {
            if (d2 > cp) {
                start[r] = dst;
                cap[r] = (int32_t)slack_cap(d2);
                atomicAdd(moved, 1ull);
            }
            deg[r] = d2;
        }
    }
}

// Exclusive prefix sums of up to three arrays of `count` values in one block
// of 1,024 threads (thread t sums its own contiguous run, one block scan of
// the run totals, then each run is written); out[count] = total.  For the
// small batches, where three kernels per scan would cost more than the data.
template <class T, int NA>
__global__ void small_scan_kernel(const T* __restrict__ in0, const T* __restrict__ in1, const T* __restrict__ in2,
                                  T* __restrict__ out0, T* __restrict__ out1, T* __restrict__ out2, int64_t count) {
    __shared__ T s_w[NA][32];
    const T* in[3] = {in0, in1, in2};
    T* out[3] = {out0, out1, out2};
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int64_t per = (count + blockDim.x - 1) / blockDim.x;
    const int64_t lo = min(count, (int64_t)threadIdx.x * per), hi = min(count, lo + per);
    T sum[NA], incl[NA];
#pragma unroll
    for (int a = 0; a < NA; ++a) {
        sum[a] = 0;
        for (int64_t i = lo; i < hi; ++i) sum[a] += in[a][i];
        incl[a] = sum[a];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const T x = __shfl_up_sync(0xffffffffu, incl[a], off);
            if (lane >= off) incl[a] += x;
        }
        if (lane == 31) s_w[a][wid] = incl[a];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int a = 0; a < NA; ++a) {
            T w = lane < nw ? s_w[a][lane] : 0;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const T x = __shfl_up_sync(0xffffffffu, w, off);
                if (lane >= off) w += x;
            }
            if (lane < nw) s_w[a][lane] = w;
        }
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NA; ++a) {
        T run = (wid ? s_w[a][wid - 1] : 0) + incl[a] - sum[a];
        for (int64_t i = lo; i < hi; ++i) {
            const T x = in[a][i];
            out[a][i] = run;
            run += x;
        }
        if (threadIdx.x == 0) out[a][count] = s_w[a][nw - 1];
    }
}

// Existing entries of the long rows: warp per kBigChunk-entry chunk, chunk c
// of row big[i] for bex[i] <= c < bex[i + 1].
__global__ void big_scatter_old_kernel(const int32_t* __restrict__ big, const int32_t* __restrict__ big_tail,
                                       const int32_t* __restrict__ bex, const int32_t* __restrict__ row_id,
                                       const int32_t* __restrict__ row_first, const int32_t* __restrict__ scrX,
                                       const int32_t* __restrict__ exX, const uint64_t* __restrict__ skey,
                                       const int8_t* __restrict__ typ, const int32_t* __restrict__ insX,
                                       const int32_t* __restrict__ delX, const int64_t* __restrict__ start,
                                       const int32_t* __restrict__ col, const double* __restrict__ val,
                                       int32_t* __restrict__ scol, double* __restrict__ sval,
                                       const int64_t* __restrict__ dst_start,
                                       unsigned long long* __restrict__ bad_rank) {
    const int lane = lane_id();
    const int32_t nb = *big_tail;
    const int64_t C = bex[nb];
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t ch = warp; ch < C; ch += nwarps) {
        const int64_t i = seg_of(bex, nb, ch);
        const int32_t k = big[i];
        const int32_t r = row_id[k];
        const int32_t d = exX[k + 1] - exX[k], d2 = scrX[k + 1] - scrX[k];
        const int32_t a = row_first[k], z = row_first[k + 1];
        const int64_t s = start[r];
        const int64_t o = dst_start ? dst_start[r] : (int64_t)scrX[k];
        const int32_t j0 = (int32_t)(ch - bex[i]) * kBigChunk;
        unsigned long long bad = 0;
#pragma unroll 2
        for (int u = 0; u < kBigChunk / 32; ++u) {
            const int32_t j = j0 + u * 32 + lane;
            if (j >= d) break;
            const int32_t c = col[s + j];
            const int32_t rk = old_rank(skey, typ, insX, delX, a, z, (uint32_t)r, c, j);
            if (rk < 0) continue;
            if (rk >= d2) {
                ++bad;
                continue;
            }
            scol[o + rk] = c;
            sval[o + rk] = val[s + j];
        }
        if (bad) atomicAdd(bad_rank, bad);
    }
}

// Inserts into the long rows.
__global__ void big_scatter_new_kernel(const uint64_t* __restrict__ skey, const uint32_t* __restrict__ sidx,
                                       const double* __restrict__ values, const int8_t* __restrict__ typ,
                                       const int32_t* __restrict__ pos, const int32_t* __restrict__ headX,
                                       const int32_t* __restrict__ row_first, const int32_t* __restrict__ insX,
                                       const int32_t* __restrict__ delX, const int32_t* __restrict__ scrX,
                                       const int8_t* __restrict__ big_flag, int64_t b, int32_t* __restrict__ scol,
                                       double* __restrict__ sval, const int32_t* __restrict__ row_id,
                                       const int64_t* __restrict__ dst_start,
                                       unsigned long long* __restrict__ bad_rank) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < b; i += (int64_t)gridDim.x * blockDim.x) {
        if (typ[i] != kIns) continue;
        const int32_t k = headX[i + 1] - 1;
        if (!big_flag[k]) continue;
        const int32_t rk = new_rank(pos, insX, delX, row_first[k], (int32_t)i);
        if (rk < 0 || rk >= scrX[k + 1] - scrX[k]) {
            atomicAdd(bad_rank, 1ull);
            continue;
        }
        const int64_t o = dst_start ? dst_start[row_id[k]] : (int64_t)scrX[k];
        scol[o + rk] = (int32_t)(uint32_t)skey[i];
        sval[o + rk] = values[sidx[i]];
    }
}

// Long rows: scratch -> their slots (in place when they fit, else fresh
// ones), warp per kBigChunk-entry chunk as above (chunks of the new rows).
__global__ void big_copy_kernel(const int32_t* __restrict__ big, const int32_t* __restrict__ big_tail,
                                const int32_t* __restrict__ bsz, const int32_t* __restrict__ row_id,
                                const int32_t* __restrict__ scrX, const int64_t* __restrict__ relX,
                                const int64_t* __restrict__ start, const int32_t* __restrict__ cap, int64_t base,
                                const int32_t* __restrict__ scol, const double* __restrict__ sval,
                                int32_t* __restrict__ col, double* __restrict__ val) {
    const int lane = lane_id();
    const int32_t nb = *big_tail;
    const int64_t C = bsz[nb];
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t ch = warp; ch < C; ch += nwarps) {
        const int64_t i = seg_of(bsz, nb, ch);
        const int32_t k = big[i];
        const int32_t r = row_id[k];
        const int32_t d2 = scrX[k + 1] - scrX[k];
        const int64_t dst = d2 <= cap[r] ? start[r] : base + relX[k];
        const int32_t o = scrX[k];
        const int32_t j0 = (int32_t)(ch - bsz[i]) * kBigChunk;
        constexpr int kPer = kBigChunk / 32;
        int32_t cv[kPer];
        double wv[kPer];
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int32_t j = j0 + u * 32 + lane;
            if (j < d2) {
                cv[u] = scol[o + j];
                wv[u] = sval[o + j];
            }
        }
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int32_t j = j0 + u * 32 + lane;
            if (j < d2) {
                col[dst + j] = cv[u];
                val[dst + j] = wv[u];
            }
        }
    }
}

__global__ void big_finalize_kernel(const int32_t* __restrict__ big, const int32_t* __restrict__ big_tail,
                                    const int32_t* __restrict__ row_id, const int32_t* __restrict__ scrX,
                                    const int64_t* __restrict__ relX, int64_t base, int64_t* __restrict__ start,
                                    int32_t* __restrict__ deg, int32_t* __restrict__ cap,
                                    unsigned long long* __restrict__ moved) {
    const int32_t nb = *big_tail;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
        const int32_t k = big[i];
        const int32_t r = row_id[k];
        const int32_t d2 = scrX[k + 1] - scrX[k];
        if (d2 > cap[r]) {
            start[r] = base + relX[k];
            cap[r] = (int32_t)slack_cap(d2);
            atomicAdd(moved, 1ull);
        }
        deg[r] = d2;
    }
}

// Merge rebuild helpers over the batch's rows k < K: changed rows get slots
// for their new degree, are left out of the copy of the unchanged rows, and
// take their new degree at the end.
__global__ void want_changed_kernel(const int32_t* __restrict__ row_id, const int32_t* __restrict__ headX,
                                    const int32_t* __restrict__ scrX, const int32_t* __restrict__ exX, int64_t b,
                                    int64_t* __restrict__ want, int32_t* __restrict__ deg_copy) {
    const int64_t K = headX[b];
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = exX[k + 1] - exX[k], d2 = scrX[k + 1] - scrX[k];
        if (d == 0 && d2 == 0) continue;
        const int32_t r = row_id[k];
        want[r] = slack_cap(d2);
        deg_copy[r] = 0;
    }
}

__global__ void set_changed_deg_kernel(const int32_t* __restrict__ row_id, const int32_t* __restrict__ headX,
                                       const int32_t* __restrict__ scrX, const int32_t* __restrict__ exX, int64_t b,
                                       int32_t* __restrict__ deg) {
    const int64_t K = headX[b];
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = exX[k + 1] - exX[k], d2 = scrX[k + 1] - scrX[k];
        if (d == 0 && d2 == 0) continue;
        deg[row_id[k]] = d2;
    }
}

// ------------------------------------------------------ repack and snapshot

__global__ void want_cap_kernel(const int32_t* __restrict__ deg, int32_t n, int64_t* __restrict__ want) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        want[v] = slack_cap(deg[v]);
}

// Rows that this batch grows get room for their new degree.
__global__ void want_batch_kernel(const int32_t* __restrict__ row_id, const int32_t* __restrict__ headX,
                                  const int32_t* __restrict__ scrX, int64_t b, int64_t* __restrict__ want) {
    const int64_t K = headX[b];
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < K; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t w = slack_cap(scrX[k + 1] - scrX[k]);
        const int32_t r = row_id[k];
        if (w > want[r]) want[r] = w;
    }
}

__global__ void set_caps_kernel(const int64_t* __restrict__ want, int32_t n, int32_t* __restrict__ cap) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        cap[v] = (int32_t)want[v];
}

// Copy every row shorter than kCopyChunk (sstart/deg in the arena) to
// dst_off[v].  A warp takes 32 consecutive rows, scans their lengths and
// copies the concatenation, four 32-entry steps per round (each lane finds
// its row by a 5-step shuffle search; the loads of a round are issued before
// its stores).  Longer rows only get their chunk count, cc[v], for
// row_copy_chunk_kernel.
template <class DstOff>
__global__ void row_copy_kernel(int32_t n, const int64_t* __restrict__ sstart, const int32_t* __restrict__ deg,
                                const int32_t* __restrict__ scol, const double* __restrict__ sval,
                                const DstOff* __restrict__ dst_off, int32_t* __restrict__ dcol,
                                double* __restrict__ dval, int32_t* __restrict__ cc) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = warp * 32; base < n; base += nwarps * 32) {
        const int64_t v = base + lane;
        int32_t d = 0;
        int64_t s = 0, o = 0;
        if (v < n) {
            d = deg[v];
            s = sstart[v];
            o = (int64_t)dst_off[v];
            cc[v] = d >= kCopyChunk ? (d + kCopyChunk - 1) / kCopyChunk : 0;
            if (d >= kCopyChunk) d = 0;
        }
        int32_t incl = d;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int32_t x = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += x;
        }
        const int32_t excl = incl - d;
        const int32_t tot = __shfl_sync(0xffffffffu, incl, 31);
        for (int32_t q0 = 0; q0 < tot; q0 += 128) {
            int64_t src[4], dst[4];
            int32_t cv[4];
            double wv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int32_t q = q0 + 32 * u + lane;
                int w = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const int32_t x = __shfl_sync(0xffffffffu, incl, w + step - 1);
                    if (x <= q) w += step;
                }
                const int64_t sw = __shfl_sync(0xffffffffu, s, w);
                const int64_t ow = __shfl_sync(0xffffffffu, o, w);
                const int32_t ew = __shfl_sync(0xffffffffu, excl, w);
                src[u] = q < tot ? sw + (q - ew) : -1;
                dst[u] = ow + (q - ew);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (src[u] >= 0) {
                    cv[u] = scol[src[u]];
                    if (dval) wv[u] = sval[src[u]];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (src[u] >= 0) {
                    dcol[dst[u]] = cv[u];
                    if (dval) dval[dst[u]] = wv[u];
                }
            }
        }
    }
}

// chunk_row[c] = v for the chunks coff[v] <= c < coff[v + 1] of each long
// row, so a chunk finds its row with one load.
__global__ void chunk_rows_kernel(int32_t n, const int32_t* __restrict__ cc, const int32_t* __restrict__ coff,
                                  int32_t* __restrict__ chunk_row) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = cc[v];
        for (int32_t i = 0; i < k; ++i) chunk_row[coff[v] + i] = (int32_t)v;
    }
}

// Chunks of the long rows, one warp each (8 entries per lane, loads first).
template <class DstOff>
__global__ void row_copy_chunk_kernel(int32_t n, const int32_t* __restrict__ coff,
                                      const int32_t* __restrict__ chunk_row, const int64_t* __restrict__ sstart,
                                      const int32_t* __restrict__ deg, const int32_t* __restrict__ scol,
                                      const double* __restrict__ sval, const DstOff* __restrict__ dst_off,
                                      int32_t* __restrict__ dcol, double* __restrict__ dval) {
    const int lane = lane_id();
    const int64_t C = coff[n];
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = warp; c < C; c += nwarps) {
        const int32_t v = chunk_row[c];
        const int32_t d = deg[v];
        const int32_t j0 = (int32_t)(c - coff[v]) * kCopyChunk;
        const int64_t s = sstart[v] + j0, o = (int64_t)dst_off[v] + j0;
        const int32_t len = min(kCopyChunk, d - j0);
        constexpr int kPer = kCopyChunk / 32;
        int32_t cv[kPer];
        double wv[kPer];
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int32_t j = u * 32 + lane;
            if (j < len) {
                cv[u] = scol[s + j];
                if (dval) wv[u] = sval[s + j];
            }
        }
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int32_t j = u * 32 + lane;
            if (j < len) {
                dcol[o + j] = cv[u];
                if (dval) dval[o + j] = wv[u];
            }
        }
    }
}

__global__ void find_kernel(const int64_t* __restrict__ start, const int32_t* __restrict__ deg,
                            const int32_t* __restrict__ col, const double* __restrict__ val, int32_t n,
                            const uint64_t* __restrict__ keys, int64_t count, double* __restrict__ out,
                            unsigned long long* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        const uint64_t r = k >> 32, c = k & 0xffffffffull;
        double v = 0.0;
        if (r < (uint64_t)n && c < (uint64_t)n) {
            const int32_t* row = col + start[r];
            int32_t lo = 0, hi = deg[r];
            while (lo < hi) {
                const int32_t mid = (lo + hi) >> 1;
                if ((uint32_t)row[mid] < (uint32_t)c) lo = mid + 1;
                else hi = mid;
            }
            if (lo < deg[r] && (uint32_t)row[lo] == (uint32_t)c) v = val[start[r] + lo];
        } else {
            atomicAdd(bad, 1ull);
        }
        out[i] = v;
    }
}

// Rows of a CSR must be strictly increasing and inside [0, n); a weight of 0
// would mark a deleted entry, so it is refused too.
__global__ void csr_check_kernel(const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                                 const double* __restrict__ w, int32_t n, int64_t m,
                                 unsigned long long* __restrict__ bad) {
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long mine = 0;
    for (int64_t v = warp; v < n; v += nwarps) {
        const int32_t b = rp[v], e = rp[v + 1];
        if (e < b || b < 0 || (int64_t)e > m) {
            if (lane_id() == 0) ++mine;
            continue;
        }
        for (int32_t j = b + lane_id(); j < e; j += 32) {
            const int32_t c = col[j];
            if (c < 0 || c >= n || (j > b && col[j - 1] >= c) || (w && w[j] == 0.0)) ++mine;
        }
    }
    if (mine) atomicAdd(bad, mine);
}

__global__ void deg_from_rowptr_kernel(const int32_t* __restrict__ rp, int32_t n, int32_t* __restrict__ deg) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        deg[v] = rp[v + 1] - rp[v];
}

__global__ void widen_rowptr_kernel(const int32_t* __restrict__ rp, int32_t n, int64_t* __restrict__ out) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        out[v] = rp[v];
}

__global__ void fill_f64_kernel(double* __restrict__ p, int64_t count, double x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = x;
}

// ------------------------------------------------------------------ host

unsigned grid_of(ghb_workspace* ws, int64_t items, int threads = 256) {
    return grid_for(items, threads, (int64_t)ws->num_sms * 16);
}

// Copy n rows (sstart/deg into scol/sval) to dst offsets (int32 CSR offsets
// or int64 arena starts).  `list` holds n + 2 int32.
// Chunk slots copy_rows needs for a graph of m entries: each long row has at
// most one partial chunk, and a long row has at least kCopyChunk entries.
inline int64_t copy_chunk_slots(int64_t m) { return 2 * (m / kCopyChunk) + 1; }

template <class DstOff>
int copy_rows(ghb_workspace* ws, int32_t n, const int64_t* sstart, const int32_t* deg, const int32_t* scol,
              const double* sval, const DstOff* dst_off, int32_t* dcol, double* dval, int32_t* cc, int32_t* coff,
              int32_t* chunk_row, int64_t* block_sums) {
    const unsigned grid = grid_for(((int64_t)n + 31) / 32 * 32, 256, (int64_t)ws->num_sms * 8);
    const double* sv = dval ? sval : nullptr;
    GHB_TRY(launch(ws, row_copy_kernel<DstOff>, dim3(grid), dim3(256), 0, n, sstart, deg, scol, sv, dst_off, dcol,
                   dval, cc));
    GHB_TRY(scan_exclusive_i32(ws, cc, coff, n, block_sums));
    GHB_TRY(launch(ws, chunk_rows_kernel, dim3(grid_for(n, 256, (int64_t)ws->num_sms * 8)), dim3(256), 0, n,
                   (const int32_t*)cc, (const int32_t*)coff, chunk_row));
    GHB_TRY(launch(ws, row_copy_chunk_kernel<DstOff>, dim3(ws->num_sms * 8), dim3(256), 0, n, (const int32_t*)coff,
                   (const int32_t*)chunk_row, sstart, deg, scol, sv, dst_off, dcol, dval));
    return GHB_OK;
}

// Copy the rows (src_start, g->deg, src_col, src_val; `entries` in all) into a fresh arena with
// want[v] slots for row v and `headroom` spare slots at its end.  On success
// g->start / cap / col / val / slots / used describe the new arena; the old
// col / val arrays are freed when they belong to the graph (free_old).
int repack(ghb_workspace* ws, ghb_gpma* g, const int64_t* src_start, const int32_t* src_col,
           const double* src_val, int64_t* want, int64_t headroom, bool free_old, int64_t entries) {
    const int32_t n = g->n;
    int64_t* nstart = nullptr;
    int32_t* big = nullptr;
    char* tmp = nullptr;
    int32_t* ncol = nullptr;
    double* nval = nullptr;
    size_t tmp_bytes = 0;
    int st = GHB_OK;
    do {
        if ((st = dev_alloc(&nstart, (int64_t)n + 1))) break;
        // cc, coff (n + 1 int32 each), the scan's block sums, the chunk rows
        if ((st = dev_alloc(&big, 2 * ((int64_t)n + 1) + 2 * scan_scratch_words(n) + copy_chunk_slots(entries))))
            break;
        // nstart = exclusive scan of want; nstart[n] = total slots.
        cudaError_t e = cudaMemsetAsync(want + n, 0, sizeof(int64_t), ws->stream);
        if (e == cudaSuccess)
            e = cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, want, nstart, (int64_t)n + 1, ws->stream);
        if (e != cudaSuccess) {
            set_error(std::string("repack scan: ") + cudaGetErrorString(e));
            st = GHB_ERR_CUDA;
            break;
        }
        if ((st = dev_alloc(&tmp, (int64_t)std::max<size_t>(tmp_bytes, 1)))) break;
        int64_t total = 0;
        e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, want, nstart, (int64_t)n + 1, ws->stream);
        ws->launches++;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&total, nstart + n, sizeof(int64_t), cudaMemcpyDeviceToHost, ws->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ws->stream);
        if (e != cudaSuccess) {
            set_error(std::string("repack scan: ") + cudaGetErrorString(e));
            st = GHB_ERR_CUDA;
            break;
        }
        const int64_t slots = total + headroom;
        if ((st = dev_alloc(&ncol, slots))) break;
        if ((st = dev_alloc(&nval, slots))) break;
        if ((st = copy_rows<int64_t>(ws, n, src_start, g->deg, src_col, src_val, nstart, ncol, nval, big,
                                     big + n + 1, big + 2 * ((int64_t)n + 1) + 2 * scan_scratch_words(n),
                                     reinterpret_cast<int64_t*>(big + 2 * ((int64_t)n + 1)))))
            break;
        if ((st = launch(ws, set_caps_kernel, dim3(grid_of(ws, n)), dim3(256), 0, (const int64_t*)want, n, g->cap)))
            break;
        e = cudaMemcpyAsync(g->start, nstart, sizeof(int64_t) * (size_t)n, cudaMemcpyDeviceToDevice, ws->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ws->stream);
        if (e != cudaSuccess) {
            set_error(std::string("repack copy: ") + cudaGetErrorString(e));
            st = GHB_ERR_CUDA;
            break;
        }
        if (free_old) {
            dev_free(g->col);
            dev_free(g->val);
        }
        g->col = ncol;
        g->val = nval;
        ncol = nullptr;
        nval = nullptr;
        g->slots = slots;
        g->used = total;
        g->stats[5]++;
    } while (false);
    dev_free(ncol);
    dev_free(nval);
    dev_free(nstart);
    dev_free(big);
    dev_free(tmp);
    return st;
}

int bbuf_reserve(ghb_gpma* g, size_t bytes) {
    if (bytes <= g->bbuf_cap) return GHB_OK;
    dev_free(reinterpret_cast<char*&>(g->bbuf));
    g->bbuf_cap = 0;
    size_t cap = (bytes + (16ull << 20) - 1) & ~((16ull << 20) - 1);
    GHB_CUDA_TRY(cudaMalloc(&g->bbuf, cap));
    g->bbuf_cap = cap;
    return GHB_OK;
}

struct PassArrays {
    uint64_t* skey;
    uint32_t *idx, *sidx;
    int32_t *ins, *del, *head, *pos;
    int8_t* typ;
    int32_t *insX, *delX, *headX, *row_id, *row_first, *scrn, *exn, *scrX, *exX;
    int64_t *reln, *relX, *block_sums;
    int32_t *big, *big_tail, *big_d, *big_d2, *bex, *bsz;
    int8_t* big_flag;
    void* tmp;
    int32_t* scol;
    double* sval;
};

void carve_pass(Carver& c, int64_t b, size_t tmp_bytes, PassArrays& a) {
    a.skey = c.take<uint64_t>(b);
    a.idx = c.take<uint32_t>(b);
    a.sidx = c.take<uint32_t>(b);
    a.ins = c.take<int32_t>(b);
    a.del = c.take<int32_t>(b);
    a.head = c.take<int32_t>(b);
    a.pos = c.take<int32_t>(b);
    a.typ = c.take<int8_t>(b);
    a.insX = c.take<int32_t>(b + 1);
    a.delX = c.take<int32_t>(b + 1);
    a.headX = c.take<int32_t>(b + 1);
    a.row_id = c.take<int32_t>(b + 1);
    a.row_first = c.take<int32_t>(b + 1);
    a.scrn = c.take<int32_t>(b);
    a.exn = c.take<int32_t>(b);
    a.scrX = c.take<int32_t>(b + 1);
    a.exX = c.take<int32_t>(b + 1);
    a.reln = c.take<int64_t>(b + 1);
    a.relX = c.take<int64_t>(b + 1);
    a.block_sums = c.take<int64_t>(scan_scratch_words(b + 1));
    a.bex = c.take<int32_t>(b + 1);
    a.bsz = c.take<int32_t>(b + 1);
    a.big = c.take<int32_t>(b);
    a.big_d = c.take<int32_t>(b);
    a.big_d2 = c.take<int32_t>(b);
    a.big_tail = c.take<int32_t>(1);
    a.big_flag = c.take<int8_t>(b);
    a.tmp = c.take<char>(tmp_bytes);
}

// The merge rebuild of one pass (see apply_pass): new slots for every row
// (changed rows sized for their new degree), the unchanged rows copied, the
// changed ones rebuilt straight into the new arena, then the row table.
int merge_rebuild(ghb_workspace* ws, ghb_gpma* g, const PassArrays& a, const double* values, int64_t b,
                  int64_t live_after, int64_t n_modified, int64_t n_ins, int64_t n_long_rows, bool small_b,
                  int32_t row_warp_max, int64_t K, unsigned long long* bad_rank) {
    const int32_t n = g->n;
    const unsigned gr = grid_of(ws, b);
    const unsigned gn = grid_of(ws, n);
    const unsigned wide = (unsigned)ws->num_sms * 16;
    const int64_t ssw = scan_scratch_words(n);
    // Row-table temporaries in the workspace scratch (this pass needs no
    // other scratch there): want and nstart (n + 1 int64 each), the copy's
    // row lengths, its cc / coff / block sums / chunk rows, the scan's temp.
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, (int64_t*)nullptr, (int64_t*)nullptr, (int64_t)n + 1,
                                  ws->stream);
    auto carve = [&](Carver& c, int64_t** want, int64_t** nstart, int32_t** degc, int32_t** tmp32, char** tmp) {
        *want = c.take<int64_t>((int64_t)n + 1);
        *nstart = c.take<int64_t>((int64_t)n + 1);
        *degc = c.take<int32_t>(n);
        *tmp32 = c.take<int32_t>(2 * ((int64_t)n + 1) + 2 * ssw + copy_chunk_slots(g->m));
        *tmp = c.take<char>(std::max<size_t>(tmp_bytes, 1));
    };
    int64_t *want = nullptr, *nstart = nullptr;
    int32_t *degc = nullptr, *tmp32 = nullptr;
    char* tmp = nullptr;
    Carver sizing(nullptr);
    carve(sizing, &want, &nstart, &degc, &tmp32, &tmp);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    carve(c, &want, &nstart, &degc, &tmp32, &tmp);
    int32_t* ncol = nullptr;
    double* nval = nullptr;
    int st = GHB_OK;
    cudaError_t e = cudaSuccess;
    do {
        // Weight changes in place first: both copies below read them.
        if (n_modified > 0 &&
            (st = launch(ws, upd_modify_kernel, dim3(gr), dim3(256), 0, (const uint64_t*)a.skey,
                         (const uint32_t*)a.sidx, values, (const int8_t*)a.typ, (const int32_t*)a.pos,
                         (const int64_t*)g->start, b, g->val)))
            break;
        if ((st = launch(ws, want_cap_kernel, dim3(gn), dim3(256), 0, (const int32_t*)g->deg, n, want))) break;
        if ((e = cudaMemcpyAsync(degc, g->deg, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToDevice, ws->stream)))
            break;
        if ((st = launch(ws, want_changed_kernel, dim3(gr), dim3(256), 0, (const int32_t*)a.row_id,
                         (const int32_t*)a.headX, (const int32_t*)a.scrX, (const int32_t*)a.exX, b, want, degc)))
            break;
        if ((e = cudaMemsetAsync(want + n, 0, sizeof(int64_t), ws->stream))) break;
        if ((e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, want, nstart, (int64_t)n + 1, ws->stream))) break;
        ws->launches++;
        int64_t total = 0;
        if ((e = cudaMemcpyAsync(&total, nstart + n, sizeof(int64_t), cudaMemcpyDeviceToHost, ws->stream))) break;
        if ((e = cudaStreamSynchronize(ws->stream))) break;
        // The new arena: the spare one when it holds the rows with a little
        // room to grow, else a fresh one with an eighth of the entries to
        // spare (the next rebuild can then reuse this one's predecessor).
        int64_t slots = total + live_after / 8 + 4096;
        if (g->spare_slots >= total + live_after / 32 + 4096) {
            ncol = g->spare_col;
            nval = g->spare_val;
            slots = g->spare_slots;
            g->spare_col = nullptr;
            g->spare_val = nullptr;
            g->spare_slots = 0;
        } else {
            dev_free(g->spare_col);
            dev_free(g->spare_val);
            g->spare_slots = 0;
            if ((st = dev_alloc(&ncol, slots))) break;
            if ((st = dev_alloc(&nval, slots))) break;
        }
        if ((st = copy_rows<int64_t>(ws, n, g->start, degc, g->col, g->val, nstart, ncol, nval, tmp32,
                                     tmp32 + n + 1, tmp32 + 2 * ((int64_t)n + 1) + 2 * ssw,
                                     reinterpret_cast<int64_t*>(tmp32 + 2 * ((int64_t)n + 1)))))
            break;
        if ((e = cudaMemsetAsync(a.big_tail, 0, sizeof(int32_t), ws->stream))) break;
        if (n_long_rows > 0) {
            if ((e = cudaMemsetAsync(a.big_d, 0, sizeof(int32_t) * (size_t)b, ws->stream))) break;
            if ((e = cudaMemsetAsync(a.big_d2, 0, sizeof(int32_t) * (size_t)b, ws->stream))) break;
        }
        if ((st = launch(ws, upd_rows_warp_kernel, dim3(grid_for(K * 32, 256, (int64_t)ws->num_sms * 8)), dim3(256),
                         0, (const int32_t*)a.row_id, (const int32_t*)a.row_first, (const int32_t*)a.headX,
                         (const int32_t*)a.scrX, (const int32_t*)a.exX, (const int64_t*)a.relX,
                         (const uint64_t*)a.skey, (const uint32_t*)a.sidx, values, (const int8_t*)a.typ,
                         (const int32_t*)a.pos, (const int32_t*)a.insX, (const int32_t*)a.delX, (int64_t)0, b,
                         g->start, g->deg, g->cap, g->col, g->val, ncol, nval, a.big, a.big_tail, a.big_d, a.big_d2,
                         a.big_flag, row_warp_max, (const int64_t*)nstart, g->moved, bad_rank)))
            break;
        if (n_long_rows > 0) {
            if (small_b)
                st = launch(ws, small_scan_kernel<int32_t, 2>, dim3(1), dim3(1024), 0, (const int32_t*)a.big_d,
                            (const int32_t*)a.big_d2, (const int32_t*)nullptr, a.bex, a.bsz, (int32_t*)nullptr, b);
            else
                st = scan_exclusive_i32(ws, a.big_d, a.bex, b, a.block_sums);
            if (st) break;
            if ((st = launch(ws, big_scatter_old_kernel, dim3(wide), dim3(256), 0, (const int32_t*)a.big,
                             (const int32_t*)a.big_tail, (const int32_t*)a.bex, (const int32_t*)a.row_id,
                             (const int32_t*)a.row_first, (const int32_t*)a.scrX, (const int32_t*)a.exX,
                             (const uint64_t*)a.skey, (const int8_t*)a.typ, (const int32_t*)a.insX,
                             (const int32_t*)a.delX, (const int64_t*)g->start, (const int32_t*)g->col,
                             (const double*)g->val, ncol, nval, (const int64_t*)nstart, bad_rank)))
                break;
            if (n_ins > 0 &&
                (st = launch(ws, big_scatter_new_kernel, dim3(gr), dim3(256), 0, (const uint64_t*)a.skey,
                             (const uint32_t*)a.sidx, values, (const int8_t*)a.typ, (const int32_t*)a.pos,
                             (const int32_t*)a.headX, (const int32_t*)a.row_first, (const int32_t*)a.insX,
                             (const int32_t*)a.delX, (const int32_t*)a.scrX, (const int8_t*)a.big_flag, b, ncol,
                             nval, (const int32_t*)a.row_id, (const int64_t*)nstart, bad_rank)))
                break;
        }
        // The row table of the new arena.
        if ((e = cudaMemcpyAsync(g->start, nstart, sizeof(int64_t) * (size_t)n, cudaMemcpyDeviceToDevice,
                                 ws->stream)))
            break;
        if ((st = launch(ws, set_caps_kernel, dim3(gn), dim3(256), 0, (const int64_t*)want, n, g->cap))) break;
        if ((st = launch(ws, set_changed_deg_kernel, dim3(gr), dim3(256), 0, (const int32_t*)a.row_id,
                         (const int32_t*)a.headX, (const int32_t*)a.scrX, (const int32_t*)a.exX, b, g->deg)))
            break;
        if ((e = cudaStreamSynchronize(ws->stream))) break;
        // The old arena becomes the spare.
        g->spare_col = g->col;
        g->spare_val = g->val;
        g->spare_slots = g->slots;
        g->col = ncol;
        g->val = nval;
        ncol = nullptr;
        nval = nullptr;
        g->slots = slots;
        g->used = total;
        g->stats[5]++;
    } while (false);
    if (e != cudaSuccess) {
        set_error(std::string("dynamic-graph merge rebuild: ") + cudaGetErrorString(e));
        st = GHB_ERR_CUDA;
    }
    dev_free(ncol);
    dev_free(nval);
    return st;
}

// One pass of at most kPassUpdates updates.
int apply_pass(ghb_workspace* ws, ghb_gpma* g, const uint64_t* keys, const double* values, int64_t b,
               int64_t* totals) {
    const int32_t n = g->n;
    const int end_bit = 32 + key_bits(n);
    size_t sort_bytes = 0, scan_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, b, 0, end_bit, ws->stream);
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (int64_t*)nullptr, (int64_t*)nullptr, b + 1, ws->stream);
    const size_t tmp_bytes = std::max(sort_bytes, scan_bytes);
    PassArrays a;
    Carver sizing(nullptr);
    carve_pass(sizing, b, tmp_bytes, a);
    GHB_TRY(bbuf_reserve(g, sizing.off));
    Carver c(g->bbuf);
    carve_pass(c, b, tmp_bytes, a);

    // dev_small: [0..5] totals, [6] modified, [7] invalid keys, [8] ranks
    // outside their row (a consistency check of the row table), [9] rows for
    // the grid-wide rebuild.
    int64_t* small = ws->dev_small;
    unsigned long long* n_mod = reinterpret_cast<unsigned long long*>(small + 6);
    unsigned long long* n_bad = reinterpret_cast<unsigned long long*>(small + 7);
    unsigned long long* bad_rank = reinterpret_cast<unsigned long long*>(small + 8);
    unsigned long long* n_long = reinterpret_cast<unsigned long long*>(small + 9);
    GHB_CUDA_TRY(cudaMemsetAsync(small, 0, sizeof(int64_t) * 10, ws->stream));
    const unsigned gr = grid_of(ws, b);

    GHB_TRY(launch(ws, upd_prep_kernel, dim3(gr), dim3(256), 0, keys, b, n, a.idx, n_bad));
    size_t sb = sort_bytes;
    GHB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(a.tmp, sb, keys, a.skey, (const uint32_t*)a.idx, a.sidx, b, 0,
                                                 end_bit, ws->stream));
    ws->launches++;
    GHB_TRY(launch(ws, upd_classify_kernel, dim3(gr), dim3(256), 0, (const int64_t*)g->start,
                   (const int32_t*)g->deg, (const int32_t*)g->col, (const uint64_t*)a.skey,
                   (const uint32_t*)a.sidx, values, b, n, a.ins, a.del, a.head, a.pos, a.typ, n_mod));
    const bool small_b = b <= kSmallScan;
    const int32_t row_warp_max = small_b ? kRowWarpSmall : kRowWarpLarge;
    if (small_b) {
        GHB_TRY(launch(ws, small_scan_kernel<int32_t, 3>, dim3(1), dim3(1024), 0, (const int32_t*)a.ins,
                       (const int32_t*)a.del, (const int32_t*)a.head, a.insX, a.delX, a.headX, b));
    } else {
        GHB_TRY(scan_exclusive_i32(ws, a.ins, a.insX, b, a.block_sums));
        GHB_TRY(scan_exclusive_i32(ws, a.del, a.delX, b, a.block_sums));
        GHB_TRY(scan_exclusive_i32(ws, a.head, a.headX, b, a.block_sums));
    }
    GHB_TRY(launch(ws, upd_rows_kernel, dim3(gr), dim3(256), 0, (const uint64_t*)a.skey, (const int32_t*)a.head,
                   (const int32_t*)a.headX, b, a.row_id, a.row_first));
    GHB_TRY(launch(ws, upd_row_summary_kernel, dim3(gr), dim3(256), 0, (const int32_t*)a.row_id,
                   (const int32_t*)a.row_first, (const int32_t*)a.headX, (const int32_t*)a.insX,
                   (const int32_t*)a.delX, (const int32_t*)g->deg, (const int32_t*)g->cap, b, a.scrn, a.exn,
                   a.reln, row_warp_max, n_long));
    if (small_b) {
        GHB_TRY(launch(ws, small_scan_kernel<int32_t, 2>, dim3(1), dim3(1024), 0, (const int32_t*)a.scrn,
                       (const int32_t*)a.exn, (const int32_t*)nullptr, a.scrX, a.exX, (int32_t*)nullptr, b));
        GHB_TRY(launch(ws, small_scan_kernel<int64_t, 1>, dim3(1), dim3(1024), 0, (const int64_t*)a.reln,
                       (const int64_t*)nullptr, (const int64_t*)nullptr, a.relX, (int64_t*)nullptr,
                       (int64_t*)nullptr, b));
    } else {
        GHB_TRY(scan_exclusive_i32(ws, a.scrn, a.scrX, b, a.block_sums));
        GHB_TRY(scan_exclusive_i32(ws, a.exn, a.exX, b, a.block_sums));
        GHB_CUDA_TRY(cudaMemsetAsync(a.reln + b, 0, sizeof(int64_t), ws->stream));
        size_t cb = scan_bytes;
        GHB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(a.tmp, cb, a.reln, a.relX, b + 1, ws->stream));
        ws->launches++;
    }
    GHB_TRY(launch(ws, upd_totals_kernel, dim3(1), dim3(32), 0, (const int32_t*)a.insX, (const int32_t*)a.delX,
                   (const int32_t*)a.headX, (const int32_t*)a.scrX, (const int32_t*)a.exX, (const int64_t*)a.relX, b,
                   small));
    GHB_TRY(ws_read_small(ws, 10));
    const int64_t* h = ws->host_pinned;
    if (h[7]) {
        set_error("invalid argument: update key with a row or column outside [0, n)");
        return GHB_ERR_INVALID_ARGUMENT;
    }
    const int64_t n_ins = h[0], n_del = h[1], K = h[2], S = h[3], E = h[4], R = h[5], n_modified = h[6];
    const int64_t n_long_rows = h[9];
    if (g->m + n_ins - n_del > kMaxEntries) {
        set_error("dynamic graph would exceed 2^31 - 1 entries");
        return GHB_ERR_LIMIT;
    }

    // A batch whose changed rows hold more than half of the entries is
    // applied as a merge rebuild: every row is written once into a fresh
    // arena (unchanged rows copied, changed rows ranked straight into their
    // new slots), 24 bytes per entry instead of the 48 of a rebuild through
    // scratch and back in place.
    if (E > 0 && 2 * E > g->m) {
        GHB_TRY(merge_rebuild(ws, g, a, values, b, g->m + n_ins - n_del, n_modified, n_ins, n_long_rows, small_b,
                              row_warp_max, K, bad_rank));
    } else {
        // Slots for rows that outgrow theirs; repack when the arena is full.
        int64_t base = g->used;
        bool repacked = false;
        if (R > 0 && g->used + R > g->slots) {
            int64_t* want = nullptr;
            GHB_TRY(dev_alloc(&want, (int64_t)n + 1));
            int st = launch(ws, want_cap_kernel, dim3(grid_of(ws, n)), dim3(256), 0, (const int32_t*)g->deg, n, want);
            if (!st)
                st = launch(ws, want_batch_kernel, dim3(gr), dim3(256), 0, (const int32_t*)a.row_id,
                            (const int32_t*)a.headX, (const int32_t*)a.scrX, b, want);
            if (!st) {
                // Headroom for later growth: an eighth of the live entries.
                const int64_t live = g->m + n_ins - n_del;
                st = repack(ws, g, g->start, g->col, g->val, want, live / 8 + 4096, true, g->m);
            }
            dev_free(want);
            GHB_TRY(st);
            base = g->used;  // every changed row fits now; relX is not used
            repacked = true;
        }

        int32_t* scol = nullptr;
        double* sval = nullptr;
        // Scratch for the rebuilt rows (S entries) in the workspace scratch.
        if (S > 0) {
            Carver sizing2(nullptr);
            sizing2.take<int32_t>(S);
            sizing2.take<double>(S);
            GHB_TRY(ws_reserve(ws, sizing2.off));
            Carver c2(ws->scratch);
            scol = c2.take<int32_t>(S);
            sval = c2.take<double>(S);
        }
        if (n_modified > 0)
            GHB_TRY(launch(ws, upd_modify_kernel, dim3(gr), dim3(256), 0, (const uint64_t*)a.skey,
                           (const uint32_t*)a.sidx, values, (const int8_t*)a.typ, (const int32_t*)a.pos,
                           (const int64_t*)g->start, b, g->val));
        if (S > 0 || E > 0) {
            const unsigned wide = (unsigned)ws->num_sms * 16;
            GHB_CUDA_TRY(cudaMemsetAsync(a.big_tail, 0, sizeof(int32_t), ws->stream));
            if (n_long_rows > 0) {
                GHB_CUDA_TRY(cudaMemsetAsync(a.big_d, 0, sizeof(int32_t) * (size_t)b, ws->stream));
                GHB_CUDA_TRY(cudaMemsetAsync(a.big_d2, 0, sizeof(int32_t) * (size_t)b, ws->stream));
            }
            GHB_TRY(launch(ws, upd_rows_warp_kernel, dim3(grid_for(K * 32, 256, (int64_t)ws->num_sms * 8)), dim3(256), 0,
                           (const int32_t*)a.row_id,
                           (const int32_t*)a.row_first, (const int32_t*)a.headX, (const int32_t*)a.scrX,
                           (const int32_t*)a.exX, (const int64_t*)a.relX, (const uint64_t*)a.skey,
                           (const uint32_t*)a.sidx, values, (const int8_t*)a.typ, (const int32_t*)a.pos,
                           (const int32_t*)a.insX, (const int32_t*)a.delX, base, b, g->start, g->deg, g->cap, g->col,
                           g->val, scol, sval, a.big, a.big_tail, a.big_d, a.big_d2, a.big_flag, row_warp_max,
                           (const int64_t*)nullptr, g->moved, bad_rank));
            if (n_long_rows > 0) {
                // Chunk offsets of the long rows, in list order (zeros past it).
                if (small_b) {
                    GHB_TRY(launch(ws, small_scan_kernel<int32_t, 2>, dim3(1), dim3(1024), 0, (const int32_t*)a.big_d,
                                   (const int32_t*)a.big_d2, (const int32_t*)nullptr, a.bex, a.bsz, (int32_t*)nullptr,
                                   b));
                } else {
                    GHB_TRY(scan_exclusive_i32(ws, a.big_d, a.bex, b, a.block_sums));
                    GHB_TRY(scan_exclusive_i32(ws, a.big_d2, a.bsz, b, a.block_sums));
                }
                GHB_TRY(launch(ws, big_scatter_old_kernel, dim3(wide), dim3(256), 0, (const int32_t*)a.big,
                               (const int32_t*)a.big_tail, (const int32_t*)a.bex, (const int32_t*)a.row_id,
                               (const int32_t*)a.row_first, (const int32_t*)a.scrX, (const int32_t*)a.exX,
                               (const uint64_t*)a.skey, (const int8_t*)a.typ, (const int32_t*)a.insX,
                               (const int32_t*)a.delX, (const int64_t*)g->start, (const int32_t*)g->col,
                               (const double*)g->val, scol, sval, (const int64_t*)nullptr, bad_rank));
                if (n_ins > 0)
                    GHB_TRY(launch(ws, big_scatter_new_kernel, dim3(gr), dim3(256), 0, (const uint64_t*)a.skey,
                                   (const uint32_t*)a.sidx, values, (const int8_t*)a.typ, (const int32_t*)a.pos,
                                   (const int32_t*)a.headX, (const int32_t*)a.row_first, (const int32_t*)a.insX,
                                   (const int32_t*)a.delX, (const int32_t*)a.scrX, (const int8_t*)a.big_flag, b, scol,
                                   sval, (const int32_t*)a.row_id, (const int64_t*)nullptr, bad_rank));
                GHB_TRY(launch(ws, big_copy_kernel, dim3(wide), dim3(256), 0, (const int32_t*)a.big,
                               (const int32_t*)a.big_tail, (const int32_t*)a.bsz, (const int32_t*)a.row_id,
                               (const int32_t*)a.scrX, (const int64_t*)a.relX, (const int64_t*)g->start,
                               (const int32_t*)g->cap, base, (const int32_t*)scol, (const double*)sval, g->col, g->val));
                GHB_TRY(launch(ws, big_finalize_kernel, dim3(ws->num_sms), dim3(256), 0, (const int32_t*)a.big,
                               (const int32_t*)a.big_tail, (const int32_t*)a.row_id, (const int32_t*)a.scrX,
                               (const int64_t*)a.relX, base, g->start, g->deg, g->cap, g->moved));
            }
        }
        // Without a repack every row counted in R moved to its new slots.
        if (!repacked) g->used += R;
    }
    GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned + 8, small + 8, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                 ws->stream));
    GHB_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    if (ws->host_pinned[8] != 0) {
        set_error("internal: dynamic-graph row rebuild produced a rank outside its row");
        return GHB_ERR_CUDA;
    }
    g->m += n_ins - n_del;
    totals[0] += n_ins;
    totals[1] += n_del;
    totals[2] += n_modified;
    totals[3] += b - n_ins - n_del - n_modified;
    return GHB_OK;
}

int snapshot(ghb_workspace* ws, ghb_gpma* g, bool weights) {
    if (g->s_ok && (!weights || g->s_val_ok)) return GHB_OK;
    const int32_t n = g->n;
    if (!g->s_rowptr) GHB_TRY(dev_alloc(&g->s_rowptr, (int64_t)n + 1));
    if (g->s_col_cap < std::max<int64_t>(g->m, 1)) {
        dev_free(g->s_col);
        g->s_col_cap = 0;
        const int64_t c = std::max<int64_t>(g->m + g->m / 16, 1);
        GHB_TRY(dev_alloc(&g->s_col, c));
        g->s_col_cap = c;
    }
    if (weights && g->s_val_cap < std::max<int64_t>(g->m, 1)) {
        dev_free(g->s_val);
        g->s_val_cap = 0;
        const int64_t c = std::max<int64_t>(g->m + g->m / 16, 1);
        GHB_TRY(dev_alloc(&g->s_val, c));
        g->s_val_cap = c;
    }
    Carver sizing(nullptr);
    sizing.take<int64_t>(scan_scratch_words((int64_t)n));
    sizing.take<int32_t>((int64_t)n + 1);
    sizing.take<int32_t>((int64_t)n + 1);
    sizing.take<int32_t>(copy_chunk_slots(g->m));
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    int64_t* block_sums = c.take<int64_t>(scan_scratch_words((int64_t)n));
    int32_t* cc = c.take<int32_t>((int64_t)n + 1);
    int32_t* coff = c.take<int32_t>((int64_t)n + 1);
    int32_t* chunk_row = c.take<int32_t>(copy_chunk_slots(g->m));
    GHB_TRY(scan_exclusive_i32(ws, g->deg, g->s_rowptr, n, block_sums));
    GHB_TRY(copy_rows<int32_t>(ws, n, g->start, g->deg, g->col, g->val, g->s_rowptr, g->s_col,
                               weights ? g->s_val : nullptr, cc, coff, chunk_row, block_sums));
    g->s_ok = true;
    g->s_val_ok = weights;
    return GHB_OK;
}

void invalidate(ghb_gpma* g) {
    g->s_ok = false;
    g->s_val_ok = false;
    g->version++;
}

void release(ghb_gpma* g) {
    dev_free(g->start);
    dev_free(g->deg);
    dev_free(g->cap);
    dev_free(g->col);
    dev_free(g->val);
    dev_free(reinterpret_cast<char*&>(g->bbuf));
    dev_free(g->s_rowptr);
    dev_free(g->s_col);
    dev_free(g->s_val);
    dev_free(g->moved);
    dev_free(g->spare_col);
    dev_free(g->spare_val);
    g->spare_slots = 0;
}

// Empty rows, no arena.
int init_empty(ghb_workspace* ws, ghb_gpma* g) {
    const int32_t n = g->n;
    GHB_TRY(dev_alloc(&g->start, n));
    GHB_TRY(dev_alloc(&g->deg, n));
    GHB_TRY(dev_alloc(&g->cap, n));
    GHB_TRY(dev_alloc(&g->moved, 1));
    GHB_CUDA_TRY(cudaMemsetAsync(g->moved, 0, sizeof(unsigned long long), ws->stream));
    GHB_CUDA_TRY(cudaMemsetAsync(g->start, 0, sizeof(int64_t) * (size_t)n, ws->stream));
    GHB_CUDA_TRY(cudaMemsetAsync(g->deg, 0, sizeof(int32_t) * (size_t)n, ws->stream));
    GHB_CUDA_TRY(cudaMemsetAsync(g->cap, 0, sizeof(int32_t) * (size_t)n, ws->stream));
    g->m = g->slots = g->used = 0;
    return GHB_OK;
}

}  // namespace
}  // namespace ghb

using namespace ghb;

extern "C" {

int ghb_gpma_create(ghb_workspace* ws, int32_t n, ghb_gpma** out) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(out, "NULL out");
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    *out = nullptr;
    ghb_gpma* g = new ghb_gpma();
    g->n = n;
    int st = init_empty(ws, g);
    if (st == GHB_OK) {
        cudaError_t e = cudaStreamSynchronize(ws->stream);
        if (e != cudaSuccess) {
            set_error(std::string("ghb_gpma_create: ") + cudaGetErrorString(e));
            st = GHB_ERR_CUDA;
        }
    }
    if (st != GHB_OK) {
        release(g);
        delete g;
        return st;
    }
    *out = g;
    return GHB_OK;
}

int ghb_gpma_destroy(ghb_gpma* g) {
    if (!g) return GHB_OK;
    cudaDeviceSynchronize();
    release(g);
    delete g;
    return GHB_OK;
}

int ghb_gpma_clear(ghb_workspace* ws, ghb_gpma* g) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && g, "NULL workspace / graph");
    GHB_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    dev_free(g->col);
    dev_free(g->val);
    dev_free(g->spare_col);
    dev_free(g->spare_val);
    g->spare_slots = 0;
    GHB_CUDA_TRY(cudaMemsetAsync(g->start, 0, sizeof(int64_t) * (size_t)g->n, ws->stream));
    GHB_CUDA_TRY(cudaMemsetAsync(g->deg, 0, sizeof(int32_t) * (size_t)g->n, ws->stream));
    GHB_CUDA_TRY(cudaMemsetAsync(g->cap, 0, sizeof(int32_t) * (size_t)g->n, ws->stream));
    g->m = g->slots = g->used = 0;
    invalidate(g);
    return GHB_OK;
}

int ghb_gpma_clone(ghb_workspace* ws, const ghb_gpma* src, ghb_gpma** out) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && src && out, "NULL workspace / source / out");
    *out = nullptr;
    ghb_gpma* g = new ghb_gpma();
    g->n = src->n;
    int st = GHB_OK;
    do {
        if ((st = dev_alloc(&g->start, g->n))) break;
        if ((st = dev_alloc(&g->deg, g->n))) break;
        if ((st = dev_alloc(&g->cap, g->n))) break;
        if ((st = dev_alloc(&g->moved, 1))) break;
        if ((st = dev_alloc(&g->col, src->slots))) break;
        if ((st = dev_alloc(&g->val, src->slots))) break;
        const size_t n = (size_t)g->n;
        cudaError_t e = cudaMemcpyAsync(g->start, src->start, sizeof(int64_t) * n, cudaMemcpyDeviceToDevice, ws->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(g->deg, src->deg, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, ws->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(g->cap, src->cap, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, ws->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(g->moved, 0, sizeof(unsigned long long), ws->stream);
        if (e == cudaSuccess && src->used > 0)
            e = cudaMemcpyAsync(g->col, src->col, sizeof(int32_t) * (size_t)src->used, cudaMemcpyDeviceToDevice,
                                ws->stream);
        if (e == cudaSuccess && src->used > 0)
            e = cudaMemcpyAsync(g->val, src->val, sizeof(double) * (size_t)src->used, cudaMemcpyDeviceToDevice,
                                ws->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ws->stream);
        if (e != cudaSuccess) {
            set_error(std::string("ghb_gpma_clone: ") + cudaGetErrorString(e));
            st = GHB_ERR_CUDA;
        }
    } while (false);
    if (st != GHB_OK) {
        release(g);
        delete g;
        return st;
    }
    g->m = src->m;
    g->slots = src->slots;
    g->used = src->used;
    *out = g;
    return GHB_OK;
}

int ghb_gpma_update(ghb_workspace* ws, ghb_gpma* g, const uint64_t* keys, const double* values, int64_t count,
                    int64_t* totals) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && g, "NULL workspace / graph");
    GHB_REQUIRE(count >= 0, "count must be >= 0");
    GHB_REQUIRE(count == 0 || (keys && values), "NULL keys / values");
    int64_t t[4] = {0, 0, 0, 0};
    for (int64_t off = 0; off < count; off += kPassUpdates) {
        const int64_t b = std::min(kPassUpdates, count - off);
        const int st = apply_pass(ws, g, keys + off, values + off, b, t);
        if (st != GHB_OK) {
            // Refused passes change nothing; any other failure may have.
            if (t[0] + t[1] + t[2] > 0 || (st != GHB_ERR_INVALID_ARGUMENT && st != GHB_ERR_LIMIT)) invalidate(g);
            return st;
        }
    }
    if (t[0] + t[1] + t[2] > 0) invalidate(g);
    g->stats[0]++;
    g->stats[1] += t[0];
    g->stats[2] += t[1];
    g->stats[3] += t[2];
    if (totals)
        for (int i = 0; i < 4; ++i) totals[i] = t[i];
    return GHB_OK;
}

int ghb_gpma_load_csr(ghb_workspace* ws, ghb_gpma* g, const int32_t* rowptr, const int32_t* col, const double* w) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && g, "NULL workspace / graph");
    GHB_REQUIRE(rowptr, "NULL rowptr");
    const int32_t n = g->n;
    int32_t ends[2] = {0, 0};
    GHB_CUDA_TRY(cudaMemcpyAsync(&ends[0], rowptr, sizeof(int32_t), cudaMemcpyDeviceToHost, ws->stream));
    GHB_CUDA_TRY(cudaMemcpyAsync(&ends[1], rowptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, ws->stream));
    GHB_CUDA_TRY(cudaStreamSynchronize(ws->stream));
    GHB_REQUIRE(ends[0] == 0 && ends[1] >= 0, "rowptr[0] must be 0 and rowptr[n] >= 0");
    const int64_t m = ends[1];
    GHB_REQUIRE(m == 0 || col, "NULL col");
    unsigned long long* bad = reinterpret_cast<unsigned long long*>(ws->dev_small);
    GHB_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int64_t), ws->stream));
    GHB_TRY(launch(ws, csr_check_kernel, dim3(ws->num_sms * 8), dim3(256), 0, rowptr, col, w, n, m, bad));
    GHB_TRY(ws_read_small(ws, 1));
    GHB_REQUIRE(ws->host_pinned[0] == 0,
                "CSR rows must hold strictly increasing columns in [0, n) with nonzero weights");
    GHB_TRY(ghb_gpma_clear(ws, g));
    if (m == 0) return GHB_OK;
    // The caller's CSR is read as an arena without slack (start = rowptr) and
    // repacked into the graph's own arena with slack.
    GHB_TRY(launch(ws, deg_from_rowptr_kernel, dim3(grid_of(ws, n)), dim3(256), 0, rowptr, n, g->deg));
    int64_t* start64 = nullptr;
    int64_t* want = nullptr;
    double* ones = nullptr;
    int st = dev_alloc(&start64, (int64_t)n + 1);
    if (!st) st = dev_alloc(&want, (int64_t)n + 1);
    if (!st && !w) {
        st = dev_alloc(&ones, m);
        if (!st) st = launch(ws, fill_f64_kernel, dim3(grid_of(ws, m)), dim3(256), 0, ones, m, 1.0);
    }
    if (!st) st = launch(ws, widen_rowptr_kernel, dim3(grid_of(ws, n)), dim3(256), 0, rowptr, n, start64);
    if (!st) st = launch(ws, want_cap_kernel, dim3(grid_of(ws, n)), dim3(256), 0, (const int32_t*)g->deg, n, want);
    if (!st) st = repack(ws, g, start64, col, w ? w : ones, want, m / 8 + 4096, false, m);
    dev_free(start64);
    dev_free(want);
    dev_free(ones);
    GHB_TRY(st);
    g->m = m;
    invalidate(g);
    return GHB_OK;
}

int ghb_gpma_info(const ghb_gpma* g, int32_t* n, int64_t* m, int64_t* slots, int64_t* version) {
    GHB_REQUIRE(g, "NULL graph");
    if (n) *n = g->n;
    if (m) *m = g->m;
    if (slots) *slots = g->slots;
    if (version) *version = g->version;
    return GHB_OK;
}

int ghb_gpma_stats(const ghb_gpma* g, int64_t* stats) {
    GHB_REQUIRE(g && stats, "NULL graph / stats");
    for (int i = 0; i < GHB_GPMA_STATS; ++i) stats[i] = g->stats[i];
    unsigned long long moved = 0;
    GHB_CUDA_TRY(cudaMemcpy(&moved, g->moved, sizeof(moved), cudaMemcpyDeviceToHost));
    stats[4] = (int64_t)moved;
    stats[6] = g->used;
    stats[7] = g->slots;
    return GHB_OK;
}

int ghb_gpma_csr(ghb_workspace* ws, ghb_gpma* g, int32_t weights, const int32_t** rowptr, const int32_t** col,
                 const double** w) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && g, "NULL workspace / graph");
    GHB_REQUIRE(rowptr && col, "NULL rowptr / col");
    GHB_TRY(snapshot(ws, g, weights != 0));
    *rowptr = g->s_rowptr;
    *col = g->s_col;
    if (w) *w = weights ? g->s_val : nullptr;
    return GHB_OK;
}

int ghb_gpma_export(ghb_workspace* ws, ghb_gpma* g, int32_t* rowptr, int32_t* col, double* w) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && g, "NULL workspace / graph");
    GHB_REQUIRE(rowptr && (g->m == 0 || col), "NULL rowptr / col");
    GHB_TRY(snapshot(ws, g, w != nullptr));
    GHB_CUDA_TRY(cudaMemcpyAsync(rowptr, g->s_rowptr, sizeof(int32_t) * ((size_t)g->n + 1),
                                 cudaMemcpyDeviceToDevice, ws->stream));
    if (g->m > 0) {
        GHB_CUDA_TRY(cudaMemcpyAsync(col, g->s_col, sizeof(int32_t) * (size_t)g->m, cudaMemcpyDeviceToDevice,
                                     ws->stream));
        if (w)
            GHB_CUDA_TRY(cudaMemcpyAsync(w, g->s_val, sizeof(double) * (size_t)g->m, cudaMemcpyDeviceToDevice,
                                         ws->stream));
    }
    return GHB_OK;
}

int ghb_gpma_find(ghb_workspace* ws, const ghb_gpma* g, const uint64_t* keys, int64_t count, double* values) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws && g, "NULL workspace / graph");
    GHB_REQUIRE(count >= 0 && (count == 0 || (keys && values)), "NULL keys / values");
    if (count == 0) return GHB_OK;
    unsigned long long* bad = reinterpret_cast<unsigned long long*>(ws->dev_small);
    GHB_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int64_t), ws->stream));
    GHB_TRY(launch(ws, find_kernel, dim3(grid_of(ws, count)), dim3(256), 0, (const int64_t*)g->start,
                   (const int32_t*)g->deg, (const int32_t*)g->col, (const double*)g->val, g->n, keys, count, values,
                   bad));
    GHB_TRY(ws_read_small(ws, 1));
    GHB_REQUIRE(ws->host_pinned[0] == 0, "lookup key with a row or column outside [0, n)");
    return GHB_OK;
}

}  // extern "C"
