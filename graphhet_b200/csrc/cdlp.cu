// Community detection by synchronous label propagation (replaces
// GPU_CDLP_csr.cuh:28-210, which gathers every row's labels into an E-length
// array and segment-sorts all E keys each iteration).  Semantics of the CPU
// path (CPU_Community_Detection.hpp:12-64): the new label of v is the most
// frequent label among its row's entries, the smallest such label on ties; a
// vertex with an empty row keeps its label.  Labels start as vertex ids.
//
// Rows are classed by length once per call and each class has its own
// kernel, so no row pays for another's size:
//   0        keep the label
//   1..32    W lanes per row (W = 2..32): bitonic sort of the W labels in
//            registers through shuffles, run lengths by ballot
//   33..256  one warp per row, open-addressing (label -> count) table of 512
//            slots in shared memory
//   257..1024 one block per row, 2048-slot shared-memory table (16 KB, so
//            eight blocks fit an SM)
//   1025..2048 one block per row, 4096-slot shared-memory table (32 KB)
//   2049..4096 one block per row, 8192-slot shared-memory table
//   > 4096   the row is cut into chunks of 2048 entries, each a block: the
//            chunk counts its labels in a shared-memory table, then adds each
//            distinct (label, count) to the row's table in global scratch and
//            lists the slots it claimed; the last chunk of a row to finish
//            writes its label, and a write-only pass empties the claimed
//            slots.  No row waits on one block, and once labels converge a
//            chunk sends a few global atomics, not 2048.
// Every insert returns the key (count after it, -label); a label's last insert
// sees its final count, so the max-reduction of those keys yields the most
// frequent label with the smallest-label tie-break, and no table is scanned
// for it.
#include <algorithm>
#include <type_traits>
#include <vector>

#include "common.cuh"

namespace ghb {
namespace {

// 0:empty 1..5: W=2,4,8,16,32  6:warp 7:block (2048 slots) 8:block (4096 slots)
// 9:block (8192 slots) 10:chunked
constexpr int kCdlpClasses = 11;
constexpr int kSumLongSlot = 15;  // counts[15]: entries of the chunked-class rows
constexpr int32_t kEmpty = -1;
constexpr int32_t kWarpSlots = 512;
constexpr int32_t kSmallBlockSlots = 2048;
constexpr int32_t kMidBlockSlots = 4096;
constexpr int32_t kBlockSlots = 8192;
constexpr int32_t kLongRow = kBlockSlots / 2;  // longer rows are chunked
constexpr int32_t kChunk = 2048;               // entries per chunk of a chunked-class row
constexpr int32_t kChunkSlots = 2 * kChunk;    // its shared-memory table (32 KB)
constexpr int kCdlpThreads = 256;

__device__ __forceinline__ int cdlp_class(int32_t d) {
    if (d == 0) return 0;
    if (d <= 2) return 1;
    if (d <= 4) return 2;
    if (d <= 8) return 3;
    if (d <= 16) return 4;
    if (d <= 32) return 5;
    if (d <= 256) return 6;
    if (d <= 1024) return 7;
    if (d <= 2048) return 8;
    if (d <= kLongRow) return 9;
    return 10;
}

// Slots of a chunked-class row's global table: the power of two >= 2 d.
__host__ __device__ __forceinline__ uint32_t global_cap(int32_t d) {
    uint32_t c = 1;
    while (c < 2u * (uint32_t)d) c <<= 1;
    return c;
}

__device__ __forceinline__ uint32_t hash_label(int32_t x) {
    uint32_t h = (uint32_t)x * 0x9E3779B1u;
    return h ^ (h >> 16);
}

// Packs (count, label) so that a larger key = more frequent, then smaller label.
__device__ __forceinline__ unsigned long long pack_best(uint32_t count, int32_t label) {
    return ((unsigned long long)count << 32) | (unsigned long long)(0x7FFFFFFFu - (uint32_t)label);
}
__device__ __forceinline__ int32_t unpack_label(unsigned long long k) {
    return (int32_t)(0x7FFFFFFFu - (uint32_t)(k & 0xFFFFFFFFull));
}

// Insert label x (valid lanes) into an open-addressing table of `slots`
// (power of two) entries, K = labels, C = counts.  Lanes of the warp holding
// the same label are merged first (one atomic per distinct label per warp),
// which matters once labels converge and a hub's row repeats a few labels.
// Every lane of the warp must call it.  Returns, on the lane that inserted for
// its group, the key (count after this insert, label), else 0.  A label's
// count only grows and its last insert sees the final count, so the largest
// key returned over a row names its most frequent label (smallest on ties)
// without a scan of the table.
__device__ __forceinline__ unsigned long long table_insert_merged(int32_t* K, int32_t* C, uint32_t slots, int32_t x,
                                                                  bool valid) {
    const unsigned act = __ballot_sync(0xffffffffu, valid);
    if (!valid) return 0;
    const unsigned same = __match_any_sync(act, x);
    if (lane_id() != __ffs(same) - 1) return 0;
    uint32_t h = hash_label(x) & (slots - 1);
    while (true) {
        const int32_t k = atomicCAS(&K[h], kEmpty, x);
        if (k == kEmpty || k == x) {
            const int32_t c = atomicAdd(&C[h], __popc(same)) + __popc(same);
            return pack_best((uint32_t)c, x);
        }
        h = (h + 1) & (slots - 1);
    }
}

// Inserts the row entries [j0, e) taken R rounds at a time, entry
// j0 + r * stride + t on thread t of round r: the R column loads issue
// before the R label gathers and those before the inserts, so a thread has R
// loads in flight instead of a chain of R round trips.  Every lane of the
// warp must call it (rounds past e are skipped warp-uniformly).  Returns the
// largest key the inserts returned.
template <int R>
__device__ __forceinline__ unsigned long long insert_rows(int32_t* K, int32_t* C, uint32_t slots,
                                                          const int32_t* __restrict__ col,
                                                          const int32_t* __restrict__ lab, int32_t b, int32_t e,
                                                          int stride, int t) {
    unsigned long long best = 0;
    for (int64_t j0 = b; j0 < e; j0 += (int64_t)R * stride) {
        int32_t x[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int64_t j = j0 + (int64_t)r * stride + t;
            x[r] = j < e ? col[j] : -1;
        }
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = x[r] >= 0 ? lab[x[r]] : 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int64_t jr = j0 + (int64_t)r * stride;
            if (jr < e) {
                const unsigned long long key = table_insert_merged(K, C, slots, x[r], jr + t < e);
                best = key > best ? key : best;
            }
        }
    }
    return best;
}

__global__ void cdlp_count_classes_kernel(int32_t n, const int32_t* __restrict__ rp, int32_t* counts) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = rp[v + 1] - rp[v];
        const int c = cdlp_class(d);
        const unsigned same = __match_any_sync(__activemask(), c);
        const int leader = __ffs(same) - 1;
        if (lane_id() == leader) atomicAdd(&counts[c], __popc(same));
        if (c == 10) atomicAdd(&counts[kSumLongSlot], d);
    }
}

// Class lists hold each row as {v, begin, end, 0}: a row kernel reads its
// row's bounds with the row itself, one load instead of two dependent ones.
__global__ void cdlp_fill_classes_kernel(int32_t n, const int32_t* __restrict__ rp, int32_t* cursor,
                                         int4* rows) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = rp[v], e = rp[v + 1];
        const int c = cdlp_class(e - b);
        const unsigned active = __activemask();
        const unsigned same = __match_any_sync(active, c);
        const int leader = __ffs(same) - 1;
        int32_t base = 0;
        if (lane_id() == leader) base = atomicAdd(&cursor[c], __popc(same));
        base = __shfl_sync(same, base, leader);
        rows[base + __popc(same & ((1u << lane_id()) - 1u))] = make_int4((int32_t)v, b, e, 0);
    }
}

__global__ void cdlp_iota_kernel(int32_t* p, int32_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = (int32_t)i;
}

__global__ void cdlp_copy_kernel(const int4* __restrict__ rows, int32_t count,
                                 const int32_t* __restrict__ lab, int32_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = rows[i].x;
        out[v] = lab[v];
    }
}

// W lanes per row, rows of 1..W entries.  kMin: every label of a row is
// distinct (first iteration), so the row's smallest label is taken directly.
template <int W, bool kMin>
__global__ void __launch_bounds__(kCdlpThreads) cdlp_small_kernel(
    const int4* __restrict__ rows, int32_t count, const int32_t* __restrict__ col,
    const int32_t* __restrict__ lab, int32_t* __restrict__ out) {
    const int lane = lane_id();
    const int li = lane & (W - 1);
    const int64_t group = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / W;
    const int64_t ngroups = ((int64_t)gridDim.x * blockDim.x) / W;
    const int64_t rounds = ((int64_t)count + ngroups - 1) / ngroups;
    const unsigned gmask = (W == 32) ? 0xffffffffu : (((1u << W) - 1u) << (lane & ~(W - 1)));
    for (int64_t r = 0; r < rounds; ++r) {
        const int64_t i = group + r * ngroups;
        int32_t v = -1, b = 0, d = 0;
        if (i < count) {
            const int4 ri = rows[i];
            v = ri.x;
            b = ri.y;
            d = ri.z - ri.y;
        }
        int32_t x = 0x7FFFFFFF;
        if (li < d) x = lab[col[b + li]];
        if constexpr (kMin) {
#pragma unroll
            for (int o = W / 2; o > 0; o >>= 1) x = min(x, __shfl_xor_sync(0xffffffffu, x, o));
            if (li == 0 && i < count) out[v] = x;
        } else {
            // Bitonic sort, ascending, within each W-lane group.
#pragma unroll
            for (int k = 2; k <= W; k <<= 1) {
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const int32_t y = __shfl_xor_sync(0xffffffffu, x, j);
                    const bool up = (li & k) == 0;
                    const bool lower = (li & j) == 0;
                    x = (lower == up) ? min(x, y) : max(x, y);
                }
            }
            // Run starts inside the group, then run length = next start - start.
            const int32_t prev = __shfl_up_sync(0xffffffffu, x, 1);
            const bool valid = li < d;
            const bool start = valid && (li == 0 || prev != x);
            const unsigned starts = __ballot_sync(0xffffffffu, start) & gmask;
            unsigned long long best = 0;
            if (start) {
                const unsigned above = starts & ~((2u << lane) - 1u);
                const int next_li = above ? ((__ffs(above) - 1) & (W - 1)) : d;
                best = pack_best((uint32_t)(next_li - li), x);
            }
#pragma unroll
            for (int o = W / 2; o > 0; o >>= 1) {
                const unsigned long long y = __shfl_xor_sync(0xffffffffu, best, o);
                best = y > best ? y : best;
            }
            if (li == 0 && i < count) out[v] = unpack_label(best);
        }
    }
}

// One warp per row of 33..256 entries, 512-slot table per warp in shared
// memory (kMin: the row's smallest label, no table).
template <bool kMin>
__global__ void __launch_bounds__(kCdlpThreads) cdlp_warp_kernel(
    const int4* __restrict__ rows, int32_t count, const int32_t* __restrict__ col,
    const int32_t* __restrict__ lab, int32_t* __restrict__ out) {
    __shared__ int32_t keys[kCdlpThreads / 32][kWarpSlots];
    __shared__ int32_t cnts[kCdlpThreads / 32][kWarpSlots];
    const int lane = lane_id();
    const int wib = threadIdx.x >> 5;
    int32_t* K = keys[wib];
    int32_t* C = cnts[wib];
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < count; i += nwarps) {
        const int4 ri = rows[i];
        const int32_t v = ri.x, b = ri.y, e = ri.z;
        if (kMin) {
            int32_t m = 0x7FFFFFFF;
            for (int32_t j = b + lane; j < e; j += 32) m = min(m, lab[col[j]]);
            m = __reduce_min_sync(0xffffffffu, m);
            if (lane == 0) out[v] = m;
            continue;
        }
        // Table of the power of two >= 2 x the row (64..512 slots): clearing
        // it costs no more than the row's own inserts.
        uint32_t cap = 64;
        while (cap < 2u * (uint32_t)(e - b)) cap <<= 1;
        for (uint32_t s = lane; s < cap; s += 32) {
            K[s] = kEmpty;
            C[s] = 0;
        }
        __syncwarp();
        unsigned long long best = insert_rows<8>(K, C, cap, col, lab, b, e, 32, lane);
        best = warp_max(best);
        if (lane == 0) out[v] = unpack_label(best);
        __syncwarp();
    }
}

__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long x, unsigned long long* red) {
    x = warp_max(x);
    if (lane_id() == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned long long y = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0ull;
        y = warp_max(y);
        if (threadIdx.x == 0) red[0] = y;
    }
    __syncthreads();
    const unsigned long long r = red[0];
    __syncthreads();
    return r;
}

// One block per row of up to `slots` / 2 entries (classes 7 and 8); the table
// (the power of two >= 2 x the row, at least 512 slots) lives in 2 x slots
// ints of dynamic shared memory.  kMin: the row's smallest label, no table.
template <bool kMin>
__global__ void __launch_bounds__(kCdlpThreads) cdlp_block_kernel(
    const int4* __restrict__ rows, int32_t count, const int32_t* __restrict__ col,
    const int32_t* __restrict__ lab, int32_t* __restrict__ out, uint32_t slots) {
    extern __shared__ int32_t smem[];
    __shared__ unsigned long long red[32];
    int32_t* K = smem;
    int32_t* C = smem + slots;
    for (int64_t i = blockIdx.x; i < count; i += gridDim.x) {
        const int4 ri = rows[i];
        const int32_t v = ri.x, b = ri.y, e = ri.z;
        if (kMin) {
            unsigned long long m = 0;
            for (int32_t j = b + threadIdx.x; j < e; j += blockDim.x) {
                const unsigned long long key = pack_best(1, lab[col[j]]);
                m = key > m ? key : m;
            }
            m = block_max_u64(m, red);
            if (threadIdx.x == 0) out[v] = unpack_label(m);
            continue;
        }
        uint32_t cap = 512;
        while (cap < 2u * (uint32_t)(e - b) && cap < slots) cap <<= 1;
        for (uint32_t s = threadIdx.x; s < cap; s += blockDim.x) {
            K[s] = kEmpty;
            C[s] = 0;
        }
        __syncthreads();
        unsigned long long best = insert_rows<4>(K, C, cap, col, lab, b, e, blockDim.x, threadIdx.x);
        // Also orders this row's inserts before the next row's clearing.
        best = block_max_u64(best, red);
        if (threadIdx.x == 0) out[v] = unpack_label(best);
    }
}

// Global tables hold slot h as one word, label << 32 | count, empty =
// kSlotEmpty (label kEmpty, count 0): a probe, its count and the later read
// touch one 8-byte word, and a count is added with one 64-bit atomic that
// cannot carry into the label (counts stay below 2^31).
constexpr unsigned long long kSlotEmpty = 0xFFFFFFFF00000000ull;

// Adds cnt to label x in a table of cap slots (cap > 2 x the labels it can
// hold, so a free slot is always reached), probing from slot h.  Sets key to
// (count after this add, label), as table_insert_merged returns it, and
// returns the slot when this call claimed it for x, else -1.
__device__ __forceinline__ int32_t global_add_from(unsigned long long* T, uint32_t cap, uint32_t h, int32_t x,
                                                   int32_t cnt, unsigned long long& key) {
    const unsigned long long mine = ((unsigned long long)(uint32_t)x << 32) | (uint32_t)cnt;
    while (true) {
        const unsigned long long cur = atomicCAS(T + h, kSlotEmpty, mine);
        if (cur == kSlotEmpty) {
            key = pack_best((uint32_t)cnt, x);
            return (int32_t)h;
        }
        if ((uint32_t)(cur >> 32) == (uint32_t)x) {
            const unsigned long long old = atomicAdd(T + h, (unsigned long long)cnt);
            key = pack_best((uint32_t)old + (uint32_t)cnt, x);
            return -1;
        }
        h = (h + 1) & (cap - 1);
    }
}

// Chunked-class row i owns pool[tab_off[i] ...] (tab_off even): cap slot
// words, then the list of claimed slots (up to d).  chunks[2k], chunks[2k+1]
// = row index i and the chunk's first entry within the row (a multiple of
// kChunk).
struct LongRow {
    int32_t v, b, d;
    uint32_t cap;
    unsigned long long* T;
    int32_t* L;
};
__device__ __forceinline__ LongRow long_row(const int4* rows, int32_t* pool,
                                            const int64_t* tab_off, int32_t i) {
    LongRow r;
    const int4 ri = rows[i];
    r.v = ri.x;
    r.b = ri.y;
    r.d = ri.z - ri.y;
    r.cap = global_cap(r.d);
    r.T = reinterpret_cast<unsigned long long*>(pool + tab_off[i]);
    r.L = reinterpret_cast<int32_t*>(r.T + r.cap);
    return r;
}

// Called by thread 0 of a block that has finished its chunk of row i with the
// chunk's best (count, -label) key: folds it into best[i]; the row's last
// chunk writes the label and resets done[i] and best[i].
__device__ __forceinline__ void chunk_done(const LongRow& r, int32_t i, unsigned long long b, int32_t* done,
                                           unsigned long long* best, int32_t* out) {
    if (b) atomicMax(best + i, b);
    __threadfence();
    const int32_t nchunks = (r.d + kChunk - 1) / kChunk;
    if (atomicAdd(done + i, 1) == nchunks - 1) {
        __threadfence();
        out[r.v] = unpack_label(atomicExch(best + i, 0ull));
        done[i] = 0;
    }
}

// One iteration of a chunked-class row, per chunk: count the chunk's labels
// in shared memory, then add each distinct (label, count) to the row's
// global table, keeping the largest key the adds return (the row's answer once
// every chunk has added, as in table_insert_merged).  Slots claimed here are
// appended to the row's list (one atomic per warp on occ[i]) for the reset
// pass.
__global__ void __launch_bounds__(kCdlpThreads) cdlp_chunk_count_kernel(
    const int4* __restrict__ rows, const int32_t* __restrict__ col,
    const int32_t* __restrict__ lab, const int32_t* __restrict__ chunks, int32_t nch, int32_t* pool,
    const int64_t* __restrict__ tab_off, int32_t* occ, int32_t* done, unsigned long long* best,
    int32_t* __restrict__ out) {
    extern __shared__ int32_t smem[];
    __shared__ unsigned long long red[32];
    int32_t* K = smem;
    int32_t* C = smem + kChunkSlots;
    for (int64_t k = blockIdx.x; k < nch; k += gridDim.x) {
        const int32_t i = chunks[2 * k];
        const LongRow r = long_row(rows, pool, tab_off, i);
        const int32_t b = r.b + chunks[2 * k + 1];
        const int32_t e = (int32_t)min((int64_t)b + kChunk, (int64_t)r.b + r.d);
        uint32_t cap = 512;
        while (cap < 2u * (uint32_t)(e - b) && cap < (uint32_t)kChunkSlots) cap <<= 1;
        for (uint32_t s = threadIdx.x; s < cap; s += blockDim.x) {
            K[s] = kEmpty;
            C[s] = 0;
        }
        __syncthreads();
        insert_rows<4>(K, C, cap, col, lab, b, e, blockDim.x, threadIdx.x);
        __syncthreads();
        // The chunk's distinct labels go to the global table kF per thread at
        // a time: the kF home-slot CASes issue together, then the adds for
        // labels found there, and only a slot held by another label is probed
        // one step at a time.  cap is a multiple of the block size: every
        // warp runs every round.
        constexpr int kF = 4;
        unsigned long long mx = 0;
        for (uint32_t s0 = 0; s0 < cap; s0 += kF * blockDim.x) {
            int32_t x[kF], c[kF];
            uint32_t h[kF];
            unsigned long long cur[kF], old[kF];
#pragma unroll
            for (int q = 0; q < kF; ++q) {
                const uint32_t s = s0 + q * blockDim.x + threadIdx.x;
                x[q] = s < cap ? K[s] : kEmpty;
                c[q] = s < cap ? C[s] : 0;
                h[q] = hash_label(x[q]) & (r.cap - 1);
                cur[q] = x[q] != kEmpty ? atomicCAS(r.T + h[q], kSlotEmpty,
                                                    ((unsigned long long)(uint32_t)x[q] << 32) | (uint32_t)c[q])
                                        : kSlotEmpty;
            }
#pragma unroll
            for (int q = 0; q < kF; ++q) {
                old[q] = 0;
                if (x[q] != kEmpty && cur[q] != kSlotEmpty && (uint32_t)(cur[q] >> 32) == (uint32_t)x[q])
                    old[q] = atomicAdd(r.T + h[q], (unsigned long long)c[q]);
            }
#pragma unroll
            for (int q = 0; q < kF; ++q) {
                if (s0 + q * blockDim.x >= cap) break;
                int32_t claimed = -1;
                unsigned long long key = 0;
                if (x[q] != kEmpty) {
                    if (cur[q] == kSlotEmpty) {
                        claimed = (int32_t)h[q];
                        key = pack_best((uint32_t)c[q], x[q]);
                    } else if ((uint32_t)(cur[q] >> 32) == (uint32_t)x[q]) {
                        key = pack_best((uint32_t)old[q] + (uint32_t)c[q], x[q]);
                    } else {
                        claimed = global_add_from(r.T, r.cap, (h[q] + 1) & (r.cap - 1), x[q], c[q], key);
                    }
                }
                mx = key > mx ? key : mx;
                const unsigned m = __ballot_sync(0xffffffffu, claimed >= 0);
                if (m) {
                    int32_t base = 0;
                    if (lane_id() == 0) base = atomicAdd(occ + i, __popc(m));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if (claimed >= 0) r.L[base + __popc(m & ((1u << lane_id()) - 1u))] = claimed;
                }
            }
        }
        // Also orders this chunk's table reads before the next chunk's clearing.
        mx = block_max_u64(mx, red);
        if (threadIdx.x == 0) chunk_done(r, i, mx, done, best, out);
    }
}

// After the count pass: empties the slots the pass claimed, by writes only.
// A sparse table (at most cap / 8 claims, the usual case once labels
// converge) is reset through its claim list, chunk k taking list entries
// [j0, j0 + kChunk); a dense one in slot order, chunk k taking the k-th share
// of the slots.  The row's last chunk resets occ[i] and done[i].
__global__ void __launch_bounds__(kCdlpThreads) cdlp_chunk_reset_kernel(
    const int4* __restrict__ rows, const int32_t* __restrict__ chunks,
    int32_t nch, int32_t* pool, const int64_t* __restrict__ tab_off, int32_t* occ, int32_t* done) {
    for (int64_t k = blockIdx.x; k < nch; k += gridDim.x) {
        const int32_t i = chunks[2 * k];
        const LongRow r = long_row(rows, pool, tab_off, i);
        const int32_t j0 = chunks[2 * k + 1];
        const int32_t claims = __ldcg(occ + i);
        const uint32_t nchunks = (uint32_t)(r.d + kChunk - 1) / kChunk;
        if ((uint32_t)claims > r.cap / 8) {
            const uint32_t per = (r.cap + nchunks - 1) / nchunks;
            const uint32_t s0 = (uint32_t)(j0 / kChunk) * per;
            const uint32_t s1 = min(s0 + per, r.cap);
            for (uint32_t s = s0 + threadIdx.x; s < s1; s += blockDim.x) r.T[s] = kSlotEmpty;
        } else {
            const int32_t j1 = (int32_t)min((int64_t)j0 + kChunk, (int64_t)claims);
            for (int32_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) r.T[__ldcg(r.L + j)] = kSlotEmpty;
        }
        __syncthreads();  // every thread has read occ[i] before it can be reset
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicAdd(done + i, 1) == (int32_t)nchunks - 1) {
                occ[i] = 0;
                done[i] = 0;
            }
        }
    }
}

// First iteration (labels distinct, no repeated entries): each chunk's
// smallest label, folded over the row's chunks as in the pick pass.
__global__ void __launch_bounds__(kCdlpThreads) cdlp_chunk_min_kernel(
    const int4* __restrict__ rows, const int32_t* __restrict__ col,
    const int32_t* __restrict__ lab, const int32_t* __restrict__ chunks, int32_t nch, int32_t* pool,
    const int64_t* __restrict__ tab_off, int32_t* done, unsigned long long* best, int32_t* __restrict__ out) {
    __shared__ unsigned long long red[32];
    for (int64_t k = blockIdx.x; k < nch; k += gridDim.x) {
        const int32_t i = chunks[2 * k];
        const LongRow r = long_row(rows, pool, tab_off, i);
        const int32_t b = r.b + chunks[2 * k + 1];
        const int32_t e = (int32_t)min((int64_t)b + kChunk, (int64_t)r.b + r.d);
        unsigned long long m = 0;
        for (int32_t j = b + threadIdx.x; j < e; j += blockDim.x) {
            const unsigned long long key = pack_best(1, lab[col[j]]);
            m = key > m ? key : m;
        }
        m = block_max_u64(m, red);
        if (threadIdx.x == 0) chunk_done(r, i, m, done, best, out);
    }
}

// Chunked-class rows: degrees for the host's table layout.
__global__ void cdlp_long_degrees_kernel(const int4* __restrict__ rows, int32_t count, int32_t* deg) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        deg[i] = rows[i].z - rows[i].y;
    }
}

// Block per chunked-class row: every slot empty.
__global__ void cdlp_pool_clear_kernel(const int4* __restrict__ rows, int32_t count, int32_t* pool,
                                       const int64_t* __restrict__ tab_off) {
    for (int64_t i = blockIdx.x; i < count; i += gridDim.x) {
        const LongRow r = long_row(rows, pool, tab_off, (int32_t)i);
        for (uint32_t s = threadIdx.x; s < r.cap; s += blockDim.x) r.T[s] = kSlotEmpty;
    }
}

}  // namespace

// init_labels (device, may be NULL = vertex ids): starting label values.
// first_min: the rows repeat no entry and the starting labels are distinct,
// so the first iteration is a minimum over each row's labels.
int cdlp_run(ghb_workspace* ws, int32_t n, const int32_t* rp, const int32_t* col, int32_t iterations,
             int32_t* labels, const int32_t* init_labels, bool first_min) {
    cudaStream_t st = ws->stream;
    int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned);

    // Pass 1: class sizes.
    Carver pre(nullptr);
    pre.take<int32_t>(16);
    GHB_TRY(ws_reserve(ws, pre.off + (size_t)n * 4 * 3 + 4096));
    int32_t* counts = reinterpret_cast<int32_t*>(ws->scratch);
    GHB_CUDA_TRY(cudaMemsetAsync(counts, 0, 16 * sizeof(int32_t), st));
    GHB_TRY(launch(ws, cdlp_count_classes_kernel, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0, n,
                   rp, counts));
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, counts, 16 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    int32_t cls[kCdlpClasses], off[kCdlpClasses + 1];
    off[0] = 0;
    for (int k = 0; k < kCdlpClasses; ++k) {
        cls[k] = hp[k];
        off[k + 1] = off[k] + cls[k];
    }
    // Chunked-class tables: (label, count) pairs for the power of two >= 2 d
    // slots, then the claimed-slot list of d ints (rounded up to even), so
    // fewer than 9 ints per entry plus one per row.
    const int32_t nlong = cls[10];
    const int64_t long_entries = hp[kSumLongSlot];
    const int64_t pool_bound = nlong > 0 ? 9 * long_entries + nlong + 16 : 1;
    const int64_t chunk_bound = long_entries / kChunk + nlong + 1;
    Carver sizing(nullptr);
    sizing.take<int32_t>(16);
    sizing.take<int32_t>(16);
    sizing.take<int4>(n);
    sizing.take<int32_t>(n);
    sizing.take<int32_t>(pool_bound);
    sizing.take<int64_t>((size_t)nlong + 1);
    sizing.take<int32_t>(2 * chunk_bound);
    sizing.take<int32_t>((size_t)nlong + 1);
    sizing.take<int32_t>((size_t)nlong + 1);
    sizing.take<unsigned long long>((size_t)nlong + 1);
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    counts = c.take<int32_t>(16);
    int32_t* cursor = c.take<int32_t>(16);
    int4* rows = c.take<int4>(n);
    int32_t* other = c.take<int32_t>(n);
    int32_t* pool = c.take<int32_t>(pool_bound);
    int64_t* tab_off = c.take<int64_t>((size_t)nlong + 1);
    int32_t* chunks = c.take<int32_t>(2 * chunk_bound);
    int32_t* occ = c.take<int32_t>((size_t)nlong + 1);
    int32_t* done = c.take<int32_t>((size_t)nlong + 1);
    unsigned long long* best = c.take<unsigned long long>((size_t)nlong + 1);

    for (int k = 0; k < kCdlpClasses; ++k) hp[k] = off[k];
    GHB_CUDA_TRY(cudaMemcpyAsync(cursor, hp, kCdlpClasses * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    GHB_TRY(launch(ws, cdlp_fill_classes_kernel, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0, n, rp,
                   cursor, rows));
    const int4* long_rows = rows + off[10];
    int32_t nch = 0;
    if (nlong > 0) {
        // Table offsets and the chunk list on the host (a few thousand rows),
        // then empty tables and zero counters.
        GHB_TRY(launch(ws, cdlp_long_degrees_kernel, dim3(grid_for(nlong, 256, ws->num_sms)), dim3(256), 0,
                       long_rows, nlong, occ));
        std::vector<int32_t> deg((size_t)nlong);
        GHB_CUDA_TRY(cudaMemcpyAsync(deg.data(), occ, sizeof(int32_t) * nlong, cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        std::vector<int64_t> toff((size_t)nlong + 1);
        std::vector<int32_t> ch;
        ch.reserve(2 * (size_t)chunk_bound);
        int64_t acc = 0;
        for (int32_t i = 0; i < nlong; ++i) {
            // global_cap needs 2 d <= 2^31.
            GHB_REQUIRE(deg[i] <= (1 << 30), "CDLP: a row holds more than 2^30 entries");
            toff[i] = acc;
            acc += 2 * (int64_t)global_cap(deg[i]) + ((deg[i] + 1) & ~1);  // keeps every tab_off even
            for (int64_t j = 0; j < deg[i]; j += kChunk) {
                ch.push_back(i);
                ch.push_back((int32_t)j);
            }
        }
        toff[nlong] = acc;
        nch = (int32_t)(ch.size() / 2);
        GHB_REQUIRE(acc <= pool_bound && nch <= chunk_bound, "CDLP table pool bound");
        GHB_CUDA_TRY(cudaMemcpyAsync(tab_off, toff.data(), sizeof(int64_t) * (nlong + 1), cudaMemcpyHostToDevice, st));
        GHB_CUDA_TRY(cudaMemcpyAsync(chunks, ch.data(), sizeof(int32_t) * ch.size(), cudaMemcpyHostToDevice, st));
        GHB_CUDA_TRY(cudaMemsetAsync(occ, 0, sizeof(int32_t) * nlong, st));
        GHB_CUDA_TRY(cudaMemsetAsync(done, 0, sizeof(int32_t) * nlong, st));
        GHB_CUDA_TRY(cudaMemsetAsync(best, 0, sizeof(unsigned long long) * nlong, st));
        GHB_TRY(launch(ws, cdlp_pool_clear_kernel, dim3(grid_for(nlong, 1, ws->num_sms * 8)), dim3(256), 0, long_rows,
                       nlong, pool, (const int64_t*)tab_off));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));  // toff and ch are read by the copies above
    }
    if (init_labels)
        GHB_CUDA_TRY(cudaMemcpyAsync(labels, init_labels, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
    else
        GHB_TRY(launch(ws, cdlp_iota_kernel, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0, labels, n));

    // Shared-memory classes: as many blocks as fit each SM.
    const size_t small_smem = 2 * kSmallBlockSlots * sizeof(int32_t), big_smem = 2 * kBlockSlots * sizeof(int32_t);
    const size_t chunk_smem = 2 * kChunkSlots * sizeof(int32_t), mid_smem = 2 * kMidBlockSlots * sizeof(int32_t);
    GHB_CUDA_TRY(cudaFuncSetAttribute(cdlp_block_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)big_smem));
    GHB_CUDA_TRY(cudaFuncSetAttribute(cdlp_chunk_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)chunk_smem));
    int per_sm_small = 0, per_sm_mid = 0, per_sm_big = 0, per_sm_chunk = 0;
    GHB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_small, cdlp_block_kernel<false>, kCdlpThreads,
                                                               small_smem));
    GHB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_mid, cdlp_block_kernel<false>, kCdlpThreads,
                                                               mid_smem));
    GHB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_big, cdlp_block_kernel<false>, kCdlpThreads,
                                                               big_smem));
    GHB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_chunk, cdlp_chunk_count_kernel, kCdlpThreads,
                                                               chunk_smem));
    const unsigned g_small = ws->num_sms * std::max(1, per_sm_small);
    const unsigned g_mid = ws->num_sms * std::max(1, per_sm_mid);
    const unsigned g_big = ws->num_sms * std::max(1, per_sm_big);
    const unsigned g_chunk = ws->num_sms * std::max(1, per_sm_chunk);
    const unsigned g = ws->num_sms * 8;

    // One iteration: every class reads cur and writes nxt.  kMin (first
    // iteration over distinct labels): each row's smallest label.
    auto iteration = [&](auto min_tag, const int32_t* cur, int32_t* nxt) -> int {
        constexpr bool M = decltype(min_tag)::value;
        const int4* R = rows;
        if (cls[0]) GHB_TRY(launch(ws, cdlp_copy_kernel, dim3(grid_for(cls[0], 256, g)), dim3(256), 0, R + off[0], cls[0], cur, nxt));
        if (cls[1]) GHB_TRY(launch(ws, cdlp_small_kernel<2, M>, dim3(grid_for((int64_t)cls[1] * 2, kCdlpThreads, g)), dim3(kCdlpThreads), 0, R + off[1], cls[1], col, cur, nxt));
        if (cls[2]) GHB_TRY(launch(ws, cdlp_small_kernel<4, M>, dim3(grid_for((int64_t)cls[2] * 4, kCdlpThreads, g)), dim3(kCdlpThreads), 0, R + off[2], cls[2], col, cur, nxt));
        if (cls[3]) GHB_TRY(launch(ws, cdlp_small_kernel<8, M>, dim3(grid_for((int64_t)cls[3] * 8, kCdlpThreads, g)), dim3(kCdlpThreads), 0, R + off[3], cls[3], col, cur, nxt));
        if (cls[4]) GHB_TRY(launch(ws, cdlp_small_kernel<16, M>, dim3(grid_for((int64_t)cls[4] * 16, kCdlpThreads, g)), dim3(kCdlpThreads), 0, R + off[4], cls[4], col, cur, nxt));
        if (cls[5]) GHB_TRY(launch(ws, cdlp_small_kernel<32, M>, dim3(grid_for((int64_t)cls[5] * 32, kCdlpThreads, g)), dim3(kCdlpThreads), 0, R + off[5], cls[5], col, cur, nxt));
        if (cls[6]) GHB_TRY(launch(ws, cdlp_warp_kernel<M>, dim3(grid_for((int64_t)cls[6] * 32, kCdlpThreads, g)), dim3(kCdlpThreads), 0, R + off[6], cls[6], col, cur, nxt));
        if (M) {
            const int32_t nblock = cls[7] + cls[8] + cls[9];
            if (nblock) GHB_TRY(launch(ws, cdlp_block_kernel<true>, dim3(grid_for(nblock, 1, g)), dim3(kCdlpThreads), 0, R + off[7], nblock, col, cur, nxt, 0u));
            if (nlong) GHB_TRY(launch(ws, cdlp_chunk_min_kernel, dim3(grid_for(nch, 1, g)), dim3(kCdlpThreads), 0, long_rows, col, cur, (const int32_t*)chunks, nch, pool, (const int64_t*)tab_off, done, best, nxt));
            return GHB_OK;
        }
        if (cls[7]) GHB_TRY(launch(ws, cdlp_block_kernel<false>, dim3(grid_for(cls[7], 1, g_small)), dim3(kCdlpThreads), small_smem, R + off[7], cls[7], col, cur, nxt, (uint32_t)kSmallBlockSlots));
        if (cls[8]) GHB_TRY(launch(ws, cdlp_block_kernel<false>, dim3(grid_for(cls[8], 1, g_mid)), dim3(kCdlpThreads), mid_smem, R + off[8], cls[8], col, cur, nxt, (uint32_t)kMidBlockSlots));
        if (cls[9]) GHB_TRY(launch(ws, cdlp_block_kernel<false>, dim3(grid_for(cls[9], 1, g_big)), dim3(kCdlpThreads), big_smem, R + off[9], cls[9], col, cur, nxt, (uint32_t)kBlockSlots));
        if (nlong) {
            GHB_TRY(launch(ws, cdlp_chunk_count_kernel, dim3(grid_for(nch, 1, g_chunk)), dim3(kCdlpThreads), chunk_smem, long_rows, col, cur, (const int32_t*)chunks, nch, pool, (const int64_t*)tab_off, occ, done, best, nxt));
            GHB_TRY(launch(ws, cdlp_chunk_reset_kernel, dim3(grid_for(nch, 1, g)), dim3(kCdlpThreads), 0, long_rows, (const int32_t*)chunks, nch, pool, (const int64_t*)tab_off, occ, done));
        }
        return GHB_OK;
    };

    int32_t* cur = labels;
    int32_t* nxt = other;
    for (int it = 0; it < iterations; ++it) {
        if (it == 0 && first_min)
            GHB_TRY(iteration(std::true_type{}, cur, nxt));
        else
            GHB_TRY(iteration(std::false_type{}, cur, nxt));
        std::swap(cur, nxt);
    }
    if (cur != labels)
        GHB_CUDA_TRY(cudaMemcpyAsync(labels, cur, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
    return GHB_OK;
}

}  // namespace ghb

using namespace ghb;

extern "C" int ghb_cdlp(ghb_workspace* ws, int32_t n, const int32_t* all_rowptr, const int32_t* all_col,
                        int32_t iterations, int32_t* labels) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(all_rowptr && labels, "NULL argument");
    GHB_REQUIRE(iterations >= 0, "iterations < 0");
    return cdlp_run(ws, n, all_rowptr, all_col, iterations, labels, nullptr, false);
}
