// Per-vertex triangle counting (replaces GPU_TC_csr.cuh:15-68; semantics of
// CPU_TC.hpp:31-60: for every entry u->v and every w in row(u) and row(v),
// add 1 to u, v and w).
//
// Symmetric, loop-free graphs with strictly increasing rows (checked on the
// device first) take the oriented path: keep u->v only when
// (deg v, v) > (deg u, u), so every triangle is found once, at its
// lowest-ranked vertex, and oriented rows hold at most O(sqrt m) entries.
// Each oriented row N+(a) is put in a shared-memory hash and every w of
// every N+(b), b in N+(a), is probed with all lanes busy (the hash path
// below); rows too long for a block's hash, or every row when the
// workspace's tc_hash knob is 0, intersect N+(u) and N+(v) per entry by
// walking one list and galloping through the other.  A triangle adds 1 to
// each of its three vertices; the reference's count is 6x that (each
// triangle is met from its 6 ordered edges), and its int32 wraps.
//
// Any other input takes the generic path: the reference's merge over every
// entry, kept for exact parity on directed or unusual inputs.
#include <atomic>

#include "common.cuh"
#include "edge_walk.cuh"
#include "scan.cuh"

namespace ghb {
namespace {

constexpr int32_t kTcFlagLoop = 1, kTcFlagUnsorted = 2, kTcFlagAsym = 4;

// First position in [b, e) of a sorted row whose entry is >= x (e if none):
// a galloping search (probes b, b+1, b+3, b+7, ... then a binary search in the
// last gap), so a hit near b costs a few probes, not log2(e - b).
__device__ __forceinline__ int32_t lower_bound_from(const int32_t* __restrict__ col, int32_t b, int32_t e, int32_t x) {
    if (b >= e || col[b] >= x) return b;
    int32_t lo = b, step = 1;  // col[lo] < x
    while (step < e - lo && col[lo + step] < x) {
        lo += step;
        step <<= 1;
    }
    b = lo + 1;
    e = step < e - lo ? lo + step : e;  // col[e] >= x, or e is the row end
    while (b < e) {
        const int32_t mid = b + ((e - b) >> 1);
        if (col[mid] < x) b = mid + 1;
        else e = mid;
    }
    return b;
}

// First position in [b, e) of a sorted row whose entry is > x (e if none).
__device__ __forceinline__ int32_t upper_bound_pos(const int32_t* __restrict__ col, int32_t b, int32_t e, int32_t x) {
    while (b < e) {
        const int32_t mid = b + ((e - b) >> 1);
        if (col[mid] <= x) b = mid + 1;
        else e = mid;
    }
    return b;
}

__device__ __forceinline__ bool row_contains(const int32_t* __restrict__ col, int32_t b, int32_t e, int32_t x) {
    while (b < e) {
        const int32_t mid = (b + e) >> 1;
        const int32_t y = col[mid];
        if (y == x) return true;
        if (y < x) b = mid + 1;
        else e = mid;
    }
    return false;
}

struct CheckVisitor {
    const int32_t* rowptr;
    const int32_t* col;
    int32_t* flags;
    __device__ bool want_row(int32_t) const { return true; }
    __device__ void operator()(int32_t u, int32_t v, int32_t j) const {
        int32_t f = 0;
        if (u == v) f |= kTcFlagLoop;
        if (j + 1 < rowptr[u + 1] && col[j + 1] <= v) f |= kTcFlagUnsorted;
        if (!row_contains(col, rowptr[v], rowptr[v + 1], u)) f |= kTcFlagAsym;
        if (f) atomicOr(flags, f);
    }
    __device__ void finish() const {}
};

__device__ __forceinline__ bool ranks_above(const int32_t* __restrict__ rowptr, int32_t u, int32_t v) {
    const int32_t du = rowptr[u + 1] - rowptr[u], dv = rowptr[v + 1] - rowptr[v];
    return dv > du || (dv == du && v > u);
}

// Adds 1 per call to cnt[u], merged across lanes that share u.
__device__ __forceinline__ void add_count_merged(int32_t* cnt, int32_t u, int32_t inc) {
    const unsigned active = __activemask();
    const unsigned same = __match_any_sync(active, u);
    int32_t total = inc;
    // Sum inc over the lanes of `same` (inc is 0 or 1 here).
    total = __popc(__ballot_sync(same, inc != 0));
    if (lane_id() == __ffs(same) - 1 && total) atomicAdd(cnt + u, total);
}

struct KeepCountVisitor {
    const int32_t* rowptr;
    int32_t* keep;
    __device__ bool want_row(int32_t) const { return true; }
    __device__ void operator()(int32_t u, int32_t v, int32_t) const {
        add_count_merged(keep, u, ranks_above(rowptr, u, v) ? 1 : 0);
    }
    __device__ void finish() const {}
};

// Ordered fill of the oriented rows: a warp per row; rows over kWalkBig
// entries are listed in long_rows (count in [0], rows from [1]) for
// orient_fill_long_kernel.
__global__ void __launch_bounds__(256) orient_fill_kernel(int32_t n, const int32_t* __restrict__ rowptr,
                                                          const int32_t* __restrict__ col,
                                                          const int32_t* __restrict__ orp, int32_t* ocol,
                                                          int32_t* long_rows) {
    const int lane = lane_id();
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t u = warp; u < n; u += nwarps) {
        const int32_t b = rowptr[u], e = rowptr[u + 1];
        if (e - b > kWalkBig) {
            if (lane == 0) long_rows[1 + atomicAdd(long_rows, 1)] = (int32_t)u;
            continue;
        }
        int32_t out = orp[u];
        for (int32_t j0 = b; j0 < e; j0 += 32) {
            const int32_t j = j0 + lane;
            int32_t v = 0;
            bool k = false;
            if (j < e) {
                v = col[j];
                k = ranks_above(rowptr, (int32_t)u, v);
            }
            const unsigned km = __ballot_sync(0xffffffffu, k);
            if (k) ocol[out + __popc(km & ((1u << lane) - 1u))] = v;
            out += __popc(km);
        }
    }
}

// The listed long rows, a block per row: each thread takes kOrientItems
// consecutive entries per step (their loads issued together), a block scan
// of the kept counts places them in row order.
constexpr int kOrientItems = 8;
__global__ void __launch_bounds__(1024) orient_fill_long_kernel(const int32_t* __restrict__ rowptr,
                                                                const int32_t* __restrict__ col,
                                                                const int32_t* __restrict__ orp, int32_t* ocol,
                                                                const int32_t* __restrict__ long_rows) {
    __shared__ int32_t wsum[32];
    const int lane = lane_id(), wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int32_t nl = long_rows[0];
    for (int32_t r = blockIdx.x; r < nl; r += gridDim.x) {
        const int32_t u = long_rows[1 + r];
        const int32_t b = rowptr[u], e = rowptr[u + 1];
        const int32_t du = e - b;
        int32_t out = orp[u];
        for (int32_t j0 = b; j0 < e; j0 += (int32_t)blockDim.x * kOrientItems) {
            const int32_t jt = j0 + (int32_t)threadIdx.x * kOrientItems;
            int32_t v[kOrientItems];
#pragma unroll
            for (int q = 0; q < kOrientItems; ++q) v[q] = jt + q < e ? col[jt + q] : -1;
            int32_t dv[kOrientItems];
#pragma unroll
            for (int q = 0; q < kOrientItems; ++q) dv[q] = v[q] >= 0 ? rowptr[v[q] + 1] - rowptr[v[q]] : -1;
            unsigned keep = 0;
#pragma unroll
            for (int q = 0; q < kOrientItems; ++q)
                if (v[q] >= 0 && (dv[q] > du || (dv[q] == du && v[q] > u))) keep |= 1u << q;
            const int32_t c = __popc(keep);
            int32_t incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t x = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += x;
            }
            if (lane == 31) wsum[wid] = incl;
            __syncthreads();
            int32_t before = 0, all = 0;
            for (int w = 0; w < nw; ++w) {
                const int32_t x = wsum[w];
                if (w < wid) before += x;
                all += x;
            }
            int32_t pos = out + before + incl - c;
#pragma unroll
            for (int q = 0; q < kOrientItems; ++q)
                if ((keep >> q) & 1u) ocol[pos++] = v[q];
            out += all;
            __syncthreads();
        }
    }
}

struct OrientedVisitor {
    const int32_t* orp;
    const int32_t* ocol;
    unsigned long long* cnt;
    __device__ bool want_row(int32_t) const { return true; }
    __device__ void operator()(int32_t u, int32_t v, int32_t) const {
        // Walk N+(v) and search N+(u), which the lanes walking u's row share
        // (it stays in L1); both are strictly increasing, so each search
        // starts where the last ended, and the walk stops once N+(u) is
        // passed.  A long N+(v) over a much shorter N+(u) is walked the other
        // way round.  (Swapping whenever N+(v) is longer measured 4 % slower
        // on 2,000 small ER graphs and 10 % slower on RMAT scale 24; plain
        // binary searches from the last hit 1.46x slower on RMAT scale 24.)
        int32_t sb = orp[v], se = orp[v + 1];
        int32_t lb = orp[u], le = orp[u + 1];
        if (se - sb > 64 && se - sb > 4 * (le - lb)) {
            const int32_t tb = sb, te = se;
            sb = lb;
            se = le;
            lb = tb;
            le = te;
        }
        unsigned long long found = 0;
        for (int32_t k = sb; k < se && lb < le; ++k) {
            const int32_t w = ocol[k];
            lb = lower_bound_from(ocol, lb, le, w);
            if (lb < le && ocol[lb] == w) {
                atomicAdd(cnt + w, 1ull);
                ++found;
                ++lb;
            }
        }
        if (found) {
            atomicAdd(cnt + u, found);
            atomicAdd(cnt + v, found);
        }
    }
    __device__ void finish() const {}
};

// ---- hash-probe counting: one row a of the oriented CSR at a time.
//
// N+(a) goes into a shared-memory hash (open addressing, at most half
// full); the lists N+(b), b in N+(a), are then walked with every lane busy
// (lists of 32 entries or more by the whole warp, shorter ones packed
// warp-wide over a scan of their lengths) and each w probed: a hit is the
// triangle (a, b, w).  a's count is summed in registers, b's in a shared
// counter per entry of N+(a) (one global add per oriented edge that closes
// any), w's by a global add per triangle.  Rows of up to kTcWarpRow entries
// take a warp each (256-slot hash), rows up to kTcBlockRow a block each
// (hash of up to 16,384 slots); longer ones go to the galloping visitor.
constexpr int32_t kTcWarpRow = 128;
constexpr int32_t kTcWarpSlots = 256;
constexpr int32_t kTcBlockRow = 8192;
constexpr int kTcWarpBlock = 256;   // threads of the warp-per-row kernel
// A list N+(b) over kTcSearchRatio x |N+(a)| entries is searched for N+(a)'s
// entries (k binary searches) rather than probed entry by entry.
constexpr int32_t kTcSearchRatio = 16;
constexpr int kTcBlockThreads = 128;
constexpr int32_t kTcSlice = 512;     // entries of N+(a) per slice-kernel item
constexpr int32_t kTcMidRow = 1024;   // rows up to this many entries: a 2,048-slot hash
constexpr int kTcMidLog2 = 11;
constexpr int32_t kTcMid2Row = 4096;  // rows up to this many entries: an 8,192-slot hash (32 KB, six blocks per SM)
constexpr int kTcMid2Log2 = 13;
constexpr int kTcBigLog2 = 14;        // 16,384 slots for rows up to kTcBlockRow (64 KB, three blocks per SM)

__device__ __forceinline__ uint32_t tc_hash(int32_t w, int shift) {
    return ((uint32_t)w * 2654435761u) >> shift;
}

__device__ __forceinline__ void tc_insert(int32_t* keys, uint32_t mask, int shift, int32_t w) {
    uint32_t h = tc_hash(w, shift);
    while (atomicCAS(keys + h, -1, w) != -1) h = (h + 1) & mask;
}

__device__ __forceinline__ bool tc_probe(const int32_t* keys, uint32_t mask, int shift, int32_t w) {
    uint32_t h = tc_hash(w, shift);
    while (true) {
        const int32_t k = keys[h];
        if (k == w) return true;
        if (k < 0) return false;
        h = (h + 1) & mask;
    }
}

// The warp's share of row a (k entries): entries [g0, g_end) of N+(a), the
// 32-entry groups from g0 with the given stride, probing the hash `keys`.
// Adds w's hits to cnt, b's to bc[(index in N+(a)) - bc_off]; returns a's
// hits (lane 0 holds those of whole-warp lists, every lane those it probed
// itself).
__device__ __forceinline__ unsigned long long tc_row_share(const int32_t* __restrict__ orp,
                                                           const int32_t* __restrict__ ocol, int32_t ab, int32_t k,
                                                           int32_t g0, int32_t g_end, int32_t stride,
                                                           const int32_t* keys, uint32_t mask, int shift, int32_t* bc,
                                                           int32_t bc_off, unsigned long long* cnt, int32_t trim_min) {
    const int lane = lane_id();
    unsigned long long a_hits = 0;
    const int32_t amin = ocol[ab], amax = ocol[ab + k - 1];
    for (int32_t g = g0; g < g_end; g += stride) {
        const int32_t i = g + lane;
        int32_t lb = 0, le = 0;
        if (i < g_end) {
            const int32_t b = ocol[ab + i];
            lb = orp[b];
            le = orp[b + 1];
            // Only N+(b)'s entries inside [min N+(a), max N+(a)] can be in
            // N+(a) (both rows ascending): lists over trim_min entries are
            // cut to that range first (two binary searches, a chain of
            // dependent loads that short lists do not repay).
            if (le - lb > trim_min) {
                lb = lower_bound_from(ocol, lb, le, amin);
                le = upper_bound_pos(ocol, lb, le, amax);
            }
        }
        unsigned med = __ballot_sync(0xffffffffu, le - lb >= 32);
        while (med) {
            const int leader = __ffs(med) - 1;
            med &= med - 1;
            const int32_t mb = __shfl_sync(0xffffffffu, lb, leader);
            const int32_t me = __shfl_sync(0xffffffffu, le, leader);
            unsigned hits = 0;
            if (me - mb > kTcSearchRatio * k) {
                // N+(b) much longer than N+(a): look N+(a)'s own entries up
                // in N+(b) by binary search instead (the same intersection).
                for (int32_t i0 = 0; i0 < k; i0 += 32) {
                    const int32_t i = i0 + lane;
                    if (i < k) {
                        const int32_t x = ocol[ab + i];
                        const int32_t p = lower_bound_from(ocol, mb, me, x);
                        if (p < me && ocol[p] == x) {
                            ++hits;
                            atomicAdd(cnt + x, 1ull);
                        }
                    }
                }
            } else {
                for (int32_t j = mb + lane; j < me; j += 32) {
                    const int32_t w = ocol[j];
                    if (tc_probe(keys, mask, shift, w)) {
                        ++hits;
                        atomicAdd(cnt + w, 1ull);
                    }
                }
            }
            hits = warp_sum(hits);
            if (lane == 0 && hits) {
                atomicAdd(bc + g + leader - bc_off, (int32_t)hits);
                a_hits += hits;
            }
        }
        if (le - lb >= 32) le = lb;
        const int32_t d = le - lb;
        int32_t incl = d;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t x = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += x;
        }
        const int32_t excl = incl - d;
        const int32_t total = __shfl_sync(0xffffffffu, incl, 31);
        for (int32_t k0 = 0; k0 < total; k0 += 32) {
            const int32_t kk = k0 + lane;
            int owner = 0;
#pragma unroll
            for (int s = 16; s >= 1; s >>= 1) {
                const int cand = owner + s;
                const int32_t ev = __shfl_sync(0xffffffffu, excl, cand);
                if (ev <= kk) owner = cand;
            }
            const int32_t ob = __shfl_sync(0xffffffffu, lb, owner);
            const int32_t oe = __shfl_sync(0xffffffffu, excl, owner);
            if (kk < total) {
                const int32_t w = ocol[ob + (kk - oe)];
                if (tc_probe(keys, mask, shift, w)) {
                    atomicAdd(bc + g + owner - bc_off, 1);
                    atomicAdd(cnt + w, 1ull);
                    ++a_hits;
                }
            }
        }
    }
    return a_hits;
}

// Rows of 1..kTcWarpRow oriented entries, a warp each.  Longer rows, up to
// block_row <= kTcBlockRow entries, are listed for the slice kernels as
// (row, first entry) items of kTcSlice entries each, in three classes by the
// hash the row needs (items[0..]: up to kTcMidRow entries,
// items[item_cap..]: up to kTcMid2Row, items[2 item_cap..]: longer); rows
// over block_row go to huge[] for the galloping walk.
// tails: [0], [1], [2] the three item counts, [3] the huge rows.
// (Eight blocks per SM, 32 registers: 774-787 ms for RMAT-24 TC against
// 789-797 ms at six blocks.)
__global__ void __launch_bounds__(kTcWarpBlock, 8) tc_hash_warp_kernel(int32_t n, const int32_t* __restrict__ orp,
                                                                    const int32_t* __restrict__ ocol,
                                                                    unsigned long long* cnt, int2* items,
                                                                    int64_t item_cap, int32_t* huge, int32_t* tails,
                                                                    int32_t block_row, int32_t trim_min) {
    __shared__ int32_t s_keys[kTcWarpBlock / 32][kTcWarpSlots];
    __shared__ int32_t s_bc[kTcWarpBlock / 32][kTcWarpRow];
    const int lane = lane_id();
    int32_t* keys = s_keys[threadIdx.x >> 5];
    int32_t* bc = s_bc[threadIdx.x >> 5];
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t a = warp; a < n; a += nwarps) {
        const int32_t ab = orp[a], k = orp[a + 1] - ab;
        if (k == 0) continue;
        if (k > kTcWarpRow) {
            if (k <= block_row) {
                const int cls = k <= kTcMidRow ? 0 : (k <= kTcMid2Row ? 1 : 2);
                const int32_t ns = (k + kTcSlice - 1) / kTcSlice;
                int32_t pos = 0;
                if (lane == 0) pos = atomicAdd(tails + cls, ns);
                pos = __shfl_sync(0xffffffffu, pos, 0);
                for (int32_t s = lane; s < ns; s += 32)
                    items[cls * item_cap + pos + s] = make_int2((int32_t)a, s * kTcSlice);
            } else if (lane == 0) {
                huge[atomicAdd(tails + 3, 1)] = (int32_t)a;
            }
            continue;
        }
        for (int s = lane; s < kTcWarpSlots; s += 32) keys[s] = -1;
        for (int s = lane; s < k; s += 32) bc[s] = 0;
        __syncwarp();
        const int shift = 32 - 8;  // 256 slots
        for (int32_t i = lane; i < k; i += 32) tc_insert(keys, kTcWarpSlots - 1, shift, ocol[ab + i]);
        __syncwarp();
        unsigned long long a_hits =
            tc_row_share(orp, ocol, ab, k, 0, k, 32, keys, kTcWarpSlots - 1, shift, bc, 0, cnt, trim_min);
        __syncwarp();
        a_hits = warp_sum(a_hits);
        if (lane == 0 && a_hits) atomicAdd(cnt + a, a_hits);
        for (int32_t i = lane; i < k; i += 32)
            if (bc[i]) atomicAdd(cnt + ocol[ab + i], (unsigned long long)bc[i]);
        __syncwarp();
    }
}

// Slices of rows over kTcWarpRow entries (items listed by the warp kernel),
// a 128-thread block per item: the block hashes the whole row N+(a) (a
// power of two >= 2k slots, at most 2^CAP_LOG2) and probes for the
// kTcSlice entries b of its slice, four warps side by side.  Small blocks
// keep many rows in flight per SM; slices spread the longest rows over
// many blocks.  DYN: the hash lives in dynamic shared memory.
template <int CAP_LOG2, bool DYN>
__global__ void __launch_bounds__(kTcBlockThreads) tc_hash_slice_kernel(const int32_t* __restrict__ orp,
                                                                        const int32_t* __restrict__ ocol,
                                                                        unsigned long long* cnt, const int2* items,
                                                                        const int32_t* count, int32_t trim_min) {
    extern __shared__ int32_t s_dyn[];
    __shared__ int32_t s_static[DYN ? 1 : (1 << CAP_LOG2)];
    __shared__ int32_t s_bc[kTcSlice];
    __shared__ unsigned long long s_hits;
    int32_t* keys = DYN ? s_dyn : s_static;
    const int32_t nitems = *count;
    const int warp_in_block = threadIdx.x >> 5, warps = blockDim.x >> 5;
    for (int32_t r = blockIdx.x; r < nitems; r += gridDim.x) {
        const int2 it = items[r];
        const int32_t a = it.x, gs = it.y;
        const int32_t ab = orp[a], k = orp[a + 1] - ab;
        const int32_t ge = min(k, gs + kTcSlice);
        int log2cap = 1;
        while ((1 << log2cap) < 2 * k) ++log2cap;
        const uint32_t cap = 1u << log2cap;
        for (uint32_t s = threadIdx.x; s < cap; s += blockDim.x) keys[s] = -1;
        for (int32_t s = threadIdx.x; s < ge - gs; s += blockDim.x) s_bc[s] = 0;
        if (threadIdx.x == 0) s_hits = 0;
        __syncthreads();
        const int shift = 32 - log2cap;
        for (int32_t i = threadIdx.x; i < k; i += blockDim.x) tc_insert(keys, cap - 1, shift, ocol[ab + i]);
        __syncthreads();
        unsigned long long a_hits = tc_row_share(orp, ocol, ab, k, gs + warp_in_block * 32, ge, warps * 32, keys,
                                                 cap - 1, shift, s_bc, gs, cnt, trim_min);
        a_hits = warp_sum(a_hits);
        if (lane_id() == 0 && a_hits) atomicAdd(&s_hits, a_hits);
        __syncthreads();
        if (threadIdx.x == 0 && s_hits) atomicAdd(cnt + a, s_hits);
        for (int32_t i = threadIdx.x; i < ge - gs; i += blockDim.x)
            if (s_bc[i]) atomicAdd(cnt + ocol[ab + gs + i], (unsigned long long)s_bc[i]);
        __syncthreads();
    }
}

// Triangles of the oriented CSR into cnt (zeroed by the caller): the
// hash-probe kernels above, then the load-balanced walk with the galloping
// visitor below for rows longer than kTcBlockRow.  `lists` holds tc_lists_ints(n, m)
// ints of scratch.  (A warp-per-row shared-memory hash variant measured 25 % slower
// on RMAT scale 24: most oriented rows hold a few entries, so a warp per row
// leaves most lanes idle, where the walker packs short rows warp-wide.
// Handing the entries whose shorter list exceeds 32 to a warp each, through
// a list appended to by atomics, measured 4 % faster at scale 22 and 12 %
// slower at scale 24.  Counting the first 4096 ids, the hubs that are the
// highest-ranked vertex of most triangles, in per-block shared-memory
// counters measured 10 % slower at scale 22 and 17 % slower at scale 24 with
// 32-bit counters, twice as slow with 64-bit ones: the L2's same-address
// reductions keep up better than a block's shared-memory atomics.)
// Items per class of the slice kernels for a CSR of n rows and m entries.
int64_t tc_item_cap(int32_t n, int64_t m) { return (int64_t)n + m / kTcSlice + 64; }

}  // namespace

// Scratch ints that tc_count_oriented's `lists` must hold.
size_t tc_lists_ints(int32_t n, int64_t m) { return (size_t)(6 * tc_item_cap(n, m) + n + 8); }

namespace {

int tc_count_oriented(ghb_workspace* ws, int32_t n, int64_t m, const int32_t* orp, const int32_t* ocol,
                      unsigned long long* cnt, const WalkBuffers& wb, int32_t* lists) {
    if (!ws->tune.tc_hash)
        return walk(ws, orp, ocol, (const int32_t*)nullptr, (const int32_t*)nullptr, (int64_t)n, (int64_t)n, wb,
                    OrientedVisitor{orp, ocol, cnt});
    const int64_t item_cap = tc_item_cap(n, m);
    int2* items = reinterpret_cast<int2*>(lists);
    int32_t* huge = lists + 6 * item_cap;
    int32_t* tails = huge + n;
    GHB_CUDA_TRY(cudaMemsetAsync(tails, 0, 4 * sizeof(int32_t), ws->stream));
    GHB_TRY(launch(ws, tc_hash_warp_kernel, dim3(grid_for((int64_t)n * 32, kTcWarpBlock, ws->num_sms * 8)),
                   dim3(kTcWarpBlock), 0, n, orp, ocol, cnt, items, item_cap, huge, tails,
                   std::min<int32_t>(std::max<int32_t>(ws->tune.tc_block_row, kTcWarpRow), kTcBlockRow),
                   ws->tune.tc_trim_min));
    GHB_TRY(launch(ws, tc_hash_slice_kernel<kTcMidLog2, false>, dim3(ws->num_sms * ws->tune.tc_slice_blocks),
                   dim3(kTcBlockThreads), 0,
                   orp, ocol, cnt, (const int2*)items, (const int32_t*)tails, ws->tune.tc_trim_min));
    const size_t smem = sizeof(int32_t) << kTcBigLog2;
    static bool attr_set[64] = {false};
    if (ws->device >= 0 && ws->device < 64 && !attr_set[ws->device]) {
        GHB_CUDA_TRY(cudaFuncSetAttribute(tc_hash_slice_kernel<kTcBigLog2, true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set[ws->device] = true;
    }
    GHB_TRY(launch(ws, tc_hash_slice_kernel<kTcMid2Log2, false>, dim3(ws->num_sms * 6), dim3(kTcBlockThreads), 0,
                   orp, ocol, cnt, (const int2*)(items + item_cap), (const int32_t*)(tails + 1),
                   ws->tune.tc_trim_min));
    GHB_TRY(launch(ws, tc_hash_slice_kernel<kTcBigLog2, true>, dim3(ws->num_sms * 3), dim3(kTcBlockThreads), smem,
                   orp, ocol, cnt, (const int2*)(items + 2 * item_cap), (const int32_t*)(tails + 2),
                   ws->tune.tc_trim_min));
    // Rows over the block path's length: the galloping walk.
    return walk(ws, orp, ocol, (const int32_t*)huge, (const int32_t*)(tails + 3), (int64_t)0,
                (int64_t)ws->num_sms * 64, wb, OrientedVisitor{orp, ocol, cnt});
}

// The reference's merge over every entry (any CSR).
struct MergeVisitor {
    const int32_t* rowptr;
    const int32_t* col;
    unsigned long long* cnt;
    __device__ bool want_row(int32_t) const { return true; }
    __device__ void operator()(int32_t u, int32_t v, int32_t) const {
        int32_t i = rowptr[u], ie = rowptr[u + 1];
        int32_t j = rowptr[v], je = rowptr[v + 1];
        unsigned long long found = 0;
        while (i < ie && j < je) {
            const int32_t a = col[i], b = col[j];
            if (a == b) {
                atomicAdd(cnt + a, 1ull);
                ++found;
                ++i;
                ++j;
            } else if (a < b) {
                ++i;
            } else {
                ++j;
            }
        }
        if (found) {
            atomicAdd(cnt + u, found);
            atomicAdd(cnt + v, found);
        }
    }
    __device__ void finish() const {}
};

__global__ void tc_finish_kernel(int32_t n, const unsigned long long* __restrict__ cnt, int scale,
                                 int64_t* counts64, int32_t* counts32, unsigned long long* total) {
    unsigned long long s = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long c = cnt[v] * (unsigned long long)scale;
        if (counts64) counts64[v] = (int64_t)c;
        if (counts32) counts32[v] = (int32_t)(uint32_t)c;
        s += cnt[v];
    }
    s = warp_sum(s);
    if (lane_id() == 0 && s) atomicAdd(total, s);
}

}  // namespace

// The oriented CSR's columns (orp already scanned); `lists` (at least n + 1
// ints, the counting scratch, free until the count) holds the long-row list.
static int orient_fill(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, const int32_t* orp,
                       int32_t* ocol, int32_t* lists) {
    GHB_CUDA_TRY(cudaMemsetAsync(lists, 0, sizeof(int32_t), ws->stream));
    GHB_TRY(launch(ws, orient_fill_kernel, dim3(grid_for((int64_t)n * 32, 256, ws->num_sms * 8)), dim3(256), 0, n,
                   rowptr, col, orp, ocol, lists));
    GHB_TRY(launch(ws, orient_fill_long_kernel, dim3(ws->num_sms * 2), dim3(1024), 0, rowptr, col, orp, ocol,
                   (const int32_t*)lists));
    return GHB_OK;
}

// Oriented triangle counting with no host round trip and no allocation: the
// caller guarantees a symmetric, loop-free CSR with strictly increasing rows
// and m = rowptr[n] entries, and passes tc_oriented_bytes(n, m) bytes of
// device scratch at `base`.  cnt (n + 1 entries, zeroed here) gets each
// vertex's triangles and, with counts64, their sum in cnt[n]; counts64 (may
// be NULL) gets the reference's 6x count.
size_t tc_oriented_bytes(int32_t n, int64_t m) {
    Carver c(nullptr);
    WalkBuffers::carve(c, n);
    c.take<int32_t>((size_t)n + 1);
    c.take<int32_t>((size_t)n + 1);
    c.take<int64_t>(scan_scratch_words(n));
    c.take<int32_t>(m > 0 ? m : 1);
    c.take<int32_t>(tc_lists_ints(n, m));
    return c.off;
}

int tc_oriented_core(ghb_workspace* ws, int32_t n, int64_t m, const int32_t* rowptr, const int32_t* col, void* base,
                     unsigned long long* cnt, int64_t* counts64) {
    cudaStream_t st = ws->stream;
    Carver c(base);
    WalkBuffers wb = WalkBuffers::carve(c, n);
    int32_t* keep = c.take<int32_t>((size_t)n + 1);
    int32_t* orp = c.take<int32_t>((size_t)n + 1);
    int64_t* bsums = c.take<int64_t>(scan_scratch_words(n));
    int32_t* ocol = c.take<int32_t>(m > 0 ? m : 1);
    int32_t* lists = c.take<int32_t>(tc_lists_ints(n, m));
    GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * ((size_t)n + 1), st));
    GHB_CUDA_TRY(cudaMemsetAsync(keep, 0, sizeof(int32_t) * n, st));
    GHB_TRY(walk(ws, rowptr, col, (const int32_t*)nullptr, (const int32_t*)nullptr, (int64_t)n, (int64_t)n, wb,
                 KeepCountVisitor{rowptr, keep}));
    GHB_TRY(scan_exclusive_i32(ws, keep, orp, n, bsums));
    GHB_TRY(orient_fill(ws, n, rowptr, col, orp, ocol, lists));
    GHB_TRY(tc_count_oriented(ws, n, m, orp, ocol, cnt, wb, lists));
    if (counts64)
        GHB_TRY(launch(ws, tc_finish_kernel, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0, n,
                       (const unsigned long long*)cnt, 6, counts64, (int32_t*)nullptr,
                       (unsigned long long*)(cnt + n)));
    return GHB_OK;
}

// flags_cache (may be NULL): the input check's flags for this CSR, -1 when
// not yet known; a known value skips the check.
int tc_run_cached(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, int64_t* counts64,
                  int32_t* counts32, int64_t* total, std::atomic<int32_t>* flags_cache) {
    cudaStream_t st = ws->stream;
    int32_t* hp = reinterpret_cast<int32_t*>(ws->host_pinned);
    GHB_CUDA_TRY(cudaMemcpyAsync(hp, rowptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GHB_CUDA_TRY(cudaStreamSynchronize(st));
    const int64_t m = hp[0];

    Carver sizing(nullptr);
    WalkBuffers::carve(sizing, n);
    sizing.take<int32_t>(8);
    sizing.take<unsigned long long>(n);
    sizing.take<unsigned long long>(1);
    sizing.take<int32_t>((size_t)n + 1);
    sizing.take<int32_t>((size_t)n + 1);
    sizing.take<int64_t>(scan_scratch_words(n));
    sizing.take<int32_t>(m > 0 ? m : 1);
    sizing.take<int32_t>(tc_lists_ints(n, m));
    GHB_TRY(ws_reserve(ws, sizing.off));
    Carver c(ws->scratch);
    WalkBuffers wb = WalkBuffers::carve(c, n);
    int32_t* flags = c.take<int32_t>(8);
    unsigned long long* cnt = c.take<unsigned long long>(n);
    unsigned long long* tot = c.take<unsigned long long>(1);
    int32_t* keep = c.take<int32_t>((size_t)n + 1);
    int32_t* orp = c.take<int32_t>((size_t)n + 1);
    int64_t* bsums = c.take<int64_t>(scan_scratch_words(n));
    int32_t* ocol = c.take<int32_t>(m > 0 ? m : 1);
    int32_t* lists = c.take<int32_t>(tc_lists_ints(n, m));

    GHB_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * n, st));
    GHB_CUDA_TRY(cudaMemsetAsync(tot, 0, sizeof(unsigned long long), st));
    int32_t check = flags_cache ? flags_cache->load(std::memory_order_relaxed) : -1;
    if (check < 0) {
        GHB_CUDA_TRY(cudaMemsetAsync(flags, 0, sizeof(int32_t), st));
        GHB_TRY(walk(ws, rowptr, col, (const int32_t*)nullptr, (const int32_t*)nullptr, (int64_t)n, (int64_t)n, wb,
                     CheckVisitor{rowptr, col, flags}));
        GHB_CUDA_TRY(cudaMemcpyAsync(hp, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        check = hp[0];
        if (flags_cache) flags_cache->store(check, std::memory_order_relaxed);
    }
    const bool oriented = check == 0;
    if (oriented) {
        GHB_CUDA_TRY(cudaMemsetAsync(keep, 0, sizeof(int32_t) * n, st));
        GHB_TRY(walk(ws, rowptr, col, (const int32_t*)nullptr, (const int32_t*)nullptr, (int64_t)n, (int64_t)n,
                     wb, KeepCountVisitor{rowptr, keep}));
        GHB_TRY(scan_exclusive_i32(ws, keep, orp, n, bsums));
        GHB_TRY(orient_fill(ws, n, rowptr, col, orp, ocol, lists));
        GHB_TRY(tc_count_oriented(ws, n, m, orp, ocol, cnt, wb, lists));
    } else {
        GHB_TRY(walk(ws, rowptr, col, (const int32_t*)nullptr, (const int32_t*)nullptr, (int64_t)n, (int64_t)n, wb,
                     MergeVisitor{rowptr, col, cnt}));
    }
    GHB_TRY(launch(ws, tc_finish_kernel, dim3(grid_for(n, 256, ws->num_sms * 8)), dim3(256), 0, n,
                   (const unsigned long long*)cnt, oriented ? 6 : 1, counts64, counts32, tot));
    if (total) {
        GHB_CUDA_TRY(cudaMemcpyAsync(ws->host_pinned, tot, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        GHB_CUDA_TRY(cudaStreamSynchronize(st));
        const unsigned long long s = *reinterpret_cast<const unsigned long long*>(ws->host_pinned);
        // oriented: sum of per-vertex incidences = 3T; generic: 18T.
        *total = (int64_t)(oriented ? s / 3 : s / 18);
    }
    return GHB_OK;
}

int tc_run(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col, int64_t* counts64,
           int32_t* counts32, int64_t* total) {
    return tc_run_cached(ws, n, rowptr, col, counts64, counts32, total, nullptr);
}

}  // namespace ghb

using namespace ghb;

extern "C" int ghb_tc(ghb_workspace* ws, int32_t n, const int32_t* rowptr, const int32_t* col,
                      int64_t* counts64, int32_t* counts32, int64_t* total) {
    ws = ws_resolve(ws);
    GHB_REQUIRE(ws, "no workspace");
    GHB_REQUIRE(n >= 1, "n must be >= 1");
    GHB_REQUIRE(rowptr, "NULL rowptr");
    return tc_run(ws, n, rowptr, col, counts64, counts32, total);
}
