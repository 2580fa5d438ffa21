/*
 * ghb_gen.h - the seeded synthetic-graph specification shared by the CUDA
 * generators (graphhet_b200/csrc/gen.cu) and the CPU restatement used by the
 * tests.  Everything here is a pure function of (seed, counter), so the GPU
 * and the CPU produce bit-identical edge lists, vertex permutations and
 * weights for the same seed.
 *
 * These graphs stand in for the LDBC Graphalytics / Graph500 datasets that the
 * reference's batch scripts name (LDBC-GPU-csr.sh:14-29); the reference loads
 * those from text files (include/LDBC/ldbc.hpp:181-253), where an undirected
 * edge gets both directions with one weight (ldbc.hpp:237-242).  The same
 * rule holds here: the weight of an edge is a hash of its unordered endpoint
 * pair, so both directions and every duplicate carry the same value.
 *
 * RNG: SplitMix64 (Steele, Lea and Flood, "Fast splittable pseudorandom number
 * generators", OOPSLA 2014), used as a counter-based hash.
 */
#ifndef GHB_GEN_H
#define GHB_GEN_H

#include <stdint.h>

#if defined(__CUDACC__)
#define GHB_HD __host__ __device__ __forceinline__
#else
#define GHB_HD static inline
#endif

/* SplitMix64 output function applied to (z + golden gamma). */
GHB_HD uint64_t ghb_mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* Stream key for a (seed, purpose) pair. */
GHB_HD uint64_t ghb_stream(uint64_t seed, uint64_t purpose) {
    return ghb_mix64(ghb_mix64(seed) ^ (purpose * 0xD1B54A32D192ED03ULL));
}

/* Counter-based 64-bit draw. */
GHB_HD uint64_t ghb_draw(uint64_t stream, uint64_t ctr) {
    return ghb_mix64(stream ^ ghb_mix64(ctr));
}

/* Purposes (distinct streams from one seed). */
#define GHB_PURPOSE_RMAT 1ULL
#define GHB_PURPOSE_PERM 2ULL
#define GHB_PURPOSE_WEIGHT 3ULL
#define GHB_PURPOSE_ER 4ULL
#define GHB_PURPOSE_SOURCES 5ULL
#define GHB_PURPOSE_DANGLING 6ULL
#define GHB_PURPOSE_POWERLAW 7ULL

/* RMAT quadrant thresholds as 32-bit integers, so CPU and GPU compare the
 * same integers: quadrant 0 if r < t0, 1 if r < t1, 2 if r < t2, else 3. */
typedef struct {
    uint32_t t0, t1, t2;
} ghb_rmat_thresholds;

GHB_HD ghb_rmat_thresholds ghb_rmat_make_thresholds(double a, double b, double c) {
    ghb_rmat_thresholds t;
    t.t0 = (uint32_t)(a * 4294967296.0);
    t.t1 = (uint32_t)((a + b) * 4294967296.0);
    t.t2 = (uint32_t)((a + b + c) * 4294967296.0);
    return t;
}

/* RMAT edge number `e` of a 2^scale-vertex graph before permutation.  Level l
 * (0 = most significant bit) uses the high or low 32 bits of draw (e, l/2).
 * Quadrant q sets source bit (q >> 1) and destination bit (q & 1). */
GHB_HD void ghb_rmat_edge(uint64_t stream, ghb_rmat_thresholds t, int scale, uint64_t e,
                          uint32_t* src, uint32_t* dst) {
    uint32_t u = 0, v = 0;
    uint64_t r = 0;
    for (int l = 0; l < scale; ++l) {
        uint32_t x;
        if ((l & 1) == 0) {
            r = ghb_draw(stream, e * 32ULL + (uint64_t)(l >> 1));
            x = (uint32_t)(r >> 32);
        } else {
            x = (uint32_t)r;
        }
        uint32_t q = x < t.t0 ? 0u : (x < t.t1 ? 1u : (x < t.t2 ? 2u : 3u));
        u = (u << 1) | (q >> 1);
        v = (v << 1) | (q & 1u);
    }
    *src = u;
    *dst = v;
}

/* A bijection on [0, 2^bits): three rounds of (odd multiply + add) mod 2^bits
 * followed by an xorshift.  Each step is invertible on bits-bit integers. */
typedef struct {
    uint32_t mul[3], add[3];
    uint32_t mask;
    int shift;
    int bits;
} ghb_perm;

GHB_HD ghb_perm ghb_perm_make(uint64_t seed, int bits) {
    ghb_perm p;
    uint64_t s = ghb_stream(seed, GHB_PURPOSE_PERM);
    for (int i = 0; i < 3; ++i) {
        uint64_t r = ghb_draw(s, (uint64_t)i);
        p.mul[i] = ((uint32_t)r) | 1u;
        p.add[i] = (uint32_t)(r >> 32);
    }
    p.bits = bits;
    p.mask = bits >= 32 ? 0xFFFFFFFFu : ((1u << bits) - 1u);
    p.shift = bits > 1 ? (bits + 1) / 2 : 1;
    return p;
}

GHB_HD uint32_t ghb_perm_apply(const ghb_perm* p, uint32_t x) {
    if (p->bits == 0) return 0;
    for (int i = 0; i < 3; ++i) {
        x = (x * p->mul[i] + p->add[i]) & p->mask;
        x ^= x >> p->shift;
    }
    return x;
}

/* Weight modes: 1 = uniform in (0, 1] with 53-bit resolution,
 *               2 = integer-valued in [1, 100]. */
#define GHB_WEIGHT_NONE 0
#define GHB_WEIGHT_UNIFORM01 1
#define GHB_WEIGHT_INT100 2

GHB_HD double ghb_pair_weight(uint64_t wstream, uint32_t u, uint32_t v, int mode) {
    uint32_t lo = u < v ? u : v, hi = u < v ? v : u;
    uint64_t r = ghb_draw(wstream, ((uint64_t)lo << 32) | (uint64_t)hi);
    if (mode == GHB_WEIGHT_INT100) return (double)(1 + (r % 100ULL));
    if (mode == GHB_WEIGHT_UNIFORM01) return (double)((r >> 11) + 1ULL) * (1.0 / 9007199254740992.0);
    return 1.0;
}

/* Erdos-Renyi G(n, m) edge e: endpoints uniform in [0, n) by Lemire's
 * multiply-shift reduction of two 32-bit halves. */
GHB_HD void ghb_er_edge(uint64_t stream, uint32_t n, uint64_t e, uint32_t* src, uint32_t* dst) {
    uint64_t r = ghb_draw(stream, e);
    *src = (uint32_t)(((r >> 32) * (uint64_t)n) >> 32);
    *dst = (uint32_t)(((r & 0xFFFFFFFFULL) * (uint64_t)n) >> 32);
}

/* Dangling vertices for the PageRank precision workload: vertex v loses all
 * its out-edges when a 32-bit draw of (seed, v) is below fraction * 2^32. */
GHB_HD int ghb_is_dangling(uint64_t dstream, uint32_t v, uint32_t threshold) {
    return (uint32_t)(ghb_draw(dstream, v) >> 32) < threshold;
}

#endif /* GHB_GEN_H */
