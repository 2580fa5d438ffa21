// Learned schedule policy: the features of a traversal level, the network's
// parameter layout, and its block-wide evaluation inside a kernel.
#pragma once

#include <cmath>

#include "common.cuh"

namespace ghb {

// Network 12 -> 64 -> 64 (ReLU) -> 20, row-major x @ W, then the
// normalisation (mean[12], 1/std[12]) after the parameters.
constexpr int kPolIn = 12, kPolH = 64, kPolOut = 20;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kPolIn * kPolH, kOffW2 = kOffB1 + kPolH, kOffB2 = kOffW2 + kPolH * kPolH,
              kOffW3 = kOffB2 + kPolH, kOffB3 = kOffW3 + kPolH * kPolOut, kPolParams = kOffB3 + kPolOut;
constexpr int kOffNorm = kPolParams;            // mean[12], inv_std[12]
constexpr int kPolTotal = kPolParams + 2 * kPolIn;  // floats on the device
// Heads: [0,2) direction, [2,4) top-down output format, [4,20) SSSP width bin.
constexpr int kHeadDir = 0, kHeadFmt = 2, kHeadDelta = 4, kDeltaBins = 16, kDeltaBinZero = 6;

// The 12 policy features of one BFS level (also the first 12 trace
// columns), scale-free so that a network trained on scales 16-22 reads a
// scale-24 graph's levels in the same ranges.  (Giving it the graph's size
// instead, as log2(m), made its decisions at scale 24 extrapolations: it
// pushed on levels whose frontier held a hundred times the unexplored
// entries.)
//  0 log2(1+n_f) - log2(n)          frontier share of the vertices
//  1 log2(1+m_f) - log2(1+m)        frontier share of the entries
//  2 log2(1+m_u) - log2(1+m)        unexplored share of the entries
//  3 log2(1+m_f) - log2(1+m_u)      the direction rule's ratio
//  4 log2(1+mean frontier degree) - log2(1+m/n)
//  5 log2(1+std of frontier degree) - log2(1+mean frontier degree)
//  6 log2(1+max frontier degree) - log2(1+m/n)
//  7 log2(1+level)
//  8 log2(1+m/n)                    mean degree of the graph
//  9 previous direction (0 push, 1 pull)
// 10 log2(1+n_f) - log2(1+n_f of the previous level)   frontier growth
// 11 log2(1+unvisited) - log2(n)    unvisited share of the vertices
// One definition for the host-driven loop and the persistent kernel.
__host__ __device__ inline void bfs_features(float* f, double n, double m, double n_f, double m_f, double m_u,
                                             int level, double deg2, double degmax, int prev_dir, double n_f_prev,
                                             double unvisited) {
    const double nf = n_f > 0 ? n_f : 0.0;
    const double mean = nf > 0 ? m_f / nf : 0.0;
    double var = nf > 0 ? deg2 / nf - mean * mean : 0.0;
    if (var < 0) var = 0;
    const double nn = n > 0 ? n : 1.0;
    const float lm = log2f((float)(1.0 + m));
    const float ln = log2f((float)nn);
    const float lmean_g = log2f((float)(1.0 + m / nn));
    const float lnf = log2f((float)(1.0 + nf));
    const float lmf = log2f((float)(1.0 + m_f));
    const float lmu = log2f((float)(1.0 + (m_u > 0 ? m_u : 0.0)));
    const float lmean = log2f((float)(1.0 + mean));
    f[0] = lnf - ln;
    f[1] = lmf - lm;
    f[2] = lmu - lm;
    f[3] = lmf - lmu;
    f[4] = lmean - lmean_g;
    f[5] = log2f((float)(1.0 + sqrt(var))) - lmean;
    f[6] = log2f((float)(1.0 + degmax)) - lmean_g;
    f[7] = log2f((float)(1 + (level > 0 ? level : 0)));
    f[8] = lmean_g;
    f[9] = (float)prev_dir;
    f[10] = lnf - log2f((float)(1.0 + (n_f_prev > 0 ? n_f_prev : 0.0)));
    f[11] = log2f((float)(1.0 + (unvisited > 0 ? unvisited : 0.0))) - ln;
}

// The features of one SSSP call (one width decision per traversal): shares
// and ratios, plus the graph's size (feature 10); feature 3 is -1 to tell
// them from BFS levels:
//  0 log2(1+deg(src)) - log2(1+mean degree)
//  1 log2(1+mean degree)
//  2 log2(1+std of degree) - log2(1+mean degree)
//  3 -1
//  4 log2(1+max degree) - log2(1+mean degree)
//  5 log2(vertices with entries) - log2(n)
//  6 log2((max weight - min weight) / mean weight + 1/64)
//  7 log2(mean weight / base width)
//  8 log2(max weight / mean weight)
//  9 log2(mean weight / min weight)
// 10 log2(1+m)   size of the graph: the best width narrows as the graph's
//    diameter grows (grids: about 14 at 256 x 256, 11 at 2048 x 2048)
// 11 log2(1+deg(src)) - log2(1+max degree)
__host__ __device__ inline void sssp_features(float* f, double n, double m, double n_active, double deg_src,
                                              double deg2_sum, double degmax, double w_mean, double w_min,
                                              double w_max, double base_delta) {
    const double na = n_active > 0 ? n_active : 1.0;
    const double mean = m / na;
    double var = deg2_sum / na - mean * mean;
    if (var < 0) var = 0;
    const double tiny = 1e-300;
    const float lmean = log2f((float)(1.0 + mean));
    const float lsrc = log2f((float)(1.0 + deg_src));
    const float lmax = log2f((float)(1.0 + degmax));
    f[0] = lsrc - lmean;
    f[1] = lmean;
    f[2] = log2f((float)(1.0 + sqrt(var))) - lmean;
    f[3] = -1.0f;
    f[4] = lmax - lmean;
    f[5] = log2f((float)na) - log2f((float)(n > 0 ? n : 1.0));
    f[6] = (float)log2((w_max - w_min) / (w_mean + tiny) + 1.0 / 64.0);
    f[7] = (float)log2((w_mean + tiny) / (base_delta + tiny));
    f[8] = (float)log2((w_max + tiny) / (w_mean + tiny));
    f[9] = (float)log2((w_mean + tiny) / (w_min + tiny));
    f[10] = log2f((float)(1.0 + m));
    f[11] = lsrc - lmax;
}

// How far, in log2 units, the direction rule's test is from its threshold
// at a level: the rule pulls when m_f > m_u / alpha and m_f > m / gamma, and
// returns to push when n_f < n / beta.  With the learned policy the network
// chooses a level's direction and output format only where this is below
// the band (the rule's uncertain zone); farther out the rule's choices
// stand, so a network reading a graph unlike its training family cannot,
// say, push a level whose frontier holds many times the unexplored entries.
__host__ __device__ inline float rule_margin(int dir, double n, double m, double n_f, double m_f, double m_u,
                                             float alpha, float beta, float gamma) {
    const float lo = 0.5f;
    if (dir == 0) {
        const float lmf = log2f(fmaxf((float)m_f, lo));
        const float a = lmf - log2f(fmaxf((float)(m_u / alpha), lo));
        const float b = lmf - log2f(fmaxf((float)(m / gamma), lo));
        return fabsf(fminf(a, b));
    }
    return fabsf(log2f(fmaxf((float)(n / beta), lo)) - log2f(fmaxf((float)n_f, lo)));
}

// Block-wide evaluation for one feature row.  P: kPolTotal floats (shared or
// global); feat: 12 floats, h1/h2: 64, logits: 20, all in shared memory.
// Needs blockDim.x >= 512; every thread of the block must call it.
__device__ __forceinline__ void policy_eval_block(const float* P, const float* feat, float* h1, float* h2,
                                                  float* logits) {
    const int t = threadIdx.x;
    if (t < kPolH) {
        float z = P[kOffB1 + t];
#pragma unroll
        for (int i = 0; i < kPolIn; ++i)
            z = fmaf((feat[i] - P[kOffNorm + i]) * P[kOffNorm + kPolIn + i], P[kOffW1 + i * kPolH + t], z);
        h1[t] = fmaxf(z, 0.f);
    }
    __syncthreads();
    if (t < 512) {
        // 8 threads per output, 8 inputs each, reduced across the 8 lanes.
        const int o = t >> 3, part = t & 7;
        float z = 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k) z = fmaf(h1[part * 8 + k], P[kOffW2 + (part * 8 + k) * kPolH + o], z);
        z += __shfl_xor_sync(0xffffffffu, z, 1);
        z += __shfl_xor_sync(0xffffffffu, z, 2);
        z += __shfl_xor_sync(0xffffffffu, z, 4);
        if (part == 0) h2[o] = fmaxf(z + P[kOffB2 + o], 0.f);
    }
    __syncthreads();
    if (t < kPolOut * 8) {
        const int o = t >> 3, part = t & 7;
        float z = 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k) z = fmaf(h2[part * 8 + k], P[kOffW3 + (part * 8 + k) * kPolOut + o], z);
        z += __shfl_xor_sync(0xffffffffu, z, 1);
        z += __shfl_xor_sync(0xffffffffu, z, 2);
        z += __shfl_xor_sync(0xffffffffu, z, 4);
        if (part == 0) logits[o] = z + P[kOffB3 + o];
    }
    __syncthreads();
}

// Device copy of the installed network for the current device (kPolTotal
// floats), or nullptr when none is installed.
const float* policy_device_params();

// Host evaluation of the installed network: direction (0 push, 1 pull) and
// top-down output format (0 queue, 1 bitmap).  False when none is installed.
bool policy_pick_level(const float* features, int* dir, int* fmt);

// SSSP bucket width from the installed network (base_delta * 2^(bin-6)), or
// a negative value when none is installed.
double policy_pick_delta(const float* features, double base_delta);

}  // namespace ghb
