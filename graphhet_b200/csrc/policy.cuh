// Learned schedule policy: features of a traversal level and the decision
// hooks used by the BFS / SSSP drivers.
#pragma once

#include <cmath>

#include "common.cuh"

namespace ghb {

// The 12 policy features of one BFS level (also the first 12 trace columns):
//  0 log2(1+n_f)      frontier vertices
//  1 log2(1+m_f)      frontier out-edges
//  2 log2(1+m_u)      edges of unvisited vertices
//  3 level index
//  4 log2(1+mean frontier degree)
//  5 log2(1+frontier degree variance)
//  6 log2(1+max frontier degree)
//  7 log2(n)
//  8 log2(1+m)
//  9 previous direction (0 push, 1 pull)
// 10 log2(1+1000*previous level ms)
// 11 log2(1+n_f) - log2(n)
inline void bfs_features(float* f, int64_t n, int64_t m, int64_t n_f, int64_t m_f, int64_t m_u,
                         int level, double deg2, double degmax, int prev_dir, float prev_ms) {
    const double nf = (double)n_f > 0 ? (double)n_f : 0.0;
    const double mean = nf > 0 ? (double)m_f / nf : 0.0;
    double var = nf > 0 ? deg2 / nf - mean * mean : 0.0;
    if (var < 0) var = 0;
    f[0] = (float)std::log2(1.0 + nf);
    f[1] = (float)std::log2(1.0 + (double)m_f);
    f[2] = (float)std::log2(1.0 + (double)(m_u > 0 ? m_u : 0));
    f[3] = (float)level;
    f[4] = (float)std::log2(1.0 + mean);
    f[5] = (float)std::log2(1.0 + var);
    f[6] = (float)std::log2(1.0 + degmax);
    f[7] = (float)std::log2((double)(n > 0 ? n : 1));
    f[8] = (float)std::log2(1.0 + (double)m);
    f[9] = (float)prev_dir;
    f[10] = (float)std::log2(1.0 + 1000.0 * (double)prev_ms);
    f[11] = f[0] - f[7];
}

// Direction from the loaded policy network (0 push, 1 pull), or -1 when no
// network is loaded (the caller keeps the heuristic's choice).
int policy_pick_direction(const float* features);

// SSSP bucket width from the loaded network, or a negative value when no
// network is loaded.
double policy_pick_delta(const float* features, double base_delta);

}  // namespace ghb
