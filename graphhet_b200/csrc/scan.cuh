// Device-wide exclusive prefix sum (reduce, scan block totals, rescan).
#pragma once

#include "common.cuh"

namespace ghb {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int64_t kScanTile = kScanThreads * kScanItems;

inline int64_t scan_scratch_words(int64_t count) { return (count + kScanTile - 1) / kScanTile + 1; }

// out[i] = sum(in[0..i)), out[count] = total; `block_sums` holds
// scan_scratch_words(count) int64.  Sums must fit in int32.
int scan_exclusive_i32(ghb_workspace* ws, const int32_t* in, int32_t* out, int64_t count,
                       int64_t* block_sums);

}  // namespace ghb
