// GPU_gpma.hpp - drop-in GPMA for GraphHET's dynamic-graph path, backed by
// libghb's dynamic graph (ghb_gpma_*, include/ghb.h).
//
// The interface of the reference's include/GPU_gpma/GPU_gpma.hpp as its
// drivers use it (LDBC_GPU_gpma.cu, GPU_gpma_example.cu): the KEY / VALUE /
// SIZE types, constants and block-count macros (GPU_gpma.hpp:17-40), the
// thrust vector typedefs and RAW_PTR, class GPMA (:42-70) with row_num,
// row_offset, get_size() and get_V(), init_csr_gpma (:911-928),
// init_gpma_from_csr (:851-909) and update_gpma (:756-824).
//
// The graph lives in libghb (rows with slack in one arena, updated by sorted
// batches; see ghb.h); class GPMA holds its handle, and copies are deep, as
// the reference's thrust vectors are.  What differs from the reference:
//  * the packed key / value arrays are not exposed (the algorithm headers in
//    GPU_gpma/algorithm read a compact CSR of the graph instead);
//  * get_size() counts live entries, not array slots; get_V() is
//    row_num + 1, the reference's row_offset.size();
//  * row_offset is kept for source compatibility (the drivers assign it
//    before loading) and is not read;
//  * update_gpma leaves the caller's vectors as they were (the reference
//    sorts and compacts them in place);
//  * repeated keys inside one batch: the last occurrence wins.
// Update semantics otherwise match: value VALUE_NONE (0) deletes a present
// key, any other value overwrites a present key's weight or inserts it.
#pragma once

#include <thrust/device_vector.h>
#include <thrust/host_vector.h>

#include <algorithm>
#include <cstdio>

#include <ghb.h>

typedef unsigned long long KEY_TYPE;
typedef double VALUE_TYPE;
typedef unsigned int SIZE_TYPE;

typedef thrust::device_vector<KEY_TYPE> DEV_VEC_KEY;
typedef thrust::device_vector<VALUE_TYPE> DEV_VEC_VALUE;
typedef thrust::device_vector<SIZE_TYPE> DEV_VEC_SIZE;

typedef KEY_TYPE* KEY_PTR;
typedef VALUE_TYPE* VALUE_PTR;

#ifndef RAW_PTR
#define RAW_PTR(x) thrust::raw_pointer_cast((x).data())
#endif

const KEY_TYPE KEY_NONE = 0xFFFFFFFFFFFFFFFFull;
const KEY_TYPE KEY_MAX = 0xFFFFFFFFFFFFFFFEull;
const KEY_TYPE KEY_HIGH = 0xFFFFFFFF00000000ull;
const SIZE_TYPE SIZE_NONE = 0xFFFFFFFFu;
const VALUE_TYPE VALUE_NONE = 0;
const KEY_TYPE COL_IDX_NONE = 0xFFFFFFFFull;
const SIZE_TYPE MAX_BLOCKS_NUM = 96 * 8;

#ifndef CALC_BLOCKS_NUM_NOLIMIT
#define CALC_BLOCKS_NUM_NOLIMIT(ITEMS_PER_BLOCK, CALC_SIZE) (((CALC_SIZE) - 1) / (ITEMS_PER_BLOCK) + 1)
#endif
#ifndef CALC_BLOCKS_NUM
#define CALC_BLOCKS_NUM(ITEMS_PER_BLOCK, CALC_SIZE) \
    std::min<SIZE_TYPE>(MAX_BLOCKS_NUM, ((CALC_SIZE) - 1) / (ITEMS_PER_BLOCK) + 1)
#endif

namespace ghb_gpma_dropin {

// Failures are printed and the call returns, as the reference's cErr does
// (GPU_gpma.hpp:9-15).
inline bool ok(int status, const char* what) {
    if (status != GHB_OK) {
        std::fprintf(stderr, "%s failed: %s (%s)\n", what, ghb_status_string(status), ghb_last_error());
        return false;
    }
    return true;
}

inline ghb_workspace* workspace() {
    ghb_workspace* ws = ghb_default_workspace();
    if (ws) ghb_workspace_set_stream(ws, nullptr);
    return ws;
}

}  // namespace ghb_gpma_dropin

#ifndef cErr
#define cErr(errcode)                                                                                   \
    do {                                                                                                \
        cudaError_t _ghb_e = (errcode);                                                                 \
        if (_ghb_e != cudaSuccess)                                                                      \
            std::printf("GPUassert: %s %s %d\n", cudaGetErrorString(_ghb_e), __FILE__, __LINE__);      \
    } while (0)
#endif

class GPMA {
public:
    SIZE_TYPE row_num = 0;
    DEV_VEC_SIZE row_offset;
    ghb_gpma* handle = nullptr;

    GPMA() = default;
    GPMA(const GPMA& o) : row_num(o.row_num), row_offset(o.row_offset) { clone_from(o); }
    GPMA& operator=(const GPMA& o) {
        if (this != &o) {
            release();
            row_num = o.row_num;
            row_offset = o.row_offset;
            clone_from(o);
        }
        return *this;
    }
    ~GPMA() { release(); }

    // Live entries (the reference: array slots, gaps included).
    inline int get_size() {
        int64_t m = 0;
        if (handle) ghb_gpma_info(handle, nullptr, &m, nullptr, nullptr);
        return (int)m;
    }
    // row_num + 1, the size of the reference's row_offset.
    inline int get_V() { return (int)row_num + 1; }

private:
    void clone_from(const GPMA& o) {
        if (o.handle)
            ghb_gpma_dropin::ok(ghb_gpma_clone(ghb_gpma_dropin::workspace(), o.handle, &handle), "ghb_gpma_clone");
    }
    void release() {
        if (handle) ghb_gpma_destroy(handle);
        handle = nullptr;
    }
};

// An empty graph over row_num vertices.
inline void init_csr_gpma(GPMA& gpma, SIZE_TYPE row_num) {
    gpma.row_num = row_num;
    gpma.row_offset.assign((size_t)row_num + 1, 0);
    if (gpma.handle) ghb_gpma_destroy(gpma.handle);
    gpma.handle = nullptr;
    ghb_gpma_dropin::ok(ghb_gpma_create(ghb_gpma_dropin::workspace(), (int32_t)std::max<SIZE_TYPE>(row_num, 1),
                                        &gpma.handle),
                        "ghb_gpma_create");
}

// One batch of updates: key (row << 32) | col, value 0 deletes.
inline void update_gpma(GPMA& gpma, DEV_VEC_KEY& update_keys, DEV_VEC_VALUE& update_values) {
    if (!gpma.handle) {
        std::fprintf(stderr, "update_gpma: GPMA not initialised (init_csr_gpma)\n");
        return;
    }
    const int64_t count = (int64_t)std::min(update_keys.size(), update_values.size());
    ghb_workspace* ws = ghb_gpma_dropin::workspace();
    if (ghb_gpma_dropin::ok(ghb_gpma_update(ws, gpma.handle, reinterpret_cast<const uint64_t*>(RAW_PTR(update_keys)),
                                            RAW_PTR(update_values), count, nullptr),
                            "ghb_gpma_update"))
        cudaStreamSynchronize(nullptr);
}

// Replace the contents with the given entries; returns their count.
inline int init_gpma_from_csr(GPMA& gpma, DEV_VEC_KEY& init_keys, DEV_VEC_VALUE& init_values) {
    if (!gpma.handle) init_csr_gpma(gpma, gpma.row_offset.empty() ? 1 : (SIZE_TYPE)gpma.row_offset.size() - 1);
    if (!gpma.handle) return 0;
    if (!ghb_gpma_dropin::ok(ghb_gpma_clear(ghb_gpma_dropin::workspace(), gpma.handle), "ghb_gpma_clear")) return 0;
    update_gpma(gpma, init_keys, init_values);
    return (int)init_keys.size();
}
