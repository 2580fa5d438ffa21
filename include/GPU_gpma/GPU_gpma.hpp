// GPU_gpma.hpp - type-only stand-in for the reference's
// include/GPU_gpma/GPU_gpma.hpp, of which the CSR path uses only the
// typedefs and block-count macros (GPU_gpma.hpp:17-40).  The GPMA+ dynamic
// graph itself is not part of this library; GPMA is declared so that
// prototypes naming it still parse.
#pragma once

#include <algorithm>

typedef unsigned long long KEY_TYPE;
typedef double VALUE_TYPE;
typedef unsigned int SIZE_TYPE;

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

class GPMA;
