// Shared helpers of the drop-in GPMA algorithm headers (host side only):
// the compact CSR that libghb keeps for a dynamic graph, and result buffers.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include <GPU_csr/GPU_csr.hpp>
#include <GPU_csr/algorithm/ghb_dropin_util.hpp>
#include <GPU_gpma/GPU_gpma.hpp>

namespace ghb_gpma_dropin {

// Device pointers of a GPMA's compact CSR (rows sorted by column); valid
// until the next update of that GPMA.
struct CsrView {
    int n = 0;
    const int32_t* rowptr = nullptr;
    const int32_t* col = nullptr;
    const double* w = nullptr;
    bool valid = false;
};

inline CsrView csr_of(GPMA& gpma, bool weights) {
    CsrView v;
    if (!gpma.handle) {
        std::fprintf(stderr, "GPMA not initialised (init_csr_gpma)\n");
        return v;
    }
    int32_t n = 0;
    ghb_gpma_info(gpma.handle, &n, nullptr, nullptr, nullptr);
    v.n = n;
    v.valid = ok(ghb_gpma_csr(workspace(), gpma.handle, weights ? 1 : 0, &v.rowptr, &v.col, &v.w), "ghb_gpma_csr");
    return v;
}

}  // namespace ghb_gpma_dropin
