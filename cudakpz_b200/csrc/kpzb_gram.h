// kpzb_gram.h -- tensor-core limb Gram (gram_tc.cu) used by the correlator (gram.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/kpzb.h"
#include "gram_slope.cuh"

namespace kpzb {

struct GramTC {
    int64_t* d_part = nullptr;            // per-CTA partial limb Grams, [grid][192][192]
    int64_t* d_out = nullptr;             // reduced limb Gram, [192][192]
    unsigned int* d_err = nullptr;        // bounded-wait flag
    int grid = 0;
    bool ready = false;
};

// Buffers for the limb Gram of N sites (N multiple of 128, N <= 2^30).
kpzb_status gram_tc_setup(GramTC* tc, uint64_t N, int sm_count);
void gram_tc_free(GramTC* tc);
// Upper triangle (row <= col) of the 192 x 192 limb Gram of the snapshots in g, exact, into
// host out[192*192].
kpzb_status gram_tc_run(GramTC* tc, const SlopeSnapGeom& g, uint64_t N, int64_t* out, cudaStream_t st);

}  // namespace kpzb
