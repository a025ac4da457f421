// kpzb_api_internal.h -- declarations shared between api.cu and the scheduler units.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/kpzb.h"

namespace kpzb {

kpzb_status fail(kpzb_status s, const char* what);
kpzb_status cuda_fail(cudaError_t e, const char* where);
int sm_count_of(int device);

// MCS per HBM pass picked for a lattice when the caller leaves fusion at 0.
int auto_fusion(int lx, int ly);

// SCABit pass shape: k MCS per HBM pass (1 = one launch per half-step), cps CTAs per SM
// (0 = shape heuristic), and the measured cost when it came from the tuner.
struct Plan {
    int k;
    int cps;
    float ms_per_mcs;
    bool tuned;
};
bool lookup_plan(int lx, int ly, uint64_t Tp, uint64_t Tq, int sm_count, Plan* out);
Plan default_plan(int lx, int ly);
cudaError_t tune_plan(uint32_t* d_src, int lx, int ly, uint64_t seed, uint32_t stream_id,
                      uint64_t Tp, uint64_t Tq, int sm_count, unsigned int* d_err,
                      cudaStream_t st, Plan* out);

// Double-tiling random-sequential scheduler state (dt.cu).
struct DtState {
    int grid = 0;
    bool ready = false;
};
kpzb_status dt_init(DtState* s, int lx, int ly, int sm_count);
void dt_free(DtState* s);
kpzb_status dt_enqueue(DtState* s, uint32_t* d_local, int lx, int ly, uint64_t t0, int n,
                       double p, double q, uint64_t seed, uint32_t stream, cudaStream_t st,
                       unsigned long long* d_counters);

}  // namespace kpzb
