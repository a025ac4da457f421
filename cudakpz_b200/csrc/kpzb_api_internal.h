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
// (0 = shape heuristic), the measured cost when it came from the tuner, the pass kernel
// (band: scabit_fused_kernel, stream: scabit_stream_kernel, wave: scabit_wave_kernel, strip:
// scabit_strip_kernel) and, for the strip kernel, the output rows of a tile.
enum PassKernel { PASS_BAND = 0, PASS_STREAM = 1, PASS_WAVE = 2, PASS_STRIP = 3 };
struct Plan {
    int k;
    int cps;
    float ms_per_mcs;
    bool tuned;
    int kind;
    int band = 0;
};
// Pass kernel and CTAs per SM for an explicitly set fusion depth: the streaming kernel with one
// chunk per SM, unless the environment variable KPZB_PASS_KERNEL says "band" / "band1".."band3"
// (the band kernel, the shape heuristic's or the given CTAs per SM), "stream2" (two chunks per
// SM), "wave" / "wave1".."wave3" (the register-wavefront kernel, 2 or the given CTAs per SM) or
// "strip" / "strip<rows>" (the warp-tile kernel, tiles of 64 or the given output rows), or
// that shape does not fit.
Plan explicit_plan(int lx, int ly, int k, int sm_count);
bool plan_shape_ok(const Plan& p, int lx, int ly, int sm_count);
bool lookup_plan(int lx, int ly, uint64_t Tp, uint64_t Tq, int sm_count, Plan* out);
Plan default_plan(int lx, int ly, uint64_t Tp, uint64_t Tq, int sm_count);
cudaError_t tune_plan(uint32_t* d_src, int lx, int ly, uint64_t seed, uint32_t stream_id,
                      uint64_t Tp, uint64_t Tq, int sm_count, unsigned int* d_err,
                      cudaStream_t st, Plan* out);

// Philox4x32-10 on the host (the same bijection as the device stream).
void philox_host(const uint32_t ctr[4], uint64_t seed, uint32_t out[4]);

// Double-tiling random-sequential scheduler state (dt.cu).
// DT_SCHEME_DB4 is not an inner scheme of DT but the reference's DB4 scheduler
// (Kpz::Scheduler<Rng, LocalLayoutDB4>): every block at once behind a dead border.
enum DtScheme {
    DT_SCHEME_DT = 0,
    DT_SCHEME_DBSH = 1,
    DT_SCHEME_DB = 2,
    DT_SCHEME_DTDBSH = 3,
    DT_SCHEME_DBSHREP = 4,
    DT_SCHEME_DB4 = 5
};
struct DtState {
    int grid = 0;
    bool ready = false;
    int scheme = DT_SCHEME_DBSH;  // inner decomposition of a block (the reference's default)
};
kpzb_status dt_init(DtState* s, int lx, int ly, int sm_count, bool db4 = false);
void dt_free(DtState* s);
// dis (optional): ENC_LOCAL rate-class words; dis_Tp / dis_Tq: the four classes' thresholds
kpzb_status dt_enqueue(DtState* s, uint32_t* d_local, int lx, int ly, uint64_t t0, int n,
                       double p, double q, uint64_t seed, uint32_t stream, cudaStream_t st,
                       unsigned long long* d_counters, const uint32_t* dis = nullptr,
                       const uint64_t* dis_Tp = nullptr, const uint64_t* dis_Tq = nullptr);

}  // namespace kpzb
