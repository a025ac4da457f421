// kpzb_internal.h -- host-side declarations shared by the kpzb translation units.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace kpzb {

struct ScabitShape {
    int TX, TY, grid;
};

ScabitShape scabit_shape(int lx, int ly, int sm_count);
cudaError_t scabit_half(uint32_t* d_sys, int lx, int ly, int sigma, uint32_t step, uint64_t seed,
                        uint32_t stream_id, uint64_t Tp, uint64_t Tq, const ScabitShape& sh,
                        unsigned long long* d_counters, cudaStream_t st);

// Quenched disorder: one half-step with per-site rate classes (d_dis_cbbit: the class words in
// ENC_CBBIT form), thresholds Tp[c], Tq[c] for classes c = 0..3.
cudaError_t scabit_half_dis(uint32_t* d_sys, const uint32_t* d_dis_cbbit, int lx, int ly, int sigma,
                            uint32_t step, uint64_t seed, uint32_t stream_id, const uint64_t Tp[4],
                            const uint64_t Tq[4], const ScabitShape& sh, unsigned long long* d_counters,
                            cudaStream_t st);

// Temporal-blocked SCABit: k MCS (2k half-steps) per HBM pass over a band of rows.
struct FusedShape {
    int band;      // output rows per CTA band
    int halo;      // halo rows each side (= 2 * mcs_per_pass)
    int mcs;       // MCS per pass
    int threads;   // threads per CTA
    size_t smem;   // dynamic shared memory bytes
    int grid;
    bool ok;
};
FusedShape scabit_fused_shape(int lx, int ly, int mcs_per_pass, int sm_count, size_t smem_optin);
FusedShape scabit_fused_shape_cps(int lx, int ly, int mcs_per_pass, int ctas_per_sm,
                                  size_t smem_optin);
cudaError_t scabit_fused(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0,
                         uint64_t seed, uint32_t stream_id, uint64_t Tp, uint64_t Tq,
                         const FusedShape& sh, unsigned long long* d_counters, unsigned int* d_err,
                         cudaStream_t st);

// Streaming (wavefront) temporal blocking: k MCS per HBM pass, a chunk of rows per CTA.
struct StreamShape {
    int mcs;       // MCS per pass
    int slots;     // ring slots (rows of all four quadrants) in shared memory
    int prefetch;  // rows loaded ahead of first use (beyond the one-tick minimum)
    int threads;   // threads per CTA
    size_t smem;   // dynamic shared memory bytes
    int grid;      // chunks (CTAs)
    bool ok;
};
StreamShape scabit_stream_shape(int lx, int ly, int mcs_per_pass, int sm_count, int ctas_per_sm);
cudaError_t scabit_stream(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0,
                          uint64_t seed, uint32_t stream_id, uint64_t Tp, uint64_t Tq,
                          const StreamShape& sh, unsigned long long* d_counters, unsigned int* d_err,
                          cudaStream_t st);

// Register-wavefront temporal blocking (scabit_wave.cu): k MCS per HBM pass, one CTA per band
// of rows spanning the full quadrant-row width, the half-steps in registers.
struct WaveShape {
    int mcs;       // MCS per pass (2, 4, 6 or 8)
    int cps;       // CTAs per SM the bands and registers are sized for
    int threads;   // threads per CTA = words per quadrant row
    int band;      // output rows per CTA
    int grid;      // bands (CTAs)
    size_t smem;   // dynamic shared memory bytes
    bool ok;
};
// mode: the DecMode of the rates (the kernel covers DEC_NONE and DEC_ONE)
WaveShape scabit_wave_shape(int lx, int ly, int mcs_per_pass, int sm_count, int ctas_per_sm, int mode);
cudaError_t scabit_wave(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0, uint64_t seed,
                        uint32_t stream_id, uint64_t Tp, uint64_t Tq, const WaveShape& sh,
                        unsigned long long* d_counters, unsigned int* d_err, cudaStream_t st);

// Warp-tile register-wavefront temporal blocking (scabit_strip.cu): k MCS per HBM pass, one
// warp per tile of a 32-column strip of a quadrant row and a band of rows, the half-steps in
// registers; strips overlap by two columns (one recomputed column each side).
struct StripShape {
    int mcs;           // MCS per pass (4, 6 or 8)
    int band;          // output rows per tile
    int nstrips;       // strips per quadrant row
    int ntiles;        // strips x bands (warps)
    int grid;          // CTAs
    int threads;       // threads per CTA
    bool random_plane; // strips laid out for rates with one random plane (DEC_ONE)
    bool ok;
};
// mode: the DecMode of the rates (the kernel covers DEC_NONE and DEC_ONE); band_rows even.
// A tile runs whole cycles of strip_cycle_rows(k) ticks over its band + 4k halo rows, so band
// heights of m * strip_cycle_rows(k) - 4k rows waste no tick.
int strip_cycle_rows(int mcs_per_pass);
StripShape scabit_strip_shape(int lx, int ly, int mcs_per_pass, int band_rows, int mode);
cudaError_t scabit_strip(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0, uint64_t seed,
                         uint32_t stream_id, uint64_t Tp, uint64_t Tq, const StripShape& sh,
                         unsigned long long* d_counters, cudaStream_t st);

// codec / init
cudaError_t init_homogeneous_dev(uint32_t* d, int lx, int ly, int encoding, cudaStream_t st);
cudaError_t local_to_cbbit_dev(const uint32_t* local, uint32_t* cbbit, int lx, int ly, cudaStream_t st);
cudaError_t cbbit_to_local_dev(const uint32_t* cbbit, uint32_t* local, int lx, int ly, cudaStream_t st);

// analysis on ENC_CBBIT lattices
struct AnalysisScratch {
    int32_t* rowinfo;      // 2 * rows: y-slope step at x=0 and x-slope row sum
    int64_t* rowstart;     // rows: height at the start of each row walk
    unsigned long long* acc;  // accumulators (see analysis.cu)
    size_t rows_cap;
};
cudaError_t analysis_alloc(AnalysisScratch* s, int ly);
void analysis_free(AnalysisScratch* s);
// out_i64[0..2]: S1, S2, hmin/hmax packed; out_f64[0..4]: S3..S7; corr outputs optional
struct MomentsOut {
    int64_t s1, s2;
    double s3to7[5];
    int64_t hmin, hmax;
    int64_t cross;   // sum h_sys * h_snap (correlate mode)
    int64_t agree;   // sum of +-1 slope agreements (correlate mode)
    int64_t snap_s1; // sum h_snap (correlate mode)
};
cudaError_t analysis_moments(const uint32_t* d_sys, const uint32_t* d_snap, int lx, int ly,
                             AnalysisScratch* s, MomentsOut* out, cudaStream_t st);
// The same moments left on the device: the final reduction record is written to d_rec
// (analysis_record_bytes() bytes) on stream st, with no host synchronisation; decode a host
// copy with analysis_decode_record.
size_t analysis_record_bytes();
cudaError_t analysis_moments_record(const uint32_t* d_sys, const uint32_t* d_snap, int lx, int ly,
                                    AnalysisScratch* s, void* d_rec, cudaStream_t st);
void analysis_decode_record(const void* rec, MomentsOut* out);
cudaError_t analysis_heights(const uint32_t* d_sys, int lx, int ly, AnalysisScratch* s,
                             int32_t* d_heights, cudaStream_t st);
// invariants: rep[0] bad rows, rep[1] bad columns, rep[2] bad plaquettes
cudaError_t analysis_invariants(const uint32_t* d_sys, int lx, int ly, AnalysisScratch* s,
                                int64_t rep[3], cudaStream_t st);

}  // namespace kpzb
