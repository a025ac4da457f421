/*
 * kpzb.h -- C ABI of libkpzb200.so, a B200 (sm_100a) implementation of the CudaKpz
 * octahedron-model KMC hot path.  Plain pointers and sizes only; every call returns a
 * kpzb_status; no exceptions, no exit().  File:line references point into CudaKpz.
 *
 * Lattices use the reference's word layouts exactly:
 *   ENC_LOCAL  (kpz/systemSize.h:94-124): 4x4 sites per uint32, word (y>>2)*(L/4)+(x>>2),
 *              bit ((x&3)<<1)|((y&3)<<3); bit0 = x-slope, bit1 = y-slope.
 *   ENC_CBBIT  (kpz/systemSize.h:143-165): quadrants [sub0.X|sub0.Y|sub1.X|sub1.Y] of
 *              N/64 words; site (x,y) of sublattice (x^y)&1 at word (y*L+x)>>6 of its
 *              quadrant, bit (x>>1)&31.
 *
 * Random numbers come from a counter-based stream (Philox4x32-10 keyed by the 64-bit
 * seed; counter = quadrant word group, half-step, bit plane, stream id), so results do
 * not depend on the launch geometry and a CPU restatement reproduces them bit for bit.
 *
 * Handles are not thread-safe; distinct handles are independent.  Each handle owns one
 * CUDA stream and all of its device memory.
 */
#ifndef KPZB_H
#define KPZB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    KPZB_OK = 0,
    KPZB_EINVAL = 1,      /* bad argument (size out of range, bad encoding, null pointer) */
    KPZB_ENOMEM = 2,      /* device or pinned allocation failed */
    KPZB_ECUDA = 3,       /* CUDA runtime error; kpzb_last_error() has the text */
    KPZB_ETIMEOUT = 4,    /* a bounded device wait expired */
    KPZB_ESTATE = 5,      /* call not valid in the current state (e.g. no snapshot) */
    KPZB_EUNSUPPORTED = 6 /* combination not implemented (e.g. DT on ENC_CBBIT) */
} kpzb_status;

/* Encodings, as Kpz::SchedulerService::Encoding (kpz/schedulerService.h:71). */
enum { KPZB_ENC_LOCAL = 0, KPZB_ENC_CBBIT = 1 };

/* Dynamics, as the GPU schedulers picked by SchedulerConfig::mkSchedulerGPU
 * (kpz/kpzFrontend.cpp:355-403). */
enum {
    KPZB_DYN_SCA = 0,    /* Kpz::SchedulerSCA: checkerboard SCA, ENC_LOCAL push/pop      */
    KPZB_DYN_SCABIT = 1, /* Kpz::SchedulerSCABit: bit-vectorised SCA, ENC_CBBIT push/pop */
    KPZB_DYN_DT = 2,     /* Kpz::SchedulerDT: double-tiling random-sequential, ENC_LOCAL */
    KPZB_DYN_DB4 = 3     /* Kpz::Scheduler<Rng, LocalLayoutDB4> ("db4", kpz/scheduler.cu): all
                            256x128-site blocks at once behind a 5-site dead border, ENC_LOCAL */
};

typedef struct kpzb_handle kpzb_handle;

/* Text of the last error on this thread (empty when none). Replaces the mixed
 * KmcExcept::CUDAError throws / stderr messages (kpz/schedulerSCABit.cu:66-72). */
const char* kpzb_last_error(void);
/* Library version string. */
const char* kpzb_version(void);
/* Measured integer-ALU throughput of `device` (-1: current), in thread-level operations per
 * second: a 3-input LOP3 chain and a 3-input IADD3 chain over 8 CTAs of 256 threads per SM,
 * CUDA-event timed (a few ms).  The denominator of the INT roofline of the bitwise SCA
 * update.  No counterpart in the reference (a measurement helper). */
kpzb_status kpzb_probe_alu_peak(int device, double* lop3_per_s, double* iadd3_per_s);

/* Create a scheduler for a 2^lx x 2^ly lattice on `device` (-1: current device).
 * Replaces SchedulerSCA/SchedulerSCABit/SchedulerDT constructors + SchedulerBase::initCUDA
 * (kpz/schedulerSCABit.cu:84-88, kpz/schedulerBase.cu:65-74, kpz/schedulerDT.cu:93-118).
 * Limits: 8 <= lx <= 30, 2 <= ly <= 30, 14 <= lx + ly <= 38; DT also needs lx >= 9 and
 * ly >= 8 (one double tile of 512x256 sites), DB4 ly >= 7 (one block of 256x128 sites).
 * The lattice starts flat. */
kpzb_status kpzb_create(kpzb_handle** h, int lx, int ly, int dynamics, int device);
kpzb_status kpzb_destroy(kpzb_handle* h);

/* SchedulerService::initHomogeneous (kpz/schedulerService.cpp:156-175), in the handle's
 * encoding. Does not reset the MCS counters. */
kpzb_status kpzb_init_homogeneous(kpzb_handle* h);
/* SchedulerService::setPQ(p, q, 0) (kpz/schedulerService.h:186-192). 0 <= p,q <= 1. */
kpzb_status kpzb_set_pq(kpzb_handle* h, double p, double q);
/* Seeds the counter stream and resets the device MCS counter to 0. Replaces
 * SchedulerService::supplySeed + randomize (kpz/schedulerService.cpp:472-482,
 * kpz/GPUTinyMT.cu:74-103). `stream` separates replicas sharing a seed. */
kpzb_status kpzb_seed(kpzb_handle* h, uint64_t seed, uint32_t stream);

/* DT only: the inner decomposition of a block, the reference's compile-time KPZ_INNER_DD
 * (kpz/param.h, kpz/kpzConst.h:26-35): KPZB_DT_INNER_DBSH (single-hit dead border, the
 * reference's default build (kpz/param.h:36) and the default of a new DT handle:
 * BaseDTInnerDBSH, kpz/kpzSimulationPrimitivesTemplates_BaseInnerDB.cu:110-163),
 * KPZB_DT_INNER_DT (single-hit double tiling, about twice as fast; a different
 * decomposition, so W^2(t) differs from DBSH's by about 0.5 % at early times),
 * KPZB_DT_INNER_DB (dead border without the per-round cell offset: BaseDTInnerDB, :30-74),
 * KPZB_DT_INNER_DTDBSH (double tiling with a random per-round cell offset:
 * BaseDTInnerDTDBSH, kpz/kpzSimulationPrimitivesTemplates_BaseInnerDTr.cu:30-85) or
 * KPZB_DT_INNER_DBSHREP (DBSH with border hits replaced by fresh attempts after the rounds:
 * BaseDTInnerDBSHRep, kpz/kpzSimulationPrimitivesTemplates_BaseInnerDB.cu:165-268).  The
 * scheme is saved in checkpoints. */
enum {
    KPZB_DT_INNER_DT = 0,
    KPZB_DT_INNER_DBSH = 1,
    KPZB_DT_INNER_DB = 2,
    KPZB_DT_INNER_DTDBSH = 3,
    KPZB_DT_INNER_DBSHREP = 4
};
kpzb_status kpzb_set_dt_inner(kpzb_handle* h, int inner);
/* SchedulerService::mcsScale (kpz/schedulerService.h:241): the factor the frontend reports
 * beside MCS counts -- p + q of rate class 0 for SCA/SCABit (kpz/schedulerSCA.cu:36-39,
 * kpz/schedulerSCABit.cu:39-42), the active fraction (256-5)(128-5)/(256*128) of a block for
 * DB4 (kpz/scheduler.cu:57-65), 1 for DT. */
kpzb_status kpzb_mcs_scale(kpzb_handle* h, double* scale);
/* SchedulerService::setPQ(p, q, n) for rate class n = 0..3 (kpz/schedulerService.h:186-192):
 * the rates a site of disorder class n uses in kpzb_mcs_disorder; class 0 is kpzb_set_pq's.
 * Classes never set follow class 0. */
kpzb_status kpzb_set_pq_class(kpzb_handle* h, int n, double p, double q);
/* Quenched disorder (SchedulerService::m_disorder, generateDisorder2 at
 * kpz/schedulerService.cpp:54-71): one word per lattice word in ENC_LOCAL layout for every
 * dynamics; the 2 bits at a site's slope position are its rate class (generateDisorder2 sets
 * only the low bit: classes 0 and 1). */
kpzb_status kpzb_set_disorder(kpzb_handle* h, const uint32_t* local_words);
/* mcsDisorder2SyncRng(n) (kpz/schedulerService.h:212; SCA: Disorder2SyncRng,
 * kpz/kpzSCACores.cu:217-280; DT: caller_mcsDisorder2SyncRng, kpz/kpz.cu:238-246): n MCS in
 * which a candidate site flips with its class's rate.  Same random stream as kpzb_mcs, so equal
 * rates in every class give kpzb_mcs's lattice.  One launch per half-step (SCA/SCABit). */
kpzb_status kpzb_mcs_disorder(kpzb_handle* h, int n);
kpzb_status kpzb_mcs_disorder_async(kpzb_handle* h, int n);

/* SchedulerService::mcsPQSyncRng(n) (kpz/schedulerService.h:211; SCA/SCABit doMcs at
 * kpz/schedulerSCA.cu:43-70, kpz/schedulerSCABit.cu:46-73; DT at kpz/schedulerDT.cu:38-78):
 * n Monte-Carlo steps with the rates from kpzb_set_pq. Synchronous. */
kpzb_status kpzb_mcs(kpzb_handle* h, int n);
/* mcsPQSyncRngAsync (kpz/schedulerService.h:212): enqueue and return; kpzb_join waits
 * (SchedulerService::join, kpz/schedulerService.h:161-171). */
kpzb_status kpzb_mcs_async(kpzb_handle* h, int n);
kpzb_status kpzb_join(kpzb_handle* h);
/* SCA/SCABit only: MCS per HBM pass of the temporally blocked kernel (1 = one launch per
 * half-step; 0 = automatic: the autotuner's choice).  Results are identical for every value. */
kpzb_status kpzb_set_fusion(kpzb_handle* h, int mcs_per_pass);
/* The MCS per pass the handle uses for its current rates (resolving the automatic choice,
 * which may run the autotuner once). */
kpzb_status kpzb_get_fusion(kpzb_handle* h, int* mcs_per_pass);
/* The full pass plan for the current rates: MCS per pass, CTAs per SM and the pass kernel
 * (KPZB_PASS_HALF_STEPS: one launch per half-step; KPZB_PASS_BAND: band kernel;
 * KPZB_PASS_STREAM: streaming wavefront kernel; KPZB_PASS_WAVE: register-wavefront kernel;
 * KPZB_PASS_STRIP: warp-tile register-wavefront kernel, for which ctas_per_sm reports the
 * output rows of a tile).  No counterpart in the reference (introspection of the measured
 * choice, e.g. for launch accounting). */
enum { KPZB_PASS_HALF_STEPS = 0, KPZB_PASS_BAND = 1, KPZB_PASS_STREAM = 2, KPZB_PASS_WAVE = 3, KPZB_PASS_STRIP = 4 };
kpzb_status kpzb_get_plan(kpzb_handle* h, int* mcs_per_pass, int* ctas_per_sm, int* pass_kernel);
/* Time every pass shape (MCS per pass x CTAs per SM) on scratch copies of the current
 * lattice and cache the fastest for this size and rate class (in memory, and in the file
 * named by KPZB_TUNE_CACHE if set).  The lattice itself is not modified.  No reference
 * counterpart: replaces the fixed LocalLayout presets (kpz/schedulerDT.h:32-47) and the
 * per-architecture block counts (kpz/kpzSCABit.cu:63-106) with measured choices. */
kpzb_status kpzb_autotune(kpzb_handle* h, int* mcs_per_pass, int* ctas_per_sm, float* ms_per_mcs);

/* SchedulerService::pushSystem / popSystem (kpz/schedulerBase.cu:35-52): copy host words
 * in the handle's encoding (kpzb_size_words words) to / from the device. */
kpzb_status kpzb_push(kpzb_handle* h, const uint32_t* words);
kpzb_status kpzb_pop(kpzb_handle* h, uint32_t* words);
/* Asynchronous push/pop: enqueued on the handle's stream behind earlier work, returning at
 * once; the host buffer must stay valid until kpzb_join.  With page-locked host buffers the
 * copies overlap other handles' MCS.  For the SCABit, DT and DB4 dynamics kpzb_push_async
 * copies into a stage buffer of the handle on a copy stream of its own, so the copy also
 * overlaps this handle's queued MCS, pops and roughness, which still see the previous
 * lattice; work enqueued after the push sees the new one.  (The reference copies
 * synchronously after join(): kpz/schedulerBase.cu:35-52.) */
kpzb_status kpzb_push_async(kpzb_handle* h, const uint32_t* words);
kpzb_status kpzb_pop_async(kpzb_handle* h, uint32_t* words);
/* Same, with device buffers of the caller (cudaMemcpyDeviceToDevice on the handle's stream). */
kpzb_status kpzb_push_device(kpzb_handle* h, const uint32_t* d_words);
kpzb_status kpzb_pop_device(kpzb_handle* h, uint32_t* d_words);
size_t kpzb_size_words(const kpzb_handle* h);
int kpzb_encoding(const kpzb_handle* h);

/* SchedulerService::roughness (kpz/schedulerService.cpp:292-297, kpz/correlator.cpp:607-697):
 * out[0] = W^2, out[1..7] = <h^k> of the path-relative heights (kpz/correlator.cpp:47-96). */
kpzb_status kpzb_roughness(kpzb_handle* h, double out[8]);
/* SchedulerService::roughnessAsync / joinRoughness (kpz/schedulerService.h:150-170): enqueue
 * the roughness of the lattice as it will be after the work already enqueued, on the handle's
 * stream, and return at once; kpzb_roughness_join waits for the handle's stream and returns it
 * (out as kpzb_roughness).  One result is held at a time: a second kpzb_roughness_async before
 * the join replaces the first. */
kpzb_status kpzb_roughness_async(kpzb_handle* h);
kpzb_status kpzb_roughness_join(kpzb_handle* h, double out[8]);
/* Roughness (as kpzb_roughness) of a caller's device ENC_CBBIT lattice, without allocating:
 * no cudaMalloc/cudaFree or allocating library call; scratch lives in a fixed device array
 * of about 1.2 MB held by every GPU that loads the library's module.  For callers that
 * cannot allocate device memory at measurement time (their allocator owns the device, or an
 * allocation would synchronize the device inside a timing loop).  No counterpart in the
 * reference.  Limit: ly <= 16.  Calls overlapping on the GPU race on the shared scratch.
 * Set-up: the scratch's device address is looked up once per device and CUDA context (again
 * after the caller recreates the context, e.g. by cudaDeviceReset); that first call may also
 * load the library's module with its array, so a caller whose no-allocation window must see
 * no allocation at all makes one call before the window, and the first call on a device
 * should precede any stream capture.  `stream` is a cudaStream_t (NULL: default stream);
 * synchronous. */
kpzb_status kpzb_roughness_noalloc(const uint32_t* d_cbbit, int lx, int ly, double out[8], void* stream);
/* Exact power sums of the relative heights: s12[0] = sum h, s12[1] = sum h^2,
 * hminmax[0..1] = min/max height. */
kpzb_status kpzb_height_sums(kpzb_handle* h, int64_t s12[2], int64_t hminmax[2]);

/* SchedulerService::correlateTag (kpz/schedulerService.cpp:200-213, Correlator::set at
 * kpz/correlator.cpp:37-106): store the current lattice as the snapshot; out[8] as roughness. */
kpzb_status kpzb_corr_tag(kpzb_handle* h, double out[8]);
/* SchedulerService::correlate with one tag (Correlator::correlate, kpz/correlator.cpp:463-477):
 * out[0..7] roughness of the current lattice, out[8] = ch, out[9] = cs. */
kpzb_status kpzb_correlate(kpzb_handle* h, double out[10]);

/* Device-side MCS counter (m_deviceMcs, kpz/schedulerService.h:244) and the reported MCS
 * (SchedulerService::mcs/setMcs, kpz/schedulerService.h:242-243). */
kpzb_status kpzb_get_mcs(const kpzb_handle* h, uint64_t* device_mcs);
kpzb_status kpzb_set_mcs(kpzb_handle* h, uint64_t device_mcs);

/* Deposition / desorption counters accumulated by the SCA/SCABit kernels since the last
 * reset (for the height-balance invariant sum(dh) = 2*(dep - des)). */
kpzb_status kpzb_counters(kpzb_handle* h, int64_t dep_des[2], int reset);
kpzb_status kpzb_enable_counters(kpzb_handle* h, int on);

/* SchedulerService::consitencyCheck (kpz/schedulerService.cpp:721-854) for both encodings:
 * rep[0] rows with nonzero x-slope sum, rep[1] columns with nonzero y-slope sum,
 * rep[2] plaquettes whose height loop does not close. All zero for a valid lattice. */
kpzb_status kpzb_check_invariants(kpzb_handle* h, int64_t rep[3]);

/* Device pointer to the lattice in the handle's internal layout (ENC_CBBIT for SCA and
 * SCABit, ENC_LOCAL for DT) for tests and zero-copy callers.  The lattice moves between the
 * handle's buffers on an MCS and on kpzb_push_async: ask again after either. */
kpzb_status kpzb_device_ptr(kpzb_handle* h, uint32_t** d_words, size_t* nwords);
/* The CUDA stream the handle enqueues on (as void*, a cudaStream_t). */
void* kpzb_stream(kpzb_handle* h);
/* Enqueue on the caller's stream from now on (NULL: back to the handle's own stream).
 * The caller keeps ownership of the stream and must keep it alive while the handle uses it. */
kpzb_status kpzb_set_stream(kpzb_handle* h, void* stream);

/* ---------------- batched replicas ----------------
 * Many independent SCABit lattices of uneven size advance together: one launch per
 * half-step over a work list of (replica, row) items, replayed from a CUDA graph per MCS
 * chunk.  Per-replica results are bit-identical to single runs with the same
 * (lx, p, q, seed, stream).  Replaces the per-lattice loop of kpz/kpzScaling.cpp:194-215
 * run once per replica. */
typedef struct kpzb_batch kpzb_batch;
kpzb_status kpzb_batch_create(kpzb_batch** b, int n, const int* lx, const double* p,
                              const double* q, const uint64_t* seed, const uint32_t* stream,
                              int device);
kpzb_status kpzb_batch_destroy(kpzb_batch* b);
kpzb_status kpzb_batch_init_homogeneous(kpzb_batch* b);
/* n MCS for every replica (synchronous).  Square lattices only, 8 <= lx <= 16. */
kpzb_status kpzb_batch_mcs(kpzb_batch* b, int n);
/* MCS per pass (1..32) and passes per captured CUDA graph (1..256; default 8).  Results are
 * identical for every choice.  A batch whose caller sets neither this nor the CTAs per SM is
 * tuned on its first kpzb_batch_mcs (kpzb_batch_autotune; KPZB_AUTOTUNE=0: 8 MCS per pass at
 * one CTA per SM).  No counterpart in the reference (its frontend runs one lattice per
 * scheduler; the launch shaping it replaces is kpz/kpzSCABit.cu:63-106). */
kpzb_status kpzb_batch_set_fusion(kpzb_batch* b, int mcs_per_pass, int passes_per_graph);
/* Persistent CTAs per SM of the pass kernel: 1 (512 threads, 226 KB of shared memory each), 2 or
 * 3 (256 threads and a half or a third of the SM's shared memory each). */
kpzb_status kpzb_batch_set_ctas_per_sm(kpzb_batch* b, int ctas_per_sm);
kpzb_status kpzb_batch_get_plan(const kpzb_batch* b, int* mcs_per_pass, int* ctas_per_sm);
/* Times every (MCS per pass in {2,4,6,8}, CTAs per SM in {1,2,3}) shape on the replicas as they
 * are, keeps the fastest (cached per set of replica sizes and rate classes) and restores the
 * replicas and the MCS count, so tuning changes no result.  Outputs may be NULL. */
kpzb_status kpzb_batch_autotune(kpzb_batch* b, int* mcs_per_pass, int* ctas_per_sm, float* ms_per_mcs);
kpzb_status kpzb_batch_get_mcs(const kpzb_batch* b, uint64_t* mcs);
kpzb_status kpzb_batch_push(kpzb_batch* b, int i, const uint32_t* words);
kpzb_status kpzb_batch_pop(kpzb_batch* b, int i, uint32_t* words);
/* W^2 of every replica, out[n]. */
kpzb_status kpzb_batch_roughness(kpzb_batch* b, double* w2);

/* ---------------- checkpoint / resume ----------------
 * kpzb_save writes SchedulerService::saveBit's file (kpz/schedulerService.cpp:389-401):
 * "<lx>\n<ly>\n" + meta + '\0' + the lattice words in the handle's encoding, and appends a
 * trailer that a saveBit reader never reaches: "KPZBCKPT", version, dynamics, lx, ly, device
 * MCS, seed, stream id, p, q, fusion and, when a correlator tag is held, its ENC_CBBIT snapshot
 * words and mean height.  With the counter-based stream that is the complete state, so a run
 * resumed from the file continues bit for bit (the reference keeps its RNG state in HDF5,
 * kpz/schedulerService.cpp:582-611, and its loadBit is an empty stub, :86-89).
 * kpzb_load reads such a file into a handle of the same size; a plain saveBit file (no
 * trailer) restores the lattice words only. */
kpzb_status kpzb_save(kpzb_handle* h, const char* path, const char* meta);
kpzb_status kpzb_load(kpzb_handle* h, const char* path);

/* ---------------- measurement scheduling ----------------
 * The reference's frontend loop (kpz/kpzScaling.cpp:194-215) advances the scheduler to the
 * next measurement time of its sampling mode (SamplingParam::nextEval, kpz/sampling.h:84-100),
 * pops the whole lattice to the host and analyses it there (SchedulerService::correlate,
 * kpz/schedulerService.cpp:292-297).  kpzb_measure_run keeps that schedule but leaves the
 * analysis on the device: the MCS chunks and the height reductions of every measurement are
 * enqueued back to back on the handle's stream, with one copy of the result records at the end
 * and no lattice transfer. */
enum { KPZB_SAMPLE_EXP = 0, KPZB_SAMPLE_LINEAR = 1, KPZB_SAMPLE_RANDOM = 2 };
typedef struct {
    int mode;              /* KPZB_SAMPLE_* */
    double density;        /* EXP: next = ceil(exp(log(t + 10) + density)); reference default 0.1 */
    uint32_t interval;     /* LINEAR: next = t + interval (> 0) */
    double random_mean;    /* RANDOM: next = t + (unsigned)(u * mean + mean), u uniform in [0, 1)
                              from the counter stream keyed by `seed` (the reference draws u from
                              the scheduler's dSFMT, SchedulerService::genrand_close_open); at
                              least t + 1 */
    uint64_t seed;         /* RANDOM only */
} kpzb_sampling;
/* The measurement times after `start` up to `end`, `end` included (the reference's EndEvent,
 * kpz/kpzFrontend.cpp:744-752).  Writes at most `max` times; *n = the full count. */
kpzb_status kpzb_sample_times(const kpzb_sampling* s, uint64_t start, uint64_t end, uint64_t* times,
                              int max, int* n);
/* Advance the handle from its device MCS to `end`, measuring at every sample time.  Row i of
 * `rows` (11 doubles) = {t, W^2, <h^1>..<h^7>, ch, cs} as kpzb_roughness / kpzb_correlate give
 * them.  Correlator tag (SchedulerService::correlateTag, kpz/schedulerService.h:151): when
 * corr_start >= the current MCS, a snapshot is taken at t = corr_start (which is also a row)
 * and rows with corr_start < t <= corr_stop carry ch and cs; elsewhere they are NaN
 * (corr_start < 0: no tag).  *n_rows = number of rows; KPZB_EINVAL when max_rows is smaller
 * (nothing is run).  Synchronous. */
kpzb_status kpzb_measure_run(kpzb_handle* h, const kpzb_sampling* s, uint64_t end, int64_t corr_start,
                             uint64_t corr_stop, double* rows, int max_rows, int* n_rows);

/* ---------------- exact height autocorrelator ----------------
 * Snapshots of one lattice (ENC_CBBIT words) are turned into relative heights, shifted by
 * a common integer offset and split into signed int8 limbs; the full Gram
 * G[s][t] = sum_sites h_s * h_t is computed on tcgen05 INT8 tensor cores with int32
 * accumulation and exact int64 recombination.  Replaces the per-pair loop of
 * Correlator::correlateThreaded (kpz/correlator.cpp:491-593) and correlateKernelCBBit
 * (kpz/correlatorCuda.cu:276-369). */
typedef struct kpzb_gram kpzb_gram;
kpzb_status kpzb_gram_create(kpzb_gram** g, int lx, int ly, int max_snapshots, int device);
kpzb_status kpzb_gram_destroy(kpzb_gram* g);
/* Add a snapshot from a device ENC_CBBIT lattice (e.g. kpzb_device_ptr of an SCABit handle). */
kpzb_status kpzb_gram_add_device(kpzb_gram* g, const uint32_t* d_cbbit);
kpzb_status kpzb_gram_add_host(kpzb_gram* g, const uint32_t* cbbit);
/* G (n x n, row-major int64) of the n snapshots added so far, and the per-snapshot sums
 * S1[s] = sum h_s. method 0 = tcgen05 INT8 tensor cores, 1 = int64 CUDA-core reference. */
kpzb_status kpzb_gram_compute(kpzb_gram* g, int method, int64_t* G, int64_t* S1);
int kpzb_gram_count(const kpzb_gram* g);

#ifdef __cplusplus
}
#endif
#endif /* KPZB_H */
