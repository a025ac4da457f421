// api.cu -- the C ABI (include/kpzb.h): handle lifecycle, MCS loop, push/pop, analysis.
//
// Mirrors Kpz::SchedulerService (kpz/schedulerService.h:73-255) and the GPU scheduler base
// (kpz/schedulerBase.cu:35-99).  Differences by design: one CUDA stream per handle, no
// busy-wait event loop, integer status codes instead of exceptions/exit, counter-based RNG
// keyed by (seed, stream) instead of per-thread TinyMT/SLCG state.
#include <algorithm>
#include <cmath>
#include <vector>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/kpzb.h"
#include "kpzb_api_internal.h"
#include "kpzb_common.cuh"
#include "kpzb_internal.h"

namespace kpzb {
thread_local std::string g_err;

kpzb_status fail(kpzb_status s, const char* what)
{
    g_err = what;
    return s;
}

kpzb_status cuda_fail(cudaError_t e, const char* where)
{
    g_err = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? KPZB_ENOMEM : KPZB_ECUDA;
}

int sm_count_of(int device)
{
    int n = 148;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
    return n;
}
}  // namespace kpzb

using namespace kpzb;

struct kpzb_handle {
    int lx = 0, ly = 0, dyn = 0, device = 0, sm_count = 148;
    cudaStream_t st = nullptr;      // stream in use
    cudaStream_t own_st = nullptr;  // stream created by the handle
    uint32_t* d_sys = nullptr;   // internal layout: CBBIT (SCA, SCABIT) or LOCAL (DT)
    uint32_t* d_tmp = nullptr;   // scratch lattice (transcoding, fused double buffer)
    uint32_t* d_snap = nullptr;  // correlator snapshot, CBBIT
    // kpzb_push_async of the SCABit and random-sequential dynamics: the host words land in a
    // third lattice buffer on a copy stream, which then trades places with d_sys.  ev_ready
    // (copy done) gates the handle's stream; ev_free (recorded on the handle's stream at the
    // trade) gates the next copy into the buffer that d_sys was, until every read of it
    // enqueued before the trade (a pop, a roughness) has run.
    uint32_t* d_stage = nullptr;
    cudaStream_t copy_st = nullptr;
    cudaEvent_t ev_ready = nullptr, ev_free = nullptr;
    double snap_mean = 0.0;
    bool has_snap = false;
    uint64_t seed = 0;
    uint32_t stream_id = 0;
    double p = 1.0, q = 0.0;
    uint64_t tdev = 0;
    int fusion = 0;
    bool count = false;
    unsigned long long* d_counters = nullptr;
    // quenched disorder: rate-class words (ENC_LOCAL for DT, ENC_CBBIT form for SCA/SCABit)
    // and the rates of classes 0..3 (class 0 = p, q)
    uint32_t* d_dis = nullptr;
    // asynchronous roughness (kpzb_roughness_async / kpzb_roughness_join): the reduction's
    // final record on the device and its pinned host copy
    void* d_rough = nullptr;
    void* h_rough = nullptr;
    bool rough_pending = false;
    double pc[4] = {1.0, 1.0, 1.0, 1.0}, qc[4] = {0.0, 0.0, 0.0, 0.0};
    bool class_set[4] = {true, false, false, false};
    AnalysisScratch an{};
    ScabitShape shape{};
    DtState dt{};
    size_t words() const { return (size_t)1 << (lx + ly - 4); }
    int encoding() const { return dyn == KPZB_DYN_SCABIT ? KPZB_ENC_CBBIT : KPZB_ENC_LOCAL; }
    // random-sequential dynamics (DT, DB4): ENC_LOCAL on the device, driven by dt_enqueue
    bool rs() const { return dyn == KPZB_DYN_DT || dyn == KPZB_DYN_DB4; }
};

#define KPZB_CHECK_H(h)                                              \
    do {                                                             \
        if (!(h)) return fail(KPZB_EINVAL, "null handle");           \
        cudaError_t _e = cudaSetDevice((h)->device);                 \
        if (_e != cudaSuccess) return cuda_fail(_e, "cudaSetDevice"); \
    } while (0)

#define KPZB_CU(call, where)                                   \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return cuda_fail(_e, where);    \
    } while (0)

extern "C" const char* kpzb_last_error(void) { return g_err.c_str(); }
extern "C" const char* kpzb_version(void) { return "kpzb200 1.0 (sm_100a)"; }

static kpzb_status ensure_tmp(kpzb_handle* h)
{
    if (!h->d_tmp) KPZB_CU(cudaMalloc(&h->d_tmp, h->words() * 4), "cudaMalloc(tmp)");
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_create(kpzb_handle** out, int lx, int ly, int dynamics, int device)
{
    if (!out) return fail(KPZB_EINVAL, "null output pointer");
    *out = nullptr;
    if (dynamics < KPZB_DYN_SCA || dynamics > KPZB_DYN_DB4) return fail(KPZB_EINVAL, "bad dynamics");
    // lx >= 8: a quadrant row holds at least one 4-word Philox group; lx + ly >= 14: every
    // launch is made of whole warps (the kernels' shuffles use full-warp masks)
    if (lx < 8 || lx > 30 || ly < 2 || ly > 30 || lx + ly > 38 || lx + ly < 14)
        return fail(KPZB_EINVAL,
                    "lattice size out of range (8<=lx<=30, 2<=ly<=30, 14<=lx+ly<=38)");
    if (dynamics == KPZB_DYN_DT && (lx < 9 || ly < 8))
        return fail(KPZB_EINVAL, "DT needs lx >= 9 and ly >= 8 (one double tile of 512x256 sites)");
    if (dynamics == KPZB_DYN_DB4 && (lx < 8 || ly < 7))
        return fail(KPZB_EINVAL, "DB4 needs lx >= 8 and ly >= 7 (one block of 256x128 sites)");
    int dev = device;
    if (dev < 0) {
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    }
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    kpzb_handle* h = new kpzb_handle();
    h->lx = lx;
    h->ly = ly;
    h->dyn = dynamics;
    h->device = dev;
    h->sm_count = sm_count_of(dev);
    h->shape = scabit_shape(lx, ly, h->sm_count);
    auto bail = [&](kpzb_status s) {
        kpzb_destroy(h);
        return s;
    };
    if ((e = cudaStreamCreateWithFlags(&h->own_st, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(cuda_fail(e, "cudaStreamCreate"));
    h->st = h->own_st;
    if ((e = cudaMalloc(&h->d_sys, h->words() * 4)) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(lattice)"));
    if ((e = cudaMalloc(&h->d_counters, 4 * sizeof(unsigned long long))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(counters)"));
    cudaMemsetAsync(h->d_counters, 0, 4 * sizeof(unsigned long long), h->st);
    if ((e = analysis_alloc(&h->an, ly)) != cudaSuccess) return bail(cuda_fail(e, "analysis_alloc"));
    if (h->rs()) {
        kpzb_status s = dt_init(&h->dt, lx, ly, h->sm_count, dynamics == KPZB_DYN_DB4);
        if (s != KPZB_OK) return bail(s);
    }
    kpzb_status s = kpzb_init_homogeneous(h);
    if (s != KPZB_OK) return bail(s);
    if ((e = cudaStreamSynchronize(h->st)) != cudaSuccess) return bail(cuda_fail(e, "create sync"));
    *out = h;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_destroy(kpzb_handle* h)
{
    if (!h) return KPZB_OK;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    if (h->copy_st) cudaStreamSynchronize(h->copy_st);
    cudaFree(h->d_sys);
    cudaFree(h->d_tmp);
    cudaFree(h->d_stage);
    if (h->ev_ready) cudaEventDestroy(h->ev_ready);
    if (h->ev_free) cudaEventDestroy(h->ev_free);
    if (h->copy_st) cudaStreamDestroy(h->copy_st);
    cudaFree(h->d_snap);
    cudaFree(h->d_counters);
    cudaFree(h->d_dis);
    cudaFree(h->d_rough);
    if (h->h_rough) cudaFreeHost(h->h_rough);
    if (h->an.rowinfo) analysis_free(&h->an);
    dt_free(&h->dt);
    if (h->own_st) cudaStreamDestroy(h->own_st);
    delete h;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_init_homogeneous(kpzb_handle* h)
{
    KPZB_CHECK_H(h);
    // SCA keeps ENC_CBBIT internally; the flat start is the same surface in both encodings
    const int internal = h->rs() ? KPZB_ENC_LOCAL : KPZB_ENC_CBBIT;
    KPZB_CU(init_homogeneous_dev(h->d_sys, h->lx, h->ly, internal, h->st), "init_homogeneous");
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_set_pq(kpzb_handle* h, double p, double q)
{
    if (!h) return fail(KPZB_EINVAL, "null handle");
    if (!(p >= 0.0 && p <= 1.0 && q >= 0.0 && q <= 1.0)) return fail(KPZB_EINVAL, "p, q must lie in [0,1]");
    h->p = p;
    h->q = q;
    for (int c = 0; c < 4; ++c)
        if (c == 0 || !h->class_set[c]) {
            h->pc[c] = p;
            h->qc[c] = q;
        }
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_set_dt_inner(kpzb_handle* h, int inner)
{
    if (!h) return fail(KPZB_EINVAL, "null handle");
    if (h->dyn != KPZB_DYN_DT) return fail(KPZB_EUNSUPPORTED, "the inner decomposition applies to DT handles");
    static const int scheme_of[] = {DT_SCHEME_DT, DT_SCHEME_DBSH, DT_SCHEME_DB, DT_SCHEME_DTDBSH, DT_SCHEME_DBSHREP};
    if (inner < KPZB_DT_INNER_DT || inner > KPZB_DT_INNER_DBSHREP) return fail(KPZB_EINVAL, "unknown DT inner scheme");
    h->dt.scheme = scheme_of[inner];
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_mcs_scale(kpzb_handle* h, double* scale)
{
    if (!h || !scale) return fail(KPZB_EINVAL, "null argument");
    if (h->dyn == KPZB_DYN_DT) *scale = 1.0;
    else if (h->dyn == KPZB_DYN_DB4) *scale = (256.0 - 5.0) * (128.0 - 5.0) / (256.0 * 128.0);
    else *scale = h->p + h->q;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_set_pq_class(kpzb_handle* h, int n, double p, double q)
{
    if (!h) return fail(KPZB_EINVAL, "null handle");
    if (n < 0 || n > 3) return fail(KPZB_EINVAL, "rate class must be 0..3");
    if (n == 0) return kpzb_set_pq(h, p, q);
    if (!(p >= 0.0 && p <= 1.0 && q >= 0.0 && q <= 1.0)) return fail(KPZB_EINVAL, "p, q must lie in [0,1]");
    h->pc[n] = p;
    h->qc[n] = q;
    h->class_set[n] = true;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_set_disorder(kpzb_handle* h, const uint32_t* local_words)
{
    KPZB_CHECK_H(h);
    if (!local_words) return fail(KPZB_EINVAL, "null disorder words");
    if (!h->d_dis) KPZB_CU(cudaMalloc(&h->d_dis, h->words() * 4), "cudaMalloc(disorder)");
    if (h->rs()) {
        KPZB_CU(cudaMemcpyAsync(h->d_dis, local_words, h->words() * 4, cudaMemcpyHostToDevice, h->st),
                "disorder copy");
    } else {
        kpzb_status s = ensure_tmp(h);
        if (s != KPZB_OK) return s;
        KPZB_CU(cudaMemcpyAsync(h->d_tmp, local_words, h->words() * 4, cudaMemcpyHostToDevice, h->st),
                "disorder copy");
        KPZB_CU(local_to_cbbit_dev(h->d_tmp, h->d_dis, h->lx, h->ly, h->st), "disorder transcode");
    }
    KPZB_CU(cudaStreamSynchronize(h->st), "disorder sync");
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_seed(kpzb_handle* h, uint64_t seed, uint32_t stream)
{
    if (!h) return fail(KPZB_EINVAL, "null handle");
    h->seed = seed;
    h->stream_id = stream;
    h->tdev = 0;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_set_fusion(kpzb_handle* h, int mcs_per_pass)
{
    if (!h) return fail(KPZB_EINVAL, "null handle");
    if (mcs_per_pass < 0 || mcs_per_pass > 64) return fail(KPZB_EINVAL, "fusion must be in [0,64]");
    h->fusion = mcs_per_pass;
    return KPZB_OK;
}

static kpzb_status resolve_plan(kpzb_handle* h, Plan* plan);

extern "C" kpzb_status kpzb_get_fusion(kpzb_handle* h, int* mcs_per_pass)
{
    if (!h || !mcs_per_pass) return fail(KPZB_EINVAL, "null argument");
    if (h->rs()) {
        *mcs_per_pass = 1;
        return KPZB_OK;
    }
    Plan p;
    kpzb_status s = resolve_plan(h, &p);
    if (s != KPZB_OK) return s;
    *mcs_per_pass = plan_shape_ok(p, h->lx, h->ly, h->sm_count) ? p.k : 1;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_get_plan(kpzb_handle* h, int* mcs_per_pass, int* ctas_per_sm, int* pass_kernel)
{
    if (!h || !mcs_per_pass || !ctas_per_sm || !pass_kernel) return fail(KPZB_EINVAL, "null argument");
    *mcs_per_pass = 1;
    *ctas_per_sm = 0;
    *pass_kernel = KPZB_PASS_HALF_STEPS;
    if (h->rs()) return KPZB_OK;
    Plan p;
    kpzb_status s = resolve_plan(h, &p);
    if (s != KPZB_OK) return s;
    if (p.k > 1 && plan_shape_ok(p, h->lx, h->ly, h->sm_count)) {
        *mcs_per_pass = p.k;
        *ctas_per_sm = p.kind == PASS_STRIP ? p.band : p.kind == PASS_STREAM && p.cps == 0 ? 1 : p.cps;
        *pass_kernel = p.kind == PASS_STREAM  ? KPZB_PASS_STREAM
                       : p.kind == PASS_WAVE  ? KPZB_PASS_WAVE
                       : p.kind == PASS_STRIP ? KPZB_PASS_STRIP
                                              : KPZB_PASS_BAND;
    }
    return KPZB_OK;
}

static uint64_t thresh_of(double p)
{
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return 1ull << 32;
    double t = std::ceil(p * 4294967296.0);
    if (t >= 4294967296.0) return 1ull << 32;
    return (uint64_t)t;
}

// The pass shape used for the current rates: the caller's choice, else the tuner's cached
// or freshly measured choice (KPZB_AUTOTUNE=0 disables measuring), else the heuristic.
static kpzb_status resolve_plan_raw(kpzb_handle* h, Plan* plan)
{
    if (h->fusion > 0) {
        *plan = explicit_plan(h->lx, h->ly, h->fusion, h->sm_count);
        return KPZB_OK;
    }
    const uint64_t Tp = thresh_of(h->p), Tq = thresh_of(h->q);
    if (lookup_plan(h->lx, h->ly, Tp, Tq, h->sm_count, plan)) return KPZB_OK;
    const char* env = getenv("KPZB_AUTOTUNE");
    if (env && env[0] == '0') {
        *plan = default_plan(h->lx, h->ly, Tp, Tq, h->sm_count);
        return KPZB_OK;
    }
    KPZB_CU(tune_plan(h->d_sys, h->lx, h->ly, h->seed, h->stream_id, Tp, Tq, h->sm_count,
                      reinterpret_cast<unsigned int*>(h->d_counters + 2), h->st, plan),
            "autotune");
    return KPZB_OK;
}

static kpzb_status resolve_plan(kpzb_handle* h, Plan* plan)
{
    kpzb_status s = resolve_plan_raw(h, plan);
    if (s != KPZB_OK) return s;
    // the register-wavefront kernel covers rates of at most one random plane; other rates
    // run the same depth as band passes
    if (plan->kind == PASS_WAVE) {
        const int mode = dec_mode(make_thresh(thresh_of(h->p)), make_thresh(thresh_of(h->q)));
        if (!scabit_wave_shape(h->lx, h->ly, plan->k, h->sm_count, plan->cps, mode).ok) {
            plan->kind = PASS_BAND;
            plan->cps = 0;
        }
    }
    if (plan->kind == PASS_STRIP) {
        const int mode = dec_mode(make_thresh(thresh_of(h->p)), make_thresh(thresh_of(h->q)));
        if (!scabit_strip_shape(h->lx, h->ly, plan->k, plan->band, mode).ok) {
            plan->kind = PASS_BAND;
            plan->cps = 0;
        }
    }
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_autotune(kpzb_handle* h, int* mcs_per_pass, int* ctas_per_sm,
                                     float* ms_per_mcs)
{
    KPZB_CHECK_H(h);
    if (h->rs()) return fail(KPZB_EUNSUPPORTED, "the tuner covers SCA/SCABit passes");
    Plan p;
    KPZB_CU(tune_plan(h->d_sys, h->lx, h->ly, h->seed, h->stream_id, thresh_of(h->p), thresh_of(h->q),
                      h->sm_count, reinterpret_cast<unsigned int*>(h->d_counters + 2), h->st, &p),
            "autotune");
    if (mcs_per_pass) *mcs_per_pass = p.k;
    if (ctas_per_sm) *ctas_per_sm = p.cps;
    if (ms_per_mcs) *ms_per_mcs = p.ms_per_mcs;
    return KPZB_OK;
}

static kpzb_status enqueue_sca(kpzb_handle* h, int n)
{
    const uint64_t Tp = thresh_of(h->p), Tq = thresh_of(h->q);
    unsigned long long* cnt = h->count ? h->d_counters : nullptr;
    int done = 0;
    Plan plan;
    kpzb_status ps = resolve_plan(h, &plan);
    if (ps != KPZB_OK) return ps;
    const int k = plan.k;
    const int mode = dec_mode(make_thresh(Tp), make_thresh(Tq));
    const WaveShape ws = plan.kind == PASS_WAVE ? scabit_wave_shape(h->lx, h->ly, k, h->sm_count, plan.cps, mode)
                                                : WaveShape{};
    const StripShape tile = plan.kind == PASS_STRIP ? scabit_strip_shape(h->lx, h->ly, k, plan.band, mode)
                                                    : StripShape{};
    if (k > 1 && plan.kind == PASS_STRIP && tile.ok) {
        kpzb_status s = ensure_tmp(h);
        if (s != KPZB_OK) return s;
        while (n - done >= k) {
            KPZB_CU(scabit_strip(h->d_sys, h->d_tmp, h->lx, h->ly, (uint32_t)(h->tdev + done), h->seed,
                                 h->stream_id, Tp, Tq, tile, cnt, h->st),
                    "scabit_strip");
            std::swap(h->d_sys, h->d_tmp);
            done += k;
        }
    } else if (k > 1 && plan.kind == PASS_WAVE && ws.ok) {
        kpzb_status s = ensure_tmp(h);
        if (s != KPZB_OK) return s;
        while (n - done >= k) {
            KPZB_CU(scabit_wave(h->d_sys, h->d_tmp, h->lx, h->ly, (uint32_t)(h->tdev + done), h->seed,
                                h->stream_id, Tp, Tq, ws, cnt, reinterpret_cast<unsigned int*>(h->d_counters + 2),
                                h->st),
                    "scabit_wave");
            std::swap(h->d_sys, h->d_tmp);
            done += k;
        }
    } else if (k > 1 && plan.kind == PASS_STREAM) {
        const StreamShape ss = scabit_stream_shape(h->lx, h->ly, k, h->sm_count, plan.cps ? plan.cps : 1);
        if (ss.ok) {
            kpzb_status s = ensure_tmp(h);
            if (s != KPZB_OK) return s;
            while (n - done >= k) {
                KPZB_CU(scabit_stream(h->d_sys, h->d_tmp, h->lx, h->ly, (uint32_t)(h->tdev + done),
                                      h->seed, h->stream_id, Tp, Tq, ss, cnt,
                                      reinterpret_cast<unsigned int*>(h->d_counters + 2), h->st),
                        "scabit_stream");
                std::swap(h->d_sys, h->d_tmp);
                done += k;
            }
        }
    } else if (k > 1) {
        FusedShape fs = scabit_fused_shape_cps(h->lx, h->ly, k, plan.cps, 0);
        if (fs.ok) {
            kpzb_status s = ensure_tmp(h);
            if (s != KPZB_OK) return s;
            while (n - done >= k) {
                KPZB_CU(scabit_fused(h->d_sys, h->d_tmp, h->lx, h->ly, (uint32_t)(h->tdev + done),
                                     h->seed, h->stream_id, Tp, Tq, fs, cnt,
                                     reinterpret_cast<unsigned int*>(h->d_counters + 2), h->st),
                        "scabit_fused");
                std::swap(h->d_sys, h->d_tmp);
                done += k;
            }
        }
    }
    for (; done < n; ++done) {
        const uint64_t t = h->tdev + done;
        for (int sg = 0; sg < 2; ++sg)
            KPZB_CU(scabit_half(h->d_sys, h->lx, h->ly, sg, (uint32_t)(2 * t + sg), h->seed,
                                h->stream_id, Tp, Tq, h->shape, cnt, h->st),
                    "scabit_half");
    }
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_mcs_async(kpzb_handle* h, int n)
{
    KPZB_CHECK_H(h);
    if (n < 0) return fail(KPZB_EINVAL, "negative MCS count");
    if (n == 0) return KPZB_OK;
    if (h->tdev + (uint64_t)n >= (1ull << 31)) return fail(KPZB_EINVAL, "device MCS counter limit 2^31");
    kpzb_status s;
    if (h->rs())
        s = dt_enqueue(&h->dt, h->d_sys, h->lx, h->ly, h->tdev, n, h->p, h->q, h->seed, h->stream_id,
                       h->st, h->count ? h->d_counters : nullptr);
    else
        s = enqueue_sca(h, n);
    if (s != KPZB_OK) return s;
    h->tdev += (uint64_t)n;
    return KPZB_OK;
}

static uint64_t thresh_of(double p);

extern "C" kpzb_status kpzb_mcs_disorder_async(kpzb_handle* h, int n)
{
    KPZB_CHECK_H(h);
    if (n < 0) return fail(KPZB_EINVAL, "negative MCS count");
    // Kpz::Scheduler::mcsDisorder2SyncRng prints "[BUG] ... not implemented" (kpz/scheduler.h:75-78)
    if (h->dyn == KPZB_DYN_DB4) return fail(KPZB_EUNSUPPORTED, "DB4 has no disorder dynamics");
    if (!h->d_dis) return fail(KPZB_ESTATE, "no disorder set (kpzb_set_disorder)");
    if (h->tdev + (uint64_t)n >= (1ull << 31)) return fail(KPZB_EINVAL, "device MCS counter limit 2^31");
    uint64_t Tp[4], Tq[4];
    for (int c = 0; c < 4; ++c) {
        Tp[c] = thresh_of(h->pc[c]);
        Tq[c] = thresh_of(h->qc[c]);
    }
    unsigned long long* cnt = h->count ? h->d_counters : nullptr;
    if (h->rs()) {
        kpzb_status s = dt_enqueue(&h->dt, h->d_sys, h->lx, h->ly, h->tdev, n, h->p, h->q, h->seed, h->stream_id,
                                   h->st, cnt, h->d_dis, Tp, Tq);
        if (s != KPZB_OK) return s;
    } else {
        for (int i = 0; i < n; ++i) {
            const uint64_t t = h->tdev + (uint64_t)i;
            for (int sg = 0; sg < 2; ++sg)
                KPZB_CU(scabit_half_dis(h->d_sys, h->d_dis, h->lx, h->ly, sg, (uint32_t)(2 * t + sg), h->seed,
                                        h->stream_id, Tp, Tq, h->shape, cnt, h->st),
                        "scabit_half_dis");
        }
    }
    h->tdev += (uint64_t)n;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_mcs_disorder(kpzb_handle* h, int n)
{
    kpzb_status s = kpzb_mcs_disorder_async(h, n);
    if (s != KPZB_OK) return s;
    return kpzb_join(h);
}

extern "C" kpzb_status kpzb_join(kpzb_handle* h)
{
    KPZB_CHECK_H(h);
    unsigned int flag = 0;
    KPZB_CU(cudaMemcpyAsync(&flag, h->d_counters + 2, sizeof flag, cudaMemcpyDeviceToHost, h->st),
            "join flag");
    KPZB_CU(cudaStreamSynchronize(h->st), "join");
    KPZB_CU(cudaGetLastError(), "join");
    if (flag) {
        cudaMemsetAsync(h->d_counters + 2, 0, sizeof(unsigned long long), h->st);
        cudaStreamSynchronize(h->st);
        return fail(KPZB_ETIMEOUT, "a bounded device wait (TMA mbarrier) expired");
    }
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_mcs(kpzb_handle* h, int n)
{
    kpzb_status s = kpzb_mcs_async(h, n);
    if (s != KPZB_OK) return s;
    return kpzb_join(h);
}

extern "C" size_t kpzb_size_words(const kpzb_handle* h) { return h ? h->words() : 0; }
extern "C" int kpzb_encoding(const kpzb_handle* h) { return h ? h->encoding() : -1; }

// Asynchronous host push without a transcode: copy into the stage buffer on the copy stream
// while the handle's stream still runs (an MCS, a pop of the previous lattice), then make the
// stage the lattice.  The copy waits only for the reads of its target enqueued before the
// previous trade.
static kpzb_status push_staged(kpzb_handle* h, const uint32_t* src)
{
    if (!h->d_stage) KPZB_CU(cudaMalloc(&h->d_stage, h->words() * 4), "cudaMalloc(stage)");
    if (!h->copy_st) KPZB_CU(cudaStreamCreateWithFlags(&h->copy_st, cudaStreamNonBlocking), "copy stream");
    if (!h->ev_ready) KPZB_CU(cudaEventCreateWithFlags(&h->ev_ready, cudaEventDisableTiming), "event");
    // a fresh stage has no readers: waiting on the not yet recorded ev_free is a no-op
    if (!h->ev_free) KPZB_CU(cudaEventCreateWithFlags(&h->ev_free, cudaEventDisableTiming), "event");
    KPZB_CU(cudaStreamWaitEvent(h->copy_st, h->ev_free, 0), "stage wait");
    KPZB_CU(cudaMemcpyAsync(h->d_stage, src, h->words() * 4, cudaMemcpyHostToDevice, h->copy_st), "push copy");
    KPZB_CU(cudaEventRecord(h->ev_ready, h->copy_st), "event record");
    KPZB_CU(cudaStreamWaitEvent(h->st, h->ev_ready, 0), "stage ready");
    std::swap(h->d_sys, h->d_stage);
    KPZB_CU(cudaEventRecord(h->ev_free, h->st), "event record");
    return KPZB_OK;
}

static kpzb_status push_from(kpzb_handle* h, const uint32_t* src, cudaMemcpyKind kind, bool sync = true)
{
    if (!sync && kind == cudaMemcpyHostToDevice && h->dyn != KPZB_DYN_SCA) return push_staged(h, src);
    if (h->dyn == KPZB_DYN_SCA) {
        kpzb_status s = ensure_tmp(h);
        if (s != KPZB_OK) return s;
        KPZB_CU(cudaMemcpyAsync(h->d_tmp, src, h->words() * 4, kind, h->st), "push copy");
        KPZB_CU(local_to_cbbit_dev(h->d_tmp, h->d_sys, h->lx, h->ly, h->st), "local_to_cbbit");
    } else {
        KPZB_CU(cudaMemcpyAsync(h->d_sys, src, h->words() * 4, kind, h->st), "push copy");
    }
    if (sync) KPZB_CU(cudaStreamSynchronize(h->st), "push sync");
    return KPZB_OK;
}

static kpzb_status pop_to(kpzb_handle* h, uint32_t* dst, cudaMemcpyKind kind, bool sync = true)
{
    if (h->dyn == KPZB_DYN_SCA) {
        kpzb_status s = ensure_tmp(h);
        if (s != KPZB_OK) return s;
        KPZB_CU(cbbit_to_local_dev(h->d_sys, h->d_tmp, h->lx, h->ly, h->st), "cbbit_to_local");
        KPZB_CU(cudaMemcpyAsync(dst, h->d_tmp, h->words() * 4, kind, h->st), "pop copy");
    } else {
        KPZB_CU(cudaMemcpyAsync(dst, h->d_sys, h->words() * 4, kind, h->st), "pop copy");
    }
    if (sync) KPZB_CU(cudaStreamSynchronize(h->st), "pop sync");
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_push(kpzb_handle* h, const uint32_t* words)
{
    KPZB_CHECK_H(h);
    if (!words) return fail(KPZB_EINVAL, "null buffer");
    return push_from(h, words, cudaMemcpyHostToDevice);
}
extern "C" kpzb_status kpzb_pop(kpzb_handle* h, uint32_t* words)
{
    KPZB_CHECK_H(h);
    if (!words) return fail(KPZB_EINVAL, "null buffer");
    return pop_to(h, words, cudaMemcpyDeviceToHost);
}
extern "C" kpzb_status kpzb_push_async(kpzb_handle* h, const uint32_t* words)
{
    KPZB_CHECK_H(h);
    if (!words) return fail(KPZB_EINVAL, "null buffer");
    return push_from(h, words, cudaMemcpyHostToDevice, false);
}
extern "C" kpzb_status kpzb_pop_async(kpzb_handle* h, uint32_t* words)
{
    KPZB_CHECK_H(h);
    if (!words) return fail(KPZB_EINVAL, "null buffer");
    return pop_to(h, words, cudaMemcpyDeviceToHost, false);
}
extern "C" kpzb_status kpzb_push_device(kpzb_handle* h, const uint32_t* d_words)
{
    KPZB_CHECK_H(h);
    if (!d_words) return fail(KPZB_EINVAL, "null buffer");
    return push_from(h, d_words, cudaMemcpyDeviceToDevice);
}
extern "C" kpzb_status kpzb_pop_device(kpzb_handle* h, uint32_t* d_words)
{
    KPZB_CHECK_H(h);
    if (!d_words) return fail(KPZB_EINVAL, "null buffer");
    return pop_to(h, d_words, cudaMemcpyDeviceToDevice);
}

// CBBIT view of the current lattice (DT keeps ENC_LOCAL and is transcoded into d_tmp).
static kpzb_status cbbit_view(kpzb_handle* h, const uint32_t** view)
{
    if (!h->rs()) {
        *view = h->d_sys;
        return KPZB_OK;
    }
    kpzb_status s = ensure_tmp(h);
    if (s != KPZB_OK) return s;
    KPZB_CU(local_to_cbbit_dev(h->d_sys, h->d_tmp, h->lx, h->ly, h->st), "local_to_cbbit");
    *view = h->d_tmp;
    return KPZB_OK;
}

static void fill_roughness(const MomentsOut& m, int lx, int ly, double out[8], long double* h0)
{
    const long double N = (long double)((uint64_t)1 << (lx + ly));
    long double h[7];
    h[0] = (long double)m.s1 / N;
    h[1] = (long double)m.s2 / N;
    for (int k = 0; k < 5; ++k) h[2 + k] = (long double)m.s3to7[k] / N;
    out[0] = (double)(h[1] - h[0] * h[0]);
    for (int k = 0; k < 7; ++k) out[1 + k] = (double)h[k];
    if (h0) *h0 = h[0];
}

extern "C" kpzb_status kpzb_roughness(kpzb_handle* h, double out[8])
{
    KPZB_CHECK_H(h);
    if (!out) return fail(KPZB_EINVAL, "null output");
    const uint32_t* v;
    kpzb_status s = cbbit_view(h, &v);
    if (s != KPZB_OK) return s;
    MomentsOut m;
    KPZB_CU(analysis_moments(v, nullptr, h->lx, h->ly, &h->an, &m, h->st), "roughness");
    fill_roughness(m, h->lx, h->ly, out, nullptr);
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_roughness_async(kpzb_handle* h)
{
    KPZB_CHECK_H(h);
    const size_t rb = analysis_record_bytes();
    if (!h->d_rough) KPZB_CU(cudaMalloc(&h->d_rough, rb), "cudaMalloc(roughness record)");
    if (!h->h_rough) KPZB_CU(cudaMallocHost(&h->h_rough, rb), "cudaMallocHost(roughness record)");
    const uint32_t* v;
    kpzb_status s = cbbit_view(h, &v);
    if (s != KPZB_OK) return s;
    KPZB_CU(analysis_moments_record(v, nullptr, h->lx, h->ly, &h->an, h->d_rough, h->st), "roughness");
    KPZB_CU(cudaMemcpyAsync(h->h_rough, h->d_rough, rb, cudaMemcpyDeviceToHost, h->st), "roughness record");
    h->rough_pending = true;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_roughness_join(kpzb_handle* h, double out[8])
{
    KPZB_CHECK_H(h);
    if (!out) return fail(KPZB_EINVAL, "null output");
    if (!h->rough_pending) return fail(KPZB_ESTATE, "no asynchronous roughness pending");
    kpzb_status s = kpzb_join(h);
    if (s != KPZB_OK) return s;
    MomentsOut m;
    analysis_decode_record(h->h_rough, &m);
    fill_roughness(m, h->lx, h->ly, out, nullptr);
    h->rough_pending = false;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_height_sums(kpzb_handle* h, int64_t s12[2], int64_t hminmax[2])
{
    KPZB_CHECK_H(h);
    if (!s12 || !hminmax) return fail(KPZB_EINVAL, "null output");
    const uint32_t* v;
    kpzb_status s = cbbit_view(h, &v);
    if (s != KPZB_OK) return s;
    MomentsOut m;
    KPZB_CU(analysis_moments(v, nullptr, h->lx, h->ly, &h->an, &m, h->st), "height sums");
    s12[0] = m.s1;
    s12[1] = m.s2;
    hminmax[0] = m.hmin;
    hminmax[1] = m.hmax;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_corr_tag(kpzb_handle* h, double out[8])
{
    KPZB_CHECK_H(h);
    const uint32_t* v;
    kpzb_status s = cbbit_view(h, &v);
    if (s != KPZB_OK) return s;
    if (!h->d_snap) KPZB_CU(cudaMalloc(&h->d_snap, h->words() * 4), "cudaMalloc(snapshot)");
    KPZB_CU(cudaMemcpyAsync(h->d_snap, v, h->words() * 4, cudaMemcpyDeviceToDevice, h->st), "snapshot");
    MomentsOut m;
    KPZB_CU(analysis_moments(h->d_snap, nullptr, h->lx, h->ly, &h->an, &m, h->st), "snapshot moments");
    double r[8];
    long double h0;
    fill_roughness(m, h->lx, h->ly, r, &h0);
    h->snap_mean = (double)h0;
    h->has_snap = true;
    if (out) memcpy(out, r, sizeof r);
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_correlate(kpzb_handle* h, double out[10])
{
    KPZB_CHECK_H(h);
    if (!out) return fail(KPZB_EINVAL, "null output");
    if (!h->has_snap) return fail(KPZB_ESTATE, "no correlator snapshot (call kpzb_corr_tag first)");
    const uint32_t* v;
    kpzb_status s = cbbit_view(h, &v);
    if (s != KPZB_OK) return s;
    MomentsOut m;
    KPZB_CU(analysis_moments(v, h->d_snap, h->lx, h->ly, &h->an, &m, h->st), "correlate");
    long double h0;
    fill_roughness(m, h->lx, h->ly, out, &h0);
    const long double N = (long double)((uint64_t)1 << (h->lx + h->ly));
    out[8] = (double)((long double)(double)m.cross / N - h0 * (long double)h->snap_mean);
    out[9] = (double)((long double)m.agree / N / 2.0L);
    return KPZB_OK;
}

// ---------------------------------------------------------------------------------
// Checkpoint / resume (saveBit layout, kpz/schedulerService.cpp:389-401, plus a trailer)
// ---------------------------------------------------------------------------------
namespace {
const char CKPT_MAGIC[8] = {'K', 'P', 'Z', 'B', 'C', 'K', 'P', 'T'};
struct CkptTrailer {  // little-endian, written field by field
    uint32_t version, dyn, lx, ly;
    uint64_t tdev, seed;
    uint32_t stream_id, fusion;
    double p, q;
    uint32_t has_snap, dt_scheme;  // dt_scheme: the DT inner scheme (0 in files of other dynamics)
    double snap_mean;
};
}  // namespace

extern "C" kpzb_status kpzb_save(kpzb_handle* h, const char* path, const char* meta)
{
    KPZB_CHECK_H(h);
    if (!path) return fail(KPZB_EINVAL, "null path");
    std::vector<uint32_t> words(h->words());
    kpzb_status st = kpzb_pop(h, words.data());
    if (st != KPZB_OK) return st;
    std::vector<uint32_t> snap;
    if (h->has_snap) {
        snap.resize(h->words());
        KPZB_CU(cudaMemcpyAsync(snap.data(), h->d_snap, snap.size() * 4, cudaMemcpyDeviceToHost, h->st), "snapshot");
        KPZB_CU(cudaStreamSynchronize(h->st), "snapshot");
    }
    FILE* f = fopen(path, "wb");
    if (!f) return fail(KPZB_EINVAL, "cannot open the checkpoint file for writing");
    bool ok = fprintf(f, "%d\n%d\n", h->lx, h->ly) > 0;
    if (meta) ok = ok && fputs(meta, f) >= 0;
    ok = ok && fputc('\0', f) != EOF;
    ok = ok && fwrite(words.data(), 4, words.size(), f) == words.size();
    CkptTrailer t{};
    t.version = 1;
    t.dyn = (uint32_t)h->dyn;
    t.lx = (uint32_t)h->lx;
    t.ly = (uint32_t)h->ly;
    t.tdev = h->tdev;
    t.seed = h->seed;
    t.stream_id = h->stream_id;
    t.fusion = (uint32_t)h->fusion;
    t.p = h->p;
    t.q = h->q;
    t.has_snap = h->has_snap ? 1u : 0u;
    t.dt_scheme = h->dyn == KPZB_DYN_DT ? (uint32_t)h->dt.scheme : 0u;
    t.snap_mean = h->snap_mean;
    ok = ok && fwrite(CKPT_MAGIC, 1, 8, f) == 8 && fwrite(&t, sizeof t, 1, f) == 1;
    if (h->has_snap) ok = ok && fwrite(snap.data(), 4, snap.size(), f) == snap.size();
    ok = (fclose(f) == 0) && ok;
    return ok ? KPZB_OK : fail(KPZB_EINVAL, "checkpoint write failed");
}

extern "C" kpzb_status kpzb_load(kpzb_handle* h, const char* path)
{
    KPZB_CHECK_H(h);
    if (!path) return fail(KPZB_EINVAL, "null path");
    FILE* f = fopen(path, "rb");
    if (!f) return fail(KPZB_EINVAL, "cannot open the checkpoint file");
    int lx = -1, ly = -1;
    bool ok = fscanf(f, "%d\n%d", &lx, &ly) == 2;
    if (ok) {  // rest of the second line, then the meta text up to its '\0'
        int c;
        while ((c = fgetc(f)) != EOF && c != '\n') {
        }
        while ((c = fgetc(f)) != EOF && c != '\0') {
        }
        ok = c == '\0';
    }
    if (!ok || lx != h->lx || ly != h->ly) {
        fclose(f);
        return fail(KPZB_EINVAL, "not a lattice file of this handle's size");
    }
    std::vector<uint32_t> words(h->words());
    if (fread(words.data(), 4, words.size(), f) != words.size()) {
        fclose(f);
        return fail(KPZB_EINVAL, "truncated lattice words");
    }
    char magic[8];
    CkptTrailer t{};
    std::vector<uint32_t> snap;
    const bool has_trailer = fread(magic, 1, 8, f) == 8 && memcmp(magic, CKPT_MAGIC, 8) == 0;
    if (has_trailer) {
        ok = fread(&t, sizeof t, 1, f) == 1 && t.version == 1 && t.lx == (uint32_t)h->lx &&
             t.ly == (uint32_t)h->ly && t.dyn == (uint32_t)h->dyn && t.dt_scheme <= (uint32_t)DT_SCHEME_DBSHREP;
        if (ok && t.has_snap) {
            snap.resize(h->words());
            ok = fread(snap.data(), 4, snap.size(), f) == snap.size();
        }
    }
    fclose(f);
    if (!ok) return fail(KPZB_EINVAL, "bad checkpoint trailer (other dynamics, size or version)");
    kpzb_status st = kpzb_push(h, words.data());
    if (st != KPZB_OK) return st;
    if (has_trailer) {
        h->tdev = t.tdev;
        h->seed = t.seed;
        h->stream_id = t.stream_id;
        h->fusion = (int)t.fusion;
        h->p = t.p;
        h->q = t.q;
        h->has_snap = t.has_snap != 0;
        h->snap_mean = t.snap_mean;
        if (h->dyn == KPZB_DYN_DT) h->dt.scheme = (int)t.dt_scheme;
        if (h->has_snap) {
            if (!h->d_snap) KPZB_CU(cudaMalloc(&h->d_snap, h->words() * 4), "cudaMalloc(snapshot)");
            KPZB_CU(cudaMemcpyAsync(h->d_snap, snap.data(), snap.size() * 4, cudaMemcpyHostToDevice, h->st), "snapshot");
            KPZB_CU(cudaStreamSynchronize(h->st), "snapshot");
        }
    }
    return KPZB_OK;
}

// ---------------------------------------------------------------------------------
// Measurement scheduling (kpz/sampling.h:84-100, kpz/kpzScaling.cpp:194-215)
// ---------------------------------------------------------------------------------
constexpr uint32_t TAG_SAMPLE = 6u;

static bool next_sample(const kpzb_sampling* s, uint64_t t, uint64_t index, uint64_t* next)
{
    double v;
    if (s->mode == KPZB_SAMPLE_LINEAR) {
        *next = t + s->interval;
        return true;
    }
    if (s->mode == KPZB_SAMPLE_EXP) {
        v = std::ceil(std::exp(std::log((double)t + 10.0) + s->density));
    } else {
        const uint32_t ctr[4] = {(uint32_t)index, (uint32_t)(index >> 32), TAG_SAMPLE << 24, 0u};
        uint32_t r[4];
        philox_host(ctr, s->seed, r);
        const double u = (double)r[0] * (1.0 / 4294967296.0);
        v = (double)t + std::floor(u * s->random_mean + s->random_mean);
    }
    if (!(v < 1.8e19)) return false;
    uint64_t n = (uint64_t)v;
    *next = n > t ? n : t + 1;
    return true;
}

static kpzb_status check_sampling(const kpzb_sampling* s)
{
    if (!s) return fail(KPZB_EINVAL, "null sampling");
    if (s->mode == KPZB_SAMPLE_LINEAR && s->interval == 0) return fail(KPZB_EINVAL, "linear interval 0");
    if (s->mode == KPZB_SAMPLE_EXP && !(s->density > 0.0)) return fail(KPZB_EINVAL, "exp density <= 0");
    if (s->mode == KPZB_SAMPLE_RANDOM && !(s->random_mean > 0.0)) return fail(KPZB_EINVAL, "random mean <= 0");
    if (s->mode < KPZB_SAMPLE_EXP || s->mode > KPZB_SAMPLE_RANDOM) return fail(KPZB_EINVAL, "unknown mode");
    return KPZB_OK;
}

static kpzb_status sample_times(const kpzb_sampling* s, uint64_t start, uint64_t end, std::vector<uint64_t>* out)
{
    kpzb_status st = check_sampling(s);
    if (st != KPZB_OK) return st;
    out->clear();
    uint64_t t = start, idx = 0;
    while (t < end) {
        uint64_t n;
        if (!next_sample(s, t, idx++, &n)) return fail(KPZB_EINVAL, "sample time overflow");
        t = n < end ? n : end;
        out->push_back(t);
        if (out->size() > (1u << 26)) return fail(KPZB_EINVAL, "more than 2^26 sample times");
    }
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_sample_times(const kpzb_sampling* s, uint64_t start, uint64_t end, uint64_t* times,
                                         int max, int* n)
{
    if (!n || (max > 0 && !times)) return fail(KPZB_EINVAL, "null argument");
    std::vector<uint64_t> v;
    kpzb_status st = sample_times(s, start, end, &v);
    if (st != KPZB_OK) return st;
    for (size_t i = 0; i < v.size() && (int)i < max; ++i) times[i] = v[i];
    *n = (int)v.size();
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_measure_run(kpzb_handle* h, const kpzb_sampling* s, uint64_t end, int64_t corr_start,
                                        uint64_t corr_stop, double* rows, int max_rows, int* n_rows)
{
    KPZB_CHECK_H(h);
    if (!n_rows || (max_rows > 0 && !rows)) return fail(KPZB_EINVAL, "null argument");
    if (end >= (1ull << 31)) return fail(KPZB_EINVAL, "device MCS counter limit 2^31");
    const uint64_t t_now = h->tdev;
    std::vector<uint64_t> times;
    kpzb_status st = sample_times(s, t_now, end, &times);
    if (st != KPZB_OK) return st;
    const bool tag = corr_start >= 0 && (uint64_t)corr_start >= t_now && (uint64_t)corr_start <= end;
    if (tag && (uint64_t)corr_start > t_now &&
        !std::binary_search(times.begin(), times.end(), (uint64_t)corr_start)) {
        times.insert(std::upper_bound(times.begin(), times.end(), (uint64_t)corr_start), (uint64_t)corr_start);
    }
    const bool tag_now = tag && (uint64_t)corr_start == t_now;  // snapshot before any MCS
    *n_rows = (int)times.size() + (tag_now ? 1 : 0);
    if (*n_rows > max_rows) return fail(KPZB_EINVAL, "rows buffer too small (see *n_rows)");
    if (tag_now) times.insert(times.begin(), t_now);
    if (times.empty()) return KPZB_OK;

    const size_t rb = analysis_record_bytes();
    unsigned char* d_rec = nullptr;
    KPZB_CU(cudaMallocAsync(&d_rec, rb * times.size(), h->st), "cudaMallocAsync(records)");
    if (tag && !h->d_snap) KPZB_CU(cudaMalloc(&h->d_snap, h->words() * 4), "cudaMalloc(snapshot)");
    kpzb_status rs = KPZB_OK;
    int snap_row = -1;
    for (size_t i = 0; i < times.size() && rs == KPZB_OK; ++i) {
        const uint64_t t = times[i];
        if (t > h->tdev) {
            rs = kpzb_mcs_async(h, (int)(t - h->tdev));
            if (rs != KPZB_OK) break;
        }
        const uint32_t* v;
        rs = cbbit_view(h, &v);
        if (rs != KPZB_OK) break;
        const bool corr = tag && snap_row >= 0 && t > (uint64_t)corr_start && t <= corr_stop;
        cudaError_t e = analysis_moments_record(v, corr ? h->d_snap : nullptr, h->lx, h->ly, &h->an, d_rec + i * rb, h->st);
        if (e == cudaSuccess && tag && t == (uint64_t)corr_start) {
            e = cudaMemcpyAsync(h->d_snap, v, h->words() * 4, cudaMemcpyDeviceToDevice, h->st);
            snap_row = (int)i;
        }
        if (e != cudaSuccess) rs = cuda_fail(e, "measurement");
    }
    std::vector<unsigned char> host(rb * times.size());
    cudaError_t e = cudaMemcpyAsync(host.data(), d_rec, host.size(), cudaMemcpyDeviceToHost, h->st);
    cudaFreeAsync(d_rec, h->st);
    kpzb_status js = kpzb_join(h);  // also reports a bounded device wait that expired
    if (rs != KPZB_OK) return rs;
    if (e != cudaSuccess) return cuda_fail(e, "measurement records");
    if (js != KPZB_OK) return js;
    const long double N = (long double)((uint64_t)1 << (h->lx + h->ly));
    long double snap_mean = 0.0L;
    for (size_t i = 0; i < times.size(); ++i) {
        MomentsOut m;
        analysis_decode_record(host.data() + i * rb, &m);
        double* row = rows + 11 * i;
        long double h0;
        row[0] = (double)times[i];
        fill_roughness(m, h->lx, h->ly, row + 1, &h0);
        row[9] = row[10] = std::nan("");
        if ((int)i == snap_row) {
            snap_mean = h0;
            h->snap_mean = (double)h0;
            h->has_snap = true;
        } else if (snap_row >= 0 && (int)i > snap_row && times[i] <= corr_stop) {
            row[9] = (double)((long double)(double)m.cross / N - h0 * (long double)(double)snap_mean);
            row[10] = (double)((long double)m.agree / N / 2.0L);
        }
    }
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_get_mcs(const kpzb_handle* h, uint64_t* device_mcs)
{
    if (!h || !device_mcs) return fail(KPZB_EINVAL, "null argument");
    *device_mcs = h->tdev;
    return KPZB_OK;
}
extern "C" kpzb_status kpzb_set_mcs(kpzb_handle* h, uint64_t device_mcs)
{
    if (!h) return fail(KPZB_EINVAL, "null handle");
    if (device_mcs >= (1ull << 31)) return fail(KPZB_EINVAL, "device MCS counter limit 2^31");
    h->tdev = device_mcs;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_enable_counters(kpzb_handle* h, int on)
{
    if (!h) return fail(KPZB_EINVAL, "null handle");
    h->count = on != 0;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_counters(kpzb_handle* h, int64_t dep_des[2], int reset)
{
    KPZB_CHECK_H(h);
    if (!dep_des) return fail(KPZB_EINVAL, "null output");
    unsigned long long c[2];
    KPZB_CU(cudaMemcpyAsync(c, h->d_counters, sizeof c, cudaMemcpyDeviceToHost, h->st), "counters");
    if (reset) KPZB_CU(cudaMemsetAsync(h->d_counters, 0, sizeof c, h->st), "counters reset");
    KPZB_CU(cudaStreamSynchronize(h->st), "counters sync");
    dep_des[0] = (int64_t)c[0];
    dep_des[1] = (int64_t)c[1];
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_check_invariants(kpzb_handle* h, int64_t rep[3])
{
    KPZB_CHECK_H(h);
    if (!rep) return fail(KPZB_EINVAL, "null output");
    const uint32_t* v;
    kpzb_status s = cbbit_view(h, &v);
    if (s != KPZB_OK) return s;
    KPZB_CU(analysis_invariants(v, h->lx, h->ly, &h->an, rep, h->st), "invariants");
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_device_ptr(kpzb_handle* h, uint32_t** d_words, size_t* nwords)
{
    if (!h || !d_words) return fail(KPZB_EINVAL, "null argument");
    *d_words = h->d_sys;
    if (nwords) *nwords = h->words();
    return KPZB_OK;
}

extern "C" void* kpzb_stream(kpzb_handle* h) { return h ? (void*)h->st : nullptr; }

extern "C" kpzb_status kpzb_set_stream(kpzb_handle* h, void* stream)
{
    KPZB_CHECK_H(h);
    KPZB_CU(cudaStreamSynchronize(h->st), "set_stream sync");
    h->st = stream ? (cudaStream_t)stream : h->own_st;
    return KPZB_OK;
}
