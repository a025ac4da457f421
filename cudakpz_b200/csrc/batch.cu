// batch.cu -- many independent SCABit lattices of uneven size in one persistent kernel.
//
// Replaces the per-lattice launch loop (one SchedulerSCABit per lattice, two launches per
// MCS each: kpz/schedulerSCABit.cu:46-73, driven by kpz/kpzScaling.cpp:194-215) with a work
// queue: every pass advances ALL replicas by k MCS.  Work items are (replica, band) pairs,
// sorted by cost, pulled by persistent CTAs (one per SM) from a global atomic counter.
// Lattices that fit in shared memory are resident (whole lattice, periodic, no halo);
// larger ones are cut into bands with a 2k-row halo (scabit_band.cuh).  The pass index
// (t, buffer parity) lives in device memory and a one-thread kernel advances it after each
// pass, so a chunk of passes is captured once as a CUDA graph and replayed.
// Per-replica results are bit-identical to single runs: the random stream depends only on
// (seed, stream, half-step, site).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "kpzb_api_internal.h"
#include "kpzb_common.cuh"
#include "kpzb_internal.h"
#include "scabit_band.cuh"

namespace kpzb {

constexpr int BATCH_THREADS = 512;  // threads of a CTA at one CTA per SM; 256 at two or three
constexpr size_t BATCH_SMEM = 227 * 1024 - 1024;

// shared memory of one CTA at `cps` CTAs per SM (the SM's 228 KB split, 1 KB each reserved)
inline size_t batch_smem(int cps) { return cps <= 1 ? BATCH_SMEM : ((228 * 1024) / (size_t)cps - 1024) & ~(size_t)127; }
inline int batch_threads(int cps) { return cps <= 1 ? BATCH_THREADS : 256; }

struct RepDesc {
    uint32_t* buf[2];  // double buffer; buf[parity] holds the current state
    int lx, ly;
    int B;             // band rows (rows when resident)
    int resident;
    Key key;
    uint32_t stream;
    Thresh tp, tq;
};

struct Item {
    int rep;
    int band;
};

struct PassState {
    uint32_t t;       // MCS index of the next pass
    uint32_t parity;  // buffer holding the current state
    uint32_t queue;   // work-queue head for the running pass
    uint32_t err;     // set when a bounded wait expired
};

template <int THREADS>
__global__ void __launch_bounds__(THREADS)
batch_pass_kernel(const RepDesc* __restrict__ reps, const Item* __restrict__ items, int nitems,
                  PassState* st, int k)
{
    extern __shared__ __align__(128) uint32_t smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int abort_flag;
    __shared__ int cur;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const uint32_t t0 = st->t;
    const uint32_t par = st->parity;
    uint32_t phase = 0;
    unsigned long long nd = 0, nr = 0;
    for (;;) {
        if (threadIdx.x == 0) cur = (int)atomicAdd(&st->queue, 1u);
        __syncthreads();
        const int i = cur;
        __syncthreads();
        if (i >= nitems) break;
        const Item it = items[i];
        const RepDesc r = reps[it.rep];
        const BandCtl ctl{&bar, &abort_flag, phase};
        const BandGeom g{r.buf[par], r.buf[par ^ 1u], r.lx, r.ly, (int64_t)it.band * r.B, r.B, k,
                         r.resident != 0, t0, r.key, r.stream, r.tp, r.tq};
        // rates differ between replicas of one launch: the run-time decision mode (a per-item
        // dispatch to rate-specialised copies measured 2-5 % slower: larger code, more registers)
        if (!scabit_band<-1, true, false, THREADS>(smem, ctl, g, nd, nr, &st->err)) return;
        phase ^= 1u;
    }
}

__global__ void batch_advance_kernel(PassState* st, int k)
{
    st->t += (uint32_t)k;
    st->parity ^= 1u;
    st->queue = 0;
}

}  // namespace kpzb

using namespace kpzb;

struct kpzb_batch {
    int n = 0, device = 0, sm_count = 148;
    cudaStream_t st = nullptr;
    std::vector<int> lx;
    std::vector<double> p, q;
    std::vector<uint64_t> seed;
    std::vector<uint32_t> stream;
    std::vector<RepDesc> reps;  // host copy
    RepDesc* d_reps = nullptr;
    Item* d_items = nullptr;
    int nitems = 0;
    PassState* d_state = nullptr;
    uint32_t t = 0, parity = 0;  // host mirror of the pass state
    int k = 8;                   // MCS per pass
    int chunk = 8;               // passes per graph replay
    int cps = 1;                 // CTAs per SM (1: 512 threads, 2 or 3: 256 threads each)
    bool planned = false;        // k and cps set by the caller or the tuner (else tuned on first MCS)
    cudaGraphExec_t graph = nullptr;
    AnalysisScratch an{};
    int max_ly = 0;
};

static uint64_t thresh_b(double p)
{
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return 1ull << 32;
    const double t = std::ceil(p * 4294967296.0);
    return t >= 4294967296.0 ? (1ull << 32) : (uint64_t)t;
}

// (Re)build the band layout and work list for MCS-per-pass k.
static kpzb_status batch_layout(kpzb_batch* b)
{
    // passes in flight read the descriptor table and the work list
    if (b->st) {
        const cudaError_t se = cudaStreamSynchronize(b->st);
        if (se != cudaSuccess) return cuda_fail(se, "batch sync");
    }
    std::vector<std::pair<double, Item>> work;
    for (int i = 0; i < b->n; ++i) {
        RepDesc& r = b->reps[i];
        const uint64_t Wr = 1ull << (r.lx - 6);
        const uint64_t row_bytes = 16ull * Wr;
        const int64_t rows = 1ll << r.ly;
        const size_t smem = batch_smem(b->cps);
        if ((uint64_t)rows * row_bytes <= smem) {
            r.resident = 1;
            r.B = (int)rows;
            work.push_back({(double)rows * Wr, Item{i, 0}});
            continue;
        }
        r.resident = 0;
        const int Rmax = (int)(smem / row_bytes);
        const int Bmax = Rmax - 4 * b->k;
        if (Bmax < 1) return fail(KPZB_EINVAL, "batch: lattice rows too wide for the pass depth");
        const int nb = (int)((rows + Bmax - 1) / Bmax);
        r.B = (int)((rows + nb - 1) / nb);
        for (int band = 0; band < nb; ++band)
            work.push_back({(double)(r.B + 4 * b->k) * Wr, Item{i, band}});
    }
    std::stable_sort(work.begin(), work.end(),
                     [](const std::pair<double, Item>& a, const std::pair<double, Item>& c) {
                         return a.first > c.first;
                     });
    std::vector<Item> items;
    for (auto& w : work) items.push_back(w.second);
    b->nitems = (int)items.size();
    cudaFree(b->d_items);
    b->d_items = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&b->d_items, items.size() * sizeof(Item))) != cudaSuccess)
        return cuda_fail(e, "cudaMalloc(items)");
    cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(Item), cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_reps, b->reps.data(), b->reps.size() * sizeof(RepDesc), cudaMemcpyHostToDevice);
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return KPZB_OK;
}

static cudaError_t enqueue_pass(kpzb_batch* b)
{
    if (b->cps <= 1)
        batch_pass_kernel<BATCH_THREADS><<<b->sm_count, BATCH_THREADS, BATCH_SMEM, b->st>>>(
            b->d_reps, b->d_items, b->nitems, b->d_state, b->k);
    else
        batch_pass_kernel<256><<<b->sm_count * b->cps, 256, batch_smem(b->cps), b->st>>>(
            b->d_reps, b->d_items, b->nitems, b->d_state, b->k);
    batch_advance_kernel<<<1, 1, 0, b->st>>>(b->d_state, b->k);
    return cudaGetLastError();
}

#define BCHECK(b)                                                       \
    do {                                                                \
        if (!(b)) return fail(KPZB_EINVAL, "null batch");               \
        cudaError_t _e = cudaSetDevice((b)->device);                    \
        if (_e != cudaSuccess) return cuda_fail(_e, "cudaSetDevice");   \
    } while (0)

extern "C" kpzb_status kpzb_batch_create(kpzb_batch** out, int n, const int* lx, const double* p,
                                         const double* q, const uint64_t* seed,
                                         const uint32_t* stream, int device)
{
    if (!out || n <= 0 || !lx || !p || !q || !seed) return fail(KPZB_EINVAL, "bad batch arguments");
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        if (lx[i] < 8 || lx[i] > 16 || 2 * lx[i] < 14)
            return fail(KPZB_EINVAL, "batch lattices are square with 8 <= lx <= 16");
        if (!(p[i] >= 0 && p[i] <= 1 && q[i] >= 0 && q[i] <= 1)) return fail(KPZB_EINVAL, "p, q in [0,1]");
    }
    int dev = device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return fail(KPZB_ECUDA, "cudaGetDevice");
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    kpzb_batch* b = new kpzb_batch();
    b->n = n;
    b->device = dev;
    b->sm_count = sm_count_of(dev);
    auto bail = [&](kpzb_status s) {
        kpzb_batch_destroy(b);
        return s;
    };
    if ((e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(cuda_fail(e, "cudaStreamCreate"));
    b->reps.resize(n);
    for (int i = 0; i < n; ++i) {
        b->lx.push_back(lx[i]);
        b->p.push_back(p[i]);
        b->q.push_back(q[i]);
        b->seed.push_back(seed[i]);
        b->stream.push_back(stream ? stream[i] : 0u);
        RepDesc& r = b->reps[i];
        r.lx = r.ly = lx[i];
        r.key = make_key(seed[i]);
        r.stream = stream ? stream[i] : 0u;
        r.tp = make_thresh(thresh_b(p[i]));
        r.tq = make_thresh(thresh_b(q[i]));
        const size_t bytes = (size_t)1 << (2 * lx[i] - 2);
        for (int s = 0; s < 2; ++s)
            if ((e = cudaMalloc(&r.buf[s], bytes)) != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(replica)"));
        b->max_ly = std::max(b->max_ly, lx[i]);
    }
    if ((e = cudaMalloc(&b->d_reps, n * sizeof(RepDesc))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(reps)"));
    if ((e = cudaMalloc(&b->d_state, sizeof(PassState))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(state)"));
    cudaMemset(b->d_state, 0, sizeof(PassState));
    if ((e = analysis_alloc(&b->an, b->max_ly)) != cudaSuccess) return bail(cuda_fail(e, "analysis_alloc"));
    if ((e = cudaFuncSetAttribute(batch_pass_kernel<BATCH_THREADS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)BATCH_SMEM)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(batch_pass_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)batch_smem(2))) != cudaSuccess)
        return bail(cuda_fail(e, "smem attribute"));
    kpzb_status s = batch_layout(b);
    if (s != KPZB_OK) return bail(s);
    s = kpzb_batch_init_homogeneous(b);
    if (s != KPZB_OK) return bail(s);
    *out = b;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_batch_destroy(kpzb_batch* b)
{
    if (!b) return KPZB_OK;
    cudaSetDevice(b->device);
    if (b->st) cudaStreamSynchronize(b->st);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (auto& r : b->reps) {
        cudaFree(r.buf[0]);
        cudaFree(r.buf[1]);
    }
    cudaFree(b->d_reps);
    cudaFree(b->d_items);
    cudaFree(b->d_state);
    if (b->an.rowinfo) analysis_free(&b->an);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_batch_init_homogeneous(kpzb_batch* b)
{
    BCHECK(b);
    for (auto& r : b->reps) {
        cudaError_t e = init_homogeneous_dev(r.buf[b->parity], r.lx, r.ly, KPZB_ENC_CBBIT, b->st);
        if (e != cudaSuccess) return cuda_fail(e, "batch init");
    }
    const cudaError_t e = cudaStreamSynchronize(b->st);
    return e == cudaSuccess ? KPZB_OK : cuda_fail(e, "batch init sync");
}

extern "C" kpzb_status kpzb_batch_set_fusion(kpzb_batch* b, int mcs_per_pass, int passes_per_graph)
{
    BCHECK(b);
    if (mcs_per_pass < 1 || mcs_per_pass > 32 || passes_per_graph < 1 || passes_per_graph > 256)
        return fail(KPZB_EINVAL, "batch fusion: 1 <= mcs_per_pass <= 32, 1 <= passes_per_graph <= 256");
    b->k = mcs_per_pass;
    b->chunk = passes_per_graph;
    b->planned = true;
    return batch_layout(b);
}

extern "C" kpzb_status kpzb_batch_set_ctas_per_sm(kpzb_batch* b, int ctas_per_sm)
{
    BCHECK(b);
    if (ctas_per_sm < 1 || ctas_per_sm > 3) return fail(KPZB_EINVAL, "batch: 1 <= ctas_per_sm <= 3");
    b->cps = ctas_per_sm;
    b->planned = true;
    return batch_layout(b);
}

extern "C" kpzb_status kpzb_batch_get_plan(const kpzb_batch* b, int* mcs_per_pass, int* ctas_per_sm)
{
    if (!b || !mcs_per_pass || !ctas_per_sm) return fail(KPZB_EINVAL, "null argument");
    *mcs_per_pass = b->k;
    *ctas_per_sm = b->cps;
    return KPZB_OK;
}

namespace {
std::mutex g_batch_mu;
std::map<std::string, std::pair<int, int>> g_batch_plans;  // batch signature -> (k, cps)

// the replicas' sizes and rate classes (random planes the decision needs), and the SM count:
// what the cost of a pass depends on
std::string batch_signature(const kpzb_batch* b)
{
    std::map<std::pair<int, int>, int> census;
    for (const RepDesc& r : b->reps) {
        const int planes = std::max(r.tp.planes, r.tq.planes);
        census[{r.lx, planes == 0 ? 0 : planes == 1 ? 1 : planes <= 4 ? 2 : 3}]++;
    }
    std::string key = "batch1:sm" + std::to_string(b->sm_count);
    for (auto& c : census)
        key += ":" + std::to_string(c.first.first) + "r" + std::to_string(c.first.second) + "x" +
               std::to_string(c.second);
    return key;
}
}  // namespace

// Times every (MCS per pass, CTAs per SM) shape on the replicas as they are and keeps the
// fastest; the replicas and the pass state are restored afterwards, so tuning changes no
// result (every shape gives bit-identical replicas).  Cached per batch signature.
extern "C" kpzb_status kpzb_batch_autotune(kpzb_batch* b, int* mcs_per_pass, int* ctas_per_sm, float* ms_per_mcs)
{
    BCHECK(b);
    cudaError_t e;
    if ((e = cudaStreamSynchronize(b->st)) != cudaSuccess) return cuda_fail(e, "batch sync");
    // snapshot of every replica's current buffer and of the pass state
    size_t total = 0;
    for (const RepDesc& r : b->reps) total += (size_t)1 << (2 * r.lx - 2);
    unsigned char* snap = nullptr;
    if ((e = cudaMalloc(&snap, total)) != cudaSuccess) return cuda_fail(e, "cudaMalloc(tune snapshot)");
    PassState saved{};
    size_t off = 0;
    for (const RepDesc& r : b->reps) {
        const size_t bytes = (size_t)1 << (2 * r.lx - 2);
        cudaMemcpyAsync(snap + off, r.buf[b->parity], bytes, cudaMemcpyDeviceToDevice, b->st);
        off += bytes;
    }
    cudaMemcpyAsync(&saved, b->d_state, sizeof saved, cudaMemcpyDeviceToHost, b->st);
    if ((e = cudaStreamSynchronize(b->st)) != cudaSuccess) {
        cudaFree(snap);
        return cuda_fail(e, "batch tune snapshot");
    }
    const int k0 = b->k, cps0 = b->cps;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int bk = k0, bc = cps0;
    kpzb_status st = KPZB_OK;
    const bool verbose = getenv("KPZB_TUNE_VERBOSE") != nullptr;
    for (int cps = 1; cps <= 3 && st == KPZB_OK; ++cps)
        for (int k : {2, 4, 6, 8}) {
            b->k = k;
            b->cps = cps;
            if ((st = batch_layout(b)) != KPZB_OK) {
                if (st == KPZB_EINVAL) {  // a lattice row too wide for this depth: not a candidate
                    st = KPZB_OK;
                    continue;
                }
                break;
            }
            const int passes = std::max(1, (16 + k - 1) / k);
            if ((e = enqueue_pass(b)) != cudaSuccess) break;  // warm-up
            cudaEventRecord(e0, b->st);
            for (int i = 0; i < passes && e == cudaSuccess; ++i) e = enqueue_pass(b);
            cudaEventRecord(e1, b->st);
            if (e != cudaSuccess || (e = cudaEventSynchronize(e1)) != cudaSuccess) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            const float per = ms / (float)(passes * k);
            if (verbose) fprintf(stderr, "kpzb batch tune k=%d cps=%d: %.4f ms/MCS\n", k, cps, per);
            if (per < best) {
                best = per;
                bk = k;
                bc = cps;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // restore the replicas and the pass state
    off = 0;
    for (const RepDesc& r : b->reps) {
        const size_t bytes = (size_t)1 << (2 * r.lx - 2);
        cudaMemcpyAsync(r.buf[b->parity], snap + off, bytes, cudaMemcpyDeviceToDevice, b->st);
        off += bytes;
    }
    PassState hs;
    cudaMemcpyAsync(&hs, b->d_state, sizeof hs, cudaMemcpyDeviceToHost, b->st);
    const cudaError_t se = cudaStreamSynchronize(b->st);
    const bool timed_out = se == cudaSuccess && hs.err != 0;
    saved.queue = 0;
    cudaMemcpy(b->d_state, &saved, sizeof saved, cudaMemcpyHostToDevice);
    cudaFree(snap);
    b->k = (e == cudaSuccess && st == KPZB_OK && best < 1e30f) ? bk : k0;
    b->cps = (e == cudaSuccess && st == KPZB_OK && best < 1e30f) ? bc : cps0;
    const kpzb_status ls = batch_layout(b);
    if (e != cudaSuccess) return cuda_fail(e, "batch tune");
    if (se != cudaSuccess) return cuda_fail(se, "batch tune restore");
    if (st != KPZB_OK) return st;
    if (ls != KPZB_OK) return ls;
    if (timed_out) return fail(KPZB_ETIMEOUT, "a bounded device wait (TMA mbarrier) expired while tuning");
    b->planned = true;
    {
        std::lock_guard<std::mutex> lk(g_batch_mu);
        g_batch_plans[batch_signature(b)] = {b->k, b->cps};
    }
    if (mcs_per_pass) *mcs_per_pass = b->k;
    if (ctas_per_sm) *ctas_per_sm = b->cps;
    if (ms_per_mcs) *ms_per_mcs = best;
    return KPZB_OK;
}

// the plan of a batch whose caller set none: a cached tuning of the same signature, else a
// fresh tuning (KPZB_AUTOTUNE=0: the fixed default, 8 MCS per pass at one CTA per SM)
static kpzb_status batch_resolve_plan(kpzb_batch* b)
{
    if (b->planned) return KPZB_OK;
    {
        std::lock_guard<std::mutex> lk(g_batch_mu);
        auto it = g_batch_plans.find(batch_signature(b));
        if (it != g_batch_plans.end()) {
            b->k = it->second.first;
            b->cps = it->second.second;
            b->planned = true;
        }
    }
    if (b->planned) return batch_layout(b);
    const char* env = getenv("KPZB_AUTOTUNE");
    if (env && env[0] == '0') {
        b->planned = true;
        return KPZB_OK;
    }
    return kpzb_batch_autotune(b, nullptr, nullptr, nullptr);
}

// n MCS for every replica: whole passes of k MCS (graph replays of `chunk` passes, then
// single passes), and a final pass of n mod k MCS.
extern "C" kpzb_status kpzb_batch_mcs(kpzb_batch* b, int n)
{
    BCHECK(b);
    if (n < 0) return fail(KPZB_EINVAL, "negative MCS count");
    if ((uint64_t)b->t + (uint64_t)n >= (1ull << 31)) return fail(KPZB_EINVAL, "MCS counter limit 2^31");
    if (n > 0) {
        const kpzb_status ps = batch_resolve_plan(b);
        if (ps != KPZB_OK) return ps;
    }
    cudaError_t e;
    int passes = n / b->k;
    const int rem = n % b->k;
    while (passes >= b->chunk) {
        if (!b->graph) {
            cudaGraph_t g;
            if ((e = cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
                return cuda_fail(e, "begin capture");
            for (int i = 0; i < b->chunk; ++i) enqueue_pass(b);
            if ((e = cudaStreamEndCapture(b->st, &g)) != cudaSuccess) return cuda_fail(e, "end capture");
            e = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
        }
        if ((e = cudaGraphLaunch(b->graph, b->st)) != cudaSuccess) return cuda_fail(e, "graph launch");
        passes -= b->chunk;
        b->t += (uint32_t)(b->chunk * b->k);
        b->parity ^= (uint32_t)(b->chunk & 1);
    }
    for (; passes > 0; --passes) {
        if ((e = enqueue_pass(b)) != cudaSuccess) return cuda_fail(e, "batch pass");
        b->t += (uint32_t)b->k;
        b->parity ^= 1u;
    }
    if (rem) {
        // one shorter pass: temporarily rebuild the bands for depth rem
        const int k = b->k;
        b->k = rem;
        kpzb_status s = batch_layout(b);
        if (s == KPZB_OK) {
            e = enqueue_pass(b);
            b->t += (uint32_t)rem;
            b->parity ^= 1u;
        }
        b->k = k;
        kpzb_status s2 = batch_layout(b);
        if (s != KPZB_OK) return s;
        if (s2 != KPZB_OK) return s2;
        if (e != cudaSuccess) return cuda_fail(e, "batch pass");
    }
    PassState hs;
    if ((e = cudaMemcpyAsync(&hs, b->d_state, sizeof hs, cudaMemcpyDeviceToHost, b->st)) != cudaSuccess)
        return cuda_fail(e, "batch state");
    if ((e = cudaStreamSynchronize(b->st)) != cudaSuccess) return cuda_fail(e, "batch sync");
    if (hs.err) return fail(KPZB_ETIMEOUT, "a bounded device wait (TMA mbarrier) expired");
    if (hs.t != b->t || hs.parity != b->parity) return fail(KPZB_ESTATE, "batch pass state out of step");
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_batch_push(kpzb_batch* b, int i, const uint32_t* words)
{
    BCHECK(b);
    if (i < 0 || i >= b->n || !words) return fail(KPZB_EINVAL, "bad replica index or buffer");
    const RepDesc& r = b->reps[i];
    cudaError_t e = cudaStreamSynchronize(b->st);
    if (e != cudaSuccess) return cuda_fail(e, "batch sync");
    e = cudaMemcpy(r.buf[b->parity], words, (size_t)1 << (2 * r.lx - 2), cudaMemcpyHostToDevice);
    return e == cudaSuccess ? KPZB_OK : cuda_fail(e, "batch push");
}

extern "C" kpzb_status kpzb_batch_pop(kpzb_batch* b, int i, uint32_t* words)
{
    BCHECK(b);
    if (i < 0 || i >= b->n || !words) return fail(KPZB_EINVAL, "bad replica index or buffer");
    const RepDesc& r = b->reps[i];
    cudaError_t e = cudaStreamSynchronize(b->st);
    if (e != cudaSuccess) return cuda_fail(e, "batch sync");
    e = cudaMemcpy(words, r.buf[b->parity], (size_t)1 << (2 * r.lx - 2), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? KPZB_OK : cuda_fail(e, "batch pop");
}

extern "C" kpzb_status kpzb_batch_roughness(kpzb_batch* b, double* w2)
{
    BCHECK(b);
    if (!w2) return fail(KPZB_EINVAL, "null output");
    for (int i = 0; i < b->n; ++i) {
        const RepDesc& r = b->reps[i];
        MomentsOut m;
        const cudaError_t e = analysis_moments(r.buf[b->parity], nullptr, r.lx, r.ly, &b->an, &m, b->st);
        if (e != cudaSuccess) return cuda_fail(e, "batch roughness");
        const long double N = (long double)((uint64_t)1 << (2 * r.lx));
        const long double h1 = (long double)m.s1 / N, h2 = (long double)m.s2 / N;
        w2[i] = (double)(h2 - h1 * h1);
    }
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_batch_get_mcs(const kpzb_batch* b, uint64_t* mcs)
{
    if (!b || !mcs) return fail(KPZB_EINVAL, "null argument");
    *mcs = b->t;
    return KPZB_OK;
}
