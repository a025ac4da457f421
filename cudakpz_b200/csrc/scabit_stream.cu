// scabit_stream.cu -- temporally blocked SCABit in streaming (wavefront) form (sm_100a).
//
// Same dynamics as the one-launch-per-half-step kernel and the band kernel: the rule of
// kpz/kpzSCABit.cu:179-290 with the masks of kpz/kpzSCABitCores.cu:69-74,139-145, the
// counter-based decision of kpzb_common.cuh, k MCS (2k half-steps) per HBM pass.
//
// A CTA owns a chunk of Hc consecutive full-width rows and walks it top to bottom with all
// 2k half-steps in flight at once: at tick tau, half-step h works on chunk row
//     r_h(tau) = tau - 2k - 2h,
// i.e. each half-step trails the previous one by two rows.  Half-step h at row r reads and
// writes rows r and r+1 only, and needs half-step h-1 done at rows r-1..r+1; the two-row skew
// gives exactly that, and the rows worked on in one tick are two apart, so all 2k half-steps
// of a tick run in parallel with one barrier per tick.  Half-step h covers chunk rows
// [h - 2k, Hc + 2k - 1 - h) -- the same trapezoid as the band kernel, whose middle Hc rows
// are exact after 2k half-steps -- so every (half-step, row) update is the one the band and
// per-half-step kernels perform, in an order that respects every dependence between them.
//
// Rows live in a ring of nb = 4k + 1 + P + Lg slots (each slot: one row of all four
// ENC_CBBIT quadrants) in shared memory.  Lane 0 of an extra warp, which computes nothing,
// streams rows in with TMA bulk copies (cp.async.bulk, local HBM only) P+1 ticks before their
// first use, each slot with its own mbarrier and a bounded wait, and streams each row out with
// a bulk store the tick after it becomes final; a slot is refilled only after
// cp.async.bulk.wait_group.read has seen its store read out (at most Lg store groups in
// flight).  P is as deep as shared memory allows, up to 16 rows.  Compared with the band kernel, the
// recomputed halo is 4k rows per chunk instead of per band of B rows, and copies overlap
// compute.
#include <cstdio>

#include "kpzb_api_internal.h"
#include "kpzb_common.cuh"
#include "kpzb_internal.h"
#include "scabit_band.cuh"

namespace kpzb {

constexpr int STREAM_THREADS = 1024;
constexpr int STREAM_MIN_PREFETCH = 3;   // P: rows loaded P+1 ticks before first use (P >= 3)
constexpr int STREAM_MAX_PREFETCH = 16;  // deeper is never needed to cover the copy latency
constexpr int STREAM_STORE_LAG = 8;      // Lg: bulk-store groups allowed to be reading shared memory
constexpr int STREAM_MAX_K = 8;
constexpr int STREAM_MAX_SLOTS = 4 * STREAM_MAX_K + 1 + STREAM_MAX_PREFETCH + STREAM_STORE_LAG;

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_lag()
{
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(STREAM_STORE_LAG) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

template <int MODE, bool USEQ, bool COUNT>
__global__ void __launch_bounds__(STREAM_THREADS, 1)
scabit_stream_kernel(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, int lx, int ly,
                     int k, int nb, int pf, uint32_t t0, Key key, uint32_t stream, Thresh tp, Thresh tq,
                     unsigned long long* __restrict__ counters, unsigned int* __restrict__ err)
{
    extern __shared__ __align__(128) uint32_t ring[];  // nb slots x 4 quadrants x Wr words
    __shared__ __align__(8) uint64_t bars[STREAM_MAX_SLOTS];

    const int tid = threadIdx.x;
    const int NT = (int)blockDim.x - 32;  // compute threads; the last warp streams rows
    const bool copier = tid == NT;        // lane 0 of the last warp issues every copy
    const uint32_t Wr = 1u << (lx - 6);        // words per quadrant row
    const int lgG = lx - 8;                     // log2 of 4-word groups per row
    const uint32_t G = 1u << lgG;
    const uint64_t Q = 1ull << (lx + ly - 6);   // words per quadrant
    const uint32_t rows = 1u << ly;
    const uint32_t rmask = rows - 1u;
    const uint32_t slot_words = 4u * Wr;
    const int K2 = 2 * k;
    const int64_t c = blockIdx.x, nch = gridDim.x;
    const int y0 = (int)(c * rows / nch);
    const int Hc = (int)((c + 1) * rows / nch) - y0;
    const int rlo = -K2, rhi = Hc + K2;  // chunk rows ever loaded: [rlo, rhi)
    const int T = Hc + 3 * K2 - 2;       // ticks

    // thread 0's view of the copy pipeline
    int next_load = rlo;   // next chunk row to load
    int next_wait = rlo;   // next chunk row whose load completion has not been observed

    auto slot_of = [&](int r) -> int { return (r + K2) % nb; };
    auto issue_load = [&](int r) {
        const int s = slot_of(r);
        uint64_t* bar = &bars[s];
        mbar_expect_tx(bar, 16u * Wr);
        const uint64_t grow = (uint64_t)((uint32_t)(y0 + r) & rmask) * Wr;
        uint32_t* dstp = ring + (uint32_t)s * slot_words;
#pragma unroll
        for (int qd = 0; qd < 4; ++qd) bulk_g2s(dstp + qd * Wr, src + qd * Q + grow, 4u * Wr, bar);
    };
    auto wait_row = [&](int r) -> bool {
        const int s = slot_of(r);
        const uint32_t parity = (uint32_t)((r + K2) / nb) & 1u;
        uint32_t spins = 0;
        while (!mbar_try_wait(&bars[s], parity))
            if (++spins > MBAR_SPIN_LIMIT) return false;
        return true;
    };

    if (copier) {
        for (int s = 0; s < nb; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (; next_load <= rlo + 1 + pf && next_load < rhi; ++next_load) issue_load(next_load);
    }
    __syncthreads();

    const int mode_items = K2 << lgG;
    unsigned long long ndep = 0, ndes = 0;
    int tm = 0;  // tau mod nb

    bool aborted = false;
    for (int tau = 0; tau < T; ++tau) {
        bool timed_out = false;
        if (copier) {
            // rows first needed at this tick: tau - 2k + 1 (and row -2k at tick 0)
            const int need = tau - K2 + 1 < rhi - 1 ? tau - K2 + 1 : rhi - 1;
            for (; next_wait <= need; ++next_wait)
                if (!wait_row(next_wait)) {
                    timed_out = true;
                    break;
                }
        }
        // the barrier itself carries the decision, so every thread leaves at the same tick
        if (__syncthreads_or(timed_out)) {
            aborted = true;
            break;
        }
        if (copier) {
            // store the row that became final in the previous tick, then refill one slot
            const int yf = tau - 3 * K2 + 1;
            if (yf >= 0 && yf < Hc) {
                const uint64_t grow = (uint64_t)((uint32_t)(y0 + yf) & rmask) * Wr;
                const uint32_t* srcp = ring + (uint32_t)slot_of(yf) * slot_words;
#pragma unroll
                for (int qd = 0; qd < 4; ++qd) bulk_s2g(dst + qd * Q + grow, srcp + qd * Wr, 4u * Wr);
            }
            bulk_commit();
            if (next_load < rhi && next_load <= tau - K2 + 2 + pf) {
                bulk_wait_read_lag();
                issue_load(next_load);
                ++next_load;
            }
        }

        for (int i = tid; i < mode_items && tid < NT; i += NT) {
            const int h = i >> lgG;
            const uint32_t g = (uint32_t)i & (G - 1u);
            const int r = tau - K2 - 2 * h;
            if (r < h - K2 || r >= Hc + K2 - 1 - h) continue;
            int s = tm - 2 * h;
            if (s < 0) s += nb;
            const int s1 = (s + 1 == nb) ? 0 : s + 1;
            const int sigma = h & 1;
            const uint32_t step = 2u * (t0 + (uint32_t)(h >> 1)) + (uint32_t)sigma;
            const uint32_t gy = (uint32_t)(y0 + r) & rmask;
            uint32_t* row = ring + (uint32_t)s * slot_words;
            uint32_t* row1 = ring + (uint32_t)s1 * slot_words;
            const uint32_t w0 = 4u * g;
            uint32_t* StX = row + (sigma ? 2u : 0u) * Wr;
            uint32_t* SoX = row + (sigma ? 0u : 2u) * Wr;
            sca_update_group<MODE, USEQ, COUNT>(StX + w0, StX + Wr + w0, SoX + w0,
                                                row1 + (sigma ? 1u : 3u) * Wr + w0, SoX + ((w0 + 4u) & (Wr - 1u)),
                                                sigma != (int)(gy & 1u), MODE, tp, tq, key, (gy << lgG) + g, step,
                                                stream, r >= 0 && r < Hc, ndep, ndes);
            // the last half-step's writes are the only ones a bulk store reads (its rows become
            // final here and are stored next tick): order them before that async-proxy read
            if (h == K2 - 1) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        if (++tm == nb) tm = 0;
    }

    __syncthreads();
    if (copier) {
        if (aborted) {
            atomicExch(err, 1u);
            // let every load already issued land in this CTA's shared memory (bounded) before exit
            for (; next_wait < next_load; ++next_wait)
                if (!wait_row(next_wait)) break;
        } else {
            const int yf = T - 3 * K2 + 1;  // the row finished in the last tick
            if (yf >= 0 && yf < Hc) {
                const uint64_t grow = (uint64_t)((uint32_t)(y0 + yf) & rmask) * Wr;
                const uint32_t* srcp = ring + (uint32_t)slot_of(yf) * slot_words;
#pragma unroll
                for (int qd = 0; qd < 4; ++qd) bulk_s2g(dst + qd * Q + grow, srcp + qd * Wr, 4u * Wr);
            }
            bulk_commit();
        }
        bulk_wait_all();
    }
    if (COUNT) {
        for (int o = 16; o > 0; o >>= 1) {
            ndep += __shfl_xor_sync(0xffffffffu, ndep, o);
            ndes += __shfl_xor_sync(0xffffffffu, ndes, o);
        }
        if ((tid & 31) == 0 && (ndep | ndes)) {
            atomicAdd(&counters[0], ndep);
            atomicAdd(&counters[1], ndes);
        }
    }
}

// ctas_per_sm: chunks per SM (1 or 2); two CTAs share an SM only when both fit.
StreamShape scabit_stream_shape(int lx, int ly, int mcs_per_pass, int sm_count, int ctas_per_sm)
{
    StreamShape s{};
    s.ok = false;
    const int k = mcs_per_pass;
    if (k < 1 || k > STREAM_MAX_K || lx < 8) return s;
    const uint64_t Wr = 1ull << (lx - 6);
    if (ctas_per_sm < 1 || ctas_per_sm > 2) return s;
    // as deep a prefetch as the shared-memory budget allows (it hides the copy latency)
    const size_t budget = ctas_per_sm == 1 ? 227 * 1024 - 1024 : 228 * 1024 / 2 - 2048;
    const int max_slots = (int)(budget / (16ull * Wr));
    int pf = max_slots - (4 * k + 1 + STREAM_STORE_LAG);
    if (pf > STREAM_MAX_PREFETCH) pf = STREAM_MAX_PREFETCH;
    if (pf < STREAM_MIN_PREFETCH) return s;
    const int nb = 4 * k + 1 + pf + STREAM_STORE_LAG;
    const size_t smem = (size_t)nb * 16ull * Wr;
    const int64_t rows = 1ll << ly;
    const int items = (2 * k) << (lx - 8);
    int threads = items < STREAM_THREADS - 32 ? items : STREAM_THREADS - 32;
    threads = (threads + 31) / 32 * 32 + 32;  // + the copy warp
    s.mcs = k;
    s.slots = nb;
    s.prefetch = pf;
    s.smem = smem;
    s.threads = threads;
    if (ctas_per_sm == 2 && threads > STREAM_THREADS / 2 + 32) return s;
    const int64_t chunks = (int64_t)sm_count * ctas_per_sm;
    s.grid = (int)(rows < chunks ? rows : chunks);
    s.ok = true;
    return s;
}

template <int MODE, bool USEQ, bool COUNT>
static cudaError_t launch_stream(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0,
                                 Key key, uint32_t stream_id, Thresh tp, Thresh tq, const StreamShape& sh,
                                 unsigned long long* d_counters, unsigned int* d_err, cudaStream_t st)
{
    auto kern = scabit_stream_kernel<MODE, USEQ, COUNT>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem);
    if (e != cudaSuccess) return e;
    kern<<<sh.grid, sh.threads, sh.smem, st>>>(d_src, d_dst, lx, ly, sh.mcs, sh.slots, sh.prefetch, t0, key, stream_id,
                                               tp, tq, d_counters, d_err);
    return cudaGetLastError();
}

template <int MODE, bool USEQ>
static cudaError_t launch_stream_c(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0,
                                   Key key, uint32_t stream_id, Thresh tp, Thresh tq, const StreamShape& sh,
                                   unsigned long long* d_counters, unsigned int* d_err, cudaStream_t st)
{
    if (d_counters)
        return launch_stream<MODE, USEQ, true>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh,
                                               d_counters, d_err, st);
    return launch_stream<MODE, USEQ, false>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, nullptr,
                                            d_err, st);
}

cudaError_t scabit_stream(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0,
                          uint64_t seed, uint32_t stream_id, uint64_t Tp, uint64_t Tq, const StreamShape& sh,
                          unsigned long long* d_counters, unsigned int* d_err, cudaStream_t st)
{
    const Key key = make_key(seed);
    const Thresh tp = make_thresh(Tp), tq = make_thresh(Tq);
    const int mode = dec_mode(tp, tq);
    const bool useq = tq.always || tq.planes > 0;
#define KPZB_STREAM_CASE(M)                                                                                   \
    return useq ? launch_stream_c<M, true>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, d_counters, \
                                           d_err, st)                                                        \
                : launch_stream_c<M, false>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, d_counters, \
                                            d_err, st)
    if (mode == DEC_NONE) KPZB_STREAM_CASE(DEC_NONE);
    if (mode == DEC_ONE) KPZB_STREAM_CASE(DEC_ONE);
    KPZB_STREAM_CASE(DEC_GENERAL);
#undef KPZB_STREAM_CASE
}

}  // namespace kpzb
