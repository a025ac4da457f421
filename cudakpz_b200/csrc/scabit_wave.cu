// scabit_wave.cu -- SCABit k-MCS pass with the half-steps kept in registers (sm_100a).
//
// The temporally blocked pass of scabit_fused_kernel (a band of B output rows plus 2k halo
// rows on each side, 2k half-steps, rows [2k, 2k + B) exact afterwards) with the lattice
// words held in registers instead of shared memory:
//   * a CTA spans the full width of a quadrant row, one word column per thread (Wr = L/64
//     threads, lx in [11, 14]);
//   * the 2k half-steps run as a diagonal wavefront: at tick tau, half-step h updates local
//     row tau - h.  An update of row r touches rows r and r + 1 only, and reads row r + 1 as
//     left by half-step h - 1 at tick tau - 1 (same thread), so one tick's updates touch
//     disjoint rows and depend on earlier ticks only; each thread keeps a window of 2k + 5
//     rows of its four quadrant words in registers (one row enters and one leaves per tick);
//   * within a tick every update is shifted or none is (row parity xor sublattice is
//     (y_lo + tau) mod 2), so the one-bit x-carry of shifted rows -- read from the next word,
//     and the flip of the next word's bit 0 -- moves between lanes by warp shuffles, and
//     between warps through shared memory: lane 0 of each warp publishes the words its left
//     neighbour will read in the next tick, lane 31 publishes its carry flips, and the
//     receiving lane 0 applies them at the next tick (before anything reads that bit); one
//     __syncthreads per tick;
//   * rows arrive through a ring of shared-memory slots filled by TMA bulk copies (one per
//     quadrant row, local HBM only) with per-slot mbarriers and bounded waits; finished rows
//     are stored straight from registers (coalesced).
// The updates -- which (half-step, row) pairs run, on which words, with which random words --
// are exactly those of the band kernel, so the output is bit-identical to every other pass
// shape and to the one-half-step kernel (kpz/kpzSCABit.cu:179-290 with the masks of
// kpz/kpzSCABitCores.cu:69-74,139-145).  Decision modes DEC_NONE and DEC_ONE; with DEC_ONE the
// four lanes of a 4-word Philox group each compute one half-step's call and exchange the
// words through shared memory.
#include <cstdint>

#include "kpzb_common.cuh"
#include "kpzb_internal.h"
#include "scabit_band.cuh"

namespace kpzb {

constexpr int WAVE_SLOTS = 8;  // TMA ring depth (rows of all four quadrants)
// bounded mbarrier wait: polls before a row counts as lost (each try_wait may itself suspend
// for a while, so this is far above any real copy time yet ends within a second or so)
constexpr uint32_t WAVE_SPIN_LIMIT = 1u << 18;

struct WaveSmem {
    // byte offsets into the dynamic shared memory
    uint32_t ring, xbuf, fbuf, rnd, bars, total;
};

__host__ __device__ inline WaveSmem wave_smem(int Wr, int K)
{
    const int nwarps = Wr / 32;
    WaveSmem s;
    s.ring = 0;
    s.xbuf = s.ring + (uint32_t)WAVE_SLOTS * 4u * (uint32_t)Wr * 4u;
    s.fbuf = s.xbuf + 2u * (uint32_t)nwarps * (uint32_t)(2 * K) * 4u;
    s.rnd = s.fbuf + 2u * (uint32_t)nwarps * 16u;
    s.bars = (s.rnd + (uint32_t)nwarps * 128u * 4u + 7u) & ~7u;
    s.total = s.bars + (uint32_t)WAVE_SLOTS * 8u;
    return s;
}

constexpr int WAVE_MAX_THREADS = 256;  // lx <= 14: a quadrant row of at most 256 words

// MINB: CTAs per SM the register allocation is sized for (the tuner's CTAs-per-SM choice)
template <int MODE, bool USEQ, bool COUNT, int K, int MINB>
__global__ void __launch_bounds__(WAVE_MAX_THREADS, MINB)
scabit_wave_kernel(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, int lx, int ly, int B,
                   uint32_t t0, Key key, uint32_t stream, Thresh tp, Thresh tq,
                   unsigned long long* __restrict__ counters, unsigned int* __restrict__ err)
{
    constexpr int H = 2 * K;       // halo rows on each side of the band
    constexpr int NH = 2 * K;      // half-steps per pass
    constexpr int NW = 2 * K + 5;  // register window rows (a unit of 4 ticks)
    extern __shared__ __align__(128) unsigned char wsm[];
    const int Wr = (int)blockDim.x;
    const int w = (int)threadIdx.x, lane = w & 31, warp = w >> 5, nwarps = Wr >> 5;
    const WaveSmem L = wave_smem(Wr, K);
    uint32_t* ring = reinterpret_cast<uint32_t*>(wsm + L.ring);
    uint32_t* xbuf = reinterpret_cast<uint32_t*>(wsm + L.xbuf);
    uint32_t* fbuf = reinterpret_cast<uint32_t*>(wsm + L.fbuf);
    uint32_t* rnd = reinterpret_cast<uint32_t*>(wsm + L.rnd) + warp * 128;
    uint64_t* bars = reinterpret_cast<uint64_t*>(wsm + L.bars);

    const int64_t rows = 1ll << ly;
    const uint64_t Q = 1ull << (lx + ly - 6);  // words per quadrant
    const uint32_t rmask = (uint32_t)rows - 1u;
    const int64_t y0 = (int64_t)blockIdx.x * B;
    const int Bc = (int)(rows - y0 < B ? rows - y0 : B);
    const int R = Bc + 2 * H;
    const uint32_t ylo = (uint32_t)((y0 - H) & (int64_t)rmask);  // global row of local row 0
    const int lgG = lx - 8;
    const uint32_t gword = (uint32_t)w >> 2;  // 4-word group of this column
    const int right = (warp + 1) % nwarps, left = (warp + nwarps - 1) % nwarps;

    if (w == 0) {
        for (int s = 0; s < WAVE_SLOTS; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // local row rho -> ring slot rho % WAVE_SLOTS (thread 0)
    auto issue = [&](int rho) {
        if (rho >= R) return;
        const int s = rho % WAVE_SLOTS;
        const uint64_t gy = (uint64_t)((ylo + (uint32_t)rho) & rmask);
        mbar_expect_tx(&bars[s], 16u * (uint32_t)Wr);
        for (int q = 0; q < 4; ++q)
            bulk_g2s(ring + ((size_t)s * 4 + q) * Wr, src + q * Q + gy * (uint64_t)Wr, 4u * (uint32_t)Wr, &bars[s]);
    };
    // wait (bounded) for local row rho; false when the copy did not arrive in time
    auto wait_row = [&](int rho) -> bool {
        const int s = rho % WAVE_SLOTS;
        const uint32_t parity = (uint32_t)(rho / WAVE_SLOTS) & 1u;
        uint32_t spins = 0;
        while (!mbar_try_wait(&bars[s], parity))
            if (++spins > WAVE_SPIN_LIMIT) return false;
        return true;
    };
    int issued_hi = -1;  // thread 0: highest local row issued to the ring
    if (w == 0)
        for (int rho = 0; rho < WAVE_SLOTS && rho < R; ++rho) {
            issue(rho);
            issued_hi = rho;
        }

    uint32_t win[4][NW];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int s = 0; s < NW; ++s) win[q][s] = 0u;
    bool timed_out = !wait_row(0);
    if (!timed_out) {
#pragma unroll
        for (int q = 0; q < 4; ++q) win[q][H] = ring[(size_t)q * Wr + w];
    }
    unsigned long long ndep = 0, ndes = 0;
    const uint32_t ap = tp.always ? 0xFFFFFFFFu : 0u, aq = tq.always ? 0xFFFFFFFFu : 0u;
    const uint32_t hp = tp.planes ? 0xFFFFFFFFu : 0u, hq = tq.planes ? 0xFFFFFFFFu : 0u;
    const int par0 = (int)(ylo & 1u);  // (y_lo + tau) & 1: the tick's updates are shifted
    const uint32_t keep0 = lane ? 0xFFFFFFFFu : 0u;  // lane 0's carry-in comes from the left warp
    // a shifted first tick reads the right warp's row-0 word (half-step 0's is the tick's only
    // exact update; the others read whatever the buffer holds and feed only inexact rows)
    if (par0 && lane == 0) xbuf[warp * NH] = win[2][H];

    if (__syncthreads_or(timed_out)) goto abort;
    // row 0 has left its slot
    if (w == 0 && WAVE_SLOTS < R) {
        issue(WAVE_SLOTS);
        issued_hi = WAVE_SLOTS;
    }

    for (int tau0 = 0; tau0 < R; tau0 += 4) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int tau = tau0 + i;
            const bool shifted = ((par0 + tau) & 1) != 0;
            // (1) row tau + 1 enters the window
            if (tau + 1 < R) {
                if (!wait_row(tau + 1)) timed_out = true;
                const int s = (tau + 1) % WAVE_SLOTS;
#pragma unroll
                for (int q = 0; q < 4; ++q) win[q][H + i + 1] = ring[((size_t)s * 4 + q) * Wr + w];
            }
            // (2) lane 0 applies the carry flips the left warp's lane 31 made in tick tau - 1
            // (one word: bit NH - 1 - h is half-step h's flip)
            if (tau >= 1 && !shifted && lane == 0) {
                const uint32_t fb = fbuf[(((tau - 1) & 1) * nwarps + left) * 4];
#pragma unroll
                for (int h = 0; h < NH; ++h) win[2 * (1 - (h & 1))][H + i - 1 - h] ^= (fb >> (NH - 1 - h)) & 1u;
            }
            // the right warp's published words, for lane 31's carries in a shifted tick
            const uint32_t* xr = xbuf + ((tau & 1) * nwarps + right) * NH;
            uint32_t fbits = 0;  // lane 31: this tick's carry flips into the right warp
            // random words of DEC_ONE: lane j of each 4-word group computes half-step hb + j's
            // Philox call; the four words of each call are exchanged through shared memory
            uint32_t rw[NH];
            if (MODE == DEC_ONE) {
#pragma unroll
                for (int hb = 0; hb < NH; hb += 4) {
                    const int hj = hb + (lane & 3);
                    const uint32_t gy = (ylo + (uint32_t)(tau - hj)) & rmask;
                    const uint32_t step = 2u * (t0 + (uint32_t)(hj >> 1)) + (uint32_t)(hj & 1);
                    const uint4 c = philox4x32_10(make_uint4((gy << lgG) + gword, step, TAG_SCA << 8, stream), key);
                    __syncwarp();
                    *reinterpret_cast<uint4*>(rnd + (lane >> 2) * 16 + (lane & 3) * 4) = c;
                    __syncwarp();
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (hb + u < NH) rw[hb + u] = rnd[(lane >> 2) * 16 + u * 4 + (lane & 3)];
                }
            }
            // (3) the tick's updates.  Every half-step runs at every tick, also on rows outside
            // its exact range [h, R - 1 - h) (the band's edges, or rows not loaded yet / any
            // more): those results only ever feed rows outside the next half-step's exact range,
            // never an exact row, and are never stored or counted, so skipping them is not
            // needed -- and the branch-free body lets the updates of a tick interleave.
#pragma unroll
            for (int h = 0; h < NH; ++h) {
                const int r = tau - h;
                {
                    const int sg = h & 1;
                    const int s = H + i - h;  // window slot of row r
                    const uint32_t tX = win[2 * sg][s], tY = win[2 * sg + 1][s];
                    const uint32_t oX = win[2 * (1 - sg)][s], oY = win[2 * (1 - sg) + 1][s + 1];
                    uint32_t xX = oX;
                    if (shifted) {
                        uint32_t nb = __shfl_down_sync(0xFFFFFFFFu, oX, 1);
                        if (lane == 31) nb = xr[h];
                        xX = __funnelshift_r(oX, nb, 1);
                    }
                    const uint32_t cp = ~(tX | tY) & xX & oY;
                    const uint32_t cq = USEQ ? (tX & tY & ~(xX | oY)) : 0u;
                    uint32_t m;
                    if (MODE == DEC_NONE) {
                        m = (cp & ap) | (cq & aq);
                    } else {
                        const uint32_t rr = rw[h];
                        m = (cp & (ap | (hp & ~rr))) | (cq & (aq | (hq & ~rr)));
                    }
                    if (COUNT && r >= H && r < H + Bc) {
                        ndep += __popc(m & cp);
                        if (USEQ) ndes += __popc(m & cq);
                    }
                    win[2 * sg][s] = tX ^ m;
                    win[2 * sg + 1][s] = tY ^ m;
                    win[2 * (1 - sg) + 1][s + 1] = oY ^ m;
                    if (shifted) {
                        const uint32_t cin = __shfl_up_sync(0xFFFFFFFFu, m >> 31, 1);
                        win[2 * (1 - sg)][s] = oX ^ (m << 1) ^ (cin & keep0);
                        fbits = __funnelshift_l(m, fbits, 1);
                    } else {
                        win[2 * (1 - sg)][s] = oX ^ m;
                    }
                }
            }
            // (4) row tau - 2k is final: store it if it is one of the band's rows
            {
                const int rho = tau - H;
                if (rho >= H && rho < H + Bc) {
                    const uint64_t gy = (uint64_t)((ylo + (uint32_t)rho) & rmask);
#pragma unroll
                    for (int q = 0; q < 4; ++q) dst[q * Q + gy * (uint64_t)Wr + w] = win[q][i];
                }
            }
            if (shifted && lane == 31) fbuf[((tau & 1) * nwarps + warp) * 4] = fbits;
            // (5) lane 0 publishes the words its left neighbour reads in the next (shifted) tick
            if (!shifted && lane == 0) {
                uint4* xb = reinterpret_cast<uint4*>(xbuf + (((tau + 1) & 1) * nwarps + warp) * NH);
#pragma unroll
                for (int h4 = 0; h4 < NH / 4; ++h4)
                    xb[h4] = make_uint4(win[2 * (1 - ((4 * h4) & 1))][H + i + 1 - 4 * h4],
                                        win[2 * (1 - ((4 * h4 + 1) & 1))][H + i - 4 * h4],
                                        win[2 * (1 - ((4 * h4 + 2) & 1))][H + i - 1 - 4 * h4],
                                        win[2 * (1 - ((4 * h4 + 3) & 1))][H + i - 2 - 4 * h4]);
            }
            // (6) one barrier per tick (the timeout vote every fourth); the ring slot of row
            // tau + 1 is free again
            if (i == 3) {
                if (__syncthreads_or(timed_out)) goto abort;
            } else {
                __syncthreads();
            }
            if (w == 0 && tau + 1 + WAVE_SLOTS < R) {
                issue(tau + 1 + WAVE_SLOTS);
                issued_hi = tau + 1 + WAVE_SLOTS;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int s = 0; s + 4 < NW; ++s) win[q][s] = win[q][s + 4];
    }
    if (COUNT) {
        for (int o = 16; o > 0; o >>= 1) {
            ndep += __shfl_xor_sync(0xFFFFFFFFu, ndep, o);
            ndes += __shfl_xor_sync(0xFFFFFFFFu, ndes, o);
        }
        if (lane == 0 && (ndep | ndes)) {
            atomicAdd(&counters[0], ndep);
            atomicAdd(&counters[1], ndes);
        }
    }
    return;
abort:
    // a ring copy did not arrive in time: report, and wait (bounded) for the copies this CTA
    // may still have in flight (the last WAVE_SLOTS rows issued) so none lands in shared memory
    // after the CTA retires
    if (w == 0) {
        atomicExch(err, 1u);
        for (int rho = issued_hi - WAVE_SLOTS + 1; rho <= issued_hi; ++rho)
            if (rho >= 0) (void)wait_row(rho);
    }
}

WaveShape scabit_wave_shape(int lx, int ly, int mcs_per_pass, int sm_count, int ctas_per_sm, int mode)
{
    WaveShape s{};
    s.ok = false;
    const int k = mcs_per_pass;
    if (lx < 11 || (1 << (lx - 6)) > WAVE_MAX_THREADS || (k != 2 && k != 4 && k != 6 && k != 8)) return s;
    if (mode != DEC_NONE && mode != DEC_ONE) return s;
    if (ctas_per_sm < 1 || ctas_per_sm > 3) return s;
    const int Wr = 1 << (lx - 6);
    const int64_t rows = 1ll << ly;
    const int64_t target = (int64_t)sm_count * ctas_per_sm;
    int64_t B = (rows + target - 1) / target;
    if (B < 8) B = 8;
    if (B > rows) B = rows;
    s.mcs = k;
    s.cps = ctas_per_sm;
    s.threads = Wr;
    s.band = (int)B;
    s.grid = (int)((rows + B - 1) / B);
    s.smem = wave_smem(Wr, k).total;
    s.ok = true;
    return s;
}

template <int MODE, bool USEQ, bool COUNT, int K, int MINB>
static cudaError_t launch_wave_kb(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0, Key key,
                                  uint32_t stream_id, Thresh tp, Thresh tq, const WaveShape& sh,
                                  unsigned long long* d_counters, unsigned int* d_err, cudaStream_t st)
{
    auto kern = scabit_wave_kernel<MODE, USEQ, COUNT, K, MINB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem);
    if (e != cudaSuccess) return e;
    kern<<<sh.grid, sh.threads, sh.smem, st>>>(d_src, d_dst, lx, ly, sh.band, t0, key, stream_id, tp, tq, d_counters,
                                               d_err);
    return cudaGetLastError();
}

template <int MODE, bool USEQ, bool COUNT, int K>
static cudaError_t launch_wave_k(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0, Key key,
                                 uint32_t stream_id, Thresh tp, Thresh tq, const WaveShape& sh,
                                 unsigned long long* d_counters, unsigned int* d_err, cudaStream_t st)
{
    if (sh.cps >= 3)
        return launch_wave_kb<MODE, USEQ, COUNT, K, 3>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh,
                                                        d_counters, d_err, st);
    return launch_wave_kb<MODE, USEQ, COUNT, K, 2>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, d_counters,
                                                    d_err, st);
}

template <int MODE, bool USEQ, bool COUNT>
static cudaError_t launch_wave(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0, Key key,
                               uint32_t stream_id, Thresh tp, Thresh tq, const WaveShape& sh,
                               unsigned long long* d_counters, unsigned int* d_err, cudaStream_t st)
{
    switch (sh.mcs) {
    case 2: return launch_wave_k<MODE, USEQ, COUNT, 2>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, d_counters, d_err, st);
    case 4: return launch_wave_k<MODE, USEQ, COUNT, 4>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, d_counters, d_err, st);
    case 6: return launch_wave_k<MODE, USEQ, COUNT, 6>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, d_counters, d_err, st);
    case 8: return launch_wave_k<MODE, USEQ, COUNT, 8>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, d_counters, d_err, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t scabit_wave(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0, uint64_t seed,
                        uint32_t stream_id, uint64_t Tp, uint64_t Tq, const WaveShape& sh,
                        unsigned long long* d_counters, unsigned int* d_err, cudaStream_t st)
{
    const Key key = make_key(seed);
    const Thresh tp = make_thresh(Tp), tq = make_thresh(Tq);
    const int mode = dec_mode(tp, tq);
    const bool useq = tq.always || tq.planes > 0;
    const bool c = d_counters != nullptr;
#define KPZB_WAVE_CASE(M)                                                                                           \
    return useq ? (c ? launch_wave<M, true, true>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, d_counters, \
                                                  d_err, st)                                                        \
                     : launch_wave<M, true, false>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, nullptr,  \
                                                   d_err, st))                                                      \
                : (c ? launch_wave<M, false, true>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh,           \
                                                   d_counters, d_err, st)                                           \
                     : launch_wave<M, false, false>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, nullptr, \
                                                    d_err, st))
    if (mode == DEC_NONE) KPZB_WAVE_CASE(DEC_NONE);
    if (mode == DEC_ONE) KPZB_WAVE_CASE(DEC_ONE);
#undef KPZB_WAVE_CASE
    return cudaErrorInvalidValue;
}

}  // namespace kpzb
