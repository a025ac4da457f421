// scabit.cu -- bit-vectorised SCA half-step on the ENC_CBBIT lattice (sm_100a).
//
// Reference behaviour: kpz/kpzSCABit.cu:112-290 (kernel), kpz/kpzSCABitCores.cu:69-74,139-145
// (mask algebra), kpz/schedulerSCABit.cu:46-73 (sublattice 0 then 1 per MCS).
//
// Layout (kpz/systemSize.h:143-165): four quadrants of Q = N/64 words,
//   [sub0.X | sub0.Y | sub1.X | sub1.Y], row y of a quadrant is Wr = L/64 words,
//   bit b of word j holds site x = 2*(32*j+b) + ((sigma ^ y) & 1).
// A half-step on sublattice sigma updates every "this" site of row y from
//   thisX, thisY (row y), otherX (row y; shifted right by one bit with carry from the
//   next word when sigma != (y & 1)), otherY (row y+1), and xors the flip mask into all
//   four (otherX with the inverse shift).  Rows are independent within a half-step.
//
// Work split: a CTA owns TY rows at a time; TX threads cover a row segment of 4*TX words
// with 128-bit loads/stores (one Philox group of 4 words per thread).  Rows longer than
// one segment are walked segment by segment with the one-bit mask carry kept in shared
// memory; the carry out of the last word wraps into bit 0 of word 0 (periodic x).
#include "kpzb_api_internal.h"
#include "kpzb_common.cuh"
#include "kpzb_internal.h"
#include "scabit_band.cuh"

namespace kpzb {

constexpr int SCABIT_THREADS = 256;

// DIS: quenched disorder -- dis holds every site's 2-bit rate class in ENC_CBBIT form (class
// bit 0 in the X quadrants, bit 1 in the Y quadrants, i.e. the ENC_LOCAL class words put
// through the lattice codec), dr the four classes' thresholds (Disorder2SyncRng,
// kpz/kpzSCACores.cu:217-280).
template <bool COUNT, bool DIS>
__global__ void __launch_bounds__(SCABIT_THREADS)
scabit_half_kernel(uint32_t* __restrict__ sys, int lx, int ly, int sigma, uint32_t step, Key key,
                   uint32_t stream, Thresh tp, Thresh tq, int TX, int TY,
                   unsigned long long* __restrict__ counters, const uint32_t* __restrict__ dis,
                   DisorderRates dr)
{
    __shared__ uint32_t nxt_s[SCABIT_THREADS];
    __shared__ uint32_t carry_s[2][SCABIT_THREADS];

    const int tx = threadIdx.x, ty = threadIdx.y;
    const int lin = ty * TX + tx;
    const uint64_t Wr = 1ull << (lx - 6);
    const uint64_t Q = 1ull << (lx + ly - 6);
    const uint64_t rows = 1ull << ly;
    const int nseg = (int)(Wr / (4ull * TX));
    const uint64_t rowgroups = rows / TY;

    const uint64_t bthisX = sigma ? 2 * Q : 0;
    const uint64_t bthisY = bthisX + Q;
    const uint64_t botherX = sigma ? 0 : 2 * Q;
    const uint64_t botherY = botherX + Q;

    unsigned long long ndep = 0, ndes = 0;

    for (uint64_t rg = blockIdx.x; rg < rowgroups; rg += gridDim.x) {
        const uint64_t y = rg * TY + ty;
        const bool shifted = sigma != (int)(y & 1);
        const uint64_t roff = y * Wr;
        const uint64_t roff1 = ((y + 1) & (rows - 1)) * Wr;
        for (int seg = 0; seg < nseg; ++seg) {
            const uint64_t wi = (uint64_t)seg * 4 * TX + 4 * (uint64_t)tx;
            uint4* ptX = reinterpret_cast<uint4*>(sys + bthisX + roff + wi);
            uint4* ptY = reinterpret_cast<uint4*>(sys + bthisY + roff + wi);
            uint4* poX = reinterpret_cast<uint4*>(sys + botherX + roff + wi);
            uint4* poY = reinterpret_cast<uint4*>(sys + botherY + roff1 + wi);
            uint4 tX = *ptX, tY = *ptY, oX = *poX, oY = *poY;
            nxt_s[lin] = oX.x;
            __syncthreads();
            uint4 xX = oX;
            if (shifted) {
                uint32_t nb;
                if (tx + 1 < TX) nb = nxt_s[lin + 1];
                else nb = sys[botherX + roff + ((wi + 4) & (Wr - 1))];
                xX.x = (oX.x >> 1) | (oX.y << 31);
                xX.y = (oX.y >> 1) | (oX.z << 31);
                xX.z = (oX.z >> 1) | (oX.w << 31);
                xX.w = (oX.w >> 1) | (nb << 31);
            }
            // deposition: this site's slopes both 0, right-x and up-y slopes both 1;
            // desorption: the complement (kpz/kpzSCABitCores.cu:69-74,139-145)
            uint4 cp, cq;
            cp.x = ~(tX.x | tY.x) & xX.x & oY.x;
            cp.y = ~(tX.y | tY.y) & xX.y & oY.y;
            cp.z = ~(tX.z | tY.z) & xX.z & oY.z;
            cp.w = ~(tX.w | tY.w) & xX.w & oY.w;
            cq.x = tX.x & tY.x & ~(xX.x | oY.x);
            cq.y = tX.y & tY.y & ~(xX.y | oY.y);
            cq.z = tX.z & tY.z & ~(xX.z | oY.z);
            cq.w = tX.w & tY.w & ~(xX.w | oY.w);
            uint4 m;
            if (DIS) {
                const uint4 d0 = *reinterpret_cast<const uint4*>(dis + bthisX + roff + wi);
                const uint4 d1 = *reinterpret_cast<const uint4*>(dis + bthisY + roff + wi);
                m = decide4_dis(cp, cq, d0, d1, dr, key, (uint32_t)((roff + wi) >> 2), step, stream);
            } else {
                m = decide4_mode(dec_mode(tp, tq), cp, cq, tp, tq, key, (uint32_t)((roff + wi) >> 2), step,
                                 stream);
            }
            if (COUNT) {
                ndep += __popc(m.x & cp.x) + __popc(m.y & cp.y) + __popc(m.z & cp.z) + __popc(m.w & cp.w);
                ndes += __popc(m.x & cq.x) + __popc(m.y & cq.y) + __popc(m.z & cq.z) + __popc(m.w & cq.w);
            }
            tX = tX ^ m;
            tY = tY ^ m;
            oY = oY ^ m;
            carry_s[seg & 1][lin] = m.w >> 31;
            __syncthreads();
            if (shifted) {
                uint32_t cin = 0;
                if (tx > 0) cin = carry_s[seg & 1][lin - 1];
                else if (seg > 0) cin = carry_s[(seg - 1) & 1][lin + TX - 1];
                oX.x ^= (m.x << 1) | cin;
                oX.y ^= (m.y << 1) | (m.x >> 31);
                oX.z ^= (m.z << 1) | (m.y >> 31);
                oX.w ^= (m.w << 1) | (m.z >> 31);
            } else {
                oX = oX ^ m;
            }
            *ptX = tX;
            *ptY = tY;
            *poX = oX;
            *poY = oY;
        }
        if (shifted && tx == 0) {
            // periodic wrap: the last word's bit-31 flip lands on bit 0 of word 0
            if (carry_s[(nseg - 1) & 1][lin + TX - 1]) sys[botherX + roff] ^= 1u;
        }
    }
    if (COUNT) {
        for (int o = 16; o > 0; o >>= 1) {
            ndep += __shfl_xor_sync(0xffffffffu, ndep, o);
            ndes += __shfl_xor_sync(0xffffffffu, ndes, o);
        }
        if ((lin & 31) == 0 && (ndep | ndes)) {
            atomicAdd(&counters[0], ndep);
            atomicAdd(&counters[1], ndes);
        }
    }
}

ScabitShape scabit_shape(int lx, int ly, int sm_count)
{
    ScabitShape s;
    const uint64_t Wr = 1ull << (lx - 6);
    uint64_t tx = Wr / 4;
    if (tx > SCABIT_THREADS) tx = SCABIT_THREADS;
    uint64_t ty = SCABIT_THREADS / tx;
    const uint64_t rows = 1ull << ly;
    if (ty > rows) ty = rows;
    s.TX = (int)tx;
    s.TY = (int)ty;
    const uint64_t rowgroups = rows / ty;
    uint64_t grid = (uint64_t)sm_count * 8;
    if (grid > rowgroups) grid = rowgroups;
    s.grid = (int)grid;
    return s;
}

cudaError_t scabit_half(uint32_t* d_sys, int lx, int ly, int sigma, uint32_t step, uint64_t seed,
                        uint32_t stream_id, uint64_t Tp, uint64_t Tq, const ScabitShape& sh,
                        unsigned long long* d_counters, cudaStream_t st)
{
    const Key key = make_key(seed);
    const Thresh tp = make_thresh(Tp), tq = make_thresh(Tq);
    dim3 block(sh.TX, sh.TY);
    const DisorderRates dr{};
    if (d_counters)
        scabit_half_kernel<true, false><<<sh.grid, block, 0, st>>>(d_sys, lx, ly, sigma, step, key, stream_id,
                                                                   tp, tq, sh.TX, sh.TY, d_counters, nullptr, dr);
    else
        scabit_half_kernel<false, false><<<sh.grid, block, 0, st>>>(d_sys, lx, ly, sigma, step, key, stream_id,
                                                                    tp, tq, sh.TX, sh.TY, nullptr, nullptr, dr);
    return cudaGetLastError();
}

cudaError_t scabit_half_dis(uint32_t* d_sys, const uint32_t* d_dis_cbbit, int lx, int ly, int sigma,
                            uint32_t step, uint64_t seed, uint32_t stream_id, const uint64_t Tp[4],
                            const uint64_t Tq[4], const ScabitShape& sh, unsigned long long* d_counters,
                            cudaStream_t st)
{
    const Key key = make_key(seed);
    const DisorderRates dr = make_disorder_rates(Tp, Tq);
    dim3 block(sh.TX, sh.TY);
    if (d_counters)
        scabit_half_kernel<true, true><<<sh.grid, block, 0, st>>>(d_sys, lx, ly, sigma, step, key, stream_id,
                                                                  dr.tp[0], dr.tq[0], sh.TX, sh.TY, d_counters,
                                                                  d_dis_cbbit, dr);
    else
        scabit_half_kernel<false, true><<<sh.grid, block, 0, st>>>(d_sys, lx, ly, sigma, step, key, stream_id,
                                                                   dr.tp[0], dr.tq[0], sh.TX, sh.TY, nullptr,
                                                                   d_dis_cbbit, dr);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// Temporal blocking.  A CTA loads a band of R = B + 4k full-width rows of all four
// quadrants into shared memory with TMA bulk copies (cp.async.bulk, local HBM only),
// runs 2k half-steps there, and writes its B middle rows to the destination buffer.
// Half-step h updates local rows [h, R-1-h); after 2k half-steps rows [2k, R-2k) are
// exact (each half-step invalidates at most one row per side), so neighbouring bands
// overlap by 2k halo rows on each side.  The one-bit carry of shifted rows crosses
// thread boundaries only in the first word of each 4-word group, which is updated
// with shared-memory atomicXor; all other words have a single writer.
// ---------------------------------------------------------------------------------
constexpr int FUSED_THREADS = 512;
constexpr int FUSED_THREADS_WIDE = 1024;  // mode-specialised variants fit 64 registers

template <int MODE, bool USEQ, bool COUNT, int NT>
__global__ void __launch_bounds__(NT, 1)
scabit_fused_kernel(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, int lx, int ly,
                    uint32_t t0, Key key, uint32_t stream, Thresh tp, Thresh tq, int B, int k,
                    unsigned long long* __restrict__ counters, unsigned int* __restrict__ err)
{
    extern __shared__ __align__(128) uint32_t smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int abort_flag;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const BandCtl ctl{&bar, &abort_flag, 0u};
    const BandGeom g{src, dst, lx, ly, (int64_t)blockIdx.x * B, B, k, false, t0, key, stream, tp, tq};
    unsigned long long ndep = 0, ndes = 0;
    if (!scabit_band<MODE, USEQ, COUNT, NT>(smem, ctl, g, ndep, ndes, err)) return;
    if (COUNT) {
        for (int o = 16; o > 0; o >>= 1) {
            ndep += __shfl_xor_sync(0xffffffffu, ndep, o);
            ndes += __shfl_xor_sync(0xffffffffu, ndes, o);
        }
        if ((threadIdx.x & 31) == 0 && (ndep | ndes)) {
            atomicAdd(&counters[0], ndep);
            atomicAdd(&counters[1], ndes);
        }
    }
}

// MCS per HBM pass when the caller leaves the choice to the library: the deepest pass whose
// band still holds at least as many output rows as halo rows (redundant work <= 2x).
int auto_fusion(int lx, int ly)
{
    int best = 1;
    for (int k = 2; k <= 8; ++k) {
        FusedShape f = scabit_fused_shape(lx, ly, k, 148, 0);
        if (f.ok && f.band >= 4 * k) best = k;
    }
    return best;
}

FusedShape scabit_fused_shape(int lx, int ly, int mcs_per_pass, int sm_count, size_t smem_optin)
{
    return scabit_fused_shape_cps(lx, ly, mcs_per_pass, 0, smem_optin);
}

// ctas_per_sm: 1 or 2 CTAs resident per SM (2 lets one CTA's TMA load overlap the other's
// compute); 0 picks 2 when the band stays at least as tall as the halo, else 1; 3 = one CTA
// per SM of 1024 threads (the rate-specialised kernels; the general decision keeps 512).
FusedShape scabit_fused_shape_cps(int lx, int ly, int mcs_per_pass, int ctas_per_sm,
                                  size_t smem_optin)
{
    const bool wide = ctas_per_sm == 3;
    if (wide) ctas_per_sm = 1;
    FusedShape f{};
    f.ok = false;
    if (smem_optin == 0) smem_optin = 227 * 1024;
    const uint64_t Wr = 1ull << (lx - 6);
    const uint64_t row_bytes = 16ull * Wr;  // four quadrants
    const int64_t rows = 1ll << ly;
    const int k = mcs_per_pass;
    if (k < 1) return f;
    const size_t budget2 = (228 * 1024) / 2 - 2048;
    const size_t budget1 = smem_optin - 1024;
    int R;
    if (ctas_per_sm == 2) R = (int)(budget2 / row_bytes);
    else if (ctas_per_sm == 1) R = (int)(budget1 / row_bytes);
    else {
        R = (int)(budget2 / row_bytes);
        if (R - 4 * k < 4 * k) R = (int)(budget1 / row_bytes);
    }
    int B = R - 4 * k;
    if (B < 1) return f;
    if (B > rows) B = (int)rows;
    R = B + 4 * k;
    if ((uint64_t)R * Wr * 16 > 0xFFFFFFFFull) return f;
    f.band = B;
    f.halo = 2 * k;
    f.mcs = k;
    f.threads = wide ? FUSED_THREADS_WIDE : FUSED_THREADS;
    f.smem = (size_t)R * row_bytes;
    f.grid = (int)((rows + B - 1) / B);
    f.ok = true;  // the load loop handles halos that wrap the lattice more than once
    return f;
}

template <int MODE, bool USEQ, bool COUNT>
static cudaError_t launch_fused(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0, Key key,
                                uint32_t stream_id, Thresh tp, Thresh tq, const FusedShape& sh,
                                unsigned long long* d_counters, unsigned int* d_err, cudaStream_t st)
{
    // the general bit-serial decision keeps 512 threads (its registers do not fit 64)
    auto kern = scabit_fused_kernel<MODE, USEQ, COUNT, FUSED_THREADS>;
    int nt = FUSED_THREADS;
    if constexpr (MODE != DEC_GENERAL) {
        if (sh.threads == FUSED_THREADS_WIDE) {
            kern = scabit_fused_kernel<MODE, USEQ, COUNT, FUSED_THREADS_WIDE>;
            nt = FUSED_THREADS_WIDE;
        }
    }
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem);
    if (e != cudaSuccess) return e;
    kern<<<sh.grid, nt, sh.smem, st>>>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh.band, sh.mcs,
                                       d_counters, d_err);
    return cudaGetLastError();
}

template <int MODE, bool USEQ>
static cudaError_t launch_fused_c(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0, Key key,
                                  uint32_t stream_id, Thresh tp, Thresh tq, const FusedShape& sh,
                                  unsigned long long* d_counters, unsigned int* d_err, cudaStream_t st)
{
    if (d_counters)
        return launch_fused<MODE, USEQ, true>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, d_counters,
                                              d_err, st);
    return launch_fused<MODE, USEQ, false>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, nullptr, d_err,
                                           st);
}

cudaError_t scabit_fused(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0,
                         uint64_t seed, uint32_t stream_id, uint64_t Tp, uint64_t Tq,
                         const FusedShape& sh, unsigned long long* d_counters, unsigned int* d_err,
                         cudaStream_t st)
{
    const Key key = make_key(seed);
    const Thresh tp = make_thresh(Tp), tq = make_thresh(Tq);
    const int mode = dec_mode(tp, tq);
    const bool useq = tq.always || tq.planes > 0;
#define KPZB_FUSED_CASE(M)                                                                                    \
    return useq ? launch_fused_c<M, true>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, d_counters,   \
                                          d_err, st)                                                          \
                : launch_fused_c<M, false>(d_src, d_dst, lx, ly, t0, key, stream_id, tp, tq, sh, d_counters,  \
                                           d_err, st)
    if (mode == DEC_NONE) KPZB_FUSED_CASE(DEC_NONE);
    if (mode == DEC_ONE) KPZB_FUSED_CASE(DEC_ONE);
    KPZB_FUSED_CASE(DEC_GENERAL);
#undef KPZB_FUSED_CASE
}

}  // namespace kpzb
