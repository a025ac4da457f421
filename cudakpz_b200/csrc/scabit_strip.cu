// scabit_strip.cu -- SCABit k-MCS pass, one warp per tile, half-steps in registers (sm_100a).
//
// A tile is a strip of 32 word columns of a quadrant row (one column per lane) times a band
// of B output rows plus 2k halo rows on each side.  Its warp runs the 2k half-steps of the
// pass as a diagonal wavefront down the band (tick tau: half-step h updates local row
// tau - h; a tick's updates touch disjoint rows, and row r + 1 was left by half-step h - 1
// earlier in the same tick), keeping 2k + 4 rows of its four quadrant words in registers; rows
// arrive six ticks ahead through a per-lane ring of shared-memory slots filled by cp.async
// (each lane copies and later reads only its own words).  No two warps share data while they
// run: no barrier, no shared-memory exchange of lattice words, no wait on another warp.
//
// The one-bit x-shift of odd rows (kpz/kpzSCABit.cu:257-274: a site's right neighbour sits
// one bit up, the top bit in the next word) moves between lanes by warp shuffles.  A strip
// that does not span the whole row recomputes one word column on each side: lane 0's carry-in
// and lane 31's right neighbour come from outside the strip and are wrong, but a wrong bit
// moves at most one bit per half-step, so after the 2k <= 16 half-steps of a pass lanes 1..30
// are exact and lanes 0 and 31 are never stored.  Consecutive strips therefore advance by 30
// columns, or by 28 when the rates need a random plane, so that each 4-word Philox group of
// the counter stream lies in one lane quad (the four lanes of a quad each compute one
// half-step's call and exchange the words through shared memory).  A 32-word row (lx = 11)
// is one periodic strip whose shuffles wrap around the warp.
//
// Which (half-step, row, site) updates run, with which random words, is exactly what the
// one-half-step kernel does (rows [2k, 2k + B) of the band are exact after the pass, as in
// the band and wave kernels), so the output is bit-identical to every other pass shape.  The
// rule and masks: kpz/kpzSCACores.cu:121-144, kpz/kpzSCABitCores.cu:69-74,139-145.
#include <cstdint>

#include "kpzb_common.cuh"
#include "kpzb_internal.h"

namespace kpzb {

constexpr int STRIP_RING = 8;      // shared-memory row slots per warp: rows arrive 6 ticks ahead
constexpr int STRIP_WARPS = 4;     // warps (independent tiles) per CTA
constexpr int STRIP_QUAD_STRIDE = 20;  // words per lane quad in the random-word exchange (padded)

// Rate kinds of the kernel: 0 = never flips, 1 = always flips, 2 = flips when the site's
// MSB plane bit is 0 (threshold 2^31, e.g. p = 1/2)
__host__ __device__ constexpr int strip_stride(bool random_plane) { return random_plane ? 28 : 30; }

__device__ __forceinline__ void cp_async4(uint32_t* smem, const uint32_t* gmem)
{
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// A flip of the updated site's own slope words: a deposition sets bits that are 0, a
// desorption clears bits that are 1, so with one kind of flip the XOR is an add or a subtract,
// done as a multiply-add by the opaque 1 / 0xFFFFFFFF in `one` / `mone` (the FMA pipe, which
// the rest of the update leaves idle); with both kinds it stays an XOR.
template <int PM, int QM>
__device__ __forceinline__ uint32_t flip_own(uint32_t x, uint32_t pm, uint32_t qm, uint32_t one, uint32_t mone)
{
    if (QM == 0) return pm * one + x;
    if (PM == 0) return qm * mone + x;
    return x ^ (pm | qm);
}
// A flip of a neighbour's slope bit (the other sublattice's X at x+1, Y at y+1): a deposition
// clears it, a desorption sets it.
template <int PM, int QM>
__device__ __forceinline__ uint32_t flip_nb(uint32_t x, uint32_t pm, uint32_t qm, uint32_t one, uint32_t mone)
{
    if (QM == 0) return pm * mone + x;
    if (PM == 0) return qm * one + x;
    return x ^ (pm | qm);
}

template <int PM, int QM, bool COUNT, int K>
__global__ void __launch_bounds__(32 * STRIP_WARPS, 4)
scabit_strip_kernel(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, int lx, int ly, int B,
                    int nstrips, int ntiles, uint32_t t0, Key key, uint32_t stream, uint32_t one, uint32_t mone,
                    unsigned long long* __restrict__ counters)
{
    constexpr int H = 2 * K;   // halo rows on each side of the band
    constexpr int NH = 2 * K;  // half-steps per pass
    constexpr int S = STRIP_RING;
    // register window rows: rows tau - 2k .. tau + 1 are live at tick tau, and a slot is
    // refilled three ticks after its row was stored; even, so a tick's shift is static
    constexpr int NW = 2 * K + 4;
    constexpr bool RND = PM == 2 || QM == 2;
    constexpr int STRIDE = strip_stride(RND);
    __shared__ __align__(16) uint32_t ring_s[STRIP_WARPS][S][4][32];
    constexpr int NG = RND ? NH / 4 : 1;  // Philox calls per lane per tick
    __shared__ __align__(16) uint32_t rnd_s[STRIP_WARPS][NG][8 * STRIP_QUAD_STRIDE];

    const int lane = (int)threadIdx.x & 31, wid = (int)threadIdx.x >> 5;
    const int tile = (int)blockIdx.x * STRIP_WARPS + wid;
    if (tile >= ntiles) return;  // whole warps only; nothing below synchronises the block
    const int strip = tile % nstrips, band = tile / nstrips;
    const uint32_t Wr = 1u << (lx - 6);
    const bool periodic = Wr == 32u;
    const uint32_t base = periodic ? 0u : (uint32_t)strip * (uint32_t)STRIDE;
    const uint32_t wcol = (base + (uint32_t)lane) & (Wr - 1u);
    const bool owned = periodic || (lane >= 1 && lane <= STRIDE && base + (uint32_t)lane <= Wr);
    const int src_up = periodic ? ((lane + 31) & 31) : (lane > 0 ? lane - 1 : 0);
    const int src_dn = periodic ? ((lane + 1) & 31) : (lane < 31 ? lane + 1 : 31);

    const int64_t rows = 1ll << ly;
    const uint32_t rmask = (uint32_t)rows - 1u;
    const uint64_t Q = 1ull << (lx + ly - 6);  // words per quadrant
    const int64_t y0 = (int64_t)band * B;
    const int Bc = (int)(rows - y0 < B ? rows - y0 : B);
    const int R = Bc + 2 * H;
    const uint32_t ylo = (uint32_t)((y0 - H) & (int64_t)rmask);  // global row of local row 0 (even)
    const uint32_t* s0 = src + wcol;
    uint32_t* d0 = dst + wcol;
    const int lgG = lx - 8;  // log2 of 4-word groups per quadrant row
    uint32_t* rs = &rnd_s[wid][0][0] + (lane >> 2) * STRIP_QUAD_STRIDE;

    // random words (RND), one tick ahead: at tick tau the lanes compute tick tau + 1's Philox
    // calls -- lane j of each quad the call of half-step 4g + j for the quad's 4-word group --
    // while tick tau's updates run, and exchange them through shared memory at its end
    uint32_t rwc[RND ? NH : 1];  // this tick's word of every half-step
    uint4 cn[NG];                // the next tick's calls
    // counter word 0 of half-step hj's call: quadrant row (ylo + tau - hj) mod rows times the
    // groups per row, plus this lane's group (one multiply-add and one mask per call)
    const uint32_t gpr = 1u << lgG, lane_grp = wcol >> 2;
    auto calls = [&](int tau_) {
#pragma unroll
        for (int g = 0; g < NG; ++g) {
            const int hj = 4 * g + (lane & 3);
            const uint32_t gy = (ylo - (uint32_t)hj + (uint32_t)tau_) & rmask;
            cn[g] = philox4x32_10(make_uint4(gy * gpr + lane_grp, 2u * t0 + (uint32_t)hj, TAG_SCA << 8, stream), key);
        }
    };
    auto exchange = [&]() {
        __syncwarp();
#pragma unroll
        for (int g = 0; g < NG; ++g)
            *reinterpret_cast<uint4*>(rs + g * 8 * STRIP_QUAD_STRIDE + (lane & 3) * 4) = cn[g];
        __syncwarp();
#pragma unroll
        for (int g = 0; g < NG; ++g)
#pragma unroll
            for (int u = 0; u < 4; ++u) rwc[4 * g + u] = rs[g * 8 * STRIP_QUAD_STRIDE + u * 4 + (lane & 3)];
    };
    if (RND) {
        calls(0);
        exchange();
    }
    uint32_t(*ring)[4][32] = ring_s[wid];

    // local row rho -> ring slot rho % S: this lane's four quadrant words, one copy group per row
    auto issue = [&](int rho) {
        const uint64_t gy = (ylo + (uint32_t)rho) & rmask;
        const int sl = rho % S;
#pragma unroll
        for (int q = 0; q < 4; ++q) cp_async4(&ring[sl][q][lane], s0 + q * Q + gy * Wr);
        cp_async_commit();
    };

    uint32_t win[4][NW];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int s = 1; s < NW; ++s) win[q][s] = 0u;
#pragma unroll
    for (int rho = 0; rho < S; ++rho) issue(rho);
    cp_async_wait<S - 1>();  // row 0
#pragma unroll
    for (int q = 0; q < 4; ++q) win[q][0] = ring[0][q][lane];
    unsigned long long ndep = 0, ndes = 0;

    // whole cycles of NW ticks, so that a cycle is one straight-line block the compiler can
    // interleave across ticks (the 2k updates of one tick form a dependency chain); ticks past
    // R update rows beyond the band's last exact row and store nothing
    for (int tau0 = 0; tau0 < R; tau0 += NW) {
#pragma unroll
        for (int i = 0; i < NW; ++i) {
            const int tau = tau0 + i;
            const bool shifted = (i & 1) != 0;  // (ylo + tau) & 1 with ylo and tau0 even
            // row tau + 1 enters the window (rows issued so far: 0 .. tau + S - 1)
            cp_async_wait<S - 2>();
            {
                const int sl = (tau + 1) % S;
#pragma unroll
                for (int q = 0; q < 4; ++q) win[q][(i + 1) % NW] = ring[sl][q][lane];
            }
            if (RND) calls(tau + 1);
#pragma unroll
            for (int h = 0; h < NH; ++h) {
                const int sg = h & 1;                          // sublattice updated
                const int sr = ((i - h) % NW + NW) % NW;       // slot of row tau - h
                const int sr1 = ((i - h + 1) % NW + NW) % NW;  // slot of row tau - h + 1
                const uint32_t tX = win[2 * sg][sr], tY = win[2 * sg + 1][sr];
                const uint32_t oX = win[2 * (1 - sg)][sr], oY = win[2 * (1 - sg) + 1][sr1];
                uint32_t xX = oX;
                if (shifted) xX = __funnelshift_r(oX, __shfl_sync(0xFFFFFFFFu, oX, src_dn), 1);
                uint32_t pm = 0u, qm = 0u;
                if (PM == 1) pm = ~(tX | tY) & xX & oY;
                if (PM == 2) pm = ~(tX | tY) & xX & oY & ~rwc[h];
                if (QM == 1) qm = tX & tY & ~(xX | oY);
                if (QM == 2) qm = tX & tY & ~(xX | oY) & ~rwc[h];
                if (PM == 2 && QM == 2 && !COUNT) {
                    // both kinds on the same random word: a candidate has tX == tY, xX == oY and
                    // tX != xX (a minimum 0,0,1,1 or a maximum 1,1,0,0), so the flip mask is
                    // ((tX ^ tY) | ~(tX ^ xX))' & ((xX ^ oY) | r)' -- three 3-input operations
                    pm = (~(tX ^ tY) & (tX ^ xX)) & (~(xX ^ oY) & ~rwc[h]);
                    qm = 0u;
                }
                if (COUNT) {
                    const int r = tau - h;
                    if (owned && r >= H && r < H + Bc) {
                        ndep += __popc(pm);
                        ndes += __popc(qm);
                    }
                }
                win[2 * sg][sr] = flip_own<PM, QM>(tX, pm, qm, one, mone);
                win[2 * sg + 1][sr] = flip_own<PM, QM>(tY, pm, qm, one, mone);
                win[2 * (1 - sg) + 1][sr1] = flip_nb<PM, QM>(oY, pm, qm, one, mone);
                if (shifted) {
                    const uint32_t m = pm | qm;
                    const uint32_t ml = __shfl_sync(0xFFFFFFFFu, m, src_up);
                    win[2 * (1 - sg)][sr] = oX ^ __funnelshift_l(ml, m, 1);
                } else {
                    win[2 * (1 - sg)][sr] = flip_nb<PM, QM>(oX, pm, qm, one, mone);
                }
            }
            // row tau - 2k is final: store it when it is one of the band's rows
            {
                const int rho = tau - H;
                const int sl = ((i - H) % NW + NW) % NW;
                if (owned && rho >= H && rho < H + Bc) {
                    const uint64_t gy = (ylo + (uint32_t)rho) & rmask;
#pragma unroll
                    for (int q = 0; q < 4; ++q) d0[q * Q + gy * Wr] = win[q][sl];
                }
            }
            // row tau + S into the ring slot row tau left a tick ago
            issue(tau + S);
            if (RND) exchange();
        }
    }
    cp_async_wait<0>();  // no copy may land in this warp's ring after it has left
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
}

int strip_cycle_rows(int mcs_per_pass) { return 2 * mcs_per_pass + 4; }

StripShape scabit_strip_shape(int lx, int ly, int mcs_per_pass, int band_rows, int mode)
{
    StripShape s{};
    s.ok = false;
    const int k = mcs_per_pass;
    if (lx < 11 || lx > 30 || (k != 4 && k != 6 && k != 8)) return s;
    if (mode != DEC_NONE && mode != DEC_ONE) return s;
    if (band_rows < 2 || (band_rows & 1)) return s;
    const int64_t Wr = 1ll << (lx - 6);
    const int64_t rows = 1ll << ly;
    const int stride = strip_stride(mode == DEC_ONE);
    const int64_t nstrips = Wr == 32 ? 1 : (Wr + stride - 1) / stride;
    const int64_t B = band_rows < rows ? band_rows : rows;
    const int64_t nbands = (rows + B - 1) / B;
    const int64_t ntiles = nstrips * nbands;
    const int64_t grid = (ntiles + STRIP_WARPS - 1) / STRIP_WARPS;
    if (grid > 0x7FFFFFFF) return s;
    s.mcs = k;
    s.band = (int)B;
    s.nstrips = (int)nstrips;
    s.ntiles = (int)ntiles;
    s.grid = (int)grid;
    s.threads = 32 * STRIP_WARPS;
    s.random_plane = mode == DEC_ONE;
    s.ok = true;
    return s;
}

template <int PM, int QM, bool COUNT, int K>
static cudaError_t launch_strip_k(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0, Key key,
                                  uint32_t stream_id, const StripShape& sh, unsigned long long* d_counters,
                                  cudaStream_t st)
{
    scabit_strip_kernel<PM, QM, COUNT, K><<<sh.grid, sh.threads, 0, st>>>(
        d_src, d_dst, lx, ly, sh.band, sh.nstrips, sh.ntiles, t0, key, stream_id, 1u, 0xFFFFFFFFu, d_counters);
    return cudaGetLastError();
}

template <int PM, int QM, bool COUNT>
static cudaError_t launch_strip(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0, Key key,
                                uint32_t stream_id, const StripShape& sh, unsigned long long* d_counters,
                                cudaStream_t st)
{
    switch (sh.mcs) {
    case 4: return launch_strip_k<PM, QM, COUNT, 4>(d_src, d_dst, lx, ly, t0, key, stream_id, sh, d_counters, st);
    case 6: return launch_strip_k<PM, QM, COUNT, 6>(d_src, d_dst, lx, ly, t0, key, stream_id, sh, d_counters, st);
    case 8: return launch_strip_k<PM, QM, COUNT, 8>(d_src, d_dst, lx, ly, t0, key, stream_id, sh, d_counters, st);
    default: return cudaErrorInvalidValue;
    }
}

template <int PM, int QM>
static cudaError_t launch_strip_c(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0, Key key,
                                  uint32_t stream_id, const StripShape& sh, unsigned long long* d_counters,
                                  cudaStream_t st)
{
    if (d_counters)
        return launch_strip<PM, QM, true>(d_src, d_dst, lx, ly, t0, key, stream_id, sh, d_counters, st);
    return launch_strip<PM, QM, false>(d_src, d_dst, lx, ly, t0, key, stream_id, sh, nullptr, st);
}

cudaError_t scabit_strip(const uint32_t* d_src, uint32_t* d_dst, int lx, int ly, uint32_t t0, uint64_t seed,
                         uint32_t stream_id, uint64_t Tp, uint64_t Tq, const StripShape& sh,
                         unsigned long long* d_counters, cudaStream_t st)
{
    const Key key = make_key(seed);
    const Thresh tp = make_thresh(Tp), tq = make_thresh(Tq);
    const int mode = dec_mode(tp, tq);
    if (!sh.ok || (mode != DEC_NONE && mode != DEC_ONE)) return cudaErrorInvalidValue;
    if (sh.random_plane != (mode == DEC_ONE)) return cudaErrorInvalidValue;  // strips made for the other stride
    // rate kinds: 0 never, 1 always, 2 the MSB plane (threshold 2^31)
    const int pk = tp.always ? 1 : tp.planes ? 2 : 0;
    const int qk = tq.always ? 1 : tq.planes ? 2 : 0;
#define KPZB_STRIP_CASE(A, C)                                                                              \
    if (pk == A && qk == C)                                                                               \
        return launch_strip_c<A, C>(d_src, d_dst, lx, ly, t0, key, stream_id, sh, d_counters, st);
    KPZB_STRIP_CASE(1, 0)
    KPZB_STRIP_CASE(0, 1)
    KPZB_STRIP_CASE(1, 1)
    KPZB_STRIP_CASE(2, 0)
    KPZB_STRIP_CASE(0, 2)
    KPZB_STRIP_CASE(2, 2)
    KPZB_STRIP_CASE(1, 2)
    KPZB_STRIP_CASE(2, 1)
#undef KPZB_STRIP_CASE
    // p = q = 0: nothing flips; the pass still leaves its lattice in the other buffer
    return cudaMemcpyAsync(d_dst, d_src, sizeof(uint32_t) << (lx + ly - 4), cudaMemcpyDeviceToDevice, st);
}

}  // namespace kpzb
