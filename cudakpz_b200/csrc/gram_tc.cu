// gram_tc.cu -- exact limb Gram of the stored snapshots on tcgen05 tensor cores (sm_100a).
//
// One persistent CTA per SM takes a contiguous range of 128-site K tiles and splits it into eight
// contiguous runs, one per producer warp.  Each producer warp owns one shared-memory stage and
// builds whole tiles in it: lane l walks snapshots l and l + 32 along the tile's row from their
// X-slope bits (gram_slope.cuh gives the walk: v(x) = b(y) + 2 #{x' in [1, x] : s_x = 1} - x,
// v(0) = z(y), v = h - c), eight sites per table lookup, and writes the values as signed int8
// limb rows in the K-major SWIZZLE_128B layout the MMA descriptors expect (limb row a * 64 + s,
// 128 bytes a row, 16-byte chunk c of row r at chunk position c ^ (r mod 8)); a
// fence.proxy.async hands the stage to the tensor core.  Warp 0 owns 256 TMEM columns and
// consumes the stages round-robin, issuing per 32-byte K step
//   D1[0:128, 0:192]   += A[0:128]   . A[0:192]^T   (M=128, N=192)
//   D2[0:128, 0:64]    += A[64:192]  . A[128:192]^T (M=128, N=64)
// (kind::i8, signed, int32 accumulators in TMEM); together they cover every (row <= col)
// entry of the symmetric 192 x 192 limb Gram.  A tile whose values all lie in [-64, 63] is its
// own low limb: its upper limb rows are zero and one M=128, N=64 MMA per K step adds all of it.
// Other tiles take balanced base-128 digits, three limbs.  Every 2^18 K elements (|l l'| <= 2^12,
// so the int32 sums stay below 2^30) warps 1-4 read the accumulators with tcgen05.ld and add
// them to the CTA's int64 partial in global memory; a final kernel sums the partials.  Only the
// slope bits cross HBM: 16 bytes per snapshot per tile.  Every mbarrier wait is bounded: on
// expiry the kernel raises a flag, stops issuing work, drains what it issued, frees its TMEM
// and returns.
#include <algorithm>
#include <cstring>

#include "gram_slope.cuh"
#include "kpzb_api_internal.h"
#include "kpzb_gram.h"
#include "scabit_band.cuh"

namespace kpzb {

constexpr int TC_ROWS = 192;
constexpr int TC_KT = GS_TILE;                    // K bytes per tile (one 128B swizzle row)
constexpr int TC_STAGE = TC_ROWS * TC_KT;         // 24 KB
constexpr int TC_WINDOW = (1 << 18) / TC_KT;      // K tiles per int32 accumulation window
constexpr int TC_PROD_WARPS = 8;                  // producer warps, one stage each
constexpr int TC_STAGES = TC_PROD_WARPS;
constexpr int TC_PROD_WARP0 = 5;                  // warps 5..12 produce, 1..4 flush, 0 issues
constexpr int TC_THREADS = (TC_PROD_WARP0 + TC_PROD_WARPS) * 32;
constexpr int TC_COLS = 256;                      // TMEM columns: D1 0..191, D2 192..255
constexpr int TC_LUT = 256;                       // 8-site slope patterns
constexpr int TC_SMEM = TC_STAGES * TC_STAGE + TC_LUT * 8 + 1024;
constexpr uint64_t TC_WAIT_NS = 4000000000ull;    // bound of every mbarrier wait (4 s)

// UMMA instruction descriptor, kind::i8: S32 accumulate (bits 4-5 = 2), signed A and B
// (bits 7-9, 10-12 = 1), both K-major, N>>3 at bit 17, M>>4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Shared-memory descriptor of a K-major SWIZZLE_128B operand: rows of 128 bytes, 8-row
// groups 1024 bytes apart (SBO), LBO 16 bytes, descriptor version 1, layout type 2.
__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// waits for the phase with the given parity; false after TC_WAIT_NS of global time
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        for (int k = 0; k < 64; ++k)
            if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > TC_WAIT_NS) return false;
    }
}

// four values' low bytes, first in the lowest byte
__device__ __forceinline__ uint32_t pack4(int32_t a, int32_t b, int32_t c, int32_t d)
{
    return __byte_perm(__byte_perm((uint32_t)a, (uint32_t)b, 0x0040), __byte_perm((uint32_t)c, (uint32_t)d, 0x0040),
                       0x5410);
}

// the 16-byte chunk `chunk` (sites 16 chunk .. +15) of limb row r in a SWIZZLE_128B stage
__device__ __forceinline__ void put_chunk(uint8_t* stage, int r, int chunk, uint4 v)
{
    *reinterpret_cast<uint4*>(stage + r * TC_KT + ((chunk ^ (r & 7)) << 4)) = v;
}

__device__ __forceinline__ void umma_i8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// Count of X-slope bits of row y in [1, x0) of one snapshot, by one thread (the running count a
// producer lane starts from when its run of tiles begins inside a row).
__device__ __forceinline__ int32_t slope_count_before(const SlopeSnapGeom& g, int s, uint64_t y, uint32_t x0)
{
    const uint64_t Wr = 1ull << (g.lx - 6);
    const uint32_t* base = g.snap + (uint64_t)s * 2 * g.Q + y * Wr;
    int32_t cnt = 0;
    for (uint32_t j = 0; j < (x0 >> 6); j += 2) {
        const uint2 a = __ldg(reinterpret_cast<const uint2*>(base + j));
        const uint2 b = __ldg(reinterpret_cast<const uint2*>(base + g.Q + j));
        cnt += __popc(a.x) + __popc(a.y) + __popc(b.x) + __popc(b.y);
    }
    // site x = 0 (sublattice y & 1, word 0, bit 0) closes the row: not part of the running count
    if (x0 > 0) cnt -= (int32_t)(__ldg(base + (y & 1) * g.Q) & 1u);
    return cnt;
}

// One snapshot's 16 values of K chunk c (sites 16 c .. 16 c + 15 of the tile) by the walk, from
// the running value `b` before the chunk; the even-x word `ew` and odd-x word `ow` are the
// tile's words (c >> 2) of the two X quadrants.  Advances b.
__device__ __forceinline__ void walk16(uint32_t ew, uint32_t ow, int c, int32_t& b, int32_t v[16])
{
    const int sh = 8 * (c & 3);
    ew >>= sh;
    ow >>= sh;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const uint32_t bit = (((i & 1) ? ow : ew) >> (i >> 1)) & 1u;
        b += 2 * (int32_t)bit - 1;
        v[i] = b;
    }
}

__global__ void __launch_bounds__(TC_THREADS, 1)
gram_tc_kernel(const SlopeSnapGeom g, uint64_t nkt, long long* __restrict__ part, unsigned int* __restrict__ err)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full[TC_STAGES], empty[TC_STAGES], accf, acce;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    // per stage: 1 when its tile has non-zero upper limbs (rows 64..191), written by the owning
    // warp before its arrival
    __shared__ volatile uint8_t upper[TC_STAGES];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    // lut[e4 | o4 << 4]: for 8 sites whose even-x bits are e4 and odd-x bits o4 (site order
    // e, o, e, o, ...), byte j = 8 + sum_{k <= j} (2 bit_k - 1), sites 0..3 in .x, 4..7 in .y
    uint2* lut = reinterpret_cast<uint2*>(smem + TC_STAGES * TC_STAGE);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // contiguous K-tile range of this CTA
    const uint64_t per = nkt / gridDim.x, rem = nkt % gridDim.x;
    const uint64_t kt0 = blockIdx.x * per + ((uint64_t)blockIdx.x < rem ? (uint64_t)blockIdx.x : rem);
    const uint64_t nloc = per + (blockIdx.x < rem ? 1 : 0);
    const uint64_t nwin = (nloc + TC_WINDOW - 1) / TC_WINDOW;

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(&full[s], 1);  // the owning warp's lane 0
            mbar_init(&empty[s], 1);
        }
        mbar_init(&accf, 1);
        mbar_init(&acce, 128);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < TC_LUT) {
        const uint32_t e4 = threadIdx.x & 15u, o4 = threadIdx.x >> 4;
        int32_t cum = 8;
        uint32_t w[2] = {0u, 0u};
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            cum += 2 * (int32_t)((((j & 1) ? o4 : e4) >> (j >> 1)) & 1u) - 1;
            w[j >> 2] |= (uint32_t)cum << (8 * (j & 3));
        }
        lut[threadIdx.x] = make_uint2(w[0], w[1]);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(TC_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = tmem_base;

    if (warp >= TC_PROD_WARP0) {
        // producer warp pw: tiles [cb0, cb1) of the CTA's range, in order, all into stage pw
        const int pw = warp - TC_PROD_WARP0;
        const uint64_t cb0 = kt0 + nloc * (uint64_t)pw / TC_PROD_WARPS;
        const uint64_t cb1 = kt0 + nloc * (uint64_t)(pw + 1) / TC_PROD_WARPS;
        uint8_t* stage = smem + pw * TC_STAGE;
        const int tpr_lg = g.lx - 7;
        const uint64_t tmask = (1ull << tpr_lg) - 1;
        // lane l: snapshots l and l + 32
        bool pres[2];
        const uint32_t* qb[2];
        const int2* rb[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int s = lane + 32 * k;
            pres[k] = s < g.n;
            qb[k] = g.snap + (uint64_t)s * 2 * g.Q;
            rb[k] = g.rows + (uint64_t)s * g.nrows;
        }
        // the next tile's words: [snapshot k][X quadrant], words 2t and 2t + 1
        uint2 nx[2][2];
        auto load = [&](uint64_t t) {
#pragma unroll
            for (int k = 0; k < 2; ++k)
#pragma unroll
                for (int q = 0; q < 2; ++q)
                    nx[k][q] = (pres[k] && t < cb1)
                                   ? __ldg(reinterpret_cast<const uint2*>(qb[k] + (uint64_t)q * g.Q + 2 * t))
                                   : make_uint2(0u, 0u);
        };
        load(cb0);
        int32_t B[2] = {0, 0}, z[2] = {0, 0};  // running value before the tile; v(0, y)
        int2 bzn[2] = {make_int2(0, 0), make_int2(0, 0)};  // {b, z} of the next row
        bool dirty = true;  // the stage's upper limb rows may hold non-zero bytes
        uint64_t m = 0;
        for (uint64_t t = cb0; t < cb1; ++t, ++m) {
            uint2 w[2][2];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                w[k][0] = nx[k][0];
                w[k][1] = nx[k][1];
            }
            load(t + 1);
            const uint64_t y = t >> tpr_lg;
            const uint32_t x0 = (uint32_t)(t & tmask) << 7;
            const bool rowstart = x0 == 0;
            if (t == cb0 || rowstart) {
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    if (!pres[k]) continue;
                    const int2 bz = (t == cb0) ? __ldg(rb[k] + y) : bzn[k];
                    if (y + 1 < g.nrows) bzn[k] = __ldg(rb[k] + y + 1);
                    z[k] = bz.y;
                    // v before site x0 (plus one at x0 = 0, whose own step is cleared below)
                    B[k] = bz.x + 1 + (rowstart ? 0 : 2 * slope_count_before(g, lane + 32 * k, y, x0) - (int32_t)x0);
                }
            }
            const int se = (int)(y & 1);  // X quadrant holding the even x of row y
            bool ok = true;
            if (lane == 0) ok = !abort_flag && mbar_wait_bounded(&empty[pw], (uint32_t)(m & 1) ^ 1u);
            if (!__shfl_sync(0xFFFFFFFFu, ok, 0)) {
                abort_flag = 1;
                break;
            }
            // low limbs, eight sites per lookup: byte = (b + 120) + lut byte = v + 128, which
            // stays in [0, 255] without carries while every group's starting value lies in
            // [-56, 55]; XOR 0x80 turns it into v's two's-complement byte
            const int32_t B0[2] = {B[0], B[1]};
            bool inrange = true;
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                uint32_t E[2] = {se ? w[k][1].x : w[k][0].x, se ? w[k][1].y : w[k][0].y};
                const uint32_t O[2] = {se ? w[k][0].x : w[k][1].x, se ? w[k][0].y : w[k][1].y};
                if (rowstart) E[0] &= ~1u;  // x = 0 closes the row in the walk
                int32_t b = B[k], bmin = b, bmax = b;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    uint32_t out[4];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int sh = 8 * (c & 3) + 4 * h;
                        const uint32_t idx = ((E[c >> 2] >> sh) & 15u) | (((O[c >> 2] >> sh) & 15u) << 4);
                        const uint2 T = lut[idx];
                        bmin = min(bmin, b);
                        bmax = max(bmax, b);
                        const uint32_t bb = (uint32_t)(b + 120) * 0x01010101u;
                        out[2 * h] = (bb + T.x) ^ 0x80808080u;
                        out[2 * h + 1] = (bb + T.y) ^ 0x80808080u;
                        b += (int32_t)(T.y >> 24) - 8;
                    }
                    if (c == 0 && rowstart) out[0] = (out[0] & ~0xFFu) | ((uint32_t)z[k] & 0xFFu);
                    const uint4 q = pres[k] ? make_uint4(out[0], out[1], out[2], out[3]) : make_uint4(0u, 0u, 0u, 0u);
                    put_chunk(stage, lane + 32 * k, c, q);
                }
                B[k] = b;
                if (pres[k])
                    inrange = inrange && bmin >= -56 && bmax <= 55 && (!rowstart || (z[k] >= -64 && z[k] <= 63));
            }
            const bool one_limb = __all_sync(0xFFFFFFFFu, inrange);
            if (!one_limb) {
                // balanced base-128 digits v = l0 + 128 l1 + 16384 l2, l_a in [-64, 63]
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    uint32_t E0 = se ? w[k][1].x : w[k][0].x;
                    const uint32_t E1 = se ? w[k][1].y : w[k][0].y;
                    const uint32_t O0 = se ? w[k][0].x : w[k][1].x, O1 = se ? w[k][0].y : w[k][1].y;
                    if (rowstart) E0 &= ~1u;
                    int32_t b = B0[k];
                    const int r = lane + 32 * k;
#pragma unroll 1
                    for (int c = 0; c < 8; ++c) {
                        int32_t v[16], l1v[16], l2v[16];
                        walk16((c >> 2) ? E1 : E0, (c >> 2) ? O1 : O0, c, b, v);
                        if (c == 0 && rowstart) v[0] = z[k];
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            const int32_t x = pres[k] ? v[j] : 0;
                            const int32_t l0 = ((x + 64) & 127) - 64;
                            const int32_t w1v = (x - l0) >> 7;
                            const int32_t l1 = ((w1v + 64) & 127) - 64;
                            v[j] = l0;
                            l1v[j] = l1;
                            l2v[j] = (w1v - l1) >> 7;
                        }
                        put_chunk(stage, r, c,
                                  make_uint4(pack4(v[0], v[1], v[2], v[3]), pack4(v[4], v[5], v[6], v[7]),
                                             pack4(v[8], v[9], v[10], v[11]), pack4(v[12], v[13], v[14], v[15])));
                        put_chunk(stage, 64 + r, c,
                                  make_uint4(pack4(l1v[0], l1v[1], l1v[2], l1v[3]),
                                             pack4(l1v[4], l1v[5], l1v[6], l1v[7]),
                                             pack4(l1v[8], l1v[9], l1v[10], l1v[11]),
                                             pack4(l1v[12], l1v[13], l1v[14], l1v[15])));
                        put_chunk(stage, 128 + r, c,
                                  make_uint4(pack4(l2v[0], l2v[1], l2v[2], l2v[3]),
                                             pack4(l2v[4], l2v[5], l2v[6], l2v[7]),
                                             pack4(l2v[8], l2v[9], l2v[10], l2v[11]),
                                             pack4(l2v[12], l2v[13], l2v[14], l2v[15])));
                    }
                }
                dirty = true;
            } else if (dirty) {
                // upper limb rows of a low-limb tile are zero
#pragma unroll 1
                for (int r = 64 + lane; r < TC_ROWS; r += 32)
#pragma unroll
                    for (int c = 0; c < 8; ++c) put_chunk(stage, r, c, make_uint4(0u, 0u, 0u, 0u));
                dirty = false;
            }
            if (lane == 0) upper[pw] = one_limb ? 0 : 1;
            // every writer makes its generic-proxy writes visible to the tensor core; the warp
            // then hands the stage over with one arrival
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&full[pw])) : "memory");
        }
    } else if (warp == 0) {
        if (lane == 0) {
            const uint32_t id1 = idesc_i8(128, 192), id2 = idesc_i8(128, 64), id0 = idesc_i8(128, 64);
            const uint64_t mmax = (nloc + TC_PROD_WARPS - 1) / TC_PROD_WARPS;
            uint64_t i = 0;  // tiles consumed
            bool stop = false;
            for (uint64_t m = 0; m < mmax && !stop; ++m) {
                for (int s = 0; s < TC_STAGES; ++s) {
                    const uint64_t ns = nloc * (uint64_t)(s + 1) / TC_PROD_WARPS - nloc * (uint64_t)s / TC_PROD_WARPS;
                    if (m >= ns) continue;
                    const uint64_t w = i / TC_WINDOW;
                    const bool first = (i % TC_WINDOW) == 0;
                    if (abort_flag || (first && w > 0 && !mbar_wait_bounded(&acce, (uint32_t)((w - 1) & 1))) ||
                        !mbar_wait_bounded(&full[s], (uint32_t)(m & 1))) {
                        abort_flag = 1;
                        stop = true;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = smem_u32(smem + s * TC_STAGE);
                    // a tile whose values all fit the low limb has zero rows 64..191: only the low
                    // limbs' 64 x 64 block is non-zero, and D1[0:128, 0:64] += A[0:128] . A[0:64]^T
                    // (rows 64..127 of A zero) adds exactly what the full products would
                    const bool full_tile = upper[s] != 0;
                    for (int kk = 0; kk < TC_KT / 32; ++kk) {
                        const uint32_t acc = (first && kk == 0) ? 0u : 1u;
                        if (full_tile || acc == 0u) {
                            umma_i8(tbase, sdesc_sw128(sa + 32 * kk), sdesc_sw128(sa + 32 * kk), id1, acc);
                            umma_i8(tbase + 192, sdesc_sw128(sa + 64 * TC_KT + 32 * kk),
                                    sdesc_sw128(sa + 128 * TC_KT + 32 * kk), id2, acc);
                        } else {
                            umma_i8(tbase, sdesc_sw128(sa + 32 * kk), sdesc_sw128(sa + 32 * kk), id0, acc);
                        }
                    }
                    umma_commit(&empty[s]);
                    if ((i % TC_WINDOW) == TC_WINDOW - 1 || i + 1 == nloc) umma_commit(&accf);
                    ++i;
                }
            }
        }
    } else {
        // epilogue: warps 1..4 own TMEM lane quarters (warp % 4)
        const int q = warp & 3;
        const int r = 32 * q + lane;  // accumulator row (TMEM lane)
        long long* prow1 = part + (uint64_t)blockIdx.x * TC_ROWS * TC_ROWS + (uint64_t)r * TC_ROWS;
        long long* prow2 = part + (uint64_t)blockIdx.x * TC_ROWS * TC_ROWS + (uint64_t)(64 + r) * TC_ROWS + 128;
        for (uint64_t w = 0; w < nwin; ++w) {
            if (!mbar_wait_bounded(&accf, (uint32_t)(w & 1))) {
                abort_flag = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int c0 = 0; c0 < TC_COLS; c0 += 32) {
                uint32_t v[32];
                const uint32_t taddr = tbase + ((uint32_t)(32 * q) << 16) + (uint32_t)c0;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                      "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                      "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (c0 < 192) {
                    for (int j = 0; j < 32; ++j) prow1[c0 + j] += (long long)(int32_t)v[j];
                } else if (r >= 64) {
                    // D2 rows 64..127 are limb rows 128..191; rows below 128 repeat D1
                    for (int j = 0; j < 32; ++j) prow2[c0 - 192 + j] += (long long)(int32_t)v[j];
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acce)) : "memory");
        }
    }
    // drain: all issued MMAs complete before the accumulator columns are released
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (abort_flag && threadIdx.x == 0) atomicExch(err, 1u);
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TC_COLS));
}

__global__ void gram_reduce_kernel(const long long* __restrict__ part, int grid, long long* __restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < TC_ROWS * TC_ROWS; i += gridDim.x * blockDim.x) {
        long long s = 0;
        for (int c = 0; c < grid; ++c) s += part[(uint64_t)c * TC_ROWS * TC_ROWS + i];
        out[i] = s;
    }
}

kpzb_status gram_tc_setup(GramTC* tc, uint64_t N, int sm_count)
{
    if (N % TC_KT || N > (1ull << 30)) return fail(KPZB_EINVAL, "gram: N must be a multiple of 128, <= 2^30");
    tc->grid = sm_count;
    cudaError_t e;
    if ((e = cudaMalloc(&tc->d_part, (size_t)tc->grid * TC_ROWS * TC_ROWS * 8)) != cudaSuccess)
        return cuda_fail(e, "cudaMalloc(gram partials)");
    if ((e = cudaMalloc(&tc->d_out, TC_ROWS * TC_ROWS * 8 + 64)) != cudaSuccess) return cuda_fail(e, "cudaMalloc(gram)");
    tc->d_err = reinterpret_cast<unsigned int*>(tc->d_out + TC_ROWS * TC_ROWS);
    if ((e = cudaFuncSetAttribute(gram_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TC_SMEM)) != cudaSuccess)
        return cuda_fail(e, "gram smem attribute");
    tc->ready = true;
    return KPZB_OK;
}

void gram_tc_free(GramTC* tc)
{
    cudaFree(tc->d_part);
    cudaFree(tc->d_out);
    tc->d_part = nullptr;
    tc->d_out = nullptr;
    tc->ready = false;
}

kpzb_status gram_tc_run(GramTC* tc, const SlopeSnapGeom& g, uint64_t N, int64_t* out, cudaStream_t st)
{
    if (!tc->ready) return fail(KPZB_ESTATE, "gram tensor path not set up");
    cudaError_t e;
    if ((e = cudaMemsetAsync(tc->d_part, 0, (size_t)tc->grid * TC_ROWS * TC_ROWS * 8, st)) != cudaSuccess)
        return cuda_fail(e, "memset partials");
    if ((e = cudaMemsetAsync(tc->d_err, 0, 4, st)) != cudaSuccess) return cuda_fail(e, "memset flag");
    gram_tc_kernel<<<tc->grid, TC_THREADS, TC_SMEM, st>>>(
        g, N / TC_KT, reinterpret_cast<long long*>(tc->d_part), tc->d_err);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "gram_tc_kernel");
    gram_reduce_kernel<<<64, 256, 0, st>>>(reinterpret_cast<const long long*>(tc->d_part), tc->grid,
                                          reinterpret_cast<long long*>(tc->d_out));
    unsigned int flag = 0;
    if ((e = cudaMemcpyAsync(out, tc->d_out, TC_ROWS * TC_ROWS * 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "gram copy");
    if ((e = cudaMemcpyAsync(&flag, tc->d_err, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "gram flag");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "gram sync");
    if (flag) return fail(KPZB_ETIMEOUT, "a bounded device wait in the tensor-core Gram expired");
    return KPZB_OK;
}

}  // namespace kpzb
