// gram_tc.cu -- exact limb Gram of the stored snapshots on tcgen05 tensor cores (sm_100a).
//
// One persistent CTA per SM takes a contiguous range of 128-site K tiles.  Eight producer warps
// rebuild each tile's heights from the snapshots' slope bits (gram_slope.cuh: 64 snapshots x 4
// lanes, 32 sites a lane), shift them by the snapshot's integer mean and split them into three
// signed int8 limbs, written straight into a shared-memory stage in the K-major SWIZZLE_128B
// layout the MMA descriptors expect (limb row a * 64 + s, 128 bytes a row, 16-byte chunk c of
// row r at chunk position c ^ (r mod 8)); a fence.proxy.async hands the stage to the tensor
// core.  Warp 0 owns 256 TMEM columns and issues, per 32-byte K step,
//   D1[0:128, 0:192]   += A[0:128]   . A[0:192]^T   (M=128, N=192)
//   D2[0:128, 0:64]    += A[64:192]  . A[128:192]^T (M=128, N=64)
// (kind::i8, signed, int32 accumulators in TMEM); together they cover every (row <= col)
// entry of the symmetric 192 x 192 limb Gram.  Every 2^18 K elements (|l l'| <= 2^12, so
// the int32 sums stay below 2^30) warps 1-4 read the accumulators with tcgen05.ld and add
// them to the CTA's int64 partial in global memory; a final kernel sums the partials.
// Only the slope bits cross HBM: 16 bytes per snapshot per tile instead of 384 bytes of
// stored limbs.  Every mbarrier wait is bounded: on expiry the kernel raises a flag, stops
// issuing work, drains what it issued, frees its TMEM and returns.
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
constexpr int TC_STAGES = 6;
constexpr int TC_WINDOW = (1 << 18) / TC_KT;      // K tiles per int32 accumulation window
constexpr int TC_PRODUCERS = 256;                 // 64 snapshots x 4 quarter tiles
constexpr int TC_PROD_WARP0 = 5;                  // warps 5..12 produce, 1..4 flush, 0 issues
constexpr int TC_THREADS = TC_PROD_WARP0 * 32 + TC_PRODUCERS;
constexpr int TC_COLS = 256;                      // TMEM columns: D1 0..191, D2 192..255
constexpr int TC_PREFETCH = 8;                    // tiles of slope words in flight per producer
constexpr int TC_SMEM = TC_STAGES * TC_STAGE + TC_PREFETCH * TC_PRODUCERS * 16 + 1024;
constexpr uint32_t TC_SPIN = 1u << 26;

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

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    uint32_t spins = 0;
    while (!mbar_try_wait(bar, parity))
        if (++spins > TC_SPIN) return false;
    return true;
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

__global__ void __launch_bounds__(TC_THREADS, 1)
gram_tc_kernel(const SlopeSnapGeom g, uint64_t nkt, long long* __restrict__ part, unsigned int* __restrict__ err)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full[TC_STAGES], empty[TC_STAGES], accf, acce;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    // per stage and producer warp: 1 when the warp wrote non-zero upper limbs (rows 64..191);
    // every warp writes its byte for every tile, before its arrival on the stage
    __shared__ __align__(8) uint8_t upper[TC_STAGES][8];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    // per producer lane, TC_PREFETCH slots of {e word, o word, b, z} filled by cp.async
    uint4* ring = reinterpret_cast<uint4*>(smem + TC_STAGES * TC_STAGE);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // contiguous K-tile range of this CTA
    const uint64_t per = nkt / gridDim.x, rem = nkt % gridDim.x;
    const uint64_t kt0 = blockIdx.x * per + ((uint64_t)blockIdx.x < rem ? (uint64_t)blockIdx.x : rem);
    const uint64_t nloc = per + (blockIdx.x < rem ? 1 : 0);
    const uint64_t nwin = (nloc + TC_WINDOW - 1) / TC_WINDOW;

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(&full[s], TC_PRODUCERS / 32);  // one arrival per producer warp
            mbar_init(&empty[s], 1);
        }
        mbar_init(&accf, 1);
        mbar_init(&acce, 128);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
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
        // producers: lane quad of snapshot s, lane qt of the quad takes a quarter of each tile
        const int p = threadIdx.x - TC_PROD_WARP0 * 32;
        const int s = p >> 2, qt = p & 3;
        SlopeCursor cur;
        slope_cursor_init(cur, s, qt);
        // tile t's words into slot t mod TC_PREFETCH, one copy group per tile (empty groups
        // past the range and for absent snapshots keep the group count uniform)
        auto issue = [&](uint64_t i) {
            if (i < nloc) {
                const SlopeQuarterAddr a = slope_quarter_addr(g, cur, kt0 + i);
                if (a.e) {
                    uint4* slot = ring + (i % TC_PREFETCH) * TC_PRODUCERS + p;
                    const uint32_t d = smem_u32(slot);
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(a.e) : "memory");
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d + 4), "l"(a.o) : "memory");
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d + 8), "l"(a.bz) : "memory");
                }
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
        };
        for (int d = 0; d < TC_PREFETCH; ++d) issue((uint64_t)d);
        for (uint64_t i = 0; i < nloc; ++i) {
            const uint64_t t = kt0 + i;
            asm volatile("cp.async.wait_group %0;" ::"n"(TC_PREFETCH - 1) : "memory");
            SlopeQuarter q{0u, 0u, make_int2(0, 0)};
            if (s < g.n) {
                const uint4 r = ring[(i % TC_PREFETCH) * TC_PRODUCERS + p];
                q = SlopeQuarter{r.x, r.y, make_int2((int32_t)r.z, (int32_t)r.w)};
            }
            int32_t v[32], lo, hi;
            slope_quarter_heights(g, cur, t, q, v, lo, hi);
            issue(i + TC_PREFETCH);  // into the slot just read (its value is in registers)
            const int st = (int)(i % TC_STAGES);
            const uint32_t ph = (uint32_t)((i / TC_STAGES) & 1);
            // lane 0 waits for the stage to be free; the warp follows it, or leaves with it
            bool ok = true;
            if (lane == 0) ok = !abort_flag && mbar_wait_bounded(&empty[st], ph ^ 1u);
            if (!__shfl_sync(0xFFFFFFFFu, ok, 0)) {
                abort_flag = 1;
                break;
            }
            uint8_t* stage = smem + st * TC_STAGE;
            const bool one_limb = __all_sync(0xFFFFFFFFu, lo >= -64 && hi <= 63);
            if (lane == 0) upper[st][warp - TC_PROD_WARP0] = one_limb ? 0 : 1;
            if (one_limb) {
                // every value is its own low limb; the two upper limbs are zero
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const int b = 16 * c;
                    put_chunk(stage, s, 2 * qt + c,
                              make_uint4(pack4(v[b], v[b + 1], v[b + 2], v[b + 3]),
                                         pack4(v[b + 4], v[b + 5], v[b + 6], v[b + 7]),
                                         pack4(v[b + 8], v[b + 9], v[b + 10], v[b + 11]),
                                         pack4(v[b + 12], v[b + 13], v[b + 14], v[b + 15])));
                    put_chunk(stage, 64 + s, 2 * qt + c, make_uint4(0u, 0u, 0u, 0u));
                    put_chunk(stage, 128 + s, 2 * qt + c, make_uint4(0u, 0u, 0u, 0u));
                }
            } else {
                // balanced base-128 digits v = l0 + 128 l1 + 16384 l2, l_a in [-64, 63]
                int32_t l1v[32], l2v[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int32_t l0 = ((v[j] + 64) & 127) - 64;
                    const int32_t w1 = (v[j] - l0) >> 7;
                    const int32_t l1 = ((w1 + 64) & 127) - 64;
                    v[j] = l0;
                    l1v[j] = l1;
                    l2v[j] = (w1 - l1) >> 7;
                }
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const int b = 16 * c;
                    put_chunk(stage, s, 2 * qt + c,
                              make_uint4(pack4(v[b], v[b + 1], v[b + 2], v[b + 3]),
                                         pack4(v[b + 4], v[b + 5], v[b + 6], v[b + 7]),
                                         pack4(v[b + 8], v[b + 9], v[b + 10], v[b + 11]),
                                         pack4(v[b + 12], v[b + 13], v[b + 14], v[b + 15])));
                    put_chunk(stage, 64 + s, 2 * qt + c,
                              make_uint4(pack4(l1v[b], l1v[b + 1], l1v[b + 2], l1v[b + 3]),
                                         pack4(l1v[b + 4], l1v[b + 5], l1v[b + 6], l1v[b + 7]),
                                         pack4(l1v[b + 8], l1v[b + 9], l1v[b + 10], l1v[b + 11]),
                                         pack4(l1v[b + 12], l1v[b + 13], l1v[b + 14], l1v[b + 15])));
                    put_chunk(stage, 128 + s, 2 * qt + c,
                              make_uint4(pack4(l2v[b], l2v[b + 1], l2v[b + 2], l2v[b + 3]),
                                         pack4(l2v[b + 4], l2v[b + 5], l2v[b + 6], l2v[b + 7]),
                                         pack4(l2v[b + 8], l2v[b + 9], l2v[b + 10], l2v[b + 11]),
                                         pack4(l2v[b + 12], l2v[b + 13], l2v[b + 14], l2v[b + 15])));
                }
            }
            // every writer makes its generic-proxy writes visible to the tensor core; the warp
            // then reports its part of the stage with one arrival
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&full[st])) : "memory");
        }
        asm volatile("cp.async.wait_all;" ::: "memory");  // no copy lands after the CTA retires
    } else if (warp == 0) {
        if (lane == 0) {
            const uint32_t id1 = idesc_i8(128, 192), id2 = idesc_i8(128, 64), id0 = idesc_i8(128, 64);
            for (uint64_t i = 0; i < nloc && !abort_flag; ++i) {
                const int s = (int)(i % TC_STAGES);
                const uint32_t ph = (uint32_t)((i / TC_STAGES) & 1);
                const uint64_t w = i / TC_WINDOW;
                const bool first = (i % TC_WINDOW) == 0;
                if (first && w > 0 && !mbar_wait_bounded(&acce, (uint32_t)((w - 1) & 1))) {
                    abort_flag = 1;
                    break;
                }
                if (!mbar_wait_bounded(&full[s], ph)) {
                    abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t sa = smem_u32(smem + s * TC_STAGE);
                // a tile whose values all fit the low limb has zero rows 64..191: only the low
                // limbs' 64 x 64 block is non-zero, and D1[0:128, 0:64] += A[0:128] . A[0:64]^T
                // (rows 64..127 of A zero) adds exactly what the full products would
                const bool full_tile = *reinterpret_cast<const volatile uint64_t*>(&upper[s][0]) != 0ull;
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
