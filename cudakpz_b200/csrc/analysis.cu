// analysis.cu -- height reconstruction, roughness moments, correlator and lattice
// invariants on ENC_CBBIT lattices (sm_100a).
//
// Heights follow the reference's path walk (kpz/correlator.cpp:47-96, :337-399):
//   row y starts at Hs(y) = h(0,y-1) + (2*s_y(0,y)-1) with h(0,-1) = 0, walks x = 1..L-1
//   adding 2*s_x(x,y)-1, and the wrap adds 2*s_x(0,y)-1 giving h(0,y) = Hs(y) + rowsum(y).
// Moments: S1 and S2 exact in int64, S3..S7 in FP64 (per 64-site chunk from exact integer
// power sums of the offsets from the chunk's first height); ch uses the exact int64 cross sum;
// cs counts equal minus different slope bits (kpz/correlator.cpp:463-477).
// Invariants extend SchedulerService::consitencyCheck (kpz/schedulerService.cpp:733-854)
// to ENC_CBBIT: x-slope row sums, y-slope column sums, plaquette loops.
//
// Three passes: (1) per-row x=0 slopes and x-slope sums, (2) one-CTA scan over rows to
// get row-start heights, (3) per-site walk with a CTA-wide scan of 64-site chunk sums.
// Per-CTA partials are reduced in a fixed order so the FP64 sums are deterministic.
#include <cstring>
#include <map>
#include <mutex>
#include "kpzb_api_internal.h"
#include "kpzb_common.cuh"
#include "kpzb_internal.h"

namespace kpzb {

constexpr int AN_THREADS = 256;
constexpr int AN_MAX_GRID = 1184;

struct Partial {
    long long s1, s2, hmin, hmax, cross, agree, snap_s1, pad;
    double s[5];
    double pad2[3];
};

// ---- pass 1: per-row x=0 slopes and x-slope row sums (one warp per row) ----
__global__ void rowinfo_kernel(const uint32_t* __restrict__ sys, int lx, int ly, int32_t* rowinfo)
{
    const uint64_t Wr = 1ull << (lx - 6);
    const uint64_t Q = 1ull << (lx + ly - 6);
    const uint64_t rows = 1ull << ly;
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t y = warp; y < rows; y += nwarps) {
        int cnt = 0;
        for (uint64_t j = lane; j < Wr; j += 32)
            cnt += __popc(sys[y * Wr + j]) + __popc(sys[2 * Q + y * Wr + j]);
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0) {
            // site (0,y) lies on sublattice y&1, word 0, bit 0
            const uint64_t b0 = (y & 1) ? 2 * Q : 0;
            const int sy0 = (int)(sys[b0 + Q + y * Wr] & 1u);
            rowinfo[2 * y] = 2 * sy0 - 1;
            rowinfo[2 * y + 1] = 2 * cnt - (int)(1ull << lx);
        }
    }
}

// ---- pass 2: row-start heights Hs(y) (single CTA, chunked Hillis-Steele scan) ----
__global__ void rowstart_kernel(const int32_t* __restrict__ rowinfo, int ly, int64_t* rowstart)
{
    __shared__ long long buf[1024];
    __shared__ long long carry;
    const uint64_t rows = 1ull << ly;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint64_t base = 0; base < rows; base += 1024) {
        const uint64_t y = base + threadIdx.x;
        // Hs(y) = sum_{y'<=y} ycol(y') + sum_{y'<y} rowsum(y')
        // contribution of row y to the inclusive scan: ycol(y) + rowsum(y-1) handled as
        // v(y) = ycol(y) + rowsum(y); Hs(y) = incl(v)(y) - rowsum(y)
        long long v = (y < rows) ? (long long)rowinfo[2 * y] + rowinfo[2 * y + 1] : 0;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            long long add = (threadIdx.x >= (unsigned)o) ? buf[threadIdx.x - o] : 0;
            __syncthreads();
            buf[threadIdx.x] += add;
            __syncthreads();
        }
        if (y < rows) rowstart[y] = carry + buf[threadIdx.x] - rowinfo[2 * y + 1];
        __syncthreads();
        if (threadIdx.x == 1023) carry += buf[1023];
        __syncthreads();
    }
}

// ---- pass 3: per-site walk ----
// MODE 0: moments; MODE 1: moments + correlate against snap; MODE 2: write heights.
template <int MODE>
__global__ void __launch_bounds__(AN_THREADS)
walk_kernel(const uint32_t* __restrict__ sys, const uint32_t* __restrict__ snap, int lx, int ly,
            const int32_t* __restrict__ rowinfo, const int64_t* __restrict__ rowstart,
            const int32_t* __restrict__ rowinfo_s, const int64_t* __restrict__ rowstart_s,
            int32_t* __restrict__ heights, Partial* __restrict__ partials)
{
    __shared__ long long wsum[AN_THREADS / 32];
    __shared__ long long wsum_s[AN_THREADS / 32];
    __shared__ long long segc[AN_THREADS];
    __shared__ long long segc_s[AN_THREADS];

    const uint64_t Wr = 1ull << (lx - 6);
    const uint64_t Q = 1ull << (lx + ly - 6);
    const uint64_t rows = 1ull << ly;
    const int TPR = (int)(Wr < AN_THREADS ? Wr : AN_THREADS);
    const int RPC = AN_THREADS / TPR;
    const int tx = threadIdx.x % TPR, ty = threadIdx.x / TPR;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nseg = (int)(Wr / TPR);
    const uint64_t groups = rows / RPC;
    const uint64_t L = 1ull << lx;

    long long s1 = 0, s2 = 0, cross = 0, agree = 0, ss1 = 0;
    long long hmin = 0x7fffffffffffffffll, hmax = -0x7fffffffffffffffll;
    double s3 = 0, s4 = 0, s5 = 0, s6 = 0, s7 = 0;

    for (uint64_t g = blockIdx.x; g < groups; g += gridDim.x) {
        const uint64_t y = g * RPC + ty;
        const uint64_t be = (y & 1) ? 2 * Q : 0, bo = (y & 1) ? 0 : 2 * Q;
        const long long Hs = rowstart[y];
        const long long rsum = rowinfo[2 * y + 1];
        long long Hs_s = 0, rsum_s = 0;
        if (MODE == 1) {
            Hs_s = rowstart_s[y];
            rsum_s = rowinfo_s[2 * y + 1];
        }
        // e0 = 2*s_x(0,y)-1 (bit 0 of the even-x word 0)
        const long long e0 = 2 * (long long)(sys[be + y * Wr] & 1u) - 1;
        long long e0_s = 0;
        if (MODE == 1) e0_s = 2 * (long long)(snap[be + y * Wr] & 1u) - 1;
        long long run = 0, run_s = 0;  // prefix carried from previous segments
        for (int seg = 0; seg < nseg; ++seg) {
            const uint64_t c = (uint64_t)seg * TPR + tx;
            const uint32_t E = sys[be + y * Wr + c], O = sys[bo + y * Wr + c];
            uint32_t Es = 0, Os = 0;
            if (MODE == 1) {
                Es = snap[be + y * Wr + c];
                Os = snap[bo + y * Wr + c];
                const uint32_t EY = sys[be + Q + y * Wr + c], OY = sys[bo + Q + y * Wr + c];
                const uint32_t EYs = snap[be + Q + y * Wr + c], OYs = snap[bo + Q + y * Wr + c];
                agree += 2 * (__popc(~(E ^ Es)) + __popc(~(O ^ Os)) + __popc(~(EY ^ EYs)) +
                              __popc(~(OY ^ OYs))) - 128;
            }
            long long v = 2 * (__popc(E) + __popc(O)) - 64;
            long long vs = (MODE == 1) ? 2 * (__popc(Es) + __popc(Os)) - 64 : 0;
            // inclusive scan of v over the TPR threads of this row
            long long incl = v, incl_s = vs;
            const int wl = TPR < 32 ? TPR : 32;
            for (int o = 1; o < wl; o <<= 1) {
                long long a = __shfl_up_sync(0xffffffffu, incl, o, wl);
                long long as = __shfl_up_sync(0xffffffffu, incl_s, o, wl);
                if ((lane % wl) >= o) {
                    incl += a;
                    incl_s += as;
                }
            }
            if (TPR > 32) {
                if (lane == 31) {
                    wsum[wid] = incl;
                    wsum_s[wid] = incl_s;
                }
                __syncthreads();
                const int w0 = (ty * TPR) >> 5;  // first warp of this row
                for (int w = w0; w < wid; ++w) {
                    incl += wsum[w];
                    incl_s += wsum_s[w];
                }
            }
            // P(x) before this chunk (inclusive prefix from x = 0)
            long long P = run + incl - v;
            long long Ps = run_s + incl_s - vs;
            // last thread of the row publishes the segment total
            if (tx == TPR - 1) {
                segc[ty] = run + incl;
                segc_s[ty] = run_s + incl_s;
            }
            __syncthreads();
            run = segc[ty];
            run_s = segc_s[ty];
            __syncthreads();
            if constexpr (MODE == 0) {
                // The chunk's heights are b + d_i with b the height before its first site and
                // |d_i| <= 64, so the power sums of d are exact in 32/64-bit integers (d^4 sums to
                // at most 64 * 64^4 < 2^31; d^5..d^7 accumulate in int64) and the moments of h
                // follow once per chunk by the binomial expansion in FP64.  The row's first site
                // (x = 0, height Hs + rowsum) is left out of the sums and added directly.
                const long long b = Hs - e0 + P;
                const bool first = c == 0;
                int d = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, dmin = 64, dmax = -64;
                long long a5 = 0, a6 = 0, a7 = 0;
#pragma unroll
                for (int i = 0; i < 64; ++i) {
                    const int bit = (int)((((i & 1) ? O : E) >> (i >> 1)) & 1u);
                    d += 2 * bit - 1;
                    if (i == 0 && first) continue;
                    const int d2 = d * d, d3 = d2 * d, d4 = d2 * d2;
                    a1 += d;
                    a2 += d2;
                    a3 += d3;
                    a4 += d4;
                    a5 += (long long)d4 * d;
                    a6 += (long long)d3 * d3;
                    a7 += (long long)d4 * d3;
                    dmin = min(dmin, d);
                    dmax = max(dmax, d);
                }
                const int n = first ? 63 : 64;
                s1 += (long long)n * b + a1;
                s2 += (long long)n * b * b + 2 * b * a1 + a2;
                hmin = min(hmin, b + dmin);
                hmax = max(hmax, b + dmax);
                const double B = (double)b, B2 = B * B, B3 = B2 * B, B4 = B2 * B2, B5 = B4 * B, B6 = B3 * B3,
                             B7 = B6 * B;
                const double n_ = n, A1 = a1, A2 = a2, A3 = a3, A4 = a4, A5 = (double)a5, A6 = (double)a6,
                             A7 = (double)a7;
                s3 += n_ * B3 + 3.0 * B2 * A1 + 3.0 * B * A2 + A3;
                s4 += n_ * B4 + 4.0 * B3 * A1 + 6.0 * B2 * A2 + 4.0 * B * A3 + A4;
                s5 += n_ * B5 + 5.0 * B4 * A1 + 10.0 * B3 * A2 + 10.0 * B2 * A3 + 5.0 * B * A4 + A5;
                s6 += n_ * B6 + 6.0 * B5 * A1 + 15.0 * B4 * A2 + 20.0 * B3 * A3 + 15.0 * B2 * A4 + 6.0 * B * A5 + A6;
                s7 += n_ * B7 + 7.0 * B6 * A1 + 21.0 * B5 * A2 + 35.0 * B4 * A3 + 35.0 * B3 * A4 + 21.0 * B2 * A5 +
                      7.0 * B * A6 + A7;
                if (first) {
                    const long long h = Hs + rsum;
                    s1 += h;
                    s2 += h * h;
                    const double dh = (double)h, dh2 = dh * dh, dh3 = dh2 * dh;
                    s3 += dh3;
                    s4 += dh2 * dh2;
                    s5 += dh3 * dh2;
                    s6 += dh3 * dh3;
                    s7 += dh3 * dh3 * dh;
                    hmin = min(hmin, h);
                    hmax = max(hmax, h);
                }
                continue;
            }
            for (int i = 0; i < 64; ++i) {
                const uint32_t bit = (((i & 1) ? O : E) >> (i >> 1)) & 1u;
                P += 2 * (long long)bit - 1;
                const uint64_t x = c * 64 + i;
                const long long h = (x == 0) ? Hs + rsum : Hs - e0 + P;
                if (MODE == 2) {
                    heights[y * L + x] = (int32_t)h;
                } else {
                    s1 += h;
                    s2 += h * h;
                    const double d = (double)h, d2 = d * d, d3 = d2 * d;
                    s3 += d3;
                    s4 += d2 * d2;
                    s5 += d3 * d2;
                    s6 += d3 * d3;
                    s7 += d3 * d3 * d;
                    hmin = min(hmin, h);
                    hmax = max(hmax, h);
                    if (MODE == 1) {
                        const uint32_t bs = (((i & 1) ? Os : Es) >> (i >> 1)) & 1u;
                        Ps += 2 * (long long)bs - 1;
                        const long long hs = (x == 0) ? Hs_s + rsum_s : Hs_s - e0_s + Ps;
                        cross += h * hs;
                        ss1 += hs;
                    }
                }
            }
        }
    }
    if constexpr (MODE != 2) {
        // block reduction in fixed order
        __shared__ Partial red[AN_THREADS / 32];
        for (int o = 16; o > 0; o >>= 1) {
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            s2 += __shfl_xor_sync(0xffffffffu, s2, o);
            cross += __shfl_xor_sync(0xffffffffu, cross, o);
            agree += __shfl_xor_sync(0xffffffffu, agree, o);
            ss1 += __shfl_xor_sync(0xffffffffu, ss1, o);
            hmin = min(hmin, __shfl_xor_sync(0xffffffffu, hmin, o));
            hmax = max(hmax, __shfl_xor_sync(0xffffffffu, hmax, o));
            s3 += __shfl_xor_sync(0xffffffffu, s3, o);
            s4 += __shfl_xor_sync(0xffffffffu, s4, o);
            s5 += __shfl_xor_sync(0xffffffffu, s5, o);
            s6 += __shfl_xor_sync(0xffffffffu, s6, o);
            s7 += __shfl_xor_sync(0xffffffffu, s7, o);
        }
        if (lane == 0) {
            Partial p;
            p.s1 = s1; p.s2 = s2; p.hmin = hmin; p.hmax = hmax; p.cross = cross; p.agree = agree;
            p.snap_s1 = ss1; p.pad = 0;
            p.s[0] = s3; p.s[1] = s4; p.s[2] = s5; p.s[3] = s6; p.s[4] = s7;
            red[wid] = p;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            Partial p = red[0];
            for (int w = 1; w < AN_THREADS / 32; ++w) {
                const Partial& q = red[w];
                p.s1 += q.s1; p.s2 += q.s2; p.cross += q.cross; p.agree += q.agree;
                p.snap_s1 += q.snap_s1;
                p.hmin = min(p.hmin, q.hmin); p.hmax = max(p.hmax, q.hmax);
                for (int k = 0; k < 5; ++k) p.s[k] += q.s[k];
            }
            partials[blockIdx.x] = p;
        }
    }
}

// Sum of the per-CTA partials in a fixed order (so repeated runs agree bit for bit): thread t
// adds partials t, t + 256, ... in turn, then a fixed pairwise tree over the 256 threads.
constexpr int FR_THREADS = 256;

__device__ __forceinline__ void merge_partial(Partial& p, const Partial& q)
{
    p.s1 += q.s1; p.s2 += q.s2; p.cross += q.cross; p.agree += q.agree;
    p.snap_s1 += q.snap_s1;
    p.hmin = min(p.hmin, q.hmin); p.hmax = max(p.hmax, q.hmax);
    for (int k = 0; k < 5; ++k) p.s[k] += q.s[k];
}

__global__ void __launch_bounds__(FR_THREADS) final_reduce_kernel(const Partial* __restrict__ partials, int n,
                                                                  Partial* out)
{
    __shared__ Partial red[FR_THREADS];
    Partial p{};
    p.hmin = 0x7fffffffffffffffll;
    p.hmax = -0x7fffffffffffffffll;
    for (int i = threadIdx.x; i < n; i += FR_THREADS) merge_partial(p, partials[i]);
    red[threadIdx.x] = p;
    __syncthreads();
    for (int w = FR_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) merge_partial(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

cudaError_t analysis_alloc(AnalysisScratch* s, int ly)
{
    const size_t rows = 1ull << ly;
    s->rows_cap = rows;
    cudaError_t e;
    // two row tables (system and snapshot) and partials + final record
    if ((e = cudaMalloc(&s->rowinfo, 4 * rows * sizeof(int32_t))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s->rowstart, 2 * rows * sizeof(int64_t))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s->acc, (AN_MAX_GRID + 1) * sizeof(Partial) + 64)) != cudaSuccess) return e;
    return cudaSuccess;
}

void analysis_free(AnalysisScratch* s)
{
    cudaFree(s->rowinfo);
    cudaFree(s->rowstart);
    cudaFree(s->acc);
    s->rowinfo = nullptr;
    s->rowstart = nullptr;
    s->acc = nullptr;
}

static int walk_grid(int lx, int ly)
{
    const uint64_t Wr = 1ull << (lx - 6);
    const int TPR = (int)(Wr < AN_THREADS ? Wr : AN_THREADS);
    const uint64_t groups = (1ull << ly) / (AN_THREADS / TPR);
    return (int)(groups < AN_MAX_GRID ? groups : AN_MAX_GRID);
}

static cudaError_t row_tables(const uint32_t* d, int lx, int ly, int32_t* ri, int64_t* rs,
                              cudaStream_t st)
{
    const uint64_t rows = 1ull << ly;
    const int grid = (int)((rows * 32 + 255) / 256 < 4096 ? (rows * 32 + 255) / 256 : 4096);
    rowinfo_kernel<<<grid, 256, 0, st>>>(d, lx, ly, ri);
    rowstart_kernel<<<1, 1024, 0, st>>>(ri, ly, rs);
    return cudaGetLastError();
}

size_t analysis_record_bytes() { return sizeof(Partial); }

void analysis_decode_record(const void* rec, MomentsOut* out)
{
    Partial h;
    memcpy(&h, rec, sizeof h);
    out->s1 = h.s1;
    out->s2 = h.s2;
    for (int k = 0; k < 5; ++k) out->s3to7[k] = h.s[k];
    out->hmin = h.hmin;
    out->hmax = h.hmax;
    out->cross = h.cross;
    out->agree = h.agree;
    out->snap_s1 = h.snap_s1;
}

cudaError_t analysis_moments_record(const uint32_t* d_sys, const uint32_t* d_snap, int lx, int ly,
                                    AnalysisScratch* s, void* d_rec, cudaStream_t st)
{
    const uint64_t rows = 1ull << ly;
    int32_t* ri = s->rowinfo;
    int32_t* ri_s = s->rowinfo + 2 * rows;
    int64_t* rs = s->rowstart;
    int64_t* rs_s = s->rowstart + rows;
    Partial* parts = reinterpret_cast<Partial*>(s->acc);
    cudaError_t e = row_tables(d_sys, lx, ly, ri, rs, st);
    if (e != cudaSuccess) return e;
    const int grid = walk_grid(lx, ly);
    if (d_snap) {
        if ((e = row_tables(d_snap, lx, ly, ri_s, rs_s, st)) != cudaSuccess) return e;
        walk_kernel<1><<<grid, AN_THREADS, 0, st>>>(d_sys, d_snap, lx, ly, ri, rs, ri_s, rs_s,
                                                    nullptr, parts);
    } else {
        walk_kernel<0><<<grid, AN_THREADS, 0, st>>>(d_sys, nullptr, lx, ly, ri, rs, nullptr,
                                                    nullptr, nullptr, parts);
    }
    final_reduce_kernel<<<1, FR_THREADS, 0, st>>>(parts, grid, reinterpret_cast<Partial*>(d_rec));
    return cudaGetLastError();
}

cudaError_t analysis_moments(const uint32_t* d_sys, const uint32_t* d_snap, int lx, int ly,
                             AnalysisScratch* s, MomentsOut* out, cudaStream_t st)
{
    const uint64_t rows = 1ull << ly;
    int32_t* ri = s->rowinfo;
    int32_t* ri_s = s->rowinfo + 2 * rows;
    int64_t* rs = s->rowstart;
    int64_t* rs_s = s->rowstart + rows;
    Partial* parts = reinterpret_cast<Partial*>(s->acc);
    Partial* fin = parts + AN_MAX_GRID;
    cudaError_t e = row_tables(d_sys, lx, ly, ri, rs, st);
    if (e != cudaSuccess) return e;
    const int grid = walk_grid(lx, ly);
    if (d_snap) {
        if ((e = row_tables(d_snap, lx, ly, ri_s, rs_s, st)) != cudaSuccess) return e;
        walk_kernel<1><<<grid, AN_THREADS, 0, st>>>(d_sys, d_snap, lx, ly, ri, rs, ri_s, rs_s,
                                                    nullptr, parts);
    } else {
        walk_kernel<0><<<grid, AN_THREADS, 0, st>>>(d_sys, nullptr, lx, ly, ri, rs, nullptr,
                                                    nullptr, nullptr, parts);
    }
    final_reduce_kernel<<<1, FR_THREADS, 0, st>>>(parts, grid, fin);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    Partial h;
    if ((e = cudaMemcpyAsync(&h, fin, sizeof(Partial), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    out->s1 = h.s1;
    out->s2 = h.s2;
    for (int k = 0; k < 5; ++k) out->s3to7[k] = h.s[k];
    out->hmin = h.hmin;
    out->hmax = h.hmax;
    out->cross = h.cross;
    out->agree = h.agree;
    out->snap_s1 = h.snap_s1;
    return cudaSuccess;
}

cudaError_t analysis_heights(const uint32_t* d_sys, int lx, int ly, AnalysisScratch* s,
                             int32_t* d_heights, cudaStream_t st)
{
    cudaError_t e = row_tables(d_sys, lx, ly, s->rowinfo, s->rowstart, st);
    if (e != cudaSuccess) return e;
    walk_kernel<2><<<walk_grid(lx, ly), AN_THREADS, 0, st>>>(d_sys, nullptr, lx, ly, s->rowinfo,
                                                             s->rowstart, nullptr, nullptr,
                                                             d_heights, nullptr);
    return cudaGetLastError();
}

// ---- invariants ----
// columns: thread per (x parity a, word column j, band of 256 rows); per-bit counters.
__global__ void colsum_kernel(const uint32_t* __restrict__ sys, int lx, int ly, int* colsum)
{
    const uint64_t Wr = 1ull << (lx - 6);
    const uint64_t Q = 1ull << (lx + ly - 6);
    const uint64_t rows = 1ull << ly;
    const uint64_t band = rows < 256 ? rows : 256;
    const uint64_t nb = rows / band;
    const uint64_t total = 2 * Wr * nb;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t j = i % Wr;
        const int a = (int)((i / Wr) & 1);
        const uint64_t b = i / (2 * Wr);
        int cnt[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) cnt[k] = 0;
        for (uint64_t y = b * band; y < (b + 1) * band; ++y) {
            const int sub = a ^ (int)(y & 1);
            const uint32_t w = sys[(sub ? 2 * Q : 0) + Q + y * Wr + j];
#pragma unroll
            for (int k = 0; k < 32; ++k) cnt[k] += (w >> k) & 1u;
        }
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            const uint64_t x = 64 * j + 2 * k + a;
            atomicAdd(&colsum[x], 2 * cnt[k] - (int)band);
        }
    }
}

__global__ void invariants_kernel(const uint32_t* __restrict__ sys, int lx, int ly,
                                  const int32_t* __restrict__ rowinfo, const int* __restrict__ colsum,
                                  unsigned long long* rep)
{
    const uint64_t Wr = 1ull << (lx - 6);
    const uint64_t Q = 1ull << (lx + ly - 6);
    const uint64_t rows = 1ull << ly;
    const uint64_t L = 1ull << lx;
    unsigned long long badr = 0, badc = 0, badp = 0;
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t y = tid; y < rows; y += nth) badr += rowinfo[2 * y + 1] != 0;
    for (uint64_t x = tid; x < L; x += nth) badc += colsum[x] != 0;
    // plaquettes: per (sublattice, row, word)
    for (uint64_t i = tid; i < 2 * Q; i += nth) {
        const int sub = (int)(i / Q);
        const uint64_t r = i % Q;
        const uint64_t y = r / Wr, j = r % Wr;
        const uint64_t bt = sub ? 2 * Q : 0, bo = sub ? 0 : 2 * Q;
        const int A = sub ^ (int)(y & 1);  // x parity of this sublattice in row y
        const uint32_t a = sys[bt + y * Wr + j];          // s_x(x,y)
        const uint32_t b = sys[bt + Q + y * Wr + j];      // s_y(x,y)
        uint32_t c;                                        // s_y(x-1,y)
        const uint32_t oy = sys[bo + Q + y * Wr + j];
        if (A) c = oy;
        else c = (oy << 1) | (sys[bo + Q + y * Wr + ((j + Wr - 1) & (Wr - 1))] >> 31);
        const uint32_t d = sys[bo + ((y + rows - 1) & (rows - 1)) * Wr + j];  // s_x(x,y-1)
        const uint32_t bad = ((a ^ c) ^ (b ^ d)) | ((a & c) ^ (b & d));
        badp += __popc(bad);
    }
    for (int o = 16; o > 0; o >>= 1) {
        badr += __shfl_xor_sync(0xffffffffu, badr, o);
        badc += __shfl_xor_sync(0xffffffffu, badc, o);
        badp += __shfl_xor_sync(0xffffffffu, badp, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&rep[0], badr);
        atomicAdd(&rep[1], badc);
        atomicAdd(&rep[2], badp);
    }
}

cudaError_t analysis_invariants(const uint32_t* d_sys, int lx, int ly, AnalysisScratch* s,
                                int64_t rep[3], cudaStream_t st)
{
    const uint64_t rows = 1ull << ly, L = 1ull << lx;
    int* colsum = nullptr;
    cudaError_t e;
    if ((e = cudaMallocAsync(&colsum, L * sizeof(int) + 64, st)) != cudaSuccess) return e;
    unsigned long long* drep = reinterpret_cast<unsigned long long*>(colsum + L);
    cudaMemsetAsync(colsum, 0, L * sizeof(int) + 64, st);
    const int grid0 = (int)((rows * 32 + 255) / 256 < 4096 ? (rows * 32 + 255) / 256 : 4096);
    rowinfo_kernel<<<grid0, 256, 0, st>>>(d_sys, lx, ly, s->rowinfo);
    colsum_kernel<<<512, 256, 0, st>>>(d_sys, lx, ly, colsum);
    invariants_kernel<<<1184, 256, 0, st>>>(d_sys, lx, ly, s->rowinfo, colsum, drep);
    unsigned long long h[3] = {0, 0, 0};
    cudaMemcpyAsync(h, drep, sizeof(h), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    cudaFreeAsync(colsum, st);
    if (e == cudaSuccess) e = cudaGetLastError();
    rep[0] = (int64_t)h[0];
    rep[1] = (int64_t)h[1];
    rep[2] = (int64_t)h[2];
    return e;
}

}  // namespace kpzb

// ---------------------------------------------------------------------------------------
// Roughness without any allocation (kpzb_roughness_noalloc).
//
// Some callers cannot allocate device memory at the point where they want a measurement:
// an application whose memory manager owns the whole device (a caching allocator that must
// see every allocation, or a budget already spent on lattices), or a timing loop that must
// not stall other streams -- cudaMalloc and cudaFree can synchronize the device.  For them
// this entry point reads a caller's device lattice and writes the caller's host output, and
// keeps its scratch (row tables and per-CTA partial sums) in one file-scope device array of
// fixed size.  Every GPU that loads the library's module holds the array until the process
// exits.
//
// Limit: ly <= NOALLOC_MAX_LY (at most 65536 rows); any lx the other entry points accept.
// The array is shared by every call: concurrent calls that overlap on the GPU (on different
// streams or host threads) race on it and must be serialized by the caller.  Every kernel
// writes each scratch word before reading it, so nothing has to be cleared between calls.
// Set-up: the array's device address is looked up with cudaGetSymbolAddress once per device
// and CUDA context, while that device is current, and cached under the context's unique id;
// a context created anew (after the caller's cudaDeviceReset) gets a fresh lookup.  That
// first call may also load the library's module, and the array with it, so a caller with a
// window in which nothing may be allocated makes one call before the window opens; the
// first call on a device should come before any stream capture the caller starts.
// ---------------------------------------------------------------------------------------
namespace kpzb {

constexpr int NOALLOC_MAX_LY = 16;
constexpr size_t NOALLOC_ROWINFO = 2ull * (1ull << NOALLOC_MAX_LY) * sizeof(int32_t);
constexpr size_t NOALLOC_ROWSTART = (1ull << NOALLOC_MAX_LY) * sizeof(int64_t);
constexpr size_t NOALLOC_PARTIALS = (AN_MAX_GRID + 1) * sizeof(Partial);
constexpr size_t NOALLOC_BYTES = NOALLOC_ROWINFO + NOALLOC_ROWSTART + NOALLOC_PARTIALS;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

namespace {
// driver entry points for the current context and its process-unique id (CUDA >= 12.0),
// resolved once through the runtime so the library needs no link against libcuda
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);
struct NoallocSetup {
    unsigned long long ctx_id = 0;
    void* addr = nullptr;
};
std::mutex g_noalloc_mu;
std::map<int, NoallocSetup> g_noalloc_setup;  // per device: context id -> symbol address
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
bool g_ctx_fns_looked_up = false;

// id of the context current on this thread; false when there is none (or it is gone)
bool current_ctx_id(unsigned long long* id)
{
    if (!g_ctx_fns_looked_up) {
        g_ctx_fns_looked_up = true;
        cudaDriverEntryPointQueryResult q1, q2;
        void* f1 = nullptr;
        void* f2 = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) ==
                cudaSuccess && q1 == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) == cudaSuccess &&
            q2 == cudaDriverEntryPointSuccess) {
            g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
            g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f2);
        }
    }
    if (!g_ctx_get_current || !g_ctx_get_id) return false;
    void* ctx = nullptr;
    if (g_ctx_get_current(&ctx) != 0 || !ctx) return false;
    return g_ctx_get_id(ctx, id) == 0;
}
}  // namespace

// The scratch array's device address on the current device (set-up once per device and
// context; see above).
static cudaError_t noalloc_scratch_addr(int dev, void** out)
{
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    unsigned long long id = 0;
    const bool have_ctx = current_ctx_id(&id);
    auto it = g_noalloc_setup.find(dev);
    if (have_ctx && it != g_noalloc_setup.end() && it->second.ctx_id == id && it->second.addr) {
        *out = it->second.addr;
        return cudaSuccess;
    }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    if (!p) return cudaErrorInvalidSymbol;
    unsigned long long id_after = 0;
    // the lookup makes the device's primary context current if none was
    if (current_ctx_id(&id_after)) g_noalloc_setup[dev] = NoallocSetup{id_after, p};
    else g_noalloc_setup.erase(dev);  // no id to key on: look up again next time
    *out = p;
    return cudaSuccess;
}

}  // namespace kpzb

extern "C" kpzb_status kpzb_roughness_noalloc(const uint32_t* d_cbbit, int lx, int ly, double out[8],
                                              void* stream)
{
    using namespace kpzb;
    if (!d_cbbit || !out) return fail(KPZB_EINVAL, "null lattice or output");
    if (lx < 8 || lx > 30 || ly < 2 || lx + ly < 14 || lx + ly > 38)
        return fail(KPZB_EINVAL, "lattice size out of range (8<=lx<=30, 14<=lx+ly<=38)");
    if (ly > NOALLOC_MAX_LY)
        return fail(KPZB_EINVAL, "ly > 16: the fixed no-allocation scratch holds at most 65536 rows");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    void* addr = nullptr;
    e = noalloc_scratch_addr(dev, &addr);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    unsigned char* base = static_cast<unsigned char*>(addr);
    AnalysisScratch view;
    view.rowinfo = reinterpret_cast<int32_t*>(base);
    view.rowstart = reinterpret_cast<int64_t*>(base + NOALLOC_ROWINFO);
    view.acc = reinterpret_cast<unsigned long long*>(base + NOALLOC_ROWINFO + NOALLOC_ROWSTART);
    view.rows_cap = 1ull << NOALLOC_MAX_LY;
    MomentsOut m;
    e = analysis_moments(d_cbbit, nullptr, lx, ly, &view, &m, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "roughness (no-alloc)");
    const long double N = (long double)((uint64_t)1 << (lx + ly));
    long double h[7];
    h[0] = (long double)m.s1 / N;
    h[1] = (long double)m.s2 / N;
    for (int k = 0; k < 5; ++k) h[2 + k] = (long double)m.s3to7[k] / N;
    out[0] = (double)(h[1] - h[0] * h[0]);
    for (int k = 0; k < 7; ++k) out[1 + k] = (double)h[k];
    return KPZB_OK;
}

