// codec.cu -- flat start and ENC_LOCAL <-> ENC_CBBIT transcoding on the device.
//
// ENC_LOCAL (kpz/systemSize.h:94-124): word (y>>2)*(L/4) + (x>>2), bit ((x&3)<<1)|((y&3)<<3),
//   bit0 = x-slope, bit1 = y-slope.
// ENC_CBBIT (kpz/systemSize.h:143-165): quadrants [sub0.X|sub0.Y|sub1.X|sub1.Y], row y of a
//   quadrant is L/64 words, site x of sublattice (x^y)&1 at word x>>6, bit (x>>1)&31.
// Flat start (kpz/schedulerService.cpp:156-175): LOCAL words 0x33CC33CC; CBBIT sub0 all 0,
//   sub1 all 1.
#include "kpzb_common.cuh"
#include "kpzb_internal.h"

namespace kpzb {

__global__ void fill_kernel(uint32_t* d, uint64_t n, uint32_t v)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        d[i] = v;
}

cudaError_t init_homogeneous_dev(uint32_t* d, int lx, int ly, int encoding, cudaStream_t st)
{
    const uint64_t sw = 1ull << (lx + ly - 4);
    const int grid = (int)((sw / 256 + 1) < 4096 ? (sw / 256 + 1) : 4096);
    if (encoding == 0) {
        fill_kernel<<<grid, 256, 0, st>>>(d, sw, 0x33CC33CCu);
    } else {
        fill_kernel<<<grid, 256, 0, st>>>(d, sw / 2, 0u);
        fill_kernel<<<grid, 256, 0, st>>>(d + sw / 2, sw / 2, 0xFFFFFFFFu);
    }
    return cudaGetLastError();
}

// One thread per (row y, 64-site chunk c): reads the 16 LOCAL words covering x in
// [64c, 64c+64) of row y, writes the four CBBIT words (sub0.X, sub0.Y, sub1.X, sub1.Y).
__global__ void local_to_cbbit_kernel(const uint32_t* __restrict__ local, uint32_t* __restrict__ cb,
                                      int lx, int ly)
{
    const uint64_t Wr = 1ull << (lx - 6);
    const uint64_t Q = 1ull << (lx + ly - 6);
    const uint64_t total = Q;  // (rows) * (chunks per row)
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t y = i >> (lx - 6);
        const uint64_t c = i & (Wr - 1);
        const uint32_t* src = local + (y >> 2) * (1ull << (lx - 2)) + c * 16;
        const int ysh = (int)(y & 3) << 3;
        uint32_t evenX = 0, evenY = 0, oddX = 0, oddY = 0;  // by x parity
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const uint32_t w = src[k] >> ysh;
            // x = 4k + {0,1,2,3}: bits at 0,2,4,6 (x-slope) and 1,3,5,7 (y-slope)
            const int b0 = 2 * k;      // site index among even x: x/2 = 2k, 2k+1
            evenX |= ((w >> 0) & 1u) << b0;
            evenY |= ((w >> 1) & 1u) << b0;
            oddX |= ((w >> 2) & 1u) << b0;
            oddY |= ((w >> 3) & 1u) << b0;
            evenX |= ((w >> 4) & 1u) << (b0 + 1);
            evenY |= ((w >> 5) & 1u) << (b0 + 1);
            oddX |= ((w >> 6) & 1u) << (b0 + 1);
            oddY |= ((w >> 7) & 1u) << (b0 + 1);
        }
        // even x belong to sublattice (y&1), odd x to sublattice (y&1)^1
        const int se = (int)(y & 1);
        const uint64_t off = y * Wr + c;
        const uint64_t be = se ? 2 * Q : 0, bo = se ? 0 : 2 * Q;
        cb[be + off] = evenX;
        cb[be + Q + off] = evenY;
        cb[bo + off] = oddX;
        cb[bo + Q + off] = oddY;
    }
}

// One thread per LOCAL word: gathers its 4x4 sites from the CBBIT quadrants.
__global__ void cbbit_to_local_kernel(const uint32_t* __restrict__ cb, uint32_t* __restrict__ local,
                                      int lx, int ly)
{
    const uint64_t Wr = 1ull << (lx - 6);
    const uint64_t Q = 1ull << (lx + ly - 6);
    const uint64_t total = 1ull << (lx + ly - 4);
    const int lxw = lx - 2;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t wy = i >> lxw, wx = i & ((1ull << lxw) - 1);
        uint32_t out = 0;
#pragma unroll
        for (int dy = 0; dy < 4; ++dy) {
            const uint64_t y = 4 * wy + dy;
#pragma unroll
            for (int dx = 0; dx < 4; ++dx) {
                const uint64_t x = 4 * wx + dx;
                const int sub = (int)((x ^ y) & 1);
                const uint64_t idx = (sub ? 2 * Q : 0) + y * Wr + (x >> 6);
                const int b = (int)((x >> 1) & 31);
                const uint32_t sx = (cb[idx] >> b) & 1u;
                const uint32_t sy = (cb[idx + Q] >> b) & 1u;
                out |= (sx | (sy << 1)) << ((dx << 1) | (dy << 3));
            }
        }
        local[i] = out;
    }
}

cudaError_t local_to_cbbit_dev(const uint32_t* local, uint32_t* cbbit, int lx, int ly, cudaStream_t st)
{
    const uint64_t n = 1ull << (lx + ly - 6);
    const int grid = (int)((n / 256 + 1) < 8192 ? (n / 256 + 1) : 8192);
    local_to_cbbit_kernel<<<grid, 256, 0, st>>>(local, cbbit, lx, ly);
    return cudaGetLastError();
}

cudaError_t cbbit_to_local_dev(const uint32_t* cbbit, uint32_t* local, int lx, int ly, cudaStream_t st)
{
    const uint64_t n = 1ull << (lx + ly - 4);
    const int grid = (int)((n / 256 + 1) < 8192 ? (n / 256 + 1) : 8192);
    cbbit_to_local_kernel<<<grid, 256, 0, st>>>(cbbit, local, lx, ly);
    return cudaGetLastError();
}

}  // namespace kpzb
