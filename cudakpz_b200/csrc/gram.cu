// gram.cu -- exact height autocorrelator over stored snapshots: snapshot -> int8 limbs,
// the int64 CUDA-core Gram, exact recombination and the C ABI (kpzb_gram_*).
//
// Reference behaviour: Correlator::correlateThreaded / correlateKernelCBBit accumulate
// sum h_snap * h_sys for one (snapshot, system) pair per call (kpz/correlator.cpp:491-593,
// kpz/correlatorCuda.cu:276-369); here the whole Gram G[s][t] = sum_sites h_s h_t over every
// stored pair is produced at once.
//
// Exactness: snapshot s keeps its path-relative heights (kpz/correlator.cpp:47-96) shifted
// by c_s = floor(<h_s>): v = h - c_s, split into three balanced base-128 digits
// v = l0 + 128 l1 + 16384 l2 with l_a in [-64, 63] (|v| < 1,056,832).  Row a*64+s of the
// limb matrix A (192 x N, int8) holds l_a of snapshot s, stored K-tile-major: the 192 rows x
// 128 sites of K tile kt are one contiguous 24 KB block (element (r, k) at
// (k / 128) * 24576 + r * 128 + k % 128), so the tensor-core kernel's TMA box of one tile is a
// single contiguous read.  The limb Gram A A^T is
// exact in int32 over windows of 2^18 sites (|l l'| <= 2^12) and summed in int64; then
//   sum v_s v_t = sum_{a,b} 128^(a+b) Glimb[a*64+s][b*64+t],
//   sum h_s h_t = sum v_s v_t + c_t S1v_s + c_s S1v_t + N c_s c_t,
// all in int64.  FP64 appears only in the caller's normalisation.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "kpzb_api_internal.h"
#include "kpzb_common.cuh"
#include "kpzb_gram.h"
#include "kpzb_internal.h"

namespace kpzb {

constexpr uint64_t LIMB_TILE = 128;                 // sites per K tile
constexpr uint64_t LIMB_TILE_BYTES = 192 * LIMB_TILE;  // one tile of all 192 rows

__host__ __device__ inline uint64_t limb_index(int row, uint64_t k)
{
    return (k / LIMB_TILE) * LIMB_TILE_BYTES + (uint64_t)row * LIMB_TILE + (k % LIMB_TILE);
}

// v = h - c split into balanced base-128 limbs (snapshot s: rows s, 64+s, 128+s); flags |v|
// too large for three limbs.
__global__ void limb_kernel(const int32_t* __restrict__ h, uint64_t n, int32_t c, int8_t* __restrict__ A, int s,
                            unsigned long long* __restrict__ sums, unsigned int* __restrict__ err)
{
    long long s0 = 0, s1 = 0, s2 = 0;
    const uint64_t n16 = n / 16;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n16;
         j += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t w[3][4];
        for (int q = 0; q < 4; ++q) {
            const int4 hv = reinterpret_cast<const int4*>(h)[4 * j + q];
            const int vals[4] = {hv.x, hv.y, hv.z, hv.w};
            uint32_t p0 = 0, p1 = 0, p2 = 0;
            for (int e = 0; e < 4; ++e) {
                const int v = vals[e] - c;
                const int l0 = ((v + 64) & 127) - 64;
                const int v1 = (v - l0) >> 7;
                const int l1 = ((v1 + 64) & 127) - 64;
                const int l2 = (v1 - l1) >> 7;
                if (l2 < -64 || l2 > 63) atomicExch(err, 1u);
                s0 += l0;
                s1 += l1;
                s2 += l2;
                p0 |= (uint32_t)(uint8_t)(int8_t)l0 << (8 * e);
                p1 |= (uint32_t)(uint8_t)(int8_t)l1 << (8 * e);
                p2 |= (uint32_t)(uint8_t)(int8_t)l2 << (8 * e);
            }
            w[0][q] = p0;
            w[1][q] = p1;
            w[2][q] = p2;
        }
        for (int a = 0; a < 3; ++a)
            *reinterpret_cast<uint4*>(A + limb_index(a * 64 + s, 16 * j)) =
                make_uint4(w[a][0], w[a][1], w[a][2], w[a][3]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&sums[0], (unsigned long long)s0);
        atomicAdd(&sums[1], (unsigned long long)s1);
        atomicAdd(&sums[2], (unsigned long long)s2);
    }
}

// Plain int64 CUDA-core Gram of v = l0 + 128 l1 + 16384 l2 over all snapshot pairs:
// a CTA stages 64 snapshots x 128 sites of v (int32) in shared memory, each of 256 threads
// owns a 4x4 block of (s,t) pairs with int64 accumulators; CTA results go to G by atomics.
constexpr int G64_KC = 128;
__global__ void __launch_bounds__(256)
gram_int64_kernel(const int8_t* __restrict__ A, uint64_t n, int ns, unsigned long long* __restrict__ G)
{
    __shared__ int32_t v[64][G64_KC + 1];
    const int ts = (threadIdx.x >> 4) * 4, tt = (threadIdx.x & 15) * 4;
    long long acc[4][4];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) acc[i][j] = 0;
    const bool active = ts < ns && tt < ns && tt + 3 >= ts;  // upper triangle (with diagonal blocks)
    for (uint64_t k0 = (uint64_t)blockIdx.x * G64_KC; k0 < n; k0 += (uint64_t)gridDim.x * G64_KC) {
        for (int e = threadIdx.x; e < 64 * G64_KC; e += 256) {
            const int s = e / G64_KC, kk = e - s * G64_KC;
            int32_t val = 0;
            if (s < ns) {
                const uint64_t idx = k0 + kk;
                val = (int32_t)A[limb_index(s, idx)] + 128 * (int32_t)A[limb_index(64 + s, idx)] +
                      16384 * (int32_t)A[limb_index(128 + s, idx)];
            }
            v[s][kk] = val;
        }
        __syncthreads();
        if (active) {
            for (int kk = 0; kk < G64_KC; ++kk) {
                int32_t a[4], b[4];
                for (int i = 0; i < 4; ++i) {
                    a[i] = v[ts + i][kk];
                    b[i] = v[tt + i][kk];
                }
                for (int i = 0; i < 4; ++i)
                    for (int j = 0; j < 4; ++j) acc[i][j] += (long long)a[i] * b[j];
            }
        }
        __syncthreads();
    }
    if (active)
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j)
                if (ts + i < ns && tt + j < ns && ts + i <= tt + j)
                    atomicAdd(&G[(ts + i) * 64 + tt + j], (unsigned long long)acc[i][j]);
}

}  // namespace kpzb

using namespace kpzb;

struct kpzb_gram {
    int lx = 0, ly = 0, device = 0, smax = 0, n = 0, sm_count = 148;
    uint64_t N = 0;
    cudaStream_t st = nullptr;
    int8_t* d_limbs = nullptr;      // [192][N]
    int32_t* d_heights = nullptr;   // scratch [N]
    uint32_t* d_tmp = nullptr;      // scratch lattice for host snapshots
    unsigned long long* d_sums = nullptr;  // [64][3] limb sums + error flag
    unsigned long long* d_g = nullptr;     // 64 x 64 int64 (CUDA-core path)
    std::vector<int64_t> shift;     // c_s
    AnalysisScratch an{};
    GramTC tc{};
};

#define GCHECK(g)                                                       \
    do {                                                                \
        if (!(g)) return fail(KPZB_EINVAL, "null gram");                \
        cudaError_t _e = cudaSetDevice((g)->device);                    \
        if (_e != cudaSuccess) return cuda_fail(_e, "cudaSetDevice");   \
    } while (0)
#define GCU(call, where)                                    \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, where); \
    } while (0)

extern "C" kpzb_status kpzb_gram_create(kpzb_gram** out, int lx, int ly, int max_snapshots, int device)
{
    if (!out) return fail(KPZB_EINVAL, "null output pointer");
    *out = nullptr;
    // 192 limb rows of N bytes each; TMA x coordinates are 32-bit
    if (lx < 8 || ly < 2 || lx + ly < 14 || lx + ly > 29)
        return fail(KPZB_EINVAL, "gram lattice size out of range (8<=lx, 14<=lx+ly<=29)");
    if (max_snapshots < 1 || max_snapshots > 64) return fail(KPZB_EINVAL, "1 <= max_snapshots <= 64");
    int dev = device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return fail(KPZB_ECUDA, "cudaGetDevice");
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    kpzb_gram* g = new kpzb_gram();
    g->lx = lx;
    g->ly = ly;
    g->device = dev;
    g->smax = max_snapshots;
    g->N = 1ull << (lx + ly);
    g->sm_count = sm_count_of(dev);
    auto bail = [&](kpzb_status s) {
        kpzb_gram_destroy(g);
        return s;
    };
    if ((e = cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(cuda_fail(e, "cudaStreamCreate"));
    // 192 limb rows always: rows of absent snapshots stay zero and add nothing
    if ((e = cudaMalloc(&g->d_limbs, 192 * g->N)) != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(limbs)"));
    if ((e = cudaMemset(g->d_limbs, 0, 192 * g->N)) != cudaSuccess) return bail(cuda_fail(e, "memset limbs"));
    if ((e = cudaMalloc(&g->d_heights, g->N * 4)) != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(heights)"));
    if ((e = cudaMalloc(&g->d_sums, (64 * 3 + 2) * 8)) != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(sums)"));
    if ((e = cudaMemset(g->d_sums, 0, (64 * 3 + 2) * 8)) != cudaSuccess) return bail(cuda_fail(e, "memset sums"));
    if ((e = cudaMalloc(&g->d_g, 64 * 64 * 8)) != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(G)"));
    if ((e = analysis_alloc(&g->an, ly)) != cudaSuccess) return bail(cuda_fail(e, "analysis_alloc"));
    kpzb_status s = gram_tc_setup(&g->tc, g->d_limbs, g->N, g->sm_count);
    if (s != KPZB_OK) return bail(s);
    *out = g;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_gram_destroy(kpzb_gram* g)
{
    if (!g) return KPZB_OK;
    cudaSetDevice(g->device);
    if (g->st) cudaStreamSynchronize(g->st);
    gram_tc_free(&g->tc);
    cudaFree(g->d_limbs);
    cudaFree(g->d_heights);
    cudaFree(g->d_tmp);
    cudaFree(g->d_sums);
    cudaFree(g->d_g);
    if (g->an.rowinfo) analysis_free(&g->an);
    if (g->st) cudaStreamDestroy(g->st);
    delete g;
    return KPZB_OK;
}

extern "C" int kpzb_gram_count(const kpzb_gram* g) { return g ? g->n : 0; }

extern "C" kpzb_status kpzb_gram_add_device(kpzb_gram* g, const uint32_t* d_cbbit)
{
    GCHECK(g);
    if (!d_cbbit) return fail(KPZB_EINVAL, "null lattice");
    if (g->n >= g->smax) return fail(KPZB_ESTATE, "snapshot capacity reached");
    const int s = g->n;
    // the snapshot's mean fixes its integer shift c_s = floor(<h>)
    MomentsOut m;
    GCU(analysis_moments(d_cbbit, nullptr, g->lx, g->ly, &g->an, &m, g->st), "snapshot moments");
    const long double mean = (long double)m.s1 / (long double)g->N;
    const int64_t c = (int64_t)std::floor((double)mean);
    if (m.hmax - c > 1000000 || c - m.hmin > 1000000) return fail(KPZB_EINVAL, "heights exceed three int8 limbs");
    GCU(analysis_heights(d_cbbit, g->lx, g->ly, &g->an, g->d_heights, g->st), "snapshot heights");
    const int grid = (int)std::min<uint64_t>(g->N / 16 / 256 + 1, (uint64_t)g->sm_count * 8);
    limb_kernel<<<grid, 256, 0, g->st>>>(g->d_heights, g->N, (int32_t)c, g->d_limbs, s, g->d_sums + 3 * s,
                                         reinterpret_cast<unsigned int*>(g->d_sums + 192));
    GCU(cudaGetLastError(), "limb_kernel");
    unsigned long long flag = 0;
    GCU(cudaMemcpyAsync(&flag, g->d_sums + 192, 8, cudaMemcpyDeviceToHost, g->st), "limb flag");
    GCU(cudaStreamSynchronize(g->st), "limb sync");
    if (flag) return fail(KPZB_EINVAL, "heights exceed three int8 limbs");
    g->shift.push_back(c);
    g->n++;
    return KPZB_OK;
}

extern "C" kpzb_status kpzb_gram_add_host(kpzb_gram* g, const uint32_t* cbbit)
{
    GCHECK(g);
    if (!cbbit) return fail(KPZB_EINVAL, "null lattice");
    if (!g->d_tmp) GCU(cudaMalloc(&g->d_tmp, g->N / 4), "cudaMalloc(tmp)");
    GCU(cudaMemcpyAsync(g->d_tmp, cbbit, g->N / 4, cudaMemcpyHostToDevice, g->st), "snapshot copy");
    return kpzb_gram_add_device(g, g->d_tmp);
}

// G_h[s][t] from the v-Gram (int64, s<=t) and the shifts; fills both triangles.
static void finish(const kpzb_gram* g, const std::vector<int64_t>& gv, const std::vector<int64_t>& s1v,
                   int64_t* G, int64_t* S1)
{
    const int n = g->n;
    const int64_t N = (int64_t)g->N;
    for (int s = 0; s < n; ++s) {
        if (S1) S1[s] = s1v[s] + N * g->shift[s];
        for (int t = s; t < n; ++t) {
            const int64_t v = gv[s * 64 + t] + g->shift[t] * s1v[s] + g->shift[s] * s1v[t] +
                              N * g->shift[s] * g->shift[t];
            G[s * n + t] = v;
            G[t * n + s] = v;
        }
    }
}

extern "C" kpzb_status kpzb_gram_compute(kpzb_gram* g, int method, int64_t* G, int64_t* S1)
{
    GCHECK(g);
    if (!G) return fail(KPZB_EINVAL, "null output");
    if (method != 0 && method != 1) return fail(KPZB_EINVAL, "method 0 (tensor) or 1 (int64)");
    const int n = g->n;
    if (n == 0) return KPZB_OK;
    std::vector<unsigned long long> sums(64 * 3);
    GCU(cudaMemcpyAsync(sums.data(), g->d_sums, 64 * 3 * 8, cudaMemcpyDeviceToHost, g->st), "limb sums");
    std::vector<int64_t> gv(64 * 64, 0), s1v(64, 0);
    if (method == 1) {
        GCU(cudaMemsetAsync(g->d_g, 0, 64 * 64 * 8, g->st), "memset G");
        const int grid = (int)std::min<uint64_t>(g->N / G64_KC, (uint64_t)g->sm_count * 4);
        gram_int64_kernel<<<grid, 256, 0, g->st>>>(g->d_limbs, g->N, n, g->d_g);
        GCU(cudaGetLastError(), "gram_int64_kernel");
        GCU(cudaMemcpyAsync(gv.data(), g->d_g, 64 * 64 * 8, cudaMemcpyDeviceToHost, g->st), "G copy");
        GCU(cudaStreamSynchronize(g->st), "gram sync");
    } else {
        std::vector<int64_t> gl(192 * 192);
        kpzb_status st = gram_tc_run(&g->tc, g->N, gl.data(), g->st);
        if (st != KPZB_OK) return st;
        // sum v_s v_t = sum_{a,b} 128^(a+b) Glimb[a*64+s][b*64+t]; the tensor kernel fills
        // the upper triangle of the limb Gram (row <= col), the rest by symmetry
        auto lg = [&](int r, int c) { return r <= c ? gl[r * 192 + c] : gl[c * 192 + r]; };
        for (int s = 0; s < n; ++s)
            for (int t = s; t < n; ++t) {
                int64_t acc = 0;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) acc += (int64_t)(1ll << (7 * (a + b))) * lg(a * 64 + s, b * 64 + t);
                gv[s * 64 + t] = acc;
            }
    }
    for (int s = 0; s < n; ++s)
        s1v[s] = (int64_t)sums[3 * s] + 128 * (int64_t)sums[3 * s + 1] + 16384 * (int64_t)sums[3 * s + 2];
    finish(g, gv, s1v, G, S1);
    return KPZB_OK;
}
