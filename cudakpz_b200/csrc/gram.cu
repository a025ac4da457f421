// gram.cu -- exact height autocorrelator over stored snapshots: snapshots kept as slope bits,
// the int64 CUDA-core Gram, exact recombination and the C ABI (kpzb_gram_*).
//
// Reference behaviour: Correlator::correlateThreaded / correlateKernelCBBit accumulate
// sum h_snap * h_sys for one (snapshot, system) pair per call (kpz/correlator.cpp:491-593,
// kpz/correlatorCuda.cu:276-369), and Correlator keeps its snapshots as lattices
// (kpz/correlator.cpp:37-106); here the whole Gram G[s][t] = sum_sites h_s h_t over every stored
// pair is produced at once.
//
// Storage: a snapshot is its two X-slope quadrants (N/8 bytes) and two int32 per row
// (gram_slope.cuh) -- 2 GiB for 64 snapshots of 16384^2, where stored int8 limbs would take
// 48 GiB.  Heights are rebuilt on the fly by the Gram kernels.
//
// Exactness: snapshot s keeps its path-relative heights (kpz/correlator.cpp:47-96) shifted
// by c_s = floor(<h_s>): v = h - c_s, split into three balanced base-128 digits
// v = l0 + 128 l1 + 16384 l2 with l_a in [-64, 63] (-1056832 <= v <= 1040447, checked when the
// snapshot is added).  Row a*64+s of the limb matrix A (192 x N, int8, built tile by tile in
// shared memory) holds l_a of snapshot s.  The limb Gram A A^T is exact in int32 over windows
// of 2^18 sites (|l l'| <= 2^12) and summed in int64; then
//   sum v_s v_t = sum_{a,b} 128^(a+b) Glimb[a*64+s][b*64+t],
//   sum h_s h_t = sum v_s v_t + c_t S1v_s + c_s S1v_t + N c_s c_t,
// all in int64, with S1v_s = S1(h_s) - N c_s exact from the height walk.  FP64 appears only in
// the caller's normalisation.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "kpzb_api_internal.h"
#include "kpzb_common.cuh"
#include "kpzb_gram.h"
#include "gram_slope.cuh"
#include "kpzb_internal.h"

namespace kpzb {

// per-row data of snapshot s: {b(y), z(y)} = {Hs(y) - c, h(0, y) - c} from the height walk's
// row starts Hs and row sums (the analysis scratch of the snapshot just measured)
__global__ void gram_rows_kernel(const int64_t* __restrict__ rowstart, const int32_t* __restrict__ rowinfo,
                                 uint64_t rows, int64_t c, int2* __restrict__ out)
{
    for (uint64_t y = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; y < rows; y += (uint64_t)gridDim.x * blockDim.x)
        out[y] = make_int2((int32_t)(rowstart[y] - c), (int32_t)(rowstart[y] + rowinfo[2 * y + 1] - c));
}

// Plain int64 CUDA-core Gram of v = h - c over all snapshot pairs, from the same slope
// snapshots: a CTA takes a contiguous range of 128-site tiles, its 256 threads rebuild the 64
// snapshots x 128 sites of each tile into shared memory (gram_slope.cuh, a lane quad per
// snapshot), then each thread owns a 4x4 block of (s,t) pairs with int64 accumulators; CTA
// results go to G by atomics.
constexpr int G64_KC = GS_TILE;
__global__ void __launch_bounds__(256)
gram_int64_kernel(const SlopeSnapGeom g, uint64_t nkt, unsigned long long* __restrict__ G)
{
    __shared__ int32_t v[64][G64_KC + 1];
    const int ts = (threadIdx.x >> 4) * 4, tt = (threadIdx.x & 15) * 4;
    const int ns = g.n;
    long long acc[4][4];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) acc[i][j] = 0;
    const bool active = ts < ns && tt < ns && tt + 3 >= ts;  // upper triangle (with diagonal blocks)
    const uint64_t per = nkt / gridDim.x, rem = nkt % gridDim.x;
    const uint64_t kt0 = blockIdx.x * per + ((uint64_t)blockIdx.x < rem ? (uint64_t)blockIdx.x : rem);
    const uint64_t nloc = per + (blockIdx.x < rem ? 1 : 0);
    const int s = threadIdx.x >> 2, qt = threadIdx.x & 3;
    SlopeCursor cur;
    slope_cursor_init(cur, s, qt);
    for (uint64_t i = 0; i < nloc; ++i) {
        const uint64_t t = kt0 + i;
        int32_t h[32], lo, hi;
        slope_quarter_heights(g, cur, t, slope_quarter_load(g, cur, t), h, lo, hi);
        for (int j = 0; j < 32; ++j) v[s][32 * qt + j] = h[j];
        __syncthreads();
        if (active) {
            for (int kk = 0; kk < G64_KC; ++kk) {
                int32_t a[4], b[4];
                for (int ii = 0; ii < 4; ++ii) {
                    a[ii] = v[ts + ii][kk];
                    b[ii] = v[tt + ii][kk];
                }
                for (int ii = 0; ii < 4; ++ii)
                    for (int jj = 0; jj < 4; ++jj) acc[ii][jj] += (long long)a[ii] * b[jj];
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
    uint64_t N = 0, Q = 0, rows = 0;
    cudaStream_t st = nullptr;
    uint32_t* d_snap = nullptr;     // [smax][2][Q] X-slope quadrants
    int2* d_rows = nullptr;         // [smax][rows] {b(y), z(y)}
    uint32_t* d_tmp = nullptr;      // scratch lattice for host snapshots
    unsigned long long* d_g = nullptr;  // 64 x 64 int64 (CUDA-core path)
    std::vector<int64_t> shift;     // c_s
    std::vector<int64_t> s1v;       // sum (h_s - c_s)
    AnalysisScratch an{};
    GramTC tc{};

    SlopeSnapGeom geom() const { return SlopeSnapGeom{d_snap, d_rows, Q, rows, lx, n}; }
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
    g->Q = g->N >> 6;
    g->rows = 1ull << ly;
    if ((e = cudaMalloc(&g->d_snap, (size_t)max_snapshots * 2 * g->Q * 4)) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(snapshots)"));
    if ((e = cudaMalloc(&g->d_rows, (size_t)max_snapshots * g->rows * sizeof(int2))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(snapshot rows)"));
    if ((e = cudaMalloc(&g->d_g, 64 * 64 * 8)) != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(G)"));
    if ((e = analysis_alloc(&g->an, ly)) != cudaSuccess) return bail(cuda_fail(e, "analysis_alloc"));
    kpzb_status s = gram_tc_setup(&g->tc, g->N, g->sm_count);
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
    cudaFree(g->d_snap);
    cudaFree(g->d_rows);
    cudaFree(g->d_tmp);
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
    // the snapshot's mean fixes its integer shift c_s = floor(<h>); the walk that measures it
    // leaves the row starts and row sums in the analysis scratch
    MomentsOut m;
    GCU(analysis_moments(d_cbbit, nullptr, g->lx, g->ly, &g->an, &m, g->st), "snapshot moments");
    const long double mean = (long double)m.s1 / (long double)g->N;
    const int64_t c = (int64_t)std::floor((double)mean);
    if (m.hmin - c < -1056832 || m.hmax - c > 1040447) return fail(KPZB_EINVAL, "heights exceed three int8 limbs");
    // the two X-slope quadrants (sublattice 0 at word 0, sublattice 1 at 2Q)
    uint32_t* dst = g->d_snap + (uint64_t)s * 2 * g->Q;
    GCU(cudaMemcpyAsync(dst, d_cbbit, g->Q * 4, cudaMemcpyDeviceToDevice, g->st), "snapshot copy");
    GCU(cudaMemcpyAsync(dst + g->Q, d_cbbit + 2 * g->Q, g->Q * 4, cudaMemcpyDeviceToDevice, g->st), "snapshot copy");
    const int grid = (int)std::min<uint64_t>(g->rows / 256 + 1, (uint64_t)g->sm_count * 4);
    gram_rows_kernel<<<grid, 256, 0, g->st>>>(g->an.rowstart, g->an.rowinfo, g->rows, c,
                                             g->d_rows + (uint64_t)s * g->rows);
    GCU(cudaGetLastError(), "gram_rows_kernel");
    GCU(cudaStreamSynchronize(g->st), "snapshot sync");
    g->shift.push_back(c);
    g->s1v.push_back(m.s1 - (int64_t)g->N * c);
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
    std::vector<int64_t> gv(64 * 64, 0), s1v(g->s1v);
    const SlopeSnapGeom geo = g->geom();
    if (method == 1) {
        GCU(cudaMemsetAsync(g->d_g, 0, 64 * 64 * 8, g->st), "memset G");
        const int grid = (int)std::min<uint64_t>(g->N / G64_KC, (uint64_t)g->sm_count * 4);
        gram_int64_kernel<<<grid, 256, 0, g->st>>>(geo, g->N / G64_KC, g->d_g);
        GCU(cudaGetLastError(), "gram_int64_kernel");
        GCU(cudaMemcpyAsync(gv.data(), g->d_g, 64 * 64 * 8, cudaMemcpyDeviceToHost, g->st), "G copy");
        GCU(cudaStreamSynchronize(g->st), "gram sync");
    } else {
        std::vector<int64_t> gl(192 * 192);
        kpzb_status st = gram_tc_run(&g->tc, geo, g->N, gl.data(), g->st);
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
    finish(g, gv, s1v, G, S1);
    return KPZB_OK;
}
