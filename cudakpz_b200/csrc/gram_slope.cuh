// gram_slope.cuh -- heights of stored slope snapshots, rebuilt on the fly for the correlator Gram.
//
// A snapshot is kept as the two X-slope quadrants of its ENC_CBBIT lattice (Q words each: the
// X quadrant of sublattice 0, then of sublattice 1; kpz/systemSize.h:143-165) plus, per row y,
// two int32: b(y) = Hs(y) - c and z(y) = h(0, y) - c, where Hs(y) is the height the reference's
// path walk (kpz/correlator.cpp:47-96) carries into row y before x = 1, h(0, y) the height it
// gives site x = 0 at the row's end, and c the snapshot's integer mean shift.  Along a row the
// walk adds 2 s_x(x, y) - 1 for x = 1, 2, ...:
//     v(x, y) = h(x, y) - c = b(y) + 2 * #{x' in [1, x] : s_x(x', y) = 1} - x      (x >= 1)
//     v(0, y) = z(y).
// K tile t (128 sites) is row y = t / (L / 128), x in [x0, x0 + 128), x0 = 128 * (t mod L/128).
// Four lanes (a lane quad) share a snapshot: lane qt takes sites x0 + 32 qt .. + 31, whose
// X-slope bits are 16 bits of one word of each X quadrant (even x on sublattice y & 1, odd x on
// the other), so a quarter tile costs two 32-bit loads.
#pragma once
#include <cstdint>

namespace kpzb {

constexpr int GS_TILE = 128;  // sites per K tile

struct SlopeSnapGeom {
    const uint32_t* snap;  // [n][2][Q] X-slope quadrants
    const int2* rows;      // [n][rows] {b(y), z(y)}
    uint64_t Q;            // words per quadrant
    uint64_t nrows;        // rows of the lattice (2^ly)
    int lx;                // log2 row length
    int n;                 // snapshots present (lanes of absent snapshots produce zeros)
};

// Running state of one lane: its snapshot, quarter, and the count of X-slope bits of its row
// in [1, x0) before the current tile (identical in the four lanes of a quad).
struct SlopeCursor {
    int s, qt;
    uint64_t last_tile;  // tile the running count was advanced past (~0: none)
    int32_t pre;
};

__device__ __forceinline__ void slope_cursor_init(SlopeCursor& c, int s, int qt)
{
    c.s = s;
    c.qt = qt;
    c.last_tile = ~0ull;
    c.pre = 0;
}

// The raw quarter words of tile t.
struct SlopeQuarter {
    uint32_t e, o;  // the X words holding this lane's 16 even-x bits (sublattice y & 1) and odd-x bits
    int2 bz;        // {b(y), z(y)}
};

// where the quarter's words lie (for loads issued ahead, e.g. by cp.async); lanes of absent
// snapshots get null pointers
struct SlopeQuarterAddr {
    const uint32_t* e;
    const uint32_t* o;
    const int2* bz;
};

__device__ __forceinline__ SlopeQuarterAddr slope_quarter_addr(const SlopeSnapGeom& g, const SlopeCursor& c, uint64_t t)
{
    if (c.s >= g.n) return SlopeQuarterAddr{nullptr, nullptr, nullptr};
    const int tpr_lg = g.lx - 7;  // log2 tiles per row
    const uint64_t y = t >> tpr_lg;
    const uint32_t x0 = (uint32_t)(t & ((1ull << tpr_lg) - 1)) << 7;
    const uint64_t Wr = 1ull << (g.lx - 6);
    const uint64_t w = y * Wr + (x0 >> 6) + (uint64_t)(c.qt >> 1);
    const uint32_t* base = g.snap + (uint64_t)c.s * 2 * g.Q;
    const int se = (int)(y & 1);
    return SlopeQuarterAddr{base + (uint64_t)se * g.Q + w, base + (uint64_t)(se ^ 1) * g.Q + w,
                            g.rows + (uint64_t)c.s * g.nrows + y};
}

__device__ __forceinline__ SlopeQuarter slope_quarter_load(const SlopeSnapGeom& g, const SlopeCursor& c, uint64_t t)
{
    const SlopeQuarterAddr a = slope_quarter_addr(g, c, t);
    if (!a.e) return SlopeQuarter{0u, 0u, make_int2(0, 0)};
    return SlopeQuarter{__ldg(a.e), __ldg(a.o), __ldg(a.bz)};
}

// Count of X-slope bits of row y in [1, x0) for the cursor's snapshot, from the row's words
// (used when a lane's tiles do not follow one another); the four lanes of the quad split the
// words and combine their counts.
__device__ __forceinline__ int32_t slope_row_prefix(const SlopeSnapGeom& g, const SlopeCursor& c, uint64_t t)
{
    const int tpr_lg = g.lx - 7;
    const uint64_t y = t >> tpr_lg;
    const uint32_t x0 = (uint32_t)(t & ((1ull << tpr_lg) - 1)) << 7;
    int32_t cnt = 0;
    if (c.s < g.n) {
        const uint64_t Wr = 1ull << (g.lx - 6);
        const uint32_t* base = g.snap + (uint64_t)c.s * 2 * g.Q + y * Wr;
        for (uint32_t j = (uint32_t)c.qt; j < (x0 >> 6); j += 4)
            cnt += __popc(__ldg(base + j)) + __popc(__ldg(base + g.Q + j));
        // site x = 0 (sublattice y & 1, word 0, bit 0) is not part of the walk's running sum
        if (c.qt == 0 && x0 > 0) cnt -= (int32_t)(__ldg(base + (y & 1) * g.Q) & 1u);
    }
    cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, 1);
    cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, 2);
    return cnt;
}

// The 32 values v = h - c of the lane's quarter of tile t, in site order, into v[0..31], and
// advances the running count.  `lo`, `hi` bound the 32 values.  All lanes of the warp call it
// together for the same tile (shuffles within each lane quad).
__device__ __forceinline__ void slope_quarter_heights(const SlopeSnapGeom& g, SlopeCursor& c, uint64_t t,
                                                      SlopeQuarter q, int32_t v[32], int32_t& lo, int32_t& hi)
{
    const int tpr_lg = g.lx - 7;
    const uint32_t x0 = (uint32_t)(t & ((1ull << tpr_lg) - 1)) << 7;
    if (x0 == 0) {
        c.pre = 0;
    } else if (c.last_tile == ~0ull || t != c.last_tile + 1) {
        c.pre = slope_row_prefix(g, c, t);
    }
    const int sh = 16 * (c.qt & 1);
    q.e = (q.e >> sh) & 0xFFFFu;
    q.o = (q.o >> sh) & 0xFFFFu;
    const bool first = x0 == 0 && c.qt == 0;
    if (first) q.e &= ~1u;  // x = 0 closes the row in the walk; its bit is not counted here
    const int32_t cnt = __popc(q.e) + __popc(q.o);
    // exclusive count of the quad's lower quarters, and the quad's total
    const int lane = (int)(threadIdx.x & 31);
    int32_t incl = cnt;
    const int32_t up1 = __shfl_up_sync(0xFFFFFFFFu, incl, 1);
    if ((lane & 3) >= 1) incl += up1;
    const int32_t up2 = __shfl_up_sync(0xFFFFFFFFu, incl, 2);
    if ((lane & 3) >= 2) incl += up2;
    const int32_t total = __shfl_sync(0xFFFFFFFFu, incl, (lane & ~3) | 3);
    const int32_t excl = incl - cnt;
    const int32_t xs = (int32_t)x0 + 32 * c.qt;
    const int32_t acc0 = q.bz.x + 2 * (c.pre + excl) - xs + 1;
    // four independent chains of 8 sites, each started from the count of the bits before it
    // (sites 8j .. 8j+7 hold even-x bits 4j .. 4j+3 and odd-x bits 4j .. 4j+3)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t below = (1u << (4 * j)) - 1u;
        int32_t acc = acc0 + 2 * (__popc(q.e & below) + __popc(q.o & below)) - 8 * j;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int i = 8 * j + k;
            const uint32_t word = (i & 1) ? q.o : q.e;
            const int32_t bit = (int32_t)((word >> (i >> 1)) & 1u);
            acc += 2 * bit - 1;
            v[i] = acc;
        }
    }
    const int32_t acc = acc0;
    lo = acc - 32;  // every step is +-1
    hi = lo + 64;
    if (first) {
        v[0] = q.bz.y;
        lo = min(lo, q.bz.y);
        hi = max(hi, q.bz.y);
    }
    if (c.s >= g.n) {
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = 0;
        lo = hi = 0;
    }
    c.pre += total;
    c.last_tile = t;
}

}  // namespace kpzb
