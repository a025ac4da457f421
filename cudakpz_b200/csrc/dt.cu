// dt.cu -- double-tiling (DT) random-sequential dynamics on ENC_LOCAL lattices (sm_100a).
//
// Reference behaviour: SchedulerDT::doMcs (kpz/schedulerDT.cu:38-78) -- per MCS a random
// origin in [0, 2*block) and a shuffled order of the four domain sets, one launch per set;
// kpzKernelTemplateDT + copyInDT/copyOutDT (kpz/kpz.cu:126-155, kpz/kpzCopy.cu:144-187) --
// each block is copied with a one-word halo into shared memory, updated, copied back; the
// inner single-hit double tiling of KpzCores::BaseDT
// (kpz/kpzSimulationPrimitivesTemplates.cu:110-141) -- per attempt round the whole block
// uses one random quadrant (sub-cell) of every thread cell, so the sites updated in a round
// never share a word and need no atomics; the per-site rule of PQSyncRng
// (kpz/kpzSimulationPrimitivesTemplates.cu:229-268).
//
// Geometry: 32x16 threads, thread cells of 8x8 sites (2x2 words), blocks of 256x128 sites
// (64x32 words), shared tile 65x33 words, 64 rounds per launch (one attempt per site per
// MCS).  All random numbers come from the counter stream (see oracle/kpz_oracle.h), so the
// CPU emulations ko_dt_mcs* reproduce every lattice bit for bit.
//
// The same kernel, with the reference's other block-level decompositions (KPZ_INNER_DD,
// kpz/kpzConst.h:26-35) as a template parameter: DTDBSH, DB, DBSH (the reference's default)
// and DBSHRep; and the reference's DB4 scheduler (Kpz::Scheduler<Rng, LocalLayoutDB4>,
// kpz/scheduler.cu:37-52, kpz/kpz.cu:95-117): per MCS two launches over every block from a
// random origin in [0, block), no halo, sites within 5 of the block's far edges dead, 32
// BaseDT rounds per launch (kpz/kpzSimulationPrimitivesTemplates.cu:74-103).
#include <cmath>
#include <type_traits>
#include <cstring>

#include "kpzb_api_internal.h"
#include "kpzb_common.cuh"
#include "kpzb_internal.h"

namespace kpzb {

constexpr uint32_t TAG_DT_SUB = 4u;
constexpr uint32_t TAG_DT_POS = 5u;
constexpr uint32_t TAG_DBSH_ORIGIN = 7u;
constexpr uint32_t TAG_DBSH_POS = 8u;
constexpr uint32_t TAG_REP_ORIGIN = 9u;
constexpr uint32_t TAG_REP_POS = 10u;
constexpr uint32_t TAG_REP_U = 11u;
constexpr uint32_t TAG_DB4_ORIGIN = 12u;
constexpr uint32_t TAG_DB4_SUB = 13u;
constexpr uint32_t TAG_DB4_POS = 14u;
constexpr uint32_t TAG_DB4_U = 15u;
constexpr int DT_TX = 32, DT_TY = 16;
constexpr int DT_THREADS = DT_TX * DT_TY;
constexpr int DT_BXW = 64, DT_BYW = 32;           // block in words
constexpr int DT_BX = 4 * DT_BXW, DT_BY = 4 * DT_BYW;  // block in sites
constexpr int DT_TW = DT_BXW + 1, DT_TH = DT_BYW + 1;  // shared tile with halo
constexpr int DT_ROUNDS = 64;
// DB4: sites of a block whose x >= 251 or y >= 123 (before the origin's offset inside a word)
// are dead, so no update reaches past the block (LocalLayoutDB4::BLOCK_BORDER_WIDTH = 5,
// kpz/LocalLayout.h:120-131)
constexpr int DB4_BORDER = 5;

__device__ __forceinline__ uint32_t pick4(const uint4& v, int i)
{
    return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

// The rule's candidates and acceptance limits for the plain rates: a site of configuration
// cfg_p (12, or an impossible 16 when p = 0) flips when its acceptance word u <= lim_p =
// T_p - 1; likewise cfg_q (3).
struct DtRule {
    uint32_t cfg_p, cfg_q, lim_p, lim_q;
};

// One attempt of the random-sequential rule (PQSyncRng::update,
// kpz/kpzSimulationPrimitivesTemplates.cu:250-281) at the site of table entry e (pack_entry_bytes)
// relative to the byte bases tb (lattice tile) and db (disorder tile): the entry gives the
// byte offsets of the site's word, its right neighbour's and its lower neighbour's, and the
// rotate amounts (used modulo 32) that bring the site's two slope bits to bits 0-1, the right
// neighbour's x-slope bit to bit 2 and the lower neighbour's y-slope bit to bit 3.
template <bool COUNT, bool DIS>
__device__ __forceinline__ void dt_attempt_at(char* tb, const char* db, uint2 e, uint32_t u, const DtRule rule,
                                              const DisorderRates& dr, unsigned long long& ndep,
                                              unsigned long long& ndes)
{
    uint32_t* pw = reinterpret_cast<uint32_t*>(tb + (e.x & 0xFFFFu));
    uint32_t* pr = reinterpret_cast<uint32_t*>(tb + (e.x >> 16));
    uint32_t* pd = reinterpret_cast<uint32_t*>(tb + (e.y & 2047u));
    const uint32_t r1 = e.y >> 11, r2 = e.y >> 16, r3 = e.y >> 21;
    const uint32_t cw = *pw, rw = *pr, dw = *pd;
    // configuration c | s_x(x+1)<<2 | s_y(y+1)<<3 (kpz/kpzSimulationPrimitivesTemplates.cu:
    // 258-260): three rotations, one mask each
    const uint32_t cfg = (__funnelshift_r(cw, cw, r1) & 3u) | (__funnelshift_r(rw, rw, r2) & 4u) |
                         (__funnelshift_r(dw, dw, r3) & 8u);
    bool flip, is_p;
    if (DIS) {
        is_p = cfg == 12u;
        flip = false;
        if (is_p || cfg == 3u) {
            const uint32_t dw0 = *reinterpret_cast<const uint32_t*>(db + (e.x & 0xFFFFu));
            const int cls = (int)(__funnelshift_r(dw0, dw0, r1) & 3u);
            const Thresh& th = is_p ? dr.tp[cls] : dr.tq[cls];
            flip = th.always || (th.planes && u < th.t);
        }
    } else {
        is_p = cfg == rule.cfg_p;
        flip = (is_p || cfg == rule.cfg_q) && u <= (is_p ? rule.lim_p : rule.lim_q);
    }
    if (flip) {
        // shared atomics: under the single-hit schemes only this thread touches these words in
        // this round (the atomics merely order its own three flips when two share a word);
        // under the dead-border schemes other threads' flips of the same phase may share them
        // (the reference's fctAtomicXor)
        atomicXor(pw, __funnelshift_l(3u, 3u, r1));
        atomicXor(pr, __funnelshift_l(4u, 4u, r2));
        atomicXor(pd, __funnelshift_l(8u, 8u, r3));
        if (COUNT) {
            if (is_p) ++ndep;
            else ++ndes;
        }
    }
}

// Site-table entry of the site (vx, vy) sites right of and below a word (a thread cell's first
// word, or the tile's): the tile words of the site, its right neighbour and its lower neighbour
// relative to that word, and the rotate amounts
//   bits 0-7: the site's shift sh (its two slope bits rotate down to bits 0-1),
//   8-15: (shr - 2) mod 32 (the right neighbour's x-slope bit rotates to bit 2),
//   16-23: (shd - 3) mod 32 (the lower neighbour's y-slope bit rotates to bit 3);
// a funnel shift uses its amount modulo 32, so no field needs a mask.
__device__ __forceinline__ uint4 site_entry(int vx, int vy)
{
    const uint32_t sh = (uint32_t)(((vx & 3) << 1) | ((vy & 3) << 3));
    const uint32_t shr = (uint32_t)((((vx + 1) & 3) << 1) | ((vy & 3) << 3));
    const uint32_t shd = (uint32_t)(((vx & 3) << 1) | (((vy + 1) & 3) << 3) | 1);
    return make_uint4((uint32_t)((vy >> 2) * DT_TW + (vx >> 2)), (uint32_t)((vy >> 2) * DT_TW + ((vx + 1) >> 2)),
                      (uint32_t)(((vy + 1) >> 2) * DT_TW + (vx >> 2)),
                      sh | (((shr - 2u) & 31u) << 8) | (((shd - 3u) & 31u) << 16));
}
constexpr int DT_VSPAN = 18;  // in-cell offsets of the shifted schemes: up to 3 + 7 + 7 (or 4 + 3 + 7 + 3)
// Row stride of the DTDBSH table: a round's 16 entries (4 x 4 in-cell offsets around one
// corner) then lie in 32 distinct banks, 8 bytes each
constexpr int DT_VROW = 20;

// An 8-byte table entry in shared memory, with byte offsets so that an address is one add to
// a byte base: x = 4 w | 4 w_right << 16, y = 4 w_down | sh << 11 | (shr - 2) << 16 |
// (shd - 3) << 21 (the rotate amounts of site_entry, each read by shifting y right and used
// modulo 32); bits 26-27 are left for flags.
__device__ __forceinline__ uint2 pack_entry_bytes(const uint4 e)
{
    return make_uint2((4u * e.x) | ((4u * e.y) << 16),
                      (4u * e.z) | ((e.w & 31u) << 11) | (((e.w >> 8) & 31u) << 16) | (((e.w >> 16) & 31u) << 21));
}

// DIS: quenched disorder (Disorder2SyncRng_shared, kpz/kpzSimulationPrimitivesTemplates.cu:
// 295-382): dis holds every site's 2-bit rate class in ENC_LOCAL words, copied into a second
// shared tile beside the lattice's; the class picks dr.tp[c] / dr.tq[c].
// SCHEME (the reference's KPZ_INNER_DD, kpz/kpzConst.h:26-35, plus its DB4 scheduler):
//   DT_SCHEME_DT      single-hit double tiling (BaseDT)
//   DT_SCHEME_DTDBSH  the same with a block-wide random offset of the thread cells per round
//   DT_SCHEME_DBSH    single-hit dead border, borders delayed to later phases of the round
//   DT_SCHEME_DB      the dead-border phases without the per-round cell offset
//   DT_SCHEME_DBSHREP DBSH with the border hits replaced by fresh attempts after the rounds
//   DT_SCHEME_DB4     every block of the lattice in one launch, a dead border of 5 sites, the
//                     inner rounds of BaseDT (32 per launch, two launches per MCS)
template <bool COUNT, bool DIS, int SCHEME>
__global__ void __launch_bounds__(DT_THREADS, 4)
dt_kernel(uint32_t* __restrict__ sys, int lxw, int lyw, int lnbx, int nblocks, int ox, int oy,
          int d, uint32_t t, Key key, uint32_t stream, Thresh tp, Thresh tq,
          unsigned long long* __restrict__ counters, const uint32_t* __restrict__ dis, DisorderRates dr)
{
    constexpr bool DB4 = SCHEME == DT_SCHEME_DB4;
    constexpr bool SHIFTED = SCHEME == DT_SCHEME_DTDBSH;
    constexpr bool REP = SCHEME == DT_SCHEME_DBSHREP;
    constexpr bool BORDER = SCHEME == DT_SCHEME_DBSH || SCHEME == DT_SCHEME_DB || REP;
    // DT and DB4 index a 64-entry table by (quadrant, position): the origin's offset inside a
    // word (ox & 3, oy & 3) is the launch's, so it is folded in.  The schemes that shift the
    // cells per round (DTDBSH and the dead-border schemes) index an 18 x 18 table by the
    // in-cell offset instead.
    constexpr int NLUT = (SHIFTED || BORDER) ? DT_VSPAN * DT_VROW : 64;
    constexpr int ROUNDS = DB4 ? DT_ROUNDS / 2 : DT_ROUNDS;
    constexpr uint32_t T_SUB = DB4 ? TAG_DB4_SUB : TAG_DT_SUB;
    constexpr uint32_t T_POS = DB4 ? TAG_DB4_POS : TAG_DT_POS;
    constexpr uint32_t T_U = DB4 ? TAG_DB4_U : TAG_DT;
    __shared__ uint32_t tile[DT_TH * DT_TW];
    __shared__ uint32_t dtile[DIS ? DT_TH * DT_TW : 1];
    __shared__ uint32_t rep_hits[REP ? DT_THREADS / 32 + 1 : 1];
    __shared__ uint2 lut[NLUT];
    const int tid = threadIdx.y * DT_TX + threadIdx.x;
    const uint32_t Wx = 1u << lxw, Wy = 1u << lyw;
    const int ax = ox & 3, ay = oy & 3;
    bool need_u = !(tp.always || tp.planes == 0) || !(tq.always || tq.planes == 0);
    if (DIS) need_u = dr.planes > 0;
    // the rule's candidates and acceptance limits: a site with configuration cfg_p (12, or an
    // impossible 16 when p = 0) flips when u <= lim_p = T_p - 1; likewise q (configuration 3)
    const uint32_t cfg_p = (tp.always || tp.planes) ? 12u : 16u, cfg_q = (tq.always || tq.planes) ? 3u : 16u;
    const uint32_t lim_p = tp.always ? 0xFFFFFFFFu : tp.t - 1u, lim_q = tq.always ? 0xFFFFFFFFu : tq.t - 1u;
    const DtRule rule{cfg_p, cfg_q, lim_p, lim_q};
    unsigned long long ndep = 0, ndes = 0;
    if (NLUT == 64) {
        if (tid < 64) {
            // bits 25 / 26 of y: the site lies at in-cell x / y >= 3, DB4's dead border when the cell
            // is the block's last in its row / column (it starts 8 sites before the block's edge)
            const int sc = tid >> 4, pb = tid & 15;
            const int ux = 4 * (sc & 1) + (pb & 3), uy = 4 * (sc >> 1) + (pb >> 2);
            uint2 e = pack_entry_bytes(site_entry(ux + ax, uy + ay));
            e.y |= (ux >= 8 - DB4_BORDER ? 1u << 26 : 0u) | (uy >= 8 - DB4_BORDER ? 1u << 27 : 0u);
            lut[tid] = e;
        }
    } else {
        for (int i = tid; i < NLUT; i += DT_THREADS) lut[i] = pack_entry_bytes(site_entry(i % DT_VROW, i / DT_VROW));
    }
    // DB4: the last thread column / row owns the block's dead border
    const uint32_t dead_mask = (threadIdx.x == DT_TX - 1 ? 1u << 26 : 0u) | (threadIdx.y == DT_TY - 1 ? 1u << 27 : 0u);
    const int tbase = 2 * threadIdx.y * DT_TW + 2 * threadIdx.x;
    // the thread cell's first word in the tiles, as byte pointers for the DT / DB4 table
    char* tcell = reinterpret_cast<char*>(tile + tbase);
    const char* dcell = reinterpret_cast<const char*>(dtile + (DIS ? tbase : 0));
    // a shifted cell whose site passes the block's right / lower edge wraps to its left / upper
    // edge (the reference masks coordinates with M_BLOCK_DIM): the cell's words move back by
    // a block's width / height
    auto wrapped_base = [&](int ex, int ey) {
        return tbase - (threadIdx.x * 8 + ex >= DT_BX ? DT_BXW : 0) - (threadIdx.y * 8 + ey >= DT_BY ? DT_BYW * DT_TW : 0);
    };

    for (int b = blockIdx.x; b < nblocks; b += gridDim.x) {
        const int bx = b & ((1 << lnbx) - 1), by = b >> lnbx;
        const uint32_t X0 = (uint32_t)ox + (uint32_t)(DB4 ? bx : 2 * bx + (d & 1)) * DT_BX;
        const uint32_t Y0 = (uint32_t)oy + (uint32_t)(DB4 ? by : 2 * by + (d >> 1)) * DT_BY;
        const uint32_t wx0 = X0 >> 2, wy0 = Y0 >> 2;
        for (int i = tid; i < DT_TH * DT_TW; i += DT_THREADS) {
            const uint32_t r = i / DT_TW, c = i - r * DT_TW;
            // DB4 blocks tile the lattice without halo: the dead border keeps every update,
            // its right and its lower neighbour inside the block's 64x32 words
            if (DB4 && (r == DT_BYW || c == DT_BXW)) continue;
            const size_t gi = (size_t)((wy0 + r) & (Wy - 1)) * Wx + ((wx0 + c) & (Wx - 1));
            tile[i] = sys[gi];
            if (DIS) dtile[i] = dis[gi];
        }
        // block-wide sub-cell sequence: 2 bits per round (every thread derives the same words)
        const uint4 sub = philox4x32_10(
            make_uint4((uint32_t)b, t, (T_SUB << 24) | ((uint32_t)d << 16), stream), key);
        const uint32_t cid = (uint32_t)b * DT_THREADS + (uint32_t)tid;
        __syncthreads();
        uint4 pos = make_uint4(0, 0, 0, 0), uu = make_uint4(0, 0, 0, 0), ow = make_uint4(0, 0, 0, 0);
        if (BORDER) {
            // the reference's default inner scheme (BaseDTInnerDBSH::systemLoopDC,
            // kpz/kpzSimulationPrimitivesTemplates_BaseInnerDB.cu:110-163): per round one
            // block-wide offset shifts every thread cell, each thread picks a site of its shifted
            // cell, and sites on a cell's last column/row wait for phases 1 (off the corner) and
            // 2 (the corner); the flips use shared-memory atomics as the reference's do.  The
            // site's words and rotations are found once per round, before the phases.
            // REP (BaseDTInnerDBSHRep, :175-268): a border hit is not done in its round but
            // counted, and after the 64 rounds the block makes that many fresh attempts, 512 per
            // repetition round, each again in the three phases.
            uint32_t hits = 0;
            for (int rb = 0; rb < DT_ROUNDS; rb += 16) {
                ow = philox4x32_10(
                    make_uint4((uint32_t)b, t, (TAG_DBSH_ORIGIN << 24) | ((uint32_t)d << 16) | (uint32_t)(rb >> 4),
                               stream), key);
                const uint4 pw = philox4x32_10(
                    make_uint4(cid, t, (TAG_DBSH_POS << 24) | ((uint32_t)d << 16) | (uint32_t)(rb >> 4), stream),
                    key);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int r = rb + j;
                    if (need_u && (j & 3) == 0)
                        uu = philox4x32_10(
                            make_uint4(cid, t, (TAG_DT << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 2), stream), key);
                    const uint32_t ob = (pick4(ow, j >> 2) >> (8 * (j & 3))) & 0xFFu;
                    const uint32_t pb = (pick4(pw, j >> 2) >> (8 * (j & 3))) & 0xFFu;
                    const int px = (int)(pb & 7u), py = (int)((pb >> 3) & 7u);
                    const int ph = (px == 7 && py == 7) ? 2 : (px == 7 || py == 7) ? 1 : 0;
                    // the site at in-cell offset (vx, vy) from the cell's first word; the table gives
                    // its words and rotations, once per round, before the phases
                    const int vx = ax + px + (SCHEME == DT_SCHEME_DB ? 0 : (int)(ob & 7u));
                    const int vy = ay + py + (SCHEME == DT_SCHEME_DB ? 0 : (int)((ob >> 3) & 7u));
                    const uint2 e = lut[vy * DT_VROW + vx];
                    const int base = wrapped_base(vx, vy);
                    char* tb = reinterpret_cast<char*>(tile + base);
                    const char* db = reinterpret_cast<const char*>(dtile + (DIS ? base : 0));
                    const uint32_t u = pick4(uu, j & 3);
                    if (REP) {
                        if (ph == 0) dt_attempt_at<COUNT, DIS>(tb, db, e, u, rule, dr, ndep, ndes);
                        else ++hits;
                        __syncthreads();
                    } else {
                        for (int phase = 0; phase < 3; ++phase) {
                            if (ph == phase) dt_attempt_at<COUNT, DIS>(tb, db, e, u, rule, dr, ndep, ndes);
                            __syncthreads();
                        }
                    }
                }
            }
            if (REP) {
                // The block's count as the reference's reduction forms it (:214-227): thread 0's
                // own hits plus the warp sums of warps 1.. -- the hits of warp 0's lanes 1-31 are
                // not repeated there, nor here.
                uint32_t ws = hits;
                for (int o = 16; o > 0; o >>= 1) ws += __shfl_xor_sync(0xffffffffu, ws, o);
                if ((tid & 31) == 0) rep_hits[1 + (tid >> 5)] = ws;
                if (tid == 0) rep_hits[0] = hits;
                __syncthreads();
                uint32_t total = rep_hits[0];
                for (int w = 1; w < DT_THREADS / 32; ++w) total += rep_hits[1 + w];
                // repetition rounds in groups of 16, unrolled like the main rounds (the offset and
                // position words serve 16 rounds, the acceptance words 4)
                for (int kb = 0; kb * DT_THREADS < (int)total; kb += 16) {
                    ow = philox4x32_10(make_uint4((uint32_t)b, t,
                                                  (TAG_REP_ORIGIN << 24) | ((uint32_t)d << 16) | (uint32_t)(kb >> 4),
                                                  stream), key);
                    const uint4 rpw = philox4x32_10(
                        make_uint4(cid, t, (TAG_REP_POS << 24) | ((uint32_t)d << 16) | (uint32_t)(kb >> 4), stream),
                        key);
                    uint4 ruu = make_uint4(0, 0, 0, 0);
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int k = kb + j;
                        if (k * DT_THREADS >= (int)total) break;
                        const bool active = k * DT_THREADS + tid < (int)total;
                        if (need_u && (j & 3) == 0)
                            ruu = philox4x32_10(
                                make_uint4(cid, t, (TAG_REP_U << 24) | ((uint32_t)d << 16) | (uint32_t)(k >> 2), stream),
                                key);
                        const uint32_t ob = (pick4(ow, j >> 2) >> (8 * (j & 3))) & 0xFFu;
                        const uint32_t pb = (pick4(rpw, j >> 2) >> (8 * (j & 3))) & 0xFFu;
                        const int px = (int)(pb & 7u), py = (int)((pb >> 3) & 7u);
                        const int ph = !active ? 3 : (px == 7 && py == 7) ? 2 : (px == 7 || py == 7) ? 1 : 0;
                        const int vx = ax + px + (int)(ob & 7u), vy = ay + py + (int)((ob >> 3) & 7u);
                        const uint2 e = lut[vy * DT_VROW + vx];
                        const int base = wrapped_base(vx, vy);
                        char* tb = reinterpret_cast<char*>(tile + base);
                        const char* db = reinterpret_cast<const char*>(dtile + (DIS ? base : 0));
                        const uint32_t u = pick4(ruu, j & 3);
                        for (int phase = 0; phase < 3; ++phase) {
                            if (ph == phase) dt_attempt_at<COUNT, DIS>(tb, db, e, u, rule, dr, ndep, ndes);
                            __syncthreads();
                        }
                    }
                }
            }
        }
#pragma unroll 4
        for (int rb = 0; rb < (BORDER ? 0 : ROUNDS); rb += 8) {
            if ((rb & 31) == 0)
                pos = philox4x32_10(
                    make_uint4(cid, t, (T_POS << 24) | ((uint32_t)d << 16) | (uint32_t)(rb >> 5), stream), key);
            if (SHIFTED && (rb & 15) == 0)
                ow = philox4x32_10(
                    make_uint4((uint32_t)b, t, (TAG_DBSH_ORIGIN << 24) | ((uint32_t)d << 16) | (uint32_t)(rb >> 4),
                               stream), key);
            const uint32_t sw = pick4(sub, rb >> 4);
            const uint32_t pw = pick4(pos, (rb & 31) >> 3);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int r = rb + j;
                if (need_u && (j & 3) == 0)
                    uu = philox4x32_10(
                        make_uint4(cid, t, (T_U << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 2), stream), key);
                const uint32_t sc = (sw >> (2 * (r & 15))) & 3u;
                const uint32_t pb = (pw >> (4 * j)) & 15u;
                const uint32_t u = pick4(uu, j & 3);
                if (SHIFTED) {
                    // BaseDTInnerDTDBSH (kpz/kpzSimulationPrimitivesTemplates_BaseInnerDTr.cu:
                    // 30-85): the quadrant and a block-wide offset in [0,8)^2 per round, the
                    // site wrapped inside the block before the origin's in-word offset is added;
                    // neighbouring threads' sites stay 4 or more sites apart, so no two share a word
                    const uint32_t ob = (pick4(ow, (r & 15) >> 2) >> (8 * (r & 3))) & 0xFFu;
                    const int ux = 4 * (int)(sc & 1u) + (int)(pb & 3u) + (int)(ob & 7u);
                    const int uy = 2 * (int)(sc & 2u) + (int)(pb >> 2) + (int)((ob >> 3) & 7u);
                    const uint2 e = lut[(uy + ay) * DT_VROW + ux + ax];
                    const int base = wrapped_base(ux, uy);
                    dt_attempt_at<COUNT, DIS>(reinterpret_cast<char*>(tile + base),
                                              reinterpret_cast<const char*>(dtile + (DIS ? base : 0)), e, u, rule, dr,
                                              ndep, ndes);
                } else {
                    const uint2 e = lut[sc * 16u + pb];
                    if (!DB4 || (e.y & dead_mask) == 0u) {
                        uint32_t* pw = reinterpret_cast<uint32_t*>(tcell + (e.x & 0xFFFFu));
                        uint32_t* pr = reinterpret_cast<uint32_t*>(tcell + (e.x >> 16));
                        uint32_t* pd = reinterpret_cast<uint32_t*>(tcell + (e.y & 2047u));
                        const uint32_t r1 = e.y >> 11, r2 = e.y >> 16, r3 = e.y >> 21;
                        const uint32_t cw = *pw, rw = *pr, dw = *pd;
                        const uint32_t cfg = (__funnelshift_r(cw, cw, r1) & 3u) | (__funnelshift_r(rw, rw, r2) & 4u) |
                                             (__funnelshift_r(dw, dw, r3) & 8u);
                        bool flip, is_p;
                        if (DIS) {
                            is_p = cfg == 12u;
                            flip = false;
                            if (is_p || cfg == 3u) {
                                const uint32_t dw0 = *reinterpret_cast<const uint32_t*>(dcell + (e.x & 0xFFFFu));
                                const int cls = (int)(__funnelshift_r(dw0, dw0, r1) & 3u);
                                const Thresh& th = is_p ? dr.tp[cls] : dr.tq[cls];
                                flip = th.always || (th.planes && u < th.t);
                            }
                        } else {
                            is_p = cfg == cfg_p;
                            flip = (is_p || cfg == cfg_q) && u <= (is_p ? lim_p : lim_q);
                        }
                        if (flip) {
                            atomicXor(pw, __funnelshift_l(3u, 3u, r1));
                            atomicXor(pr, __funnelshift_l(4u, 4u, r2));
                            atomicXor(pd, __funnelshift_l(8u, 8u, r3));
                            if (COUNT) {
                                if (is_p) ++ndep;
                                else ++ndes;
                            }
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (int i = tid; i < DT_TH * DT_TW; i += DT_THREADS) {
            const uint32_t r = i / DT_TW, c = i - r * DT_TW;
            if (DB4 && (r == DT_BYW || c == DT_BXW)) continue;
            sys[(size_t)((wy0 + r) & (Wy - 1)) * Wx + ((wx0 + c) & (Wx - 1))] = tile[i];
        }
        __syncthreads();
    }
    if (COUNT) {
        for (int o = 16; o > 0; o >>= 1) {
            ndep += __shfl_xor_sync(0xffffffffu, ndep, o);
            ndes += __shfl_xor_sync(0xffffffffu, ndes, o);
        }
        if ((tid & 31) == 0 && (ndep | ndes)) {
            atomicAdd(&counters[0], ndep);
            atomicAdd(&counters[1], ndes);
        }
    }
}

// Host copy of the Philox4x32-10 bijection for the per-MCS origin and domain-set order (and
// the random measurement spacing of kpzb_sample_times).
void philox_host(const uint32_t ctr[4], uint64_t seed, uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0;
        c1 = (uint32_t)p1;
        c2 = n2;
        c3 = (uint32_t)p0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

// Origin in [0, 2*block) sites and the Kmc::Shuffle<4> order (inc/shuffle.h:76-90).
static void dt_plan(uint64_t seed, uint32_t stream, uint32_t t, int* ox, int* oy, int order[4])
{
    const uint32_t ctr[4] = {0u, t, TAG_DT_ORIGIN << 24, stream};
    uint32_t r[4];
    philox_host(ctr, seed, r);
    *ox = (int)(r[0] & (uint32_t)(2 * DT_BX - 1));
    *oy = (int)(r[1] & (uint32_t)(2 * DT_BY - 1));
    uint32_t rnd = r[2];
    for (int a = 0; a < 4; ++a) order[a] = a;
    for (int a = 0; a < 4; ++a) {
        const int i = (int)(rnd & 3u);
        const int v = order[i];
        order[i] = order[a];
        order[a] = v;
        rnd >>= 2;
    }
}

kpzb_status dt_init(DtState* s, int lx, int ly, int sm_count, bool db4)
{
    if (db4 && (lx < 8 || ly < 7)) return fail(KPZB_EINVAL, "DB4 needs lx >= 8 and ly >= 7 (one 256x128 block)");
    if (!db4 && (lx < 9 || ly < 8))
        return fail(KPZB_EINVAL, "DT needs lx >= 9 and ly >= 8 (one 512x256 double tile)");
    const int nblocks = db4 ? (1 << (lx - 8)) * (1 << (ly - 7)) : (1 << (lx - 9)) * (1 << (ly - 8));
    // 2048 threads per SM / 512 per CTA: 4 resident CTAs per SM
    s->grid = nblocks < sm_count * 4 ? nblocks : sm_count * 4;
    if (db4) s->scheme = DT_SCHEME_DB4;
    s->ready = true;
    return KPZB_OK;
}

void dt_free(DtState* s) { s->ready = false; }

static uint64_t thresh_dt(double p)
{
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return 1ull << 32;
    const double t = std::ceil(p * 4294967296.0);
    return t >= 4294967296.0 ? (1ull << 32) : (uint64_t)t;
}

kpzb_status dt_enqueue(DtState* s, uint32_t* d_local, int lx, int ly, uint64_t t0, int n, double p,
                       double q, uint64_t seed, uint32_t stream, cudaStream_t st,
                       unsigned long long* d_counters, const uint32_t* dis, const uint64_t* dis_Tp,
                       const uint64_t* dis_Tq)
{
    if (!s->ready) return fail(KPZB_ESTATE, "DT state not initialised");
    const Key key = make_key(seed);
    const Thresh tp = make_thresh(thresh_dt(p)), tq = make_thresh(thresh_dt(q));
    const bool db4 = s->scheme == DT_SCHEME_DB4;
    const int lnbx = db4 ? lx - 8 : lx - 9;
    const int nblocks = (1 << lnbx) * (1 << (db4 ? ly - 7 : ly - 8));
    const dim3 block(DT_TX, DT_TY);
    const DisorderRates dr = dis ? make_disorder_rates(dis_Tp, dis_Tq) : DisorderRates{};
    const bool c = d_counters != nullptr, ds = dis != nullptr;
    auto launch = [&](int ox, int oy, int d, uint32_t t) {
        auto go = [&](auto kern) {
            kern<<<s->grid, block, 0, st>>>(d_local, lx - 2, ly - 2, lnbx, nblocks, ox, oy, d, t, key, stream, tp,
                                             tq, d_counters, dis, dr);
        };
        auto pick = [&](auto scheme_tag) {
            constexpr int S = decltype(scheme_tag)::value;
            if (c && ds) go(dt_kernel<true, true, S>);
            else if (c) go(dt_kernel<true, false, S>);
            else if (ds) go(dt_kernel<false, true, S>);
            else go(dt_kernel<false, false, S>);
        };
        switch (s->scheme) {
        case DT_SCHEME_DBSH: pick(std::integral_constant<int, DT_SCHEME_DBSH>{}); break;
        case DT_SCHEME_DB: pick(std::integral_constant<int, DT_SCHEME_DB>{}); break;
        case DT_SCHEME_DTDBSH: pick(std::integral_constant<int, DT_SCHEME_DTDBSH>{}); break;
        case DT_SCHEME_DBSHREP: pick(std::integral_constant<int, DT_SCHEME_DBSHREP>{}); break;
        case DT_SCHEME_DB4: pick(std::integral_constant<int, DT_SCHEME_DB4>{}); break;
        default: pick(std::integral_constant<int, DT_SCHEME_DT>{}); break;
        }
    };
    for (int i = 0; i < n; ++i) {
        const uint32_t t = (uint32_t)(t0 + (uint64_t)i);
        if (db4) {
            // Scheduler::doMcs (kpz/scheduler.cu:37-52): 2^L_MCS_DIV = 2 launches per MCS, each
            // over every block from a random origin in [0, block) sites
            for (int a = 0; a < 2; ++a) {
                const uint32_t ctr[4] = {(uint32_t)a, t, TAG_DB4_ORIGIN << 24, stream};
                uint32_t r[4];
                philox_host(ctr, seed, r);
                launch((int)(r[0] & (uint32_t)(DT_BX - 1)), (int)(r[1] & (uint32_t)(DT_BY - 1)), a, t);
            }
        } else {
            int ox, oy, order[4];
            dt_plan(seed, stream, t, &ox, &oy, order);
            for (int a = 0; a < 4; ++a) launch(ox, oy, order[a], t);
        }
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "dt_kernel");
    }
    return KPZB_OK;
}

}  // namespace kpzb
