// kpzb_common.cuh -- device helpers shared by the kpzb kernels (sm_100a).
//
// Counter-based random stream (the one the CPU oracle restates):
//   Philox4x32-10 (Salmon et al., SC'11), key = (seed lo, seed hi),
//   counter = (qword >> 2, step, plane | tag << 8, stream); output word qword & 3.
//   qword: word index inside an ENC_CBBIT quadrant; step = 2*t + sublattice;
//   plane k supplies bit (31-k) of each site's 32-bit uniform u.
// Decision: local minimum flips iff u < T(p), local maximum iff u < T(q),
//   T(x) = min(2^32, ceil(x * 2^32)).  Evaluated bit-serially from the MSB
//   plane, 32 sites per word at once, stopping when no site is undecided.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace kpzb {

constexpr uint32_t TAG_SCA = 1u;
constexpr uint32_t TAG_DT = 2u;
constexpr uint32_t TAG_DT_ORIGIN = 3u;

struct Key {
    uint32_t k0, k1;
};

__host__ __device__ __forceinline__ Key make_key(uint64_t seed)
{
    return Key{(uint32_t)seed, (uint32_t)(seed >> 32)};
}

// Philox4x32-10 round function and Weyl key schedule (SC'11, sec. 3.2).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, Key k)
{
    uint32_t k0 = k.k0, k1 = k.k1;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint32_t lo0 = 0xD2511F53u * c.x;
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
    }
    return c;
}

// Threshold as (flag, low 32 bits): always = T >= 2^32; never = T == 0;
// planes = number of MSB planes that can decide (32 - ctz(T)).
struct Thresh {
    uint32_t t;      // low 32 bits of T (T < 2^32 when !always)
    int planes;      // 0 when always or never
    bool always;
};

__host__ __device__ inline Thresh make_thresh(uint64_t T)
{
    Thresh r;
    r.always = T >= (1ull << 32);
    r.t = r.always ? 0u : (uint32_t)T;
    int planes = 0;
    if (!r.always && r.t) {
        uint32_t v = r.t;
        int ctz = 0;
        while (!(v & 1u)) {
            v >>= 1;
            ++ctz;
        }
        planes = 32 - ctz;
    }
    r.planes = planes;
    return r;
}

// Four-word decision for the 128 sites of one Philox group (qgroup = qword >> 2).
// cp: local-minimum candidates, cq: local-maximum candidates. Returns the flip mask.
__device__ __forceinline__ uint4 decide4(uint4 cp, uint4 cq, Thresh tp, Thresh tq, Key key,
                                         uint32_t qgroup, uint32_t step, uint32_t stream)
{
    uint4 ltp, eqp, ltq, eqq;
    if (tp.always) {
        ltp = cp;
        eqp = make_uint4(0, 0, 0, 0);
    } else {
        ltp = make_uint4(0, 0, 0, 0);
        eqp = tp.planes ? cp : make_uint4(0, 0, 0, 0);
    }
    if (tq.always) {
        ltq = cq;
        eqq = make_uint4(0, 0, 0, 0);
    } else {
        ltq = make_uint4(0, 0, 0, 0);
        eqq = tq.planes ? cq : make_uint4(0, 0, 0, 0);
    }
    const int kmax = max(tp.planes, tq.planes);
    for (int k = 0; k < kmax; ++k) {
        const uint32_t any = eqp.x | eqp.y | eqp.z | eqp.w | eqq.x | eqq.y | eqq.z | eqq.w;
        if (!any) break;
        const uint4 r = philox4x32_10(make_uint4(qgroup, step, (uint32_t)k | (TAG_SCA << 8), stream), key);
        const uint32_t bp = (tp.t >> (31 - k)) & 1u;
        const uint32_t bq = (tq.t >> (31 - k)) & 1u;
        // bit of T is 1: sites with u-bit 0 are below T (decided), u-bit 1 stay equal.
        // bit of T is 0: sites with u-bit 1 are above T (drop), u-bit 0 stay equal.
        if (bp) {
            ltp.x |= eqp.x & ~r.x; ltp.y |= eqp.y & ~r.y; ltp.z |= eqp.z & ~r.z; ltp.w |= eqp.w & ~r.w;
            eqp.x &= r.x; eqp.y &= r.y; eqp.z &= r.z; eqp.w &= r.w;
        } else {
            eqp.x &= ~r.x; eqp.y &= ~r.y; eqp.z &= ~r.z; eqp.w &= ~r.w;
        }
        if (bq) {
            ltq.x |= eqq.x & ~r.x; ltq.y |= eqq.y & ~r.y; ltq.z |= eqq.z & ~r.z; ltq.w |= eqq.w & ~r.w;
            eqq.x &= r.x; eqq.y &= r.y; eqq.z &= r.z; eqq.w &= r.w;
        } else {
            eqq.x &= ~r.x; eqq.y &= ~r.y; eqq.z &= ~r.z; eqq.w &= ~r.w;
        }
        if (k + 1 >= tp.planes) eqp = make_uint4(0, 0, 0, 0);
        if (k + 1 >= tq.planes) eqq = make_uint4(0, 0, 0, 0);
    }
    return make_uint4(ltp.x | ltq.x, ltp.y | ltq.y, ltp.z | ltq.z, ltp.w | ltq.w);
}

// Decision modes, chosen once per launch from the two thresholds:
//   DEC_NONE   no random plane can matter (every threshold is 0 or 2^32),
//   DEC_ONE    at most the MSB plane matters (thresholds in {0, 2^31, 2^32}, e.g. p = 1/2),
//   DEC_GENERAL anything else (bit-serial loop of decide4).
enum DecMode { DEC_NONE = 0, DEC_ONE = 1, DEC_GENERAL = 2 };

__host__ __device__ inline int dec_mode(Thresh tp, Thresh tq)
{
    const int m = tp.planes > tq.planes ? tp.planes : tq.planes;
    return m == 0 ? DEC_NONE : m == 1 ? DEC_ONE : DEC_GENERAL;
}

// decide4 with the cheap modes spelled out; identical results in every mode.
__device__ __forceinline__ uint4 decide4_mode(int mode, uint4 cp, uint4 cq, Thresh tp, Thresh tq,
                                              Key key, uint32_t qgroup, uint32_t step,
                                              uint32_t stream)
{
    if (mode == DEC_NONE) {
        const uint32_t ap = tp.always ? 0xFFFFFFFFu : 0u, aq = tq.always ? 0xFFFFFFFFu : 0u;
        return make_uint4((cp.x & ap) | (cq.x & aq), (cp.y & ap) | (cq.y & aq),
                          (cp.z & ap) | (cq.z & aq), (cp.w & ap) | (cq.w & aq));
    }
    if (mode == DEC_ONE) {
        // a threshold with one plane is 2^31: sites whose MSB of u is 0 flip
        const uint32_t any = cp.x | cp.y | cp.z | cp.w | cq.x | cq.y | cq.z | cq.w;
        uint4 r = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
        if (any) r = philox4x32_10(make_uint4(qgroup, step, TAG_SCA << 8, stream), key);
        const uint32_t ap = tp.always ? 0xFFFFFFFFu : 0u, aq = tq.always ? 0xFFFFFFFFu : 0u;
        const uint32_t hp = tp.planes ? 0xFFFFFFFFu : 0u, hq = tq.planes ? 0xFFFFFFFFu : 0u;
        return make_uint4((cp.x & (ap | (hp & ~r.x))) | (cq.x & (aq | (hq & ~r.x))),
                          (cp.y & (ap | (hp & ~r.y))) | (cq.y & (aq | (hq & ~r.y))),
                          (cp.z & (ap | (hp & ~r.z))) | (cq.z & (aq | (hq & ~r.z))),
                          (cp.w & (ap | (hp & ~r.w))) | (cq.w & (aq | (hq & ~r.w))));
    }
    return decide4(cp, cq, tp, tq, key, qgroup, step, stream);
}

// Quenched disorder (mcsDisorder2SyncRng): every site carries a 2-bit rate class c (bit 0 in
// d0, bit 1 in d1) that picks thresholds tp[c] / tq[c]; the comparison u < T(site) runs on the
// same random planes as decide4, so equal rates in every class give decide4's result.
struct DisorderRates {
    Thresh tp[4], tq[4];
    int planes;  // most planes any of the eight thresholds can need
};

inline DisorderRates make_disorder_rates(const uint64_t Tp[4], const uint64_t Tq[4])
{
    DisorderRates dr{};
    dr.planes = 0;
    for (int c = 0; c < 4; ++c) {
        dr.tp[c] = make_thresh(Tp[c]);
        dr.tq[c] = make_thresh(Tq[c]);
        if (dr.tp[c].planes > dr.planes) dr.planes = dr.tp[c].planes;
        if (dr.tq[c].planes > dr.planes) dr.planes = dr.tq[c].planes;
    }
    return dr;
}

__device__ __forceinline__ uint32_t sel_class(uint32_t d0, uint32_t d1, uint32_t b0, uint32_t b1, uint32_t b2,
                                              uint32_t b3)
{
    return (~d1 & ((~d0 & b0) | (d0 & b1))) | (d1 & ((~d0 & b2) | (d0 & b3)));
}

__device__ __forceinline__ uint32_t dis_word(uint32_t cp, uint32_t cq, uint32_t d0, uint32_t d1,
                                             const uint32_t bp[4], const uint32_t bq[4])
{
    return (cp & sel_class(d0, d1, bp[0], bp[1], bp[2], bp[3])) |
           (cq & sel_class(d0, d1, bq[0], bq[1], bq[2], bq[3]));
}

__device__ __forceinline__ uint4 decide4_dis(uint4 cp, uint4 cq, uint4 d0, uint4 d1, const DisorderRates& dr,
                                             Key key, uint32_t qgroup, uint32_t step, uint32_t stream)
{
    uint32_t ap[4], aq[4], hp[4], hq[4];
    for (int c = 0; c < 4; ++c) {
        ap[c] = dr.tp[c].always ? 0xFFFFFFFFu : 0u;
        aq[c] = dr.tq[c].always ? 0xFFFFFFFFu : 0u;
        hp[c] = dr.tp[c].planes ? 0xFFFFFFFFu : 0u;
        hq[c] = dr.tq[c].planes ? 0xFFFFFFFFu : 0u;
    }
    // decided flips (threshold 2^32) and sites still equal to their threshold's prefix
    uint4 lt = make_uint4(dis_word(cp.x, cq.x, d0.x, d1.x, ap, aq), dis_word(cp.y, cq.y, d0.y, d1.y, ap, aq),
                          dis_word(cp.z, cq.z, d0.z, d1.z, ap, aq), dis_word(cp.w, cq.w, d0.w, d1.w, ap, aq));
    uint4 eq = make_uint4(dis_word(cp.x, cq.x, d0.x, d1.x, hp, hq), dis_word(cp.y, cq.y, d0.y, d1.y, hp, hq),
                          dis_word(cp.z, cq.z, d0.z, d1.z, hp, hq), dis_word(cp.w, cq.w, d0.w, d1.w, hp, hq));
    for (int k = 0; k < dr.planes; ++k) {
        if (!(eq.x | eq.y | eq.z | eq.w)) break;
        const uint4 r = philox4x32_10(make_uint4(qgroup, step, (uint32_t)k | (TAG_SCA << 8), stream), key);
        uint32_t bp[4], bq[4], ep[4], eqn[4];
        for (int c = 0; c < 4; ++c) {
            bp[c] = ((dr.tp[c].t >> (31 - k)) & 1u) ? 0xFFFFFFFFu : 0u;
            bq[c] = ((dr.tq[c].t >> (31 - k)) & 1u) ? 0xFFFFFFFFu : 0u;
            // thresholds with no 1 bit left below this plane can no longer be exceeded from below
            ep[c] = (k + 1 >= dr.tp[c].planes) ? 0xFFFFFFFFu : 0u;
            eqn[c] = (k + 1 >= dr.tq[c].planes) ? 0xFFFFFFFFu : 0u;
        }
#define KPZB_DIS_PLANE(F)                                                   \
    {                                                                       \
        const uint32_t tb = dis_word(cp.F, cq.F, d0.F, d1.F, bp, bq);       \
        lt.F |= eq.F & tb & ~r.F;                                           \
        eq.F &= ~(tb ^ r.F);                                                \
        eq.F &= ~dis_word(cp.F, cq.F, d0.F, d1.F, ep, eqn);                 \
    }
        KPZB_DIS_PLANE(x) KPZB_DIS_PLANE(y) KPZB_DIS_PLANE(z) KPZB_DIS_PLANE(w)
#undef KPZB_DIS_PLANE
    }
    return lt;
}

__device__ __forceinline__ uint4 operator^(uint4 a, uint4 b)
{
    return make_uint4(a.x ^ b.x, a.y ^ b.y, a.z ^ b.z, a.w ^ b.w);
}

}  // namespace kpzb
