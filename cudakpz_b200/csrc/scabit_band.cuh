// scabit_band.cuh -- one band of SCABit rows advanced k MCS in shared memory (sm_100a).
//
// Shared by the single-lattice temporally blocked kernel (scabit.cu) and the batched
// replica kernel (batch.cu).  A band is R full-width rows of all four ENC_CBBIT quadrants
// (kpz/systemSize.h:143-165), loaded with TMA bulk copies (cp.async.bulk, local HBM only)
// and an mbarrier with a bounded wait.
//   halo mode:     R = B + 4k rows starting 2k rows above the band; half-step h updates
//                  local rows [h, R-1-h); rows [2k, 2k+B) are exact afterwards.
//   resident mode: the whole lattice (R = rows); every half-step updates every row with
//                  periodic y-neighbours inside shared memory; any k.
// The update rule is that of kpz/kpzSCABit.cu:179-290 with the masks of
// kpz/kpzSCABitCores.cu:69-74,139-145.  The one-bit x-carry of shifted rows crosses thread
// boundaries only in the first word of each 4-word group (shared-memory atomicXor).
#pragma once
#include "kpzb_common.cuh"

namespace kpzb {

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
                 "r"(smem_u32(src)), "r"(bytes)
                 : "memory");
}

// bounded spin on the TMA mbarrier: ~2^26 polls (far above any real copy time)
constexpr uint32_t MBAR_SPIN_LIMIT = 1u << 26;

struct BandCtl {
    uint64_t* bar;     // shared mbarrier, initialised once per CTA with count 1
    int* abort_flag;   // shared
    uint32_t phase;    // parity of the mbarrier phase this band waits on
};

struct BandGeom {
    const uint32_t* src;
    uint32_t* dst;
    int lx, ly;
    int64_t y0;      // first output row
    int B;           // output rows (halo mode) or rows (resident)
    int k;           // MCS per pass
    bool resident;
    uint32_t t0;     // MCS index of the first MCS of the pass
    Key key;
    uint32_t stream;
    Thresh tp, tq;
};

// One 4-word group (128 sites, one Philox group) of one half-step: the rule of
// kpz/kpzSCABit.cu:179-290 with the masks of kpz/kpzSCABitCores.cu:69-74,139-145.
// pTX/pTY: this sublattice's X/Y words of the row; pOX: the other sublattice's X words of the
// row; pOY: the other sublattice's Y words of the next row; nbp: the first word of the next
// group of the other X row (the one-bit carry of shifted rows).  MODE is a DecMode, or -1 to
// decide with the runtime mode `mode_rt`; USEQ false when maxima never flip (q = 0), which
// drops the maximum-candidate mask.  The carry crosses groups with shared-memory atomicXor on
// disjoint bits (bit 0 of the next group's first word; bits 1..31 of this group's), so
// neighbouring groups of a row may be updated concurrently.
// The words one group update reads (loaded ahead of the update when the caller pipelines rows).
struct GroupIn {
    uint4 tX, tY, oX, oY;
    uint32_t nb;
};

__device__ __forceinline__ GroupIn sca_load_group(const uint32_t* pTX, const uint32_t* pTY, const uint32_t* pOX,
                                                  const uint32_t* pOY, const uint32_t* nbp)
{
    GroupIn in;
    in.tX = *reinterpret_cast<const uint4*>(pTX);
    in.tY = *reinterpret_cast<const uint4*>(pTY);
    in.oX = *reinterpret_cast<const uint4*>(pOX);
    in.oY = *reinterpret_cast<const uint4*>(pOY);
    in.nb = *nbp;
    return in;
}

// Candidate masks and flip mask of one 4-word group from its words (xX: the other-X words as
// seen by this sublattice's sites, i.e. shifted for shifted rows).
template <int MODE, bool USEQ>
__device__ __forceinline__ uint4 sca_decide(const uint4& tX, const uint4& tY, const uint4& xX, const uint4& oY,
                                            int mode_rt, const Thresh& tp, const Thresh& tq, Key key,
                                            uint32_t qgroup, uint32_t step, uint32_t stream, uint4& cp, uint4& cq)
{
    cq = make_uint4(0, 0, 0, 0);
    cp.x = ~(tX.x | tY.x) & xX.x & oY.x;
    cp.y = ~(tX.y | tY.y) & xX.y & oY.y;
    cp.z = ~(tX.z | tY.z) & xX.z & oY.z;
    cp.w = ~(tX.w | tY.w) & xX.w & oY.w;
    if (USEQ) {
        cq.x = tX.x & tY.x & ~(xX.x | oY.x);
        cq.y = tX.y & tY.y & ~(xX.y | oY.y);
        cq.z = tX.z & tY.z & ~(xX.z | oY.z);
        cq.w = tX.w & tY.w & ~(xX.w | oY.w);
    }
    if (MODE == DEC_NONE) {
        const uint32_t ap = tp.always ? 0xFFFFFFFFu : 0u;
        if (!USEQ) return make_uint4(cp.x & ap, cp.y & ap, cp.z & ap, cp.w & ap);
        const uint32_t aq = tq.always ? 0xFFFFFFFFu : 0u;
        return make_uint4((cp.x & ap) | (cq.x & aq), (cp.y & ap) | (cq.y & aq), (cp.z & ap) | (cq.z & aq),
                          (cp.w & ap) | (cq.w & aq));
    }
    return decide4_mode(MODE < 0 ? mode_rt : MODE, cp, cq, tp, tq, key, qgroup, step, stream);
}

// The update of one group from its loaded words.  Within a half-step a group may be loaded
// before other groups are stored: an update reads its row's this-X/this-Y/other-X words and
// the next row's other-Y words and writes the same words, which no other row or group of the
// half-step reads or writes, except the next group's first other-X word, whose bit 0 it
// changes by an atomic XOR -- a bit the owner neither reads (the one-bit right shift drops it)
// nor stores (it XORs its own mask in atomically).
template <int MODE, bool USEQ, bool COUNT>
__device__ __forceinline__ void sca_update_loaded(const GroupIn& in, uint32_t* pTX, uint32_t* pTY, uint32_t* pOX,
                                                  uint32_t* pOY, uint32_t* nbp, bool shifted, int mode_rt,
                                                  const Thresh& tp, const Thresh& tq, Key key, uint32_t qgroup,
                                                  uint32_t step, uint32_t stream, bool count_row,
                                                  unsigned long long& ndep, unsigned long long& ndes)
{
    const uint4 tX = in.tX, tY = in.tY, oX = in.oX, oY = in.oY;
    uint4 xX = oX;
    if (shifted) {
        xX.x = __funnelshift_r(oX.x, oX.y, 1);
        xX.y = __funnelshift_r(oX.y, oX.z, 1);
        xX.z = __funnelshift_r(oX.z, oX.w, 1);
        xX.w = __funnelshift_r(oX.w, in.nb, 1);
    }
    uint4 cp, cq;
    const uint4 m = sca_decide<MODE, USEQ>(tX, tY, xX, oY, mode_rt, tp, tq, key, qgroup, step, stream, cp, cq);
    if (COUNT && count_row) {
        ndep += __popc(m.x & cp.x) + __popc(m.y & cp.y) + __popc(m.z & cp.z) + __popc(m.w & cp.w);
        if (USEQ) ndes += __popc(m.x & cq.x) + __popc(m.y & cq.y) + __popc(m.z & cq.z) + __popc(m.w & cq.w);
    }
    *reinterpret_cast<uint4*>(pTX) = tX ^ m;
    *reinterpret_cast<uint4*>(pTY) = tY ^ m;
    *reinterpret_cast<uint4*>(pOY) = oY ^ m;
    if (shifted) {
        atomicXor(pOX, m.x << 1);
        pOX[1] = oX.y ^ __funnelshift_l(m.x, m.y, 1);
        pOX[2] = oX.z ^ __funnelshift_l(m.y, m.z, 1);
        pOX[3] = oX.w ^ __funnelshift_l(m.z, m.w, 1);
        if (m.w >> 31) atomicXor(nbp, 1u);
    } else {
        *reinterpret_cast<uint4*>(pOX) = oX ^ m;
    }
}

// One 4-word group (128 sites, one Philox group) of one half-step: the rule of
// kpz/kpzSCABit.cu:179-290 with the masks of kpz/kpzSCABitCores.cu:69-74,139-145.
// pTX/pTY: this sublattice's X/Y words of the row; pOX: the other sublattice's X words of the
// row; pOY: the other sublattice's Y words of the next row; nbp: the first word of the next
// group of the other X row (the one-bit carry of shifted rows).  MODE is a DecMode, or -1 to
// decide with the runtime mode `mode_rt`; USEQ false when maxima never flip (q = 0), which
// drops the maximum-candidate mask.  The carry crosses groups with shared-memory atomicXor on
// disjoint bits (bit 0 of the next group's first word; bits 1..31 of this group's), so
// neighbouring groups of a row may be updated concurrently.
template <int MODE, bool USEQ, bool COUNT>
__device__ __forceinline__ void sca_update_group(uint32_t* pTX, uint32_t* pTY, uint32_t* pOX,
                                                 uint32_t* pOY, uint32_t* nbp, bool shifted,
                                                 int mode_rt, const Thresh& tp, const Thresh& tq,
                                                 Key key, uint32_t qgroup, uint32_t step,
                                                 uint32_t stream, bool count_row,
                                                 unsigned long long& ndep, unsigned long long& ndes)
{
    const GroupIn in = sca_load_group(pTX, pTY, pOX, pOY, nbp);
    sca_update_loaded<MODE, USEQ, COUNT>(in, pTX, pTY, pOX, pOY, nbp, shifted, mode_rt, tp, tq, key, qgroup,
                                         step, stream, count_row, ndep, ndes);
}

// Runs one band; returns false (after flagging *err) when the TMA load did not complete in
// time.  Must be called by all threads of the CTA; NT = blockDim.x.  MODE / USEQ as for
// sca_update_group (MODE -1 with USEQ true: rates known only at run time, as in a batch).
template <int MODE, bool USEQ, bool COUNT, int NT>
__device__ bool scabit_band(uint32_t* smem, const BandCtl& ctl, const BandGeom& g,
                            unsigned long long& ndep, unsigned long long& ndes,
                            unsigned int* err)
{
    const uint64_t Wr = 1ull << (g.lx - 6);
    const uint64_t Q = 1ull << (g.lx + g.ly - 6);
    const int64_t rows = 1ll << g.ly;
    const int H = g.resident ? 0 : 2 * g.k;
    const int R = g.resident ? (int)rows : g.B + 2 * H;
    const int G = (int)(Wr / 4);  // 4-word groups per row
    const int lgG = g.lx - 8;
    const uint64_t qsz = (uint64_t)R * Wr;  // words per quadrant slab in shared memory
    const int64_t y0 = g.resident ? 0 : g.y0;
    const int Bc = g.resident ? (int)rows : (int)(rows - y0 < g.B ? rows - y0 : g.B);
    const int64_t ylo = y0 - H;  // global row of local row 0

    if (threadIdx.x == 0) {
        *ctl.abort_flag = 0;
        mbar_expect_tx(ctl.bar, (uint32_t)(16ull * qsz));
        int64_t r0 = ylo & (rows - 1);
        int done = 0;
        while (done < R) {
            const int piece = (int)((int64_t)(R - done) < rows - r0 ? (int64_t)(R - done) : rows - r0);
            for (int qd = 0; qd < 4; ++qd)
                bulk_g2s(smem + qd * qsz + (uint64_t)done * Wr, g.src + qd * Q + (uint64_t)r0 * Wr,
                         (uint32_t)((uint64_t)piece * Wr * 4), ctl.bar);
            done += piece;
            r0 = 0;
        }
        uint32_t spins = 0;
        while (!mbar_try_wait(ctl.bar, ctl.phase)) {
            if (++spins > MBAR_SPIN_LIMIT) {
                *ctl.abort_flag = 1;
                break;
            }
        }
    }
    __syncthreads();
    if (*ctl.abort_flag) {
        // leave dst untouched and report; the copy in flight targets this CTA's shared
        // memory only, so wait for it (bounded) before the caller retires the CTA
        if (threadIdx.x == 0) {
            atomicExch(err, 1u);
            uint32_t spins = 0;
            while (!mbar_try_wait(ctl.bar, ctl.phase) && ++spins < MBAR_SPIN_LIMIT) {
            }
        }
        return false;
    }

    // Each thread owns one 4-word column group gi and walks rows with stride NT / G; all
    // shared-memory offsets are 32-bit (a band is at most 227 KB).  (A warp-per-row variant
    // that passes the x-carry by shuffles removed the atomics and bank conflicts but issued
    // 67 % more instructions and ran 15 % slower at 16384^2; the atomics stay.)
    const int mode_rt = MODE < 0 ? dec_mode(g.tp, g.tq) : MODE;
    const uint32_t wr = (uint32_t)Wr;
    const int gi = (G >= NT) ? (int)threadIdx.x : (int)(threadIdx.x & (G - 1));
    const int rstride = (G >= NT) ? 1 : NT >> lgG;
    const int rofs = (G >= NT) ? 0 : (int)(threadIdx.x >> lgG);
    const uint32_t rmask = (uint32_t)rows - 1u;
    const int ylo32 = (int)(ylo & (int64_t)rmask);  // ylo mod rows
    const uint32_t q32 = (uint32_t)qsz;
    for (int h = 0; h < 2 * g.k; ++h) {
        const int sigma = h & 1;
        const uint32_t step = 2u * (g.t0 + (uint32_t)(h >> 1)) + (uint32_t)sigma;
        uint32_t* StX = smem + (sigma ? 2u * q32 : 0u);
        uint32_t* StY = StX + q32;
        uint32_t* SoX = smem + (sigma ? 0u : 2u * q32);
        uint32_t* SoY = SoX + q32;
        const int ra = g.resident ? 0 : h;
        const int rb = g.resident ? R : R - 1 - h;
        // wide rows (G > NT): a thread takes several column groups of a row in turn
        for (int gg = gi; gg < G; gg += NT) {
            const uint32_t w0 = 4u * (uint32_t)gg;
            const uint32_t wnext = (w0 + 4u) & (wr - 1u);
            for (int lr = ra + rofs; lr < rb; lr += rstride) {
                const uint32_t gy = ((uint32_t)ylo32 + (uint32_t)lr) & rmask;  // periodic in y
                const uint32_t ro = (uint32_t)lr * wr;
                const uint32_t ro1 = g.resident ? (((uint32_t)lr + 1u) & rmask) * wr : ro + wr;
                sca_update_group<MODE, USEQ, COUNT>(StX + ro + w0, StY + ro + w0, SoX + ro + w0, SoY + ro1 + w0,
                                                    SoX + ro + wnext, sigma != (int)(gy & 1u), mode_rt, g.tp,
                                                    g.tq, g.key, (gy << lgG) + (uint32_t)gg, step, g.stream,
                                                    lr >= H && lr < H + Bc, ndep, ndes);
            }
        }
        __syncthreads();
    }

    // write the band's own rows [H, H + Bc) of each quadrant, then wait until the bulk
    // store has read shared memory so the caller may reuse it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int qd = 0; qd < 4; ++qd)
            bulk_s2g(g.dst + qd * Q + (uint64_t)y0 * Wr, smem + qd * qsz + (uint64_t)H * Wr,
                     (uint32_t)((uint64_t)Bc * Wr * 4));
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    return true;
}

}  // namespace kpzb
