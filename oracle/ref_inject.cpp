// ref_inject.cpp -- TEST INFRASTRUCTURE ONLY: the reference's own per-site checkerboard update
// (SchedulerCPUCBBit<Rng>::Func_MCSLocalBase::pqSyncRngUpdate,
// kpz/schedulerCPUCBBit_nested.inl:261-295, driven by doMcs, kpz/schedulerCPUCBBit.cpp:42-79)
// run with a stand-in for its random number generator that hands it, site by site, the
// decisions of this project's counter stream.
//
// With one worker thread the reference visits the sites of one sublattice row by row, x rising
// (rows [0, L/2) and then [L/2, L) of the single thread's range), and draws exactly one
// randomFloat() per site of the sublattice before it looks at the site's configuration; a
// half-step therefore consumes L*L/2 draws, sublattice 0 first.  The stand-in counts its draws,
// recovers the site and half-step from the count, takes the site's 32-bit uniform u from the
// oracle's restatement of the stream (ko_site_u) and returns a float v whose comparisons with
// the reference's rates reproduce u < T(p) and u < T(q).  Everything else -- geometry, the
// configuration test, which bits flip and in which words -- is the reference's code, unchanged,
// so the lattice it leaves equals the oracle's (and the GPU's) exactly when both implement the
// same per-site rule on the same decisions.  compiled by oracle/build_ref.py into
// oracle/_ref/kpz_ref (command cbbit-inject).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "schedulerCPUCB.cpp"
#include "schedulerCPUCBBit.cpp"
#include "schedulerCPUBaseThreadedRng.cpp"

#include "CPURngIface.h"

extern "C" {
#include "kpz_oracle.h"
}

namespace {
struct InjectConfig {
    int lx = 0;
    uint64_t seed = 0, t0 = 0;
    uint32_t stream = 0;
    double p = 0.0, q = 0.0;
    uint64_t Tp = 0, Tq = 0;
    bool bad_rates = false;  // p and q closer than the float spacing: no v separates them
};
InjectConfig g_cfg;

bool below(uint32_t u, uint64_t T) { return T >= (1ull << 32) || (uint64_t)u < T; }

// the smallest float v with (double)v >= x
float float_at_least(double x)
{
    float v = (float)x;
    if ((double)v < x) v = std::nextafterf(v, 2.0f);
    return v;
}
}  // namespace

namespace Kpz {
namespace RngIface {
// The stand-in generator: plain data (the scheduler copies it with memcpy between half-steps).
class InjectRng
{
    uint64_t m_draws = 0;

public:
    unsigned int random()
    {
        // only the bit-parallel p = 1/2, q = 0 path draws words; the per-site path never does
        std::fprintf(stderr, "InjectRng::random() called: rates not on the per-site path\n");
        std::abort();
    }
    float randomFloat()
    {
        const uint64_t half = 1ull << (2 * g_cfg.lx - 1);  // sites of one sublattice
        const uint64_t hs = m_draws / half, i = m_draws % half;
        ++m_draws;
        const int sigma = (int)(hs & 1);
        const uint64_t t = g_cfg.t0 + hs / 2;
        const int y = (int)(i >> (g_cfg.lx - 1));
        const int x = (int)(((i & ((1ull << (g_cfg.lx - 1)) - 1)) << 1) | (uint64_t)((y ^ sigma) & 1));
        const uint64_t qword = ((uint64_t)y << (g_cfg.lx - 6)) + (uint64_t)(x >> 6);
        const uint32_t u = ko_site_u(g_cfg.seed, g_cfg.stream, KO_TAG_SCA, (uint32_t)(2 * t + sigma), qword,
                                     (x >> 1) & 31);
        const bool ap = below(u, g_cfg.Tp), aq = below(u, g_cfg.Tq);
        // the reference flips a minimum iff v < p and a maximum iff v < q (kpz/schedulerCPUCBBit_nested.inl:276-287)
        if (ap && aq) return 0.0f;
        if (!ap && !aq) return 1.0f;
        const double lo = ap ? g_cfg.q : g_cfg.p, hi = ap ? g_cfg.p : g_cfg.q;  // want lo <= v < hi
        const float v = float_at_least(lo);
        if (!((double)v < hi)) g_cfg.bad_rates = true;
        return v;
    }
    void seed(unsigned int) {}
    template <class Container>
    static void initialize(Container&)
    {
    }
    template <class Container>
    static void randomize(Container&, dsfmt_t&)
    {
    }
    template <class Container>
    static void writeH5(splash::DataCollector*, int, Container&, const std::string& = "")
    {
    }
    template <class Container>
    static bool readH5(splash::DataCollector*, int, Container&, const std::string& = "")
    {
        return false;
    }
};
}  // namespace RngIface

template class SchedulerCPUCB<RngIface::InjectRng>;
template class SchedulerCPUCBBit<RngIface::InjectRng>;
}  // namespace Kpz

// n MCS of SchedulerCPUCBBit<InjectRng>::mcsPQSyncRng on the ENC_CBBIT lattice `words` (in
// place), one worker thread, the counter stream (seed, stream) starting at MCS t0.
// Returns 0, or 1 when the rates do not take the per-site path or cannot be separated.
int ref_cbbit_injected(int lx, double p, double q, int n, uint32_t* words, uint64_t seed, uint32_t stream,
                       uint64_t t0)
{
    if (q == 0.0 && p == 0.5) return 1;  // the reference's bit-parallel path (kpz/schedulerCPUCBBit.cpp:98)
    g_cfg = InjectConfig{};
    g_cfg.lx = lx;
    g_cfg.seed = seed;
    g_cfg.stream = stream;
    g_cfg.t0 = t0;
    g_cfg.p = p;
    g_cfg.q = q;
    g_cfg.Tp = ko_threshold(p);
    g_cfg.Tq = ko_threshold(q);
    Kpz::SchedulerCPUCBBit<Kpz::RngIface::InjectRng> s(lx, lx, 1);
    s.initHomogeneous(Kpz::SchedulerService::ENC_CBBIT);
    std::memcpy(s.system(), words, s.size().sizeW() * 4);
    s.pushSystem();
    s.setPQ(p, q);
    s.mcsPQSyncRng(n);
    s.popSystem();
    std::memcpy(words, s.system(), s.size().sizeW() * 4);
    return g_cfg.bad_rates ? 1 : 0;
}
