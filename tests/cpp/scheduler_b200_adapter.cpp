// SchedulerB200: the Kpz::SchedulerService subclass a maintainer adds to the CudaKpz tree to
// run the reference's frontend on this library.  It forwards the scheduler virtuals to the
// kpzb C ABI and keeps the reference's host lattice
// m_system in the reference's word layout, so the reference's own host analysis --
// SchedulerService::roughness (kpz/schedulerService.cpp:292-297) and consitencyCheck
// (:721-854) -- runs unchanged on lattices this library produced.
//
// oracle/build_ref.py compiles it against the reference's headers and CPU objects (never
// copied into this repository) into oracle/_ref/kpz_ref_adapter.  Usage:
//   kpz_ref_adapter LX P Q SEED N   ->  "RESULT <reference W2> <kpzb W2> <reference consistency ok>"
//   kpz_ref_adapter dtcurve LX P Q SEED T1 T2 ...
//       --scheduler dt through the adapter: "<t> <W2>" per time, W2 from the reference's own
//       SchedulerService::roughness on the popped lattice
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>

#include "correlator.h"
#include "kpzb.h"
#include "schedulerService.h"

// HDF5/libSplash entry points of SchedulerService are not built (not on the hot path).
bool Kpz::SchedulerService::collectH5(splash::DataCollector*, const std::string&) { return false; }
bool Kpz::SchedulerService::retrieveH5(splash::DataCollector*, const std::string&) { return false; }

namespace Kpz {
class SchedulerB200 : public SchedulerService {
    kpzb_handle* h_ = nullptr;
    static void ck(kpzb_status s)
    {
        if (s != KPZB_OK) throw std::runtime_error(kpzb_last_error());
    }

public:
    SchedulerB200(int lx, int ly, int dynamics, int device)
        : SchedulerService(lx, ly, dynamics == KPZB_DYN_SCABIT ? ENC_CBBIT : ENC_LOCAL)
    {
        ck(kpzb_create(&h_, lx, ly, dynamics, device));
        // the block-level decomposition the reference's DT scheduler is built with by
        // default (KPZ_INNER_DD = KPZ_INNER_DBSH, kpz/param.h:36), set explicitly
        if (dynamics == KPZB_DYN_DT) ck(kpzb_set_dt_inner(h_, KPZB_DT_INNER_DBSH));
    }
    ~SchedulerB200() override { kpzb_destroy(h_); }
    kpzb_handle* handle() { return h_; }
    void seed(uint64_t s) { ck(kpzb_seed(h_, s, 0)); }

    void initHomogeneous(Encoding e) override
    {
        SchedulerService::initHomogeneous(e);
        pushSystem();
    }
    bool setPQ(double p, double q, unsigned int n = 0) override
    {
        if (!SchedulerService::setPQ(p, q, n)) return false;
        return (n == 0 ? kpzb_set_pq(h_, p, q) : kpzb_set_pq_class(h_, (int)n, p, q)) == KPZB_OK;
    }
    void pushSystem() override
    {
        SchedulerService::pushSystem();
        ck(kpzb_push(h_, m_system));
    }
    void popSystem() override
    {
        SchedulerService::popSystem();
        ck(kpzb_pop(h_, m_system));
    }
    void mcsPQSyncRng(int n) override
    {
        ck(kpzb_mcs(h_, n));
        m_deviceMcs += n;
    }
    void mcsPQ(int n) override { mcsPQSyncRng(n); }
    void mcsDisorder2SyncRng(int n) override
    {
        ck(kpzb_set_disorder(h_, m_disorder));
        ck(kpzb_mcs_disorder(h_, n));
        m_deviceMcs += n;
    }
    double mcsScale() const override
    {
        double s = 1.0;
        ck(kpzb_mcs_scale(h_, &s));
        return s;
    }
    void randomize() override {}
};
}  // namespace Kpz

static int dt_curve(int argc, char** argv)
{
    const int lx = std::atoi(argv[2]);
    const double p = std::atof(argv[3]), q = std::atof(argv[4]);
    const unsigned long long seed = std::strtoull(argv[5], nullptr, 10);
    try {
        std::streambuf* keep = std::cout.rdbuf();
        std::cout.rdbuf(nullptr);
        Kpz::Correlator::setNThreads(2);
        Kpz::SchedulerB200 s(lx, lx, KPZB_DYN_DT, 0);
        s.seed(seed);
        s.initHomogeneous(Kpz::SchedulerService::ENC_LOCAL);
        s.setPQ(p, q);
        int t = 0;
        std::ostringstream out;
        out.precision(17);
        for (int i = 6; i < argc; ++i) {
            const int T = std::atoi(argv[i]);
            s.mcsPQSyncRng(T - t);
            t = T;
            s.popSystem();
            out << T << " " << (double)s.roughness().w2 << "\n";
        }
        std::cout.rdbuf(keep);
        std::cout << out.str() << std::flush;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}

int main(int argc, char** argv)
{
    if (argc >= 7 && std::string(argv[1]) == "dtcurve") return dt_curve(argc, argv);
    if (argc < 6) {
        std::cerr << "usage: kpz_ref_adapter LX P Q SEED N\n";
        return 2;
    }
    const int lx = std::atoi(argv[1]);
    const double p = std::atof(argv[2]), q = std::atof(argv[3]);
    const unsigned long long seed = std::strtoull(argv[4], nullptr, 10);
    const int n = std::atoi(argv[5]);
    try {
        std::streambuf* keep = std::cout.rdbuf();
        std::cout.rdbuf(nullptr);  // the reference prints set-up chatter
        Kpz::Correlator::setNThreads(2);
        Kpz::SchedulerB200 s(lx, lx, KPZB_DYN_SCA, 0);
        s.seed(seed);
        s.initHomogeneous(Kpz::SchedulerService::ENC_LOCAL);
        s.setPQ(p, q);
        s.mcsPQSyncRng(n);
        s.popSystem();
        const auto r = s.roughness();                  // the reference's host analysis
        const bool ok = s.consitencyCheck(true, std::cerr);  // the reference's invariants
        double ours[8];
        if (kpzb_roughness(s.handle(), ours) != KPZB_OK) throw std::runtime_error(kpzb_last_error());
        std::cout.rdbuf(keep);
        std::fflush(stdout);
        std::printf("\nRESULT %.17g %.17g %d\n", (double)r.w2, ours[0], ok ? 1 : 0);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
