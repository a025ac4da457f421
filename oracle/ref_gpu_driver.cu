// ref_gpu_driver.cu -- MEASUREMENT INFRASTRUCTURE (reference arm only, never the product).
//
// Times the reference's own GPU scheduler, SchedulerSCABit<SLCG64> (kpz/schedulerSCABit.cu,
// kpz/kpzSCABit.cu, kpz/kpzSCABitCores.cu), compiled from the CudaKpz sources by
// oracle/build_ref.py into oracle/_ref/kpz_ref_gpu, through its public SchedulerService calls
// exactly as the reference's kpzScaling driver uses them (kpz/kpzScaling.cpp:142-215):
// supplySeed, randomize, initHomogeneous, setPQ, mcsPQSyncRng, popSystem.
//
// and SchedulerDT<SLCG64, SchedulerDT_LocalLayoutDis> (kpz/schedulerDT.cu, kpz/kpz.cu, the
// default DBSH inner decomposition of kpz/param.h) and the DB4 scheduler
// Scheduler<SLCG64, Scheduler_LocalLayoutDefault> (kpz/scheduler.cu, --scheduler db4 of
// kpz/kpzFrontend.cpp:368-371) the same way.
//
// usage:
//   kpz_ref_gpu scabit LX P Q WARMUP MCS   warm-up MCS, then MCS timed; prints
//   kpz_ref_gpu dt LX P Q WARMUP MCS       "<attempted updates/ns> <seconds> <W2>"
//   kpz_ref_gpu db4 LX P Q WARMUP MCS
//   kpz_ref_gpu dtcurve LX P Q SEED T1 T2 ...      supplySeed(1, SEED); "<t> <W2> <h>" per time
//   kpz_ref_gpu db4curve LX P Q SEED T1 T2 ...
//   kpz_ref_gpu scabitcurve LX P Q SEED T1 T2 ...
//   kpz_ref_gpu scabitdump LX P Q N FILE          lattice words after N MCS (flat start)
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>

#include "GPURandom.h"
#include "correlator.h"
#include "scheduler.h"
#include "schedulerDT.h"
#include "schedulerSCABit.h"

// HDF5/libSplash entry points of SchedulerService are not built (not on the hot path).
bool Kpz::SchedulerService::collectH5(splash::DataCollector*, const std::string&) { return false; }
bool Kpz::SchedulerService::retrieveH5(splash::DataCollector*, const std::string&) { return false; }

static double now()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class Sched>
static int run(int lx, double p, double q, int warm, int n, Kpz::SchedulerService::Encoding enc)
{
    std::streambuf* keep = std::cout.rdbuf();
    std::cout.rdbuf(nullptr);  // the schedulers print set-up chatter on std::cout
    Sched s(lx, lx, 0);
    s.supplySeed(1, 1);
    s.randomize();
    s.initHomogeneous(enc);
    s.pushSystem();
    s.setPQ(p, q);
    if (warm > 0) s.mcsPQSyncRng(warm);
    const double t0 = now();
    s.mcsPQSyncRng(n);  // returns after cudaThreadSynchronize (kpz/schedulerSCABit.cu:64, schedulerDT.cu:57)
    const double t1 = now();
    s.popSystem();
    Kpz::Correlator::setNThreads(1);  // host roughness walk on one thread
    const auto r = s.roughness();
    std::cout.rdbuf(keep);
    std::cout << std::setprecision(9) << (double)s.size().size() * n / ((t1 - t0) * 1e9) << ' ' << (t1 - t0)
              << ' ' << (double)r.w2 << '\n';
    return 0;
}

// W^2 and <h> at increasing times (a growth curve): "<t> <W2> <h1>" per line.
template <class Sched>
static int curve(int lx, double p, double q, int seed, char** ts, int nt, Kpz::SchedulerService::Encoding enc)
{
    std::streambuf* keep = std::cout.rdbuf();
    std::cout.rdbuf(nullptr);
    Sched s(lx, lx, 0);
    s.supplySeed(1, seed);
    s.randomize();
    s.initHomogeneous(enc);
    s.pushSystem();
    s.setPQ(p, q);
    Kpz::Correlator::setNThreads(1);
    int t = 0;
    std::ostringstream out;
    out << std::setprecision(12);
    for (int i = 0; i < nt; ++i) {
        const int target = std::atoi(ts[i]);
        s.mcsPQSyncRng(target - t);
        t = target;
        s.popSystem();
        const auto r = s.roughness();
        out << t << ' ' << (double)r.w2 << ' ' << (double)r.h[0] << '\n';
    }
    std::cout.rdbuf(keep);
    std::cout << out.str();
    return 0;
}

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::cerr << "usage: kpz_ref_gpu scabit LX P Q WARMUP MCS\n";
        return 2;
    }
    const std::string cmd = argv[1];
    if ((cmd == "scabit" || cmd == "dt" || cmd == "db4") && argc >= 7) {
        const int lx = std::atoi(argv[2]);
        const double p = std::atof(argv[3]), q = std::atof(argv[4]);
        const int warm = std::atoi(argv[5]), n = std::atoi(argv[6]);
        if (cmd == "scabit")
            return run<Kpz::SchedulerSCABit<SLCG64>>(lx, p, q, warm, n, Kpz::SchedulerService::ENC_CBBIT);
        if (cmd == "db4")
            return run<Kpz::Scheduler<SLCG64, Kpz::Scheduler_LocalLayoutDefault>>(lx, p, q, warm, n,
                                                                               Kpz::SchedulerService::ENC_LOCAL);
        return run<Kpz::SchedulerDT<SLCG64, Kpz::SchedulerDT_LocalLayoutDis>>(lx, p, q, warm, n,
                                                                           Kpz::SchedulerService::ENC_LOCAL);
    }
    if (cmd == "scabitdump" && argc >= 7) {
        // the lattice words after N MCS from the flat start (deterministic rates only)
        const int lx = std::atoi(argv[2]);
        const double p = std::atof(argv[3]), q = std::atof(argv[4]);
        const int n = std::atoi(argv[5]);
        std::streambuf* keep = std::cout.rdbuf();
        std::cout.rdbuf(nullptr);
        Kpz::SchedulerSCABit<SLCG64> s(lx, lx, 0);
        s.supplySeed(1, 1);
        s.randomize();
        s.initHomogeneous(Kpz::SchedulerService::ENC_CBBIT);
        s.pushSystem();
        s.setPQ(p, q);
        s.mcsPQSyncRng(n);
        s.popSystem();
        std::cout.rdbuf(keep);
        FILE* f = std::fopen(argv[6], "wb");
        if (!f) return 3;
        const size_t nw = s.size().sizeW();
        const bool ok = std::fwrite(s.system(), 4, nw, f) == nw;
        std::fclose(f);
        return ok ? 0 : 3;
    }
    if ((cmd == "dtcurve" || cmd == "scabitcurve" || cmd == "db4curve") && argc >= 7) {
        const int lx = std::atoi(argv[2]);
        const double p = std::atof(argv[3]), q = std::atof(argv[4]);
        const int seed = std::atoi(argv[5]);
        if (cmd == "scabitcurve")
            return curve<Kpz::SchedulerSCABit<SLCG64>>(lx, p, q, seed, argv + 6, argc - 6,
                                                       Kpz::SchedulerService::ENC_CBBIT);
        if (cmd == "db4curve")
            return curve<Kpz::Scheduler<SLCG64, Kpz::Scheduler_LocalLayoutDefault>>(
                lx, p, q, seed, argv + 6, argc - 6, Kpz::SchedulerService::ENC_LOCAL);
        return curve<Kpz::SchedulerDT<SLCG64, Kpz::SchedulerDT_LocalLayoutDis>>(lx, p, q, seed, argv + 6, argc - 6,
                                                                              Kpz::SchedulerService::ENC_LOCAL);
    }
    std::cerr << "unknown command " << cmd << "\n";
    return 2;
}
