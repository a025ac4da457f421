// ref_driver.cpp -- command-line driver around the reference's own CPU code (CudaKpz),
// compiled with it by oracle/build_ref.py into oracle/_ref/kpz_ref.  TEST INFRASTRUCTURE
// ONLY: it produces golden vectors (tests/golden/) and times the reference CPU schedulers
// for bench.py's reference arm.  It never links into the product.
//
// Commands (lattice files are raw little-endian uint32 words in the reference layout):
//   rs LX SEED T1 [T2 ...] OUT      SchedulerCPU::mcs (kpz/schedulerCPU.cpp:35-38), flat ENC_LOCAL
//                                   start, supplySeed(1, SEED); prints "t W2 h1..h7" at each T;
//                                   writes the final lattice to OUT
//   cbbit LX P Q N IN|flat OUT THR  SchedulerCPUCBBit<TinyMT32>::mcsPQSyncRng(N) (ENC_CBBIT)
//   cb LX P Q N IN|flat OUT THR     SchedulerCPUCB<TinyMT32>::mcsPQSyncRng(N) (ENC_LOCAL SCA)
//   cbbit-inject LX P Q N IN|flat OUT SEED STREAM
//                                   SchedulerCPUCBBit::mcsPQSyncRng(N), its per-site path fed the
//                                   counter stream's decisions (ref_inject.cpp), one thread
//   rough ENC LX IN                 SchedulerService::roughness() (Correlator::roughnessThreaded)
//   corr ENC LX SNAP SYS            Correlator::set(SNAP) then Correlator::correlate() on SYS;
//                                   prints W2 h1..h7 ch cs
//   check ENC LX IN                 SchedulerService::consitencyCheck(); prints 1/0
//   bench-cbbit LX P Q N THR        time mcsPQSyncRng(N) of SchedulerCPUCBBit; prints upd/ns
//   bench-rs LX N                   time SchedulerCPU::mcs(N); prints upd/ns
//   bench-dtr LX P Q N THR          time SchedulerCPUDTr<TinyMT32>::mcsPQSyncRng(N) (the reference's
//                                   CPU double-tiling scheduler, kpz/schedulerCPUDTr.cpp); upd/ns
//   bench-corr LX THR               time one Correlator::correlate() (kpz/correlator.cpp, THR
//                                   threads) of an ENC_CBBIT lattice against a snapshot; seconds
//   savebit LX SEED N FILE [META]   SchedulerService::saveBit of the RS lattice after N MCS
//   rsdis LX SEED FILL N P0 Q0 P1 Q1 DISFILE LATFILE   generateDisorder2 + SchedulerCPU::mcsDisorder2
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "CPURngIface.h"
#include "correlator.h"
#include "schedulerCPU.h"
#include "schedulerCPUCB.h"
#include "schedulerCPUCBBit.h"
#include "schedulerCPUDTr.h"
#include "schedulerService.h"

extern "C" {
#include "kpz_oracle.h"
}
// ref_inject.cpp
int ref_cbbit_injected(int lx, double p, double q, int n, uint32_t* words, uint64_t seed, uint32_t stream,
                       uint64_t t0);

// The HDF5/libSplash and MPI entry points of SchedulerService are outside the hot path;
// the build strips their definitions, and these keep the vtables complete.
bool Kpz::SchedulerService::collectH5(splash::DataCollector*, const std::string&) { return false; }
bool Kpz::SchedulerService::retrieveH5(splash::DataCollector*, const std::string&) { return false; }

namespace {

std::vector<uint32_t> load(const char* path, size_t n)
{
    std::vector<uint32_t> v(n);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char*>(v.data()), n * 4);
    if ((size_t)f.gcount() != n * 4) {
        std::cerr << "short read " << path << "\n";
        std::exit(2);
    }
    return v;
}

void save(const char* path, const uint32_t* w, size_t n)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(w), n * 4);
}

void print_r(const Kpz::Roughness& r)
{
    std::cout << std::setprecision(17) << (double)r.w2;
    for (int k = 0; k < Kpz::Roughness::H_ORDERS; ++k) std::cout << ' ' << (double)r.h[k];
}

template <class S>
void setup(S& s, const char* in, Kpz::SchedulerService::Encoding enc)
{
    if (std::string(in) == "flat") {
        s.initHomogeneous(enc);
    } else {
        s.initHomogeneous(enc);
        auto v = load(in, s.size().sizeW());
        std::memcpy(s.system(), v.data(), v.size() * 4);
    }
    s.pushSystem();
}

double now()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

int main(int argc, char** argv)
{
    std::cout.setf(std::ios::unitbuf);
    if (argc < 2) {
        std::cerr << "usage: see header\n";
        return 2;
    }
    const std::string cmd = argv[1];
    // silence the reference's banners on stdout
    std::streambuf* keep = std::cout.rdbuf();
    std::ostringstream sink;
    auto quiet = [&]() { std::cout.rdbuf(sink.rdbuf()); };
    auto loud = [&]() { std::cout.rdbuf(keep); };

    if (cmd == "rs") {
        const int lx = std::atoi(argv[2]);
        const int seed = std::atoi(argv[3]);
        quiet();
        Kpz::SchedulerCPU s(lx, lx);
        s.supplySeed(1, seed);
        s.initHomogeneous(Kpz::SchedulerService::ENC_LOCAL);
        s.pushSystem();
        loud();
        int t = 0;
        for (int i = 4; i < argc - 1; ++i) {
            const int target = std::atoi(argv[i]);
            quiet();
            s.mcs(target - t);
            s.popSystem();
            loud();
            t = target;
            std::cout << t << ' ';
            print_r(s.roughness());
            std::cout << '\n';
        }
        save(argv[argc - 1], s.system(), s.size().sizeW());
        return 0;
    }
    if (cmd == "rsdis") {
        // generateDisorder2(fill) (kpz/schedulerService.cpp:54-71), then
        // SchedulerCPU::mcsDisorder2(N) (kpz/schedulerCPU.cpp:48-80) with classes 0 and 1
        const int lx = std::atoi(argv[2]);
        const int seed = std::atoi(argv[3]);
        const double fill = std::atof(argv[4]);
        const int n = std::atoi(argv[5]);
        const double p0 = std::atof(argv[6]), q0 = std::atof(argv[7]);
        const double p1 = std::atof(argv[8]), q1 = std::atof(argv[9]);
        quiet();
        Kpz::SchedulerCPU s(lx, lx);
        s.supplySeed(1, seed);
        s.initHomogeneous(Kpz::SchedulerService::ENC_LOCAL);
        s.pushSystem();
        s.generateDisorder2(fill);
        s.setPQ(p0, q0, 0);
        s.setPQ(p1, q1, 1);
        s.mcsDisorder2(n);
        s.popSystem();
        loud();
        save(argv[10], s.disorder(), s.size().sizeW());
        save(argv[11], s.system(), s.size().sizeW());
        return 0;
    }
    if (cmd == "savebit") {
        // SchedulerService::saveBit (kpz/schedulerService.cpp:389-401) of the RS lattice after N MCS
        const int lx = std::atoi(argv[2]);
        const int seed = std::atoi(argv[3]);
        const int n = std::atoi(argv[4]);
        quiet();
        Kpz::SchedulerCPU s(lx, lx);
        s.supplySeed(1, seed);
        s.initHomogeneous(Kpz::SchedulerService::ENC_LOCAL);
        s.pushSystem();
        s.mcs(n);
        s.popSystem();
        const bool ok = s.saveBit(argv[5], argc > 6 ? argv[6] : nullptr);
        loud();
        return ok ? 0 : 1;
    }
    if (cmd == "cbbit-inject" && argc >= 10) {
        const int lx = std::atoi(argv[2]);
        const double p = std::atof(argv[3]), q = std::atof(argv[4]);
        const int n = std::atoi(argv[5]);
        const size_t nw = (size_t)1 << (2 * lx - 4);
        std::vector<uint32_t> w(nw);
        if (std::string(argv[6]) == "flat")
            ko_init_homogeneous(w.data(), lx, lx, 1);
        else
            w = load(argv[6], nw);
        quiet();
        const int rc = ref_cbbit_injected(lx, p, q, n, w.data(), std::strtoull(argv[8], nullptr, 10),
                                          (uint32_t)std::strtoul(argv[9], nullptr, 10), 0);
        loud();
        if (rc != 0) {
            std::cerr << "cbbit-inject: rates not on the per-site path, or not separable in float\n";
            return 1;
        }
        save(argv[7], w.data(), nw);
        return 0;
    }
    if (cmd == "cbbit" || cmd == "cb") {
        const int lx = std::atoi(argv[2]);
        const double p = std::atof(argv[3]), q = std::atof(argv[4]);
        const int n = std::atoi(argv[5]);
        const int thr = argc > 8 ? std::atoi(argv[8]) : 1;
        quiet();
        if (cmd == "cbbit") {
            Kpz::SchedulerCPUCBBit<Kpz::RngIface::TinyMT32> s(lx, lx, thr);
            s.supplySeed(1, 1);
            s.randomize();
            setup(s, argv[6], Kpz::SchedulerService::ENC_CBBIT);
            s.setPQ(p, q);
            s.mcsPQSyncRng(n);
            s.popSystem();
            loud();
            save(argv[7], s.system(), s.size().sizeW());
        } else {
            Kpz::SchedulerCPUCB<Kpz::RngIface::TinyMT32> s(lx, lx, thr);
            s.supplySeed(1, 1);
            s.randomize();
            setup(s, argv[6], Kpz::SchedulerService::ENC_LOCAL);
            s.setPQ(p, q);
            s.mcsPQSyncRng(n);
            s.popSystem();
            loud();
            save(argv[7], s.system(), s.size().sizeW());
        }
        return 0;
    }
    if (cmd == "rough" || cmd == "check" || cmd == "corr") {
        const int enc = std::atoi(argv[2]);
        const int lx = std::atoi(argv[3]);
        quiet();
        Kpz::SchedulerCPU s(lx, lx);
        const auto e = enc ? Kpz::SchedulerService::ENC_CBBIT : Kpz::SchedulerService::ENC_LOCAL;
        s.initHomogeneous(e);
        // consitencyCheck divides by Correlator::nThreads(); setNThreads(n<=1) stores 0
        // (kpz/correlator.cpp:699-705, kpz/schedulerService.cpp:812-814)
        Kpz::Correlator::setNThreads(cmd == "check" ? 2 : 1);
        loud();
        if (cmd == "rough") {
            auto v = load(argv[4], s.size().sizeW());
            std::memcpy(s.system(), v.data(), v.size() * 4);
            print_r(s.roughness());
            std::cout << '\n';
        } else if (cmd == "check") {
            auto v = load(argv[4], s.size().sizeW());
            std::memcpy(s.system(), v.data(), v.size() * 4);
            quiet();
            const bool ok = s.consitencyCheck(false, sink);
            loud();
            std::cout << (ok ? 1 : 0) << '\n';
        } else {
            auto snap = load(argv[4], s.size().sizeW());
            auto sys = load(argv[5], s.size().sizeW());
            std::memcpy(s.system(), snap.data(), snap.size() * 4);
            Kpz::Correlator c(&s);
            c.set(0);
            std::memcpy(s.system(), sys.data(), sys.size() * 4);
            Kpz::Roughness r = c.correlate();
            print_r(r);
            std::cout << ' ' << std::setprecision(17) << c.ch() << ' ' << c.cs() << '\n';
        }
        return 0;
    }
    if (cmd == "dsfmt") {
        // dSFMT-19937 draws of the reference's vendored generator: SEED N [reseed]
        dsfmt_t d;
        dsfmt_init_gen_rand(&d, (uint32_t)std::atoi(argv[2]));
        if (argc > 4)
            for (int a = 0; a < 100000; ++a) dsfmt_genrand_close_open(&d);
        const int n = std::atoi(argv[3]);
        for (int i = 0; i < n; ++i)
            std::cout << std::setprecision(17) << dsfmt_genrand_close_open(&d) << '\n';
        return 0;
    }
    if (cmd == "bench-cbbit") {
        const int lx = std::atoi(argv[2]);
        const double p = std::atof(argv[3]), q = std::atof(argv[4]);
        const int n = std::atoi(argv[5]);
        const int thr = std::atoi(argv[6]);
        quiet();
        Kpz::SchedulerCPUCBBit<Kpz::RngIface::TinyMT32> s(lx, lx, thr);
        s.supplySeed(1, 1);
        s.randomize();
        s.initHomogeneous(Kpz::SchedulerService::ENC_CBBIT);
        s.pushSystem();
        s.setPQ(p, q);
        const double t0 = now();
        s.mcsPQSyncRng(n);
        const double t1 = now();
        loud();
        std::cout << std::setprecision(9) << (double)s.size().size() * n / ((t1 - t0) * 1e9) << ' '
                  << (t1 - t0) << '\n';
        return 0;
    }
    if (cmd == "bench-rs") {
        const int lx = std::atoi(argv[2]);
        const int n = std::atoi(argv[3]);
        quiet();
        Kpz::SchedulerCPU s(lx, lx);
        s.supplySeed(1, 1);
        s.initHomogeneous(Kpz::SchedulerService::ENC_LOCAL);
        s.pushSystem();
        const double t0 = now();
        s.mcs(n);
        const double t1 = now();
        loud();
        std::cout << std::setprecision(9) << (double)s.size().size() * n / ((t1 - t0) * 1e9) << ' '
                  << (t1 - t0) << '\n';
        return 0;
    }
    if (cmd == "bench-corr") {
        const int lx = std::atoi(argv[2]);
        const int thr = std::atoi(argv[3]);
        quiet();
        Kpz::SchedulerCPUCBBit<Kpz::RngIface::TinyMT32> s(lx, lx, thr);
        s.supplySeed(1, 1);
        s.randomize();
        s.initHomogeneous(Kpz::SchedulerService::ENC_CBBIT);
        s.pushSystem();
        s.setPQ(0.5, 0.5);
        s.mcsPQSyncRng(2);
        s.popSystem();
        Kpz::Correlator::setNThreads(thr);
        Kpz::Correlator c(&s);
        c.set(2);
        s.mcsPQSyncRng(1);
        s.popSystem();
        const double t0 = now();
        const Kpz::Roughness r = c.correlate();
        const double t1 = now();
        loud();
        std::cout << std::setprecision(9) << (t1 - t0) << ' ' << (double)r.w2 << '\n';
        return 0;
    }
    if (cmd == "bench-dtr") {
        const int lx = std::atoi(argv[2]);
        const double p = std::atof(argv[3]), q = std::atof(argv[4]);
        const int n = std::atoi(argv[5]);
        const int thr = std::atoi(argv[6]);
        quiet();
        Kpz::SchedulerCPUDTr<Kpz::RngIface::TinyMT32> s(lx, lx, thr);
        s.supplySeed(1, 1);
        s.randomize();
        s.initHomogeneous(Kpz::SchedulerService::ENC_LOCAL);
        s.pushSystem();
        s.setPQ(p, q);
        const double t0 = now();
        s.mcsPQSyncRng(n);
        const double t1 = now();
        loud();
        std::cout << std::setprecision(9) << (double)s.size().size() * n / ((t1 - t0) * 1e9) << ' '
                  << (t1 - t0) << '\n';
        return 0;
    }
    std::cerr << "unknown command " << cmd << "\n";
    return 2;
}
