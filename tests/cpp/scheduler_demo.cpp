// A SchedulerService-style client written against include/kpzb_scheduler.hpp, the way the
// reference's C++ frontend (kpz/kpzScaling.cpp:142-215) drives a scheduler: flat start,
// seed, MCS chunks, popSystem, roughness, correlate, consitencyCheck.
// Usage: scheduler_demo LX P Q SEED NMCS OUT.bin  -> prints "w2 h1 ch cs consistent"
#include <cstdio>
#include <cstdlib>

#include "kpzb_scheduler.hpp"

int main(int argc, char** argv)
{
    if (argc < 7) return 2;
    const int lx = std::atoi(argv[1]);
    const double p = std::atof(argv[2]), q = std::atof(argv[3]);
    const unsigned long long seed = std::strtoull(argv[4], nullptr, 10);
    const int n = std::atoi(argv[5]);
    try {
        kpzb::Scheduler s(lx, lx, kpzb::Scheduler::SCABIT, 0);
        s.initHomogeneous();
        s.setPQ(p, q);
        s.supplySeed(seed);
        s.mcsPQSyncRng(n / 2);
        s.correlateTag();
        s.mcsPQSyncRng(n - n / 2);
        double ch = 0, cs = 0;
        const kpzb::Roughness r = s.correlate(&ch, &cs);
        const bool ok = s.consitencyCheck();
        s.popSystem();
        FILE* f = std::fopen(argv[6], "wb");
        if (!f) return 3;
        std::fwrite(s.system().data(), 4, s.system().size(), f);
        std::fclose(f);
        std::printf("%.17g %.17g %.17g %.17g %d\n", r.w2, r.h[0], ch, cs, ok ? 1 : 0);
    } catch (const kpzb::Error& e) {
        std::fprintf(stderr, "kpzb error %d: %s\n", (int)e.status, e.what());
        return 1;
    }
    return 0;
}
