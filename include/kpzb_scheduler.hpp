// kpzb_scheduler.hpp -- header-only C++ front end over the kpzb C ABI, with the member
// names and semantics of Kpz::SchedulerService (kpz/schedulerService.h:73-255) and the GPU
// schedulers SchedulerSCA / SchedulerSCABit / SchedulerDT (kpz/schedulerSCA.h,
// kpz/schedulerSCABit.h, kpz/schedulerDT.h).  Errors become kpzb::Error exceptions, as the
// reference throws KmcExcept::CUDAError (kpz/schedulerSCABit.cu:66-72); the C ABI itself
// never throws.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "kpzb.h"

namespace kpzb {

struct Error : std::runtime_error {
    kpzb_status status;
    Error(kpzb_status s, const std::string& where)
        : std::runtime_error(where + ": " + kpzb_last_error()), status(s) {}
};

inline void check(kpzb_status s, const char* where)
{
    if (s != KPZB_OK) throw Error(s, where);
}

// Kpz::Roughness (kpz/schedulerService.h:52-66): W^2 and <h^k>, k = 1..7.
struct Roughness {
    double w2 = 0;
    double h[7] = {0, 0, 0, 0, 0, 0, 0};
};

class Scheduler {
public:
    enum Encoding { ENC_LOCAL = KPZB_ENC_LOCAL, ENC_CBBIT = KPZB_ENC_CBBIT };
    enum Dynamics { SCA = KPZB_DYN_SCA, SCABIT = KPZB_DYN_SCABIT, DT = KPZB_DYN_DT, DB4 = KPZB_DYN_DB4 };

    Scheduler(int lx, int ly, Dynamics dyn = SCABIT, int device = -1) : dyn_(dyn)
    {
        check(kpzb_create(&h_, lx, ly, dyn, device), "kpzb_create");
        setPQDefault();
    }
    ~Scheduler() { kpzb_destroy(h_); }
    Scheduler(const Scheduler&) = delete;
    Scheduler& operator=(const Scheduler&) = delete;

    Encoding encoding() const { return (Encoding)kpzb_encoding(h_); }
    size_t sizeW() const { return kpzb_size_words(h_); }

    void initHomogeneous() { check(kpzb_init_homogeneous(h_), "kpzb_init_homogeneous"); }
    // SchedulerService::setPQ(p, q, n): n > 0 sets the rates of quenched-disorder class n
    bool setPQ(double p, double q, int n = 0)
    {
        if (n != 0) {
            check(kpzb_set_pq_class(h_, n, p, q), "kpzb_set_pq_class");
            return true;
        }
        check(kpzb_set_pq(h_, p, q), "kpzb_set_pq");
        p_ = p;
        q_ = q;
        return true;
    }
    // SchedulerService::m_disorder: rate-class words in ENC_LOCAL layout
    void setDisorder(const std::vector<uint32_t>& words)
    {
        if (words.size() != sizeW()) throw Error(KPZB_EINVAL, "setDisorder: one word per lattice word");
        check(kpzb_set_disorder(h_, words.data()), "kpzb_set_disorder");
    }
    // DT: the block-level decomposition (KPZB_DT_INNER_*; the reference's KPZ_INNER_DD)
    void setDtInner(int inner) { check(kpzb_set_dt_inner(h_, inner), "kpzb_set_dt_inner"); }
    // SchedulerService::mcsScale (kpz/schedulerService.h:241)
    double mcsScale() const
    {
        double s = 1.0;
        check(kpzb_mcs_scale(h_, &s), "kpzb_mcs_scale");
        return s;
    }
    double rateP() const { return p_; }
    double rateQ() const { return q_; }
    void supplySeed(uint64_t seed, uint32_t stream = 0) { check(kpzb_seed(h_, seed, stream), "kpzb_seed"); }

    // dynamics (kpz/schedulerService.h:199-215)
    void mcsPQSyncRng(int n)
    {
        check(kpzb_mcs(h_, n), "kpzb_mcs");
        mcs_ += (unsigned)n;
    }
    void mcsPQ(int n) { mcsPQSyncRng(n); }
    void mcsSyncRng(int n)
    {
        setPQDefault();
        mcsPQSyncRng(n);
    }
    void mcs(int n) { mcsSyncRng(n); }
    void mcsPQSyncRngAsync(int n)
    {
        check(kpzb_mcs_async(h_, n), "kpzb_mcs_async");
        mcs_ += (unsigned)n;
    }
    void join() { check(kpzb_join(h_), "kpzb_join"); }
    void mcsDisorder2SyncRng(int n)
    {
        check(kpzb_mcs_disorder(h_, n), "kpzb_mcs_disorder");
        mcs_ += (unsigned)n;
    }

    // SchedulerService::saveBit (kpz/schedulerService.cpp:389-401) plus the resume trailer
    bool saveBit(const char* file, const char* meta = nullptr)
    {
        check(kpzb_save(h_, file, meta), "kpzb_save");
        return true;
    }
    bool loadBit(const char* file)
    {
        check(kpzb_load(h_, file), "kpzb_load");
        mcs_ = (unsigned)deviceMcs();
        return true;
    }

    // the frontend's measurement loop (kpz/kpzScaling.cpp:194-215) with device-side analysis:
    // rows of {t, W^2, <h^1..7>, ch, cs}
    std::vector<double> measureRun(uint64_t end, const kpzb_sampling& s, int64_t corrStart = -1,
                                   uint64_t corrStop = 0)
    {
        int n = 0;
        kpzb_status st = kpzb_measure_run(h_, &s, end, corrStart, corrStop, nullptr, 0, &n);
        if (st != KPZB_OK && n == 0) check(st, "kpzb_measure_run");
        std::vector<double> rows((size_t)n * 11);
        check(kpzb_measure_run(h_, &s, end, corrStart, corrStop, rows.data(), n, &n), "kpzb_measure_run");
        mcs_ = (unsigned)end;
        return rows;
    }

    // host copy (kpz/schedulerBase.cu:35-52), in the encoding of encoding()
    std::vector<uint32_t>& system() { return host_; }
    void pushSystem() { check(kpzb_push(h_, host_.data()), "kpzb_push"); }
    void popSystem()
    {
        host_.resize(sizeW());
        check(kpzb_pop(h_, host_.data()), "kpzb_pop");
    }

    // asynchronous copies from / to a caller's buffer of sizeW() words (page-locked for the
    // copies to overlap queued work), valid until join(); the reference copies synchronously
    // after join() and has no counterpart
    void pushSystemAsync(const uint32_t* words) { check(kpzb_push_async(h_, words), "kpzb_push_async"); }
    void popSystemAsync(uint32_t* words) { check(kpzb_pop_async(h_, words), "kpzb_pop_async"); }

    Roughness roughness()
    {
        double o[8];
        check(kpzb_roughness(h_, o), "kpzb_roughness");
        return toR(o);
    }
    // SchedulerService::roughnessAsync / joinRoughness
    void roughnessAsync() { check(kpzb_roughness_async(h_), "kpzb_roughness_async"); }
    Roughness joinRoughness()
    {
        double o[8];
        check(kpzb_roughness_join(h_, o), "kpzb_roughness_join");
        return toR(o);
    }
    Roughness correlateTag()
    {
        double o[8];
        check(kpzb_corr_tag(h_, o), "kpzb_corr_tag");
        return toR(o);
    }
    // Correlator::correlate: roughness of the current lattice plus ch, cs
    Roughness correlate(double* ch, double* cs)
    {
        double o[10];
        check(kpzb_correlate(h_, o), "kpzb_correlate");
        if (ch) *ch = o[8];
        if (cs) *cs = o[9];
        return toR(o);
    }
    bool consitencyCheck()
    {
        int64_t rep[3];
        check(kpzb_check_invariants(h_, rep), "kpzb_check_invariants");
        return rep[0] == 0 && rep[1] == 0 && rep[2] == 0;
    }

    unsigned int mcs() const { return mcs_; }
    void setMcs(unsigned int m) { mcs_ = m; }
    uint64_t deviceMcs() const
    {
        uint64_t t = 0;
        check(kpzb_get_mcs(h_, &t), "kpzb_get_mcs");
        return t;
    }
    kpzb_handle* handle() { return h_; }

private:
    // setPQDefault of each scheduler (kpz/schedulerSCA.h:37-39, kpz/schedulerSCABit.h:35-37);
    // SchedulerDT::mcs and Scheduler (DB4)::mcs run the p=1, q=0 core (kpz/kpz.cu:157-162,208-216)
    void setPQDefault()
    {
        if (dyn_ == SCA) setPQ(0.95, 0.0);
        else if (dyn_ == SCABIT) setPQ(0.5, 0.0);
        else setPQ(1.0, 0.0);
    }
    static Roughness toR(const double* o)
    {
        Roughness r;
        r.w2 = o[0];
        for (int k = 0; k < 7; ++k) r.h[k] = o[1 + k];
        return r;
    }

    kpzb_handle* h_ = nullptr;
    Dynamics dyn_;
    double p_ = 0, q_ = 0;
    unsigned int mcs_ = 0;
    std::vector<uint32_t> host_;
};

}  // namespace kpzb
