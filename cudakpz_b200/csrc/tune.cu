// tune.cu -- autotuner for the SCABit pass shape (MCS per HBM pass, CTAs per SM).
//
// Every shape produces bit-identical lattices (the random stream is indexed by site and
// half-step, not by thread), so the tuner is free to time real passes on scratch copies of
// the lattice and keep the fastest.  Results are cached per (lattice size, rate class,
// SM count) in memory and, when KPZB_TUNE_CACHE names a file, in that file
// (one "key kind k cps ms_per_mcs band" line per entry).
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "kpzb_api_internal.h"
#include "kpzb_common.cuh"
#include "kpzb_internal.h"

namespace kpzb {

namespace {
std::mutex g_mu;
std::map<std::string, Plan> g_plans;
bool g_file_loaded = false;

std::string plan_key(int lx, int ly, uint64_t Tp, uint64_t Tq, int sm_count)
{
    // rates enter the cost only through the number of random planes the decision needs
    const Thresh a = make_thresh(Tp), b = make_thresh(Tq);
    const int planes = a.planes > b.planes ? a.planes : b.planes;
    const int pclass = planes == 0 ? 0 : planes == 1 ? 1 : planes <= 4 ? 2 : 3;
    char buf[96];
    snprintf(buf, sizeof buf, "scabit4:%d:%d:rng%d:sm%d", lx, ly, pclass, sm_count);
    return buf;
}

void load_file()
{
    if (g_file_loaded) return;
    g_file_loaded = true;
    const char* path = getenv("KPZB_TUNE_CACHE");
    if (!path) return;
    FILE* f = fopen(path, "r");
    if (!f) return;
    char key[96];
    int kind, k, cps, band;
    float ms;
    while (fscanf(f, "%95s %d %d %d %f %d", key, &kind, &k, &cps, &ms, &band) == 6)
        g_plans[key] = Plan{k, cps, ms, true, kind, band};
    fclose(f);
}

void save_file()
{
    const char* path = getenv("KPZB_TUNE_CACHE");
    if (!path) return;
    FILE* f = fopen(path, "w");
    if (!f) return;
    for (const auto& kv : g_plans)
        fprintf(f, "%s %d %d %d %.6f %d\n", kv.first.c_str(), kv.second.kind, kv.second.k, kv.second.cps,
                kv.second.ms_per_mcs, kv.second.band);
    fclose(f);
}
}  // namespace

bool lookup_plan(int lx, int ly, uint64_t Tp, uint64_t Tq, int sm_count, Plan* out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    load_file();
    auto it = g_plans.find(plan_key(lx, ly, Tp, Tq, sm_count));
    if (it == g_plans.end()) return false;
    *out = it->second;
    return true;
}

Plan default_plan(int lx, int ly, uint64_t Tp, uint64_t Tq, int sm_count)
{
    // without measuring: the warp-tile kernel for rates of at most one random plane, in the
    // shapes measured fastest at 16384^2 on a B200 (8 MCS per pass and 128-row tiles without a
    // random plane, 4 MCS and 56-row tiles with one), else the band heuristic
    (void)sm_count;
    const int mode = dec_mode(make_thresh(Tp), make_thresh(Tq));
    if (mode == DEC_NONE && scabit_strip_shape(lx, ly, 8, 128, mode).ok) return Plan{8, 0, 0.f, false, PASS_STRIP, 128};
    if (mode == DEC_ONE && scabit_strip_shape(lx, ly, 4, 56, mode).ok) return Plan{4, 0, 0.f, false, PASS_STRIP, 56};
    const int k = auto_fusion(lx, ly);
    return Plan{k, 0, 0.f, false, PASS_BAND};
}

Plan explicit_plan(int lx, int ly, int k, int sm_count)
{
    const char* env = getenv("KPZB_PASS_KERNEL");
    const std::string v = env ? env : "";
    if (k <= 1 || v == "band") return Plan{k, 0, 0.f, false, PASS_BAND};
    // "band1" .. "band3": the band kernel with that CTAs-per-SM choice (the tuner's candidates)
    if (v.size() == 5 && v.compare(0, 4, "band") == 0 && v[4] >= '1' && v[4] <= '3')
        return Plan{k, v[4] - '0', 0.f, false, PASS_BAND};
    if (v.compare(0, 5, "strip") == 0) {
        const int band = v.size() > 5 ? atoi(v.c_str() + 5) : 64;
        Plan p{k, 0, 0.f, false, PASS_STRIP, band};
        if (scabit_strip_shape(lx, ly, k, band, DEC_NONE).ok) return p;
        return Plan{k, 0, 0.f, false, PASS_BAND};
    }
    if (v.compare(0, 4, "wave") == 0) {
        const int cps = v.size() > 4 ? v[4] - '0' : 2;
        if (scabit_wave_shape(lx, ly, k, sm_count, cps, DEC_NONE).ok) return Plan{k, cps, 0.f, false, PASS_WAVE};
        return Plan{k, 0, 0.f, false, PASS_BAND};
    }
    const int cps = v == "stream2" ? 2 : 1;
    if (scabit_stream_shape(lx, ly, k, sm_count, cps).ok) return Plan{k, cps, 0.f, false, PASS_STREAM};
    return Plan{k, 0, 0.f, false, PASS_BAND};
}

bool plan_shape_ok(const Plan& p, int lx, int ly, int sm_count)
{
    if (p.k <= 1) return true;
    if (p.kind == PASS_STREAM) return scabit_stream_shape(lx, ly, p.k, sm_count, p.cps ? p.cps : 1).ok;
    if (p.kind == PASS_WAVE) return scabit_wave_shape(lx, ly, p.k, sm_count, p.cps, DEC_NONE).ok;
    if (p.kind == PASS_STRIP) return scabit_strip_shape(lx, ly, p.k, p.band, DEC_NONE).ok;
    return scabit_fused_shape_cps(lx, ly, p.k, p.cps, 0).ok;
}

cudaError_t tune_plan(uint32_t* d_src, int lx, int ly, uint64_t seed, uint32_t stream_id,
                      uint64_t Tp, uint64_t Tq, int sm_count, unsigned int* d_err,
                      cudaStream_t st, Plan* out)
{
    const size_t bytes = (size_t)1 << (lx + ly - 2);
    uint32_t *a = nullptr, *b = nullptr;
    cudaError_t e;
    if ((e = cudaMallocAsync(&a, bytes, st)) != cudaSuccess) return e;
    if ((e = cudaMallocAsync(&b, bytes, st)) != cudaSuccess) {
        cudaFreeAsync(a, st);
        return e;
    }
    cudaMemcpyAsync(a, d_src, bytes, cudaMemcpyDeviceToDevice, st);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);

    struct Cand {
        int k, cps, kind, band;
    };
    const int mode = dec_mode(make_thresh(Tp), make_thresh(Tq));
    std::vector<Cand> cands{{1, 0, PASS_BAND, 0}};
    for (int k = 2; k <= 8; ++k)
        for (int cps = 1; cps <= 3; ++cps) {
            FusedShape f = scabit_fused_shape_cps(lx, ly, k, cps, 0);
            if (f.ok && f.band >= 2) cands.push_back({k, cps, PASS_BAND, 0});
            if (cps <= 2 && scabit_stream_shape(lx, ly, k, sm_count, cps).ok)
                cands.push_back({k, cps, PASS_STREAM, 0});
            if (scabit_wave_shape(lx, ly, k, sm_count, cps, mode).ok) cands.push_back({k, cps, PASS_WAVE, 0});
        }
    // the warp-tile kernel: depth x tile height (taller tiles recompute fewer halo rows, shorter
    // ones make more warps), heights that fill whole tick cycles; heights that leave the same
    // tiles as a shorter one are skipped
    for (int k = 4; k <= 8; k += 2) {
        int last_tiles = -1;
        for (int m = 2; m <= 12; ++m) {
            const int band = m * strip_cycle_rows(k) - 4 * k;
            if (band < 8) continue;
            const StripShape ps = scabit_strip_shape(lx, ly, k, band, mode);
            if (!ps.ok || ps.ntiles == last_tiles) continue;
            last_tiles = ps.ntiles;
            cands.push_back({k, 0, PASS_STRIP, band});
        }
    }
    Plan best{1, 0, 1e30f, true, PASS_BAND, 0};
    const ScabitShape hs = scabit_shape(lx, ly, sm_count);
    for (const Cand& c : cands) {
        // enough MCS per measurement to dwarf launch overhead, capped by lattice size
        const int target = (lx + ly >= 26) ? 16 : 32;
        auto run = [&](int mcs) -> cudaError_t {
            if (c.k == 1) {
                for (int m = 0; m < mcs; ++m)
                    for (int sg = 0; sg < 2; ++sg) {
                        cudaError_t r = scabit_half(a, lx, ly, sg, (uint32_t)(2 * m + sg), seed,
                                                    stream_id, Tp, Tq, hs, nullptr, st);
                        if (r != cudaSuccess) return r;
                    }
                return cudaSuccess;
            }
            const FusedShape f = scabit_fused_shape_cps(lx, ly, c.k, c.cps, 0);
            const StreamShape ss = scabit_stream_shape(lx, ly, c.k, sm_count, c.cps);
            const WaveShape ws = scabit_wave_shape(lx, ly, c.k, sm_count, c.cps, mode);
            const StripShape ps = scabit_strip_shape(lx, ly, c.k, c.band, mode);
            uint32_t *s = a, *d = b;
            for (int m = 0; m + c.k <= mcs; m += c.k) {
                cudaError_t r = c.kind == PASS_STRIP
                                    ? scabit_strip(s, d, lx, ly, (uint32_t)m, seed, stream_id, Tp, Tq, ps, nullptr, st)
                                : c.kind == PASS_STREAM
                                    ? scabit_stream(s, d, lx, ly, (uint32_t)m, seed, stream_id, Tp, Tq, ss,
                                                    nullptr, d_err, st)
                                : c.kind == PASS_WAVE
                                    ? scabit_wave(s, d, lx, ly, (uint32_t)m, seed, stream_id, Tp, Tq, ws, nullptr,
                                                  d_err, st)
                                    : scabit_fused(s, d, lx, ly, (uint32_t)m, seed, stream_id, Tp, Tq, f,
                                                   nullptr, d_err, st);
                if (r != cudaSuccess) return r;
                std::swap(s, d);
            }
            return cudaSuccess;
        };
        int mcs = c.k == 1 ? target / 2 : c.k * ((target + c.k - 1) / c.k);
        if ((e = run(c.k == 1 ? 1 : c.k)) != cudaSuccess) break;  // warm-up
        cudaEventRecord(e0, st);
        if ((e = run(mcs)) != cudaSuccess) break;
        cudaEventRecord(e1, st);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const float per = ms / (float)mcs;
        if (getenv("KPZB_TUNE_VERBOSE"))
            fprintf(stderr, "kpzb tune lx=%d ly=%d %s k=%d cps=%d band=%d: %.4f ms/MCS, %.1f upd/ns\n", lx, ly,
                    c.kind == PASS_STREAM  ? "stream"
                    : c.kind == PASS_WAVE  ? "wave"
                    : c.kind == PASS_STRIP ? "strip"
                                           : "band",
                    c.k, c.cps, c.band, per, (double)(1ull << (lx + ly)) / (per * 1e6));
        if (per < best.ms_per_mcs) best = Plan{c.k, c.cps, per, true, c.kind, c.band};
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(a, st);
    cudaFreeAsync(b, st);
    cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        load_file();
        g_plans[plan_key(lx, ly, Tp, Tq, sm_count)] = best;
        save_file();
    }
    *out = best;
    return cudaSuccess;
}

}  // namespace kpzb
