/*
 * kpz_oracle.h -- CPU restatement of the CudaKpz octahedron-model hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in
 * cudakpz_b200/: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load it.  The product never links or calls it.
 *
 * Everything here is plain, single-threaded C written from the reference's
 * behaviour (file:line citations are into the CudaKpz source tree):
 *   - lattice geometry / encodings        kpz/systemSize.h:94-165, kpz/lattice.h:29-95
 *   - flat start                          kpz/schedulerService.cpp:156-175
 *   - per-site octahedron rule            kpz/kpzSCACores.cu:121-144, kpz/schedulerCPUCBBit_nested.inl:261-295
 *   - SCA checkerboard order              kpz/schedulerSCABit.cu:46-73 (sublattice 0, then 1)
 *   - height walk / roughness             kpz/correlator.cpp:37-106, kpz/roughness.cpp:38-43
 *   - correlator ch / cs                  kpz/correlator.cpp:337-399, :463-477
 *   - consistency invariants              kpz/schedulerService.cpp:721-854
 *   - random-sequential CPU scheduler     kpz/schedulerCPU.inl:21-88, kpz/schedulerCPU.cpp:35-46
 *   - dSFMT-19937 (vendored, BSD)         inc/dSFMT/dSFMT.{h,cpp}, inc/dSFMT/dSFMT-params19937.h
 *
 * The counter-based random stream (shared specification with the CUDA path):
 *   Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), key = (seed lo, seed hi),
 *   counter = (qword >> 2, step, plane | tag << 8, stream), output word qword & 3.
 *   "qword" is the word index of a site inside its ENC_CBBIT quadrant,
 *   "step" = 2*t + sigma is the half-step index (t = device MCS count),
 *   plane k in [0,32) supplies bit (31-k) of the site's 32-bit uniform u.
 *   A site of bit b in that word has u = sum_k ((plane_k >> b) & 1) << (31-k).
 *   Local minimum flips iff u < T(p), local maximum iff u < T(q), with
 *   T(x) = min(2^32, ceil(x * 2^32)).
 */
#ifndef KPZ_ORACLE_H
#define KPZ_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KO_TAG_SCA 1u

/* ---- counter RNG ---- */
void ko_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
uint32_t ko_plane_word(uint64_t seed, uint32_t stream, uint32_t tag, uint32_t step,
                       uint32_t plane, uint64_t qword);
uint32_t ko_site_u(uint64_t seed, uint32_t stream, uint32_t tag, uint32_t step,
                   uint64_t qword, int bit);
uint64_t ko_threshold(double p);

/* ---- geometry ---- */
uint64_t ko_size_words(int lx, int ly);
/* ENC_LOCAL: bit0 = x-slope, bit1 = y-slope of site (x,y) */
int ko_local_get(const uint32_t* w, int lx, int x, int y);
void ko_local_flip(uint32_t* w, int lx, int x, int y, int bits);
/* ENC_CBBIT */
uint64_t ko_cbbit_xindex(int lx, int ly, int x, int y);
uint64_t ko_cbbit_yindex(int lx, int ly, int x, int y);
int ko_cbbit_get(const uint32_t* w, int lx, int ly, int x, int y);
void ko_init_homogeneous(uint32_t* w, int lx, int ly, int encoding);
void ko_local_to_cbbit(const uint32_t* local, uint32_t* cbbit, int lx, int ly);
void ko_cbbit_to_local(const uint32_t* cbbit, uint32_t* local, int lx, int ly);

/* ---- SCA (checkerboard) dynamics, per-site restatement ---- */
/* One half-step on sublattice sigma; returns #deposits in *dep, #desorptions in *des. */
void ko_sca_halfstep(uint32_t* w, int lx, int ly, int encoding, int sigma,
                     uint64_t seed, uint32_t stream, uint32_t step,
                     uint64_t Tp, uint64_t Tq, int64_t* dep, int64_t* des);
/* n MCS starting at device MCS count t0 (sublattice 0 then 1 each MCS). */
/* Quenched disorder (mcsDisorder2SyncRng): rate class c = the 2 bits of `dis` (ENC_LOCAL words,
 * SchedulerService::m_disorder's layout) at the site picks Tp[c] / Tq[c]; the random stream is
 * the same as without disorder. */
void ko_sca_halfstep_dis(uint32_t* w, int lx, int ly, int encoding, int sigma, uint64_t seed,
                         uint32_t stream, uint32_t step, const uint64_t Tp[4], const uint64_t Tq[4],
                         const uint32_t* dis, int64_t* dep, int64_t* des);
void ko_sca_mcs_dis(uint32_t* w, int lx, int ly, int encoding, uint64_t seed, uint32_t stream,
                    uint64_t t0, int n, const double p[4], const double q[4], const uint32_t* dis,
                    int64_t* dep, int64_t* des);
void ko_sca_mcs(uint32_t* w, int lx, int ly, int encoding, uint64_t seed, uint32_t stream,
                uint64_t t0, int n, double p, double q, int64_t* dep, int64_t* des);
/* The same n MCS on ENC_CBBIT words, 32 sites per word operation (same lattice and counts as
 * ko_sca_mcs with encoding ENC_CBBIT; fast enough for 16384^2 lattices). */
void ko_sca_mcs_words(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                      double p, double q, int64_t* dep, int64_t* des);

/* ---- heights, roughness, correlator ---- */
/* Relative heights along the reference's path walk; h is int32[2^(lx+ly)], row-major. */
void ko_heights(const uint32_t* w, int lx, int ly, int encoding, int32_t* h);
/* Exact power sums S_k = sum h^k, k = 1..7, as two's complement 128-bit (lo, hi) pairs. */
void ko_power_sums(const int32_t* h, uint64_t n, int64_t lo[7], int64_t hi[7]);
/* Reference-style roughness: out[0] = W^2, out[1..7] = <h^k> (long double accumulation). */
void ko_roughness(const uint32_t* w, int lx, int ly, int encoding, double out[8]);
/* Reference-style correlator of sys against snap: out[0..7] = roughness of sys,
 * out[8] = ch, out[9] = cs; snap_mean = <h_snap> from ko_roughness(snap). */
void ko_correlate(const uint32_t* sys, const uint32_t* snap, int lx, int ly, int encoding,
                  double snap_mean, double out[10]);
/* Consistency invariants: rep[0] = rows with nonzero x-sum, rep[1] = columns with nonzero
 * y-sum, rep[2] = plaquettes with nonzero loop. All zero for a valid lattice. */
void ko_check_invariants(const uint32_t* w, int lx, int ly, int encoding, int64_t rep[3]);

/* ---- double-tiling (DT) random-sequential dynamics, CPU emulation of the GPU scheme ----
 * Restates SchedulerDT::doMcs (kpz/schedulerDT.cu:65-78: random origin in [0, 2*block) and a
 * shuffled order of the 4 domain sets per MCS, kpz/kpzCopy.cu:144-187: block + halo tiles)
 * with the inner single-hit double tiling of KpzCores::BaseDT
 * (kpz/kpzSimulationPrimitivesTemplates.cu:110-141: per round one block-wide sub-cell, each
 * thread one attempt inside that quadrant of its thread cell), driven by the counter stream:
 *   origin/order : Philox(ctr=(0, t, TAG_DT_ORIGIN<<24, stream)) words 0,1,2
 *   sub-cells    : Philox(ctr=(block, t, TAG_DT_SUB<<24 | d<<16, stream)), 2 bits per round
 *   positions    : Philox(ctr=(cell, t, TAG_DT_POS<<24 | d<<16 | r>>5, stream)), 4 bits/round
 *   acceptance u : Philox(ctr=(cell, t, TAG_DT<<24 | d<<16 | r>>2, stream)), word r&3
 * Geometry: 32x16 threads, 8x8-site thread cells, blocks of 256x128 sites, 64 rounds per
 * launch (one attempt per site per MCS).  ENC_LOCAL lattice, lx >= 9, ly >= 8. */
#define KO_TAG_DT 2u
#define KO_TAG_DT_ORIGIN 3u
#define KO_TAG_DT_SUB 4u
#define KO_TAG_DT_POS 5u
void ko_dt_mcs(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
               double p, double q, int64_t* dep, int64_t* des);
void ko_dt_mcs_dis(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                   const double p[4], const double q[4], const uint32_t* dis, int64_t* dep, int64_t* des);
/* the same blocks and domain sets with the reference's default single-hit dead-border
 * inner scheme (DBSH) */
#define KO_TAG_DBSH_ORIGIN 7u
#define KO_TAG_DBSH_POS 8u
void ko_dt_mcs_dbsh(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                    const double p[4], const double q[4], const uint32_t* dis, int64_t* dep, int64_t* des);
/* the dead-border scheme without the per-round cell offset (DB) */
void ko_dt_mcs_db(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                  const double p[4], const double q[4], const uint32_t* dis, int64_t* dep, int64_t* des);
/* double tiling with a per-round block-wide offset of the thread cells (DTDBSH) */
void ko_dt_mcs_dtdbsh(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                      const double p[4], const double q[4], const uint32_t* dis, int64_t* dep, int64_t* des);
/* DBSH with border hits replaced by fresh attempts after the rounds (DBSHRep) */
#define KO_TAG_REP_ORIGIN 9u
#define KO_TAG_REP_POS 10u
#define KO_TAG_REP_U 11u
void ko_dt_mcs_dbshrep(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                       const double p[4], const double q[4], const uint32_t* dis, int64_t* dep, int64_t* des);
/* the DB4 scheduler: all 256x128 blocks per launch behind a 5-site dead border, 2 launches
 * of 32 BaseDT rounds per MCS; ENC_LOCAL lattice, lx >= 8, ly >= 7 */
#define KO_TAG_DB4_ORIGIN 12u
#define KO_TAG_DB4_SUB 13u
#define KO_TAG_DB4_POS 14u
#define KO_TAG_DB4_U 15u
void ko_db4_mcs(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n, double p,
                double q, int64_t* dep, int64_t* des);
/* the per-MCS origin (sites) and domain-set order used by ko_dt_mcs */
void ko_dt_plan(uint64_t seed, uint32_t stream, uint64_t t, int* ox, int* oy, int order[4]);

/* ---- random-sequential CPU scheduler with dSFMT-19937 ---- */
typedef struct ko_dsfmt ko_dsfmt;
size_t ko_dsfmt_size(void);
void ko_dsfmt_init(ko_dsfmt* s, uint32_t seed);
double ko_dsfmt_close_open(ko_dsfmt* s);
/* supplySeed(std, dsfmt) equivalent: init with seed, then discard 100000 draws. */
void ko_dsfmt_reseed(ko_dsfmt* s, uint32_t seed);
/* SchedulerCPU::mcs (p=1,q=0, 2 draws/attempt) if pq==0, mcsPQ (third draw only when
 * the site is active) if pq==1. ENC_LOCAL lattice. */
void ko_rs_mcs(uint32_t* w, int lx, int ly, ko_dsfmt* s, int n, int pq, double p, double q);
/* the same, also counting depositions and desorptions */
void ko_rs_mcs_count(uint32_t* w, int lx, int ly, ko_dsfmt* s, int n, int pq, double p, double q,
                     int64_t* dep, int64_t* des);
/* SchedulerService::generateDisorder2(fill) and SchedulerCPU::mcsDisorder2 with rate classes */
void ko_generate_disorder2(uint32_t* dis, int lx, int ly, ko_dsfmt* s, double fill);
void ko_rs_mcs_dis(uint32_t* w, int lx, int ly, ko_dsfmt* s, int n, const double p[4], const double q[4],
                   const uint32_t* dis, int64_t* dep, int64_t* des);

#ifdef __cplusplus
}
#endif
#endif
