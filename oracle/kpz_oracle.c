/*
 * kpz_oracle.c -- CPU restatement of the CudaKpz hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker): loaded by tests/, by
 * __graft_entry__.smoke() and by bench.py's cpu_baseline leg, never by the
 * product library.  Each function cites the reference file:line it restates.
 * Written for clarity, not speed: per-site loops, full 32-plane uniforms.
 */
#include "kpz_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Philox4x32-10, from Salmon et al., "Parallel random numbers: as easy as   */
/* 1, 2, 3" (SC'11), section 3.2: Feistel-like rounds with two 32x32->64     */
/* multiplies, Weyl key schedule.                                            */
/* ------------------------------------------------------------------------ */
void ko_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

uint32_t ko_plane_word(uint64_t seed, uint32_t stream, uint32_t tag, uint32_t step,
                       uint32_t plane, uint64_t qword)
{
    uint32_t ctr[4] = {(uint32_t)(qword >> 2), step, plane | (tag << 8), stream};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t out[4];
    ko_philox4x32_10(ctr, key, out);
    return out[qword & 3];
}

uint32_t ko_site_u(uint64_t seed, uint32_t stream, uint32_t tag, uint32_t step,
                   uint64_t qword, int bit)
{
    uint32_t u = 0;
    for (uint32_t k = 0; k < 32; ++k) {
        uint32_t w = ko_plane_word(seed, stream, tag, step, k, qword);
        u |= ((w >> bit) & 1u) << (31 - k);
    }
    return u;
}

uint64_t ko_threshold(double p)
{
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return (uint64_t)1 << 32;
    double t = ceil(p * 4294967296.0);
    if (t >= 4294967296.0) return (uint64_t)1 << 32;
    return (uint64_t)t;
}

/* ------------------------------------------------------------------------ */
/* Geometry: kpz/systemSize.h:94-165                                         */
/* ------------------------------------------------------------------------ */
uint64_t ko_size_words(int lx, int ly) { return (uint64_t)1 << (lx + ly - 4); }

/* index(x,y) = (y>>2 << lDimXW) + (x>>2); shift = ((x&3)<<1)|((y&3)<<3)   (systemSize.h:94-100) */
static inline uint64_t local_index(int lx, int x, int y)
{
    return ((uint64_t)(y >> 2) << (lx - 2)) + (uint64_t)(x >> 2);
}
static inline int local_shift(int x, int y) { return ((x & 3) << 1) | ((y & 3) << 3); }

int ko_local_get(const uint32_t* w, int lx, int x, int y)
{
    return (int)((w[local_index(lx, x, y)] >> local_shift(x, y)) & 3u);
}

void ko_local_flip(uint32_t* w, int lx, int x, int y, int bits)
{
    w[local_index(lx, x, y)] ^= (uint32_t)bits << local_shift(x, y);
}

/* quadrantIndex_CBBit = (y << (lDimX-6)) + (x >> 6); sublattice = (x^y)&1;
 * X quadrant base = sublattice * sizeW/2, Y base = sublattice*sizeW/2 + sizeW/4;
 * bit = (x>>1)&31   (systemSize.h:143-165) */
uint64_t ko_cbbit_xindex(int lx, int ly, int x, int y)
{
    uint64_t sw = ko_size_words(lx, ly);
    uint64_t qi = ((uint64_t)y << (lx - 6)) + (uint64_t)(x >> 6);
    return qi + (((x ^ y) & 1) ? (sw >> 1) : 0);
}
uint64_t ko_cbbit_yindex(int lx, int ly, int x, int y)
{
    return ko_cbbit_xindex(lx, ly, x, y) + (ko_size_words(lx, ly) >> 2);
}
int ko_cbbit_get(const uint32_t* w, int lx, int ly, int x, int y)
{
    int b = (x >> 1) & 31;
    int sx = (int)((w[ko_cbbit_xindex(lx, ly, x, y)] >> b) & 1u);
    int sy = (int)((w[ko_cbbit_yindex(lx, ly, x, y)] >> b) & 1u);
    return sx | (sy << 1);
}
static void cbbit_flip(uint32_t* w, int lx, int ly, int x, int y, int bits)
{
    int b = (x >> 1) & 31;
    if (bits & 1) w[ko_cbbit_xindex(lx, ly, x, y)] ^= 1u << b;
    if (bits & 2) w[ko_cbbit_yindex(lx, ly, x, y)] ^= 1u << b;
}

/* kpz/schedulerService.cpp:156-175 */
void ko_init_homogeneous(uint32_t* w, int lx, int ly, int encoding)
{
    uint64_t sw = ko_size_words(lx, ly);
    if (encoding == 0) {
        for (uint64_t i = 0; i < sw; ++i) w[i] = 0x33CC33CCu;
    } else {
        for (uint64_t i = 0; i < sw / 2; ++i) w[i] = 0u;
        for (uint64_t i = sw / 2; i < sw; ++i) w[i] = 0xFFFFFFFFu;
    }
}

void ko_local_to_cbbit(const uint32_t* local, uint32_t* cbbit, int lx, int ly)
{
    memset(cbbit, 0, ko_size_words(lx, ly) * 4);
    int L = 1 << lx, M = 1 << ly;
    for (int y = 0; y < M; ++y)
        for (int x = 0; x < L; ++x) {
            int v = ko_local_get(local, lx, x, y);
            cbbit_flip(cbbit, lx, ly, x, y, v);
        }
}

void ko_cbbit_to_local(const uint32_t* cbbit, uint32_t* local, int lx, int ly)
{
    memset(local, 0, ko_size_words(lx, ly) * 4);
    int L = 1 << lx, M = 1 << ly;
    for (int y = 0; y < M; ++y)
        for (int x = 0; x < L; ++x) {
            int v = ko_cbbit_get(cbbit, lx, ly, x, y);
            ko_local_flip(local, lx, x, y, v);
        }
}

static int get_site(const uint32_t* w, int lx, int ly, int enc, int x, int y)
{
    return enc == 0 ? ko_local_get(w, lx, x, y) : ko_cbbit_get(w, lx, ly, x, y);
}
static void flip_site(uint32_t* w, int lx, int ly, int enc, int x, int y, int bits)
{
    if (enc == 0) ko_local_flip(w, lx, x, y, bits);
    else cbbit_flip(w, lx, ly, x, y, bits);
}

/* ------------------------------------------------------------------------ */
/* SCA half-step, per-site form of kpz/kpzSCACores.cu:121-144 and           */
/* kpz/schedulerCPUCBBit_nested.inl:261-295: config = c | s_x(x+1,y)<<2 |     */
/* s_y(x,y+1)<<3; 12 -> deposit with prob p, 3 -> desorb with prob q; a flip */
/* xors both bits of (x,y), the x-bit of (x+1,y) and the y-bit of (x,y+1).   */
/* All sites of one sublattice are independent, so loop order is free.     */
/* ------------------------------------------------------------------------ */
/* Half-step with per-site rate classes: class c = the 2 bits of dis (ENC_LOCAL words, the
 * layout of SchedulerService::m_disorder) at the site, or 0 when dis is NULL; thresholds
 * Tp[c], Tq[c] (Disorder2SyncRng::update, kpz/kpzSCACores.cu:238-261: the site's own disorder
 * bits pick DEVICE_CONST_DISORDER2_P/Q). */
void ko_sca_halfstep_dis(uint32_t* w, int lx, int ly, int encoding, int sigma, uint64_t seed,
                         uint32_t stream, uint32_t step, const uint64_t Tp[4], const uint64_t Tq[4],
                         const uint32_t* dis, int64_t* dep, int64_t* des)
{
    int L = 1 << lx, M = 1 << ly;
    int64_t nd = 0, nr = 0;
    for (int y = 0; y < M; ++y)
        for (int x = 0; x < L; ++x) {
            if (((x ^ y) & 1) != sigma) continue;
            int c = get_site(w, lx, ly, encoding, x, y);
            int r = get_site(w, lx, ly, encoding, (x + 1) & (L - 1), y) & 1;
            int l = (get_site(w, lx, ly, encoding, x, (y + 1) & (M - 1)) >> 1) & 1;
            int config = c | (r << 2) | (l << 3);
            int cls = dis ? ko_local_get(dis, lx, x, y) : 0;
            uint64_t T;
            if (config == 12) T = Tp[cls];
            else if (config == 3) T = Tq[cls];
            else continue;
            if (T == 0) continue;
            if (T < ((uint64_t)1 << 32)) {
                /* the site's uniform: CBBit quadrant word index and bit (systemSize.h:143-165) */
                uint64_t qword = ((uint64_t)y << (lx - 6)) + (uint64_t)(x >> 6);
                uint32_t u = ko_site_u(seed, stream, KO_TAG_SCA, step, qword, (x >> 1) & 31);
                if ((uint64_t)u >= T) continue;
            }
            flip_site(w, lx, ly, encoding, x, y, 3);
            flip_site(w, lx, ly, encoding, (x + 1) & (L - 1), y, 1);
            flip_site(w, lx, ly, encoding, x, (y + 1) & (M - 1), 2);
            if (config == 12) ++nd; else ++nr;
        }
    if (dep) *dep += nd;
    if (des) *des += nr;
}

void ko_sca_halfstep(uint32_t* w, int lx, int ly, int encoding, int sigma,
                     uint64_t seed, uint32_t stream, uint32_t step,
                     uint64_t Tp, uint64_t Tq, int64_t* dep, int64_t* des)
{
    const uint64_t P[4] = {Tp, Tp, Tp, Tp}, Q[4] = {Tq, Tq, Tq, Tq};
    ko_sca_halfstep_dis(w, lx, ly, encoding, sigma, seed, stream, step, P, Q, NULL, dep, des);
}

/* kpz/schedulerSCA.cu mcsDisorder2SyncRng: n MCS with rate classes p[c], q[c] */
void ko_sca_mcs_dis(uint32_t* w, int lx, int ly, int encoding, uint64_t seed, uint32_t stream,
                    uint64_t t0, int n, const double p[4], const double q[4], const uint32_t* dis,
                    int64_t* dep, int64_t* des)
{
    uint64_t Tp[4], Tq[4];
    for (int c = 0; c < 4; ++c) {
        Tp[c] = ko_threshold(p[c]);
        Tq[c] = ko_threshold(q[c]);
    }
    for (int i = 0; i < n; ++i) {
        uint64_t t = t0 + (uint64_t)i;
        for (int s = 0; s < 2; ++s)
            ko_sca_halfstep_dis(w, lx, ly, encoding, s, seed, stream, (uint32_t)(2 * t + s), Tp, Tq, dis,
                                dep, des);
    }
}

/* kpz/schedulerSCABit.cu:46-73 (caller(0); caller(1); per MCS) */
void ko_sca_mcs(uint32_t* w, int lx, int ly, int encoding, uint64_t seed, uint32_t stream,
                uint64_t t0, int n, double p, double q, int64_t* dep, int64_t* des)
{
    uint64_t Tp = ko_threshold(p), Tq = ko_threshold(q);
    for (int i = 0; i < n; ++i) {
        uint64_t t = t0 + (uint64_t)i;
        for (int s = 0; s < 2; ++s)
            ko_sca_halfstep(w, lx, ly, encoding, s, seed, stream, (uint32_t)(2 * t + s), Tp, Tq,
                            dep, des);
    }
}

/* ------------------------------------------------------------------------ */
/* Word-parallel form of the same dynamics on ENC_CBBIT words: 32 sites of   */
/* one sublattice per word, the mask algebra of kpz/kpzSCABitCores.cu:69-74, */
/* 139-145 on the geometry of kpz/kpzSCABit.cu:120-172 (row y of sublattice */
/* sigma reads the other sublattice's X word one bit to the right when x is */
/* odd, i.e. when (y ^ sigma) & 1; kpz/schedulerCPUCBBit_nested.inl:208-257 */
/* does the same 64 sites at a time).  The decision u < T is taken plane by  */
/* plane from the MSB over the words of ko_plane_word: a site is below T at  */
/* the first plane where its bit is 0 and T's is 1, above it where its bit  */
/* is 1 and T's 0; once T has no 1 bit left below the plane, sites still    */
/* equal can no longer fall below it.  Gives ko_sca_mcs's lattice and       */
/* counts for every rate (checked on the CPU), in a few seconds at 16384^2. */
/* ------------------------------------------------------------------------ */
static uint32_t words_below(uint32_t cand, uint64_t T, uint64_t seed, uint32_t stream, uint32_t step,
                            uint64_t qword, const uint32_t* plane_cache, int* planes_done)
{
    if (!cand || T == 0) return 0;
    if (T >= ((uint64_t)1 << 32)) return cand;
    uint32_t t = (uint32_t)T, lt = 0, eq = cand;
    for (int k = 0; k < 32 && eq; ++k) {
        uint32_t r;
        if (k < *planes_done) {
            r = plane_cache[k];
        } else {
            r = ko_plane_word(seed, stream, KO_TAG_SCA, step, (uint32_t)k, qword);
            ((uint32_t*)plane_cache)[k] = r;
            *planes_done = k + 1;
        }
        if ((t >> (31 - k)) & 1u) {
            lt |= eq & ~r;
            eq &= r;
        } else {
            eq &= ~r;
        }
        if ((t & (0xFFFFFFFFu >> (k + 1))) == 0 || k == 31) eq = 0; /* no 1 bit of T below plane k */
    }
    return lt;
}

void ko_sca_mcs_words(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                      double p, double q, int64_t* dep, int64_t* des)
{
    const uint64_t Tp = ko_threshold(p), Tq = ko_threshold(q);
    const uint64_t Q = (uint64_t)1 << (lx + ly - 6), Wr = (uint64_t)1 << (lx - 6), M = (uint64_t)1 << ly;
    int64_t nd = 0, nr = 0;
    for (int i = 0; i < n; ++i)
        for (int sigma = 0; sigma < 2; ++sigma) {
            const uint32_t step = (uint32_t)(2 * (t0 + (uint64_t)i) + (uint64_t)sigma);
            uint32_t* tXq = w + (uint64_t)(2 * sigma) * Q;
            uint32_t* tYq = tXq + Q;
            uint32_t* oXq = w + (uint64_t)(2 * (1 - sigma)) * Q;
            uint32_t* oYq = oXq + Q;
            for (uint64_t y = 0; y < M; ++y) {
                const int shifted = (int)((y ^ (uint64_t)sigma) & 1u);
                uint32_t* tX = tXq + y * Wr;
                uint32_t* tY = tYq + y * Wr;
                uint32_t* oX = oXq + y * Wr;
                uint32_t* oY = oYq + ((y + 1) & (M - 1)) * Wr;
                for (uint64_t j = 0; j < Wr; ++j) {
                    const uint64_t jn = (j + 1) & (Wr - 1);
                    const uint32_t xX = shifted ? (oX[j] >> 1) | (oX[jn] << 31) : oX[j];
                    const uint32_t cp = ~tX[j] & ~tY[j] & xX & oY[j];
                    const uint32_t cq = tX[j] & tY[j] & ~xX & ~oY[j];
                    uint32_t cache[32];
                    int done = 0;
                    const uint64_t qword = y * Wr + j;
                    const uint32_t m = words_below(cp, Tp, seed, stream, step, qword, cache, &done) |
                                       words_below(cq, Tq, seed, stream, step, qword, cache, &done);
                    if (!m) continue;
                    nd += __builtin_popcount(m & cp);
                    nr += __builtin_popcount(m & cq);
                    tX[j] ^= m;
                    tY[j] ^= m;
                    oY[j] ^= m;
                    if (shifted) {
                        oX[j] ^= m << 1;
                        oX[jn] ^= m >> 31;
                    } else {
                        oX[j] ^= m;
                    }
                }
            }
        }
    if (dep) *dep += nd;
    if (des) *des += nr;
}

/* ------------------------------------------------------------------------ */
/* Heights: kpz/correlator.cpp:47-96. Start of row y adds s_y(0,y); then     */
/* x = 1..L-1 adds s_x(x,y); then the wrap adds s_x(0,y) giving h(0,y).     */
/* h(0,y) is recorded last; the value carried into row y+1 is h(0,y).       */
/* ------------------------------------------------------------------------ */
void ko_heights(const uint32_t* w, int lx, int ly, int encoding, int32_t* h)
{
    int L = 1 << lx, M = 1 << ly;
    int32_t cur = 0;
    for (int y = 0; y < M; ++y) {
        int row = get_site(w, lx, ly, encoding, 0, y);
        cur += (row & 2) ? 1 : -1;
        for (int x = 1; x < L; ++x) {
            cur += (get_site(w, lx, ly, encoding, x, y) & 1) ? 1 : -1;
            h[(size_t)y * L + x] = cur;
        }
        cur += (row & 1) ? 1 : -1;
        h[(size_t)y * L] = cur;
    }
}

void ko_power_sums(const int32_t* h, uint64_t n, int64_t lo[7], int64_t hi[7])
{
    __int128 s[7] = {0, 0, 0, 0, 0, 0, 0};
    for (uint64_t i = 0; i < n; ++i) {
        __int128 v = h[i], a = v;
        for (int k = 0; k < 7; ++k) {
            s[k] += a;
            a *= v;
        }
    }
    for (int k = 0; k < 7; ++k) {
        unsigned __int128 u = (unsigned __int128)s[k];
        lo[k] = (int64_t)(uint64_t)u;
        hi[k] = (int64_t)(uint64_t)(u >> 64);
    }
}

/* Roughness::addH / normAndSetW2 (kpz/schedulerService.h:58-64, kpz/roughness.cpp:38-43):
 * long double accumulation of double-valued powers, then division by N. */
static void add_h(long double acc[7], double ph)
{
    acc[0] += ph;
    double a = ph;
    for (int k = 1; k < 7; ++k) acc[k] += (a *= ph);
}

void ko_roughness(const uint32_t* w, int lx, int ly, int encoding, double out[8])
{
    uint64_t n = (uint64_t)1 << (lx + ly);
    int32_t* h = (int32_t*)malloc(n * sizeof(int32_t));
    ko_heights(w, lx, ly, encoding, h);
    long double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    /* the reference visits x = 1..L-1 then x = 0 per row; same order here */
    int L = 1 << lx, M = 1 << ly;
    for (int y = 0; y < M; ++y) {
        for (int x = 1; x < L; ++x) add_h(acc, h[(size_t)y * L + x]);
        add_h(acc, h[(size_t)y * L]);
    }
    for (int k = 0; k < 7; ++k) acc[k] /= (long double)n;
    out[0] = (double)(acc[1] - acc[0] * acc[0]);
    for (int k = 0; k < 7; ++k) out[1 + k] = (double)acc[k];
    free(h);
}

/* Correlator::correlate (kpz/correlator.cpp:463-477) with CorrelateData::correlateCBBit /
 * correlateCO (:180-263, :337-399): ch = sum h_snap*h_sys / N - <h_sys><h_snap>,
 * cs = (number of equal slope bits - number of different slope bits) / N / 2. */
void ko_correlate(const uint32_t* sys, const uint32_t* snap, int lx, int ly, int encoding,
                  double snap_mean, double out[10])
{
    uint64_t n = (uint64_t)1 << (lx + ly);
    int L = 1 << lx, M = 1 << ly;
    int32_t* hs = (int32_t*)malloc(n * sizeof(int32_t));
    int32_t* ht = (int32_t*)malloc(n * sizeof(int32_t));
    ko_heights(sys, lx, ly, encoding, hs);
    ko_heights(snap, lx, ly, encoding, ht);
    long double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    double ch = 0.0;
    long long tcs = 0;
    for (int y = 0; y < M; ++y) {
        for (int xi = 1; xi <= L; ++xi) {
            int x = xi & (L - 1);
            size_t i = (size_t)y * L + x;
            add_h(acc, hs[i]);
            ch += ht[i] * (double)hs[i];
            int a = get_site(sys, lx, ly, encoding, x, y);
            int b = get_site(snap, lx, ly, encoding, x, y);
            tcs += ((a & 1) == (b & 1)) ? 1 : -1;
            tcs += ((a & 2) == (b & 2)) ? 1 : -1;
        }
    }
    for (int k = 0; k < 7; ++k) acc[k] /= (long double)n;
    out[0] = (double)(acc[1] - acc[0] * acc[0]);
    for (int k = 0; k < 7; ++k) out[1 + k] = (double)acc[k];
    out[8] = ch / (double)n - (double)acc[0] * snap_mean;
    out[9] = (double)tcs / (double)n / 2.0;
    free(hs);
    free(ht);
}

/* SchedulerService::consitencyCheckThread (kpz/schedulerService.cpp:733-810), for both
 * encodings: row sums of x-slopes, column sums of y-slopes, plaquette loops
 * s_x(x,y) - s_y(x,y) + s_y(x-1,y) - s_x(x,y-1) (as +-1) = 0. */
void ko_check_invariants(const uint32_t* w, int lx, int ly, int encoding, int64_t rep[3])
{
    int L = 1 << lx, M = 1 << ly;
    int64_t badrows = 0, badcols = 0, badloops = 0;
    int64_t* colsum = (int64_t*)calloc((size_t)L, sizeof(int64_t));
    for (int y = 0; y < M; ++y) {
        int64_t rs = 0;
        for (int x = 0; x < L; ++x) {
            int c = get_site(w, lx, ly, encoding, x, y);
            int sx = (c & 1) ? 1 : -1, sy = (c & 2) ? 1 : -1;
            rs += sx;
            colsum[x] += sy;
            int syl = (get_site(w, lx, ly, encoding, (x + L - 1) & (L - 1), y) & 2) ? 1 : -1;
            int sxd = (get_site(w, lx, ly, encoding, x, (y + M - 1) & (M - 1)) & 1) ? 1 : -1;
            if (sx - sy + syl - sxd != 0) ++badloops;
        }
        if (rs != 0) ++badrows;
    }
    for (int x = 0; x < L; ++x)
        if (colsum[x] != 0) ++badcols;
    free(colsum);
    rep[0] = badrows;
    rep[1] = badcols;
    rep[2] = badloops;
}

/* ------------------------------------------------------------------------ */
/* Double tiling: see kpz_oracle.h.  Block 256x128 sites, 32x16 thread cells */
/* of 8x8 sites, 64 rounds per launch.                                      */
/* ------------------------------------------------------------------------ */
static void philox_u32(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t out[4])
{
    uint32_t ctr[4] = {c0, c1, c2, c3};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    ko_philox4x32_10(ctr, key, out);
}

void ko_dt_plan(uint64_t seed, uint32_t stream, uint64_t t, int* ox, int* oy, int order[4])
{
    uint32_t r[4];
    philox_u32(seed, 0u, (uint32_t)t, KO_TAG_DT_ORIGIN << 24, stream, r);
    *ox = (int)(r[0] & 511u); /* [0, 2 * 256) sites */
    *oy = (int)(r[1] & 255u); /* [0, 2 * 128) sites */
    /* Kmc::Shuffle<4>::shuffle (inc/shuffle.h:76-90): RC4 key-schedule style swaps */
    uint32_t rnd = r[2];
    for (int a = 0; a < 4; ++a) order[a] = a;
    for (int a = 0; a < 4; ++a) {
        int i = (int)(rnd & 3u);
        int v = order[i];
        order[i] = order[a];
        order[a] = v;
        rnd >>= 2;
    }
}

void ko_dt_mcs(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
               double p, double q, int64_t* dep, int64_t* des)
{
    const double P[4] = {p, p, p, p}, Q[4] = {q, q, q, q};
    ko_dt_mcs_dis(w, lx, ly, seed, stream, t0, n, P, Q, NULL, dep, des);
}

void ko_dt_mcs_dis(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                   const double p[4], const double q[4], const uint32_t* dis, int64_t* dep, int64_t* des)
{
    const int L = 1 << lx, M = 1 << ly;
    const int BX = 256, BY = 128;
    const int nbx = L / (2 * BX), nby = M / (2 * BY);
    uint64_t Tpc[4], Tqc[4];
    for (int c = 0; c < 4; ++c) {
        Tpc[c] = ko_threshold(p[c]);
        Tqc[c] = ko_threshold(q[c]);
    }
    int64_t nd = 0, nr = 0;
    for (int i = 0; i < n; ++i) {
        const uint64_t t = t0 + (uint64_t)i;
        int ox, oy, order[4];
        ko_dt_plan(seed, stream, t, &ox, &oy, order);
        for (int a = 0; a < 4; ++a) {
            const int d = order[a];
            for (int b = 0; b < nbx * nby; ++b) {
                const int bx = b % nbx, by = b / nbx;
                const int X0 = ox + (2 * bx + (d & 1)) * BX;
                const int Y0 = oy + (2 * by + (d >> 1)) * BY;
                uint32_t sub[4];
                philox_u32(seed, (uint32_t)b, (uint32_t)t, (KO_TAG_DT_SUB << 24) | ((uint32_t)d << 16),
                           stream, sub);
                for (int r = 0; r < 64; ++r) {
                    const int s = (int)((sub[r >> 4] >> (2 * (r & 15))) & 3u);
                    for (int cell = 0; cell < 512; ++cell) {
                        const int tx = cell & 31, ty = cell >> 5;
                        const uint32_t cid = (uint32_t)b * 512u + (uint32_t)cell;
                        uint32_t pw[4];
                        philox_u32(seed, cid, (uint32_t)t,
                                   (KO_TAG_DT_POS << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 5),
                                   stream, pw);
                        const int pos = (int)((pw[(r & 31) >> 3] >> (4 * (r & 7))) & 15u);
                        const int x = (X0 + tx * 8 + (s & 1) * 4 + (pos & 3)) & (L - 1);
                        const int y = (Y0 + ty * 8 + (s >> 1) * 4 + (pos >> 2)) & (M - 1);
                        const int c = ko_local_get(w, lx, x, y);
                        const int rr = ko_local_get(w, lx, (x + 1) & (L - 1), y) & 1;
                        const int ll = (ko_local_get(w, lx, x, (y + 1) & (M - 1)) >> 1) & 1;
                        const int config = c | (rr << 2) | (ll << 3);
                        const int cls = dis ? ko_local_get(dis, lx, x, y) : 0;
                        uint64_t T;
                        if (config == 12) T = Tpc[cls];
                        else if (config == 3) T = Tqc[cls];
                        else continue;
                        if (T == 0) continue;
                        if (T < ((uint64_t)1 << 32)) {
                            uint32_t uw[4];
                            philox_u32(seed, cid, (uint32_t)t,
                                       (KO_TAG_DT << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 2),
                                       stream, uw);
                            if ((uint64_t)uw[r & 3] >= T) continue;
                        }
                        ko_local_flip(w, lx, x, y, 3);
                        ko_local_flip(w, lx, (x + 1) & (L - 1), y, 1);
                        ko_local_flip(w, lx, x, (y + 1) & (M - 1), 2);
                        if (config == 12) ++nd; else ++nr;
                    }
                }
            }
        }
    }
    if (dep) *dep += nd;
    if (des) *des += nr;
}

/* One attempt of the RS rule at global site (x, y) with acceptance word u (used only when
 * the threshold is strictly between 0 and 2^32); class from dis. */
static void dt_attempt(uint32_t* w, int lx, int ly, int x, int y, const uint64_t* Tpc, const uint64_t* Tqc,
                       const uint32_t* dis, uint32_t u, int64_t* nd, int64_t* nr)
{
    const int L = 1 << lx, M = 1 << ly;
    const int c = ko_local_get(w, lx, x, y);
    const int rr = ko_local_get(w, lx, (x + 1) & (L - 1), y) & 1;
    const int ll = (ko_local_get(w, lx, x, (y + 1) & (M - 1)) >> 1) & 1;
    const int config = c | (rr << 2) | (ll << 3);
    const int cls = dis ? ko_local_get(dis, lx, x, y) : 0;
    uint64_t T;
    if (config == 12) T = Tpc[cls];
    else if (config == 3) T = Tqc[cls];
    else return;
    if (T == 0) return;
    if (T < ((uint64_t)1 << 32) && (uint64_t)u >= T) return;
    ko_local_flip(w, lx, x, y, 3);
    ko_local_flip(w, lx, (x + 1) & (L - 1), y, 1);
    ko_local_flip(w, lx, x, (y + 1) & (M - 1), 2);
    if (config == 12) ++*nd; else ++*nr;
}

/* DT with the single-hit dead-border inner scheme of the reference's default DT build
 * (BaseDTInnerDBSH::systemLoopDC, kpz/kpzSimulationPrimitivesTemplates_BaseInnerDB.cu:110-163):
 * the same blocks, domain sets and origins as ko_dt_mcs_dis; inside a block, every round
 * shifts all 8x8 thread cells by one block-wide offset (ox_r, oy_r) in [0,8)^2, each thread
 * picks a site (px, py) in its shifted cell, sites on the cell's last column or row are
 * delayed: phase 0 interior sites, phase 1 border sites off the corner, phase 2 the corner.
 * Site coordinates in the block tile are taken modulo the block (256 x 128 sites measured
 * from the tile's first word), as the reference masks them (`x &= M_BLOCK_DIM_X`).
 * Counter stream: offset byte r&15 of Philox(ctr=(block, t, TAG_DBSH_ORIGIN<<24 | d<<16 |
 * r>>4, stream)) word (r&15)>>2 (bits 0-2 x, 3-5 y); the position byte the same from
 * (cell, t, TAG_DBSH_POS<<24 | d<<16 | r>>4); acceptance u as ko_dt_mcs_dis. */
static void dt_mcs_border(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                          const double p[4], const double q[4], const uint32_t* dis, int shift, int64_t* dep,
                          int64_t* des);

void ko_dt_mcs_dbsh(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                    const double p[4], const double q[4], const uint32_t* dis, int64_t* dep, int64_t* des)
{
    dt_mcs_border(w, lx, ly, seed, stream, t0, n, p, q, dis, 1, dep, des);
}

/* The dead-border scheme without the per-round shift of the cells (BaseDTInnerDB,
 * kpz/kpzSimulationPrimitivesTemplates_BaseInnerDB.cu:30-74): ko_dt_mcs_dbsh with offset 0. */
void ko_dt_mcs_db(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                  const double p[4], const double q[4], const uint32_t* dis, int64_t* dep, int64_t* des)
{
    dt_mcs_border(w, lx, ly, seed, stream, t0, n, p, q, dis, 0, dep, des);
}

static void dt_mcs_border(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                          const double p[4], const double q[4], const uint32_t* dis, int shift, int64_t* dep,
                          int64_t* des)
{
    const int L = 1 << lx, M = 1 << ly;
    const int BX = 256, BY = 128;
    const int nbx = L / (2 * BX), nby = M / (2 * BY);
    uint64_t Tpc[4], Tqc[4];
    for (int c = 0; c < 4; ++c) {
        Tpc[c] = ko_threshold(p[c]);
        Tqc[c] = ko_threshold(q[c]);
    }
    int64_t nd = 0, nr = 0;
    for (int i = 0; i < n; ++i) {
        const uint64_t t = t0 + (uint64_t)i;
        int ox, oy, order[4];
        ko_dt_plan(seed, stream, t, &ox, &oy, order);
        for (int a = 0; a < 4; ++a) {
            const int d = order[a];
            for (int b = 0; b < nbx * nby; ++b) {
                const int bx = b % nbx, by = b / nbx;
                const int X0 = ox + (2 * bx + (d & 1)) * BX;
                const int Y0 = oy + (2 * by + (d >> 1)) * BY;
                for (int r = 0; r < 64; ++r) {
                    uint32_t ow[4];
                    philox_u32(seed, (uint32_t)b, (uint32_t)t,
                               (KO_TAG_DBSH_ORIGIN << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 4), stream, ow);
                    const uint32_t ob = (ow[(r & 15) >> 2] >> (8 * (r & 3))) & 0xFFu;
                    const int orx = shift ? (int)(ob & 7u) : 0, ory = shift ? (int)((ob >> 3) & 7u) : 0;
                    for (int phase = 0; phase < 3; ++phase)
                        for (int cell = 0; cell < 512; ++cell) {
                            const int tx = cell & 31, ty = cell >> 5;
                            const uint32_t cid = (uint32_t)b * 512u + (uint32_t)cell;
                            uint32_t pw[4];
                            philox_u32(seed, cid, (uint32_t)t,
                                       (KO_TAG_DBSH_POS << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 4), stream,
                                       pw);
                            const uint32_t pb = (pw[(r & 15) >> 2] >> (8 * (r & 3))) & 0xFFu;
                            const int px = (int)(pb & 7u), py = (int)((pb >> 3) & 7u);
                            const int ph = (px == 7 && py == 7) ? 2 : (px == 7 || py == 7) ? 1 : 0;
                            if (ph != phase) continue;
                            const int xt = (tx * 8 + (X0 & 3) + px + orx) & (BX - 1);
                            const int yt = (ty * 8 + (Y0 & 3) + py + ory) & (BY - 1);
                            const int x = ((X0 & ~3) + xt) & (L - 1);
                            const int y = ((Y0 & ~3) + yt) & (M - 1);
                            uint32_t uw[4];
                            philox_u32(seed, cid, (uint32_t)t,
                                       (KO_TAG_DT << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 2), stream, uw);
                            dt_attempt(w, lx, ly, x, y, Tpc, Tqc, dis, uw[r & 3], &nd, &nr);
                        }
                }
            }
        }
    }
    if (dep) *dep += nd;
    if (des) *des += nr;
}

/* Single-hit double tiling with a block-wide random offset of the thread cells per round
 * (BaseDTInnerDTDBSH::systemLoopDC, kpz/kpzSimulationPrimitivesTemplates_BaseInnerDTr.cu:
 * 56-83): per round the DT sub-cell (as ko_dt_mcs_dis) and an offset (ox_r, oy_r) in [0,8)^2
 * (the DBSH offset byte of dt_mcs_border); the site's in-block coordinates wrap modulo the
 * block before the origin's in-word offset (X0 & 3) is added; positions and acceptance words
 * as ko_dt_mcs_dis. */
void ko_dt_mcs_dtdbsh(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                      const double p[4], const double q[4], const uint32_t* dis, int64_t* dep, int64_t* des)
{
    const int L = 1 << lx, M = 1 << ly;
    const int BX = 256, BY = 128;
    const int nbx = L / (2 * BX), nby = M / (2 * BY);
    uint64_t Tpc[4], Tqc[4];
    for (int c = 0; c < 4; ++c) {
        Tpc[c] = ko_threshold(p[c]);
        Tqc[c] = ko_threshold(q[c]);
    }
    int64_t nd = 0, nr = 0;
    for (int i = 0; i < n; ++i) {
        const uint64_t t = t0 + (uint64_t)i;
        int ox, oy, order[4];
        ko_dt_plan(seed, stream, t, &ox, &oy, order);
        for (int a = 0; a < 4; ++a) {
            const int d = order[a];
            for (int b = 0; b < nbx * nby; ++b) {
                const int bx = b % nbx, by = b / nbx;
                const int X0 = ox + (2 * bx + (d & 1)) * BX;
                const int Y0 = oy + (2 * by + (d >> 1)) * BY;
                uint32_t sub[4];
                philox_u32(seed, (uint32_t)b, (uint32_t)t, (KO_TAG_DT_SUB << 24) | ((uint32_t)d << 16), stream, sub);
                for (int r = 0; r < 64; ++r) {
                    const int s = (int)((sub[r >> 4] >> (2 * (r & 15))) & 3u);
                    uint32_t ow[4];
                    philox_u32(seed, (uint32_t)b, (uint32_t)t,
                               (KO_TAG_DBSH_ORIGIN << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 4), stream, ow);
                    const uint32_t ob = (ow[(r & 15) >> 2] >> (8 * (r & 3))) & 0xFFu;
                    const int orx = (int)(ob & 7u), ory = (int)((ob >> 3) & 7u);
                    for (int cell = 0; cell < 512; ++cell) {
                        const int tx = cell & 31, ty = cell >> 5;
                        const uint32_t cid = (uint32_t)b * 512u + (uint32_t)cell;
                        uint32_t pw[4], uw[4];
                        philox_u32(seed, cid, (uint32_t)t,
                                   (KO_TAG_DT_POS << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 5), stream, pw);
                        const int pos = (int)((pw[(r & 31) >> 3] >> (4 * (r & 7))) & 15u);
                        const int xt = ((tx * 8 + (s & 1) * 4 + (pos & 3) + orx) & (BX - 1)) + (X0 & 3);
                        const int yt = ((ty * 8 + (s >> 1) * 4 + (pos >> 2) + ory) & (BY - 1)) + (Y0 & 3);
                        const int x = ((X0 & ~3) + xt) & (L - 1);
                        const int y = ((Y0 & ~3) + yt) & (M - 1);
                        philox_u32(seed, cid, (uint32_t)t, (KO_TAG_DT << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 2),
                                   stream, uw);
                        dt_attempt(w, lx, ly, x, y, Tpc, Tqc, dis, uw[r & 3], &nd, &nr);
                    }
                }
            }
        }
    }
    if (dep) *dep += nd;
    if (des) *des += nr;
}

/* DBSH with out-of-sequence replaced borders (BaseDTInnerDBSHRep::systemLoopDC,
 * kpz/kpzSimulationPrimitivesTemplates_BaseInnerDB.cu:184-268): the 64 rounds of
 * dt_mcs_border, but a site on its shifted cell's last column or row is not updated; each
 * thread counts such hits.  The block then makes R fresh attempts, where R is formed as the
 * reference's reduction forms it (:214-227): thread 0's own count plus the counts of threads
 * 32..511 (the hits of threads 1..31 are not repeated).  Repetition round k (512 attempts,
 * thread c active while 512k + c < R) draws a new block offset, a new position per active
 * thread and runs the three phases of dt_mcs_border.  Counter stream of the repetition:
 * offset byte k&15 of Philox(ctr=(block, t, TAG_REP_ORIGIN<<24 | d<<16 | k>>4, stream)),
 * position byte k&15 of (cell, t, TAG_REP_POS<<24 | d<<16 | k>>4), acceptance word k&3 of
 * (cell, t, TAG_REP_U<<24 | d<<16 | k>>2). */
void ko_dt_mcs_dbshrep(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n,
                       const double p[4], const double q[4], const uint32_t* dis, int64_t* dep, int64_t* des)
{
    const int L = 1 << lx, M = 1 << ly;
    const int BX = 256, BY = 128;
    const int nbx = L / (2 * BX), nby = M / (2 * BY);
    uint64_t Tpc[4], Tqc[4];
    for (int c = 0; c < 4; ++c) {
        Tpc[c] = ko_threshold(p[c]);
        Tqc[c] = ko_threshold(q[c]);
    }
    int64_t nd = 0, nr = 0;
    uint32_t hits[512];
    for (int i = 0; i < n; ++i) {
        const uint64_t t = t0 + (uint64_t)i;
        int ox, oy, order[4];
        ko_dt_plan(seed, stream, t, &ox, &oy, order);
        for (int a = 0; a < 4; ++a) {
            const int d = order[a];
            for (int b = 0; b < nbx * nby; ++b) {
                const int bx = b % nbx, by = b / nbx;
                const int X0 = ox + (2 * bx + (d & 1)) * BX;
                const int Y0 = oy + (2 * by + (d >> 1)) * BY;
                for (int c = 0; c < 512; ++c) hits[c] = 0;
                for (int r = 0; r < 64; ++r) {
                    uint32_t ow[4];
                    philox_u32(seed, (uint32_t)b, (uint32_t)t,
                               (KO_TAG_DBSH_ORIGIN << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 4), stream, ow);
                    const uint32_t ob = (ow[(r & 15) >> 2] >> (8 * (r & 3))) & 0xFFu;
                    for (int cell = 0; cell < 512; ++cell) {
                        const int tx = cell & 31, ty = cell >> 5;
                        const uint32_t cid = (uint32_t)b * 512u + (uint32_t)cell;
                        uint32_t pw[4], uw[4];
                        philox_u32(seed, cid, (uint32_t)t,
                                   (KO_TAG_DBSH_POS << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 4), stream, pw);
                        const uint32_t pb = (pw[(r & 15) >> 2] >> (8 * (r & 3))) & 0xFFu;
                        const int px = (int)(pb & 7u), py = (int)((pb >> 3) & 7u);
                        if (px == 7 || py == 7) {
                            ++hits[cell];
                            continue;
                        }
                        const int xt = (tx * 8 + (X0 & 3) + px + (int)(ob & 7u)) & (BX - 1);
                        const int yt = (ty * 8 + (Y0 & 3) + py + (int)((ob >> 3) & 7u)) & (BY - 1);
                        philox_u32(seed, cid, (uint32_t)t, (KO_TAG_DT << 24) | ((uint32_t)d << 16) | (uint32_t)(r >> 2),
                                   stream, uw);
                        dt_attempt(w, lx, ly, ((X0 & ~3) + xt) & (L - 1), ((Y0 & ~3) + yt) & (M - 1), Tpc, Tqc, dis,
                                   uw[r & 3], &nd, &nr);
                    }
                }
                uint32_t R = hits[0];
                for (int c = 32; c < 512; ++c) R += hits[c];
                for (int k = 0; k * 512 < (int)R; ++k) {
                    uint32_t ow[4];
                    philox_u32(seed, (uint32_t)b, (uint32_t)t,
                               (KO_TAG_REP_ORIGIN << 24) | ((uint32_t)d << 16) | (uint32_t)(k >> 4), stream, ow);
                    const uint32_t ob = (ow[(k & 15) >> 2] >> (8 * (k & 3))) & 0xFFu;
                    for (int phase = 0; phase < 3; ++phase)
                        for (int cell = 0; cell < 512 && k * 512 + cell < (int)R; ++cell) {
                            const int tx = cell & 31, ty = cell >> 5;
                            const uint32_t cid = (uint32_t)b * 512u + (uint32_t)cell;
                            uint32_t pw[4], uw[4];
                            philox_u32(seed, cid, (uint32_t)t,
                                       (KO_TAG_REP_POS << 24) | ((uint32_t)d << 16) | (uint32_t)(k >> 4), stream, pw);
                            const uint32_t pb = (pw[(k & 15) >> 2] >> (8 * (k & 3))) & 0xFFu;
                            const int px = (int)(pb & 7u), py = (int)((pb >> 3) & 7u);
                            const int ph = (px == 7 && py == 7) ? 2 : (px == 7 || py == 7) ? 1 : 0;
                            if (ph != phase) continue;
                            const int xt = (tx * 8 + (X0 & 3) + px + (int)(ob & 7u)) & (BX - 1);
                            const int yt = (ty * 8 + (Y0 & 3) + py + (int)((ob >> 3) & 7u)) & (BY - 1);
                            philox_u32(seed, cid, (uint32_t)t,
                                       (KO_TAG_REP_U << 24) | ((uint32_t)d << 16) | (uint32_t)(k >> 2), stream, uw);
                            dt_attempt(w, lx, ly, ((X0 & ~3) + xt) & (L - 1), ((Y0 & ~3) + yt) & (M - 1), Tpc, Tqc,
                                       dis, uw[k & 3], &nd, &nr);
                        }
                }
            }
        }
    }
    if (dep) *dep += nd;
    if (des) *des += nr;
}

/* The DB4 scheduler (Kpz::Scheduler<Rng, LocalLayoutDB4>::doMcs, kpz/scheduler.cu:37-52;
 * kpzKernelTemplate, kpz/kpz.cu:95-117; Base::systemLoopDC,
 * kpz/kpzSimulationPrimitivesTemplates.cu:74-103): per MCS two launches a = 0, 1, each from a
 * random origin (ox, oy) in [0,256) x [0,128) sites over every 256x128 block of the lattice
 * (block (bx, by) starts at site (ox + 256 bx, oy + 128 by)); per launch 32 BaseDT rounds (a
 * block-wide sub-cell, a position per thread cell in that quadrant), an attempt whose
 * in-block position (before the origin's in-word offset) has x >= 251 or y >= 123 is skipped
 * (LocalLayoutDB4::BLOCK_BORDER_WIDTH = 5, kpz/LocalLayout.h:120-131).  Counter stream:
 *   origin       : Philox(ctr=(a, t, TAG_DB4_ORIGIN<<24, stream)) words 0, 1
 *   sub-cells    : Philox(ctr=(block, t, TAG_DB4_SUB<<24 | a<<16, stream)), 2 bits per round
 *   positions    : Philox(ctr=(cell, t, TAG_DB4_POS<<24 | a<<16 | r>>5, stream)), 4 bits/round
 *   acceptance u : Philox(ctr=(cell, t, TAG_DB4_U<<24 | a<<16 | r>>2, stream)), word r&3 */
void ko_db4_mcs(uint32_t* w, int lx, int ly, uint64_t seed, uint32_t stream, uint64_t t0, int n, double p,
                double q, int64_t* dep, int64_t* des)
{
    const int L = 1 << lx, M = 1 << ly;
    const int BX = 256, BY = 128;
    const int nbx = L / BX, nby = M / BY;
    uint64_t Tpc[4], Tqc[4];
    for (int c = 0; c < 4; ++c) {
        Tpc[c] = ko_threshold(p);
        Tqc[c] = ko_threshold(q);
    }
    int64_t nd = 0, nr = 0;
    for (int i = 0; i < n; ++i) {
        const uint64_t t = t0 + (uint64_t)i;
        for (int a = 0; a < 2; ++a) {
            uint32_t o[4];
            philox_u32(seed, (uint32_t)a, (uint32_t)t, KO_TAG_DB4_ORIGIN << 24, stream, o);
            const int ox = (int)(o[0] & (uint32_t)(BX - 1)), oy = (int)(o[1] & (uint32_t)(BY - 1));
            for (int b = 0; b < nbx * nby; ++b) {
                const int bx = b % nbx, by = b / nbx;
                const int X0 = ox + bx * BX, Y0 = oy + by * BY;
                uint32_t sub[4];
                philox_u32(seed, (uint32_t)b, (uint32_t)t, (KO_TAG_DB4_SUB << 24) | ((uint32_t)a << 16), stream, sub);
                for (int r = 0; r < 32; ++r) {
                    const int s = (int)((sub[r >> 4] >> (2 * (r & 15))) & 3u);
                    for (int cell = 0; cell < 512; ++cell) {
                        const int tx = cell & 31, ty = cell >> 5;
                        const uint32_t cid = (uint32_t)b * 512u + (uint32_t)cell;
                        uint32_t pw[4], uw[4];
                        philox_u32(seed, cid, (uint32_t)t,
                                   (KO_TAG_DB4_POS << 24) | ((uint32_t)a << 16) | (uint32_t)(r >> 5), stream, pw);
                        const int pos = (int)((pw[(r & 31) >> 3] >> (4 * (r & 7))) & 15u);
                        const int xl = tx * 8 + (s & 1) * 4 + (pos & 3), yl = ty * 8 + (s >> 1) * 4 + (pos >> 2);
                        if (xl >= BX - 5 || yl >= BY - 5) continue;
                        philox_u32(seed, cid, (uint32_t)t,
                                   (KO_TAG_DB4_U << 24) | ((uint32_t)a << 16) | (uint32_t)(r >> 2), stream, uw);
                        dt_attempt(w, lx, ly, (X0 + xl) & (L - 1), (Y0 + yl) & (M - 1), Tpc, Tqc, NULL, uw[r & 3],
                                   &nd, &nr);
                    }
                }
            }
        }
    }
    if (dep) *dep += nd;
    if (des) *des += nr;
}

/* ------------------------------------------------------------------------ */
/* dSFMT-19937 (vendored BSD third-party code in the reference,             */
/* inc/dSFMT/dSFMT.{h,cpp}, parameters inc/dSFMT/dSFMT-params19937.h;       */
/* Saito & Matsumoto, "A PRNG specialized in double precision floating      */
/* point numbers using an affine transition", MCQMC 2008). Restated here:   */
/* 128-bit lung recursion, MT-style 32-bit seeding, exponent masking and    */
/* period certification, [1,2) doubles minus 1.                             */
/* ------------------------------------------------------------------------ */
#define KD_N 191
#define KD_POS1 117
#define KD_SL1 19
#define KD_SR 12
#define KD_MSK1 0x000ffafffffffb3fULL
#define KD_MSK2 0x000ffdfffc90fffdULL
#define KD_FIX1 0x90014964b32f4329ULL
#define KD_FIX2 0x3b8d12ac548a7c7aULL
#define KD_PCV1 0x3d84e1ac0dc82880ULL
#define KD_PCV2 0x0000000000000001ULL

struct ko_dsfmt {
    uint64_t st[KD_N + 1][2];
    int idx;
};

size_t ko_dsfmt_size(void) { return sizeof(struct ko_dsfmt); }

static void kd_recursion(uint64_t r[2], const uint64_t a[2], const uint64_t b[2], uint64_t lung[2])
{
    uint64_t t0 = a[0], t1 = a[1], L0 = lung[0], L1 = lung[1];
    lung[0] = (t0 << KD_SL1) ^ (L1 >> 32) ^ (L1 << 32) ^ b[0];
    lung[1] = (t1 << KD_SL1) ^ (L0 >> 32) ^ (L0 << 32) ^ b[1];
    r[0] = (lung[0] >> KD_SR) ^ (lung[0] & KD_MSK1) ^ t0;
    r[1] = (lung[1] >> KD_SR) ^ (lung[1] & KD_MSK2) ^ t1;
}

static void kd_gen_all(ko_dsfmt* s)
{
    uint64_t lung[2] = {s->st[KD_N][0], s->st[KD_N][1]};
    int i;
    for (i = 0; i < KD_N - KD_POS1; ++i) kd_recursion(s->st[i], s->st[i], s->st[i + KD_POS1], lung);
    for (; i < KD_N; ++i) kd_recursion(s->st[i], s->st[i], s->st[i + KD_POS1 - KD_N], lung);
    s->st[KD_N][0] = lung[0];
    s->st[KD_N][1] = lung[1];
}

void ko_dsfmt_init(ko_dsfmt* s, uint32_t seed)
{
    uint32_t v[(KD_N + 1) * 4];
    v[0] = seed;
    for (uint32_t i = 1; i < (KD_N + 1) * 4; ++i)
        v[i] = 1812433253u * (v[i - 1] ^ (v[i - 1] >> 30)) + i;
    for (int i = 0; i < KD_N + 1; ++i)
        for (int j = 0; j < 2; ++j)
            s->st[i][j] = (uint64_t)v[4 * i + 2 * j] | ((uint64_t)v[4 * i + 2 * j + 1] << 32);
    for (int i = 0; i < KD_N; ++i)
        for (int j = 0; j < 2; ++j)
            s->st[i][j] = (s->st[i][j] & 0x000FFFFFFFFFFFFFULL) | 0x3FF0000000000000ULL;
    /* period certification; PCV2 is odd, so a failing check flips bit 0 of the lung's high word */
    uint64_t t0 = s->st[KD_N][0] ^ KD_FIX1, t1 = s->st[KD_N][1] ^ KD_FIX2;
    uint64_t inner = (t0 & KD_PCV1) ^ (t1 & KD_PCV2);
    for (int i = 32; i > 0; i >>= 1) inner ^= inner >> i;
    if ((inner & 1) != 1) s->st[KD_N][1] ^= 1;
    s->idx = KD_N * 2;
}

double ko_dsfmt_close_open(ko_dsfmt* s)
{
    if (s->idx >= KD_N * 2) {
        kd_gen_all(s);
        s->idx = 0;
    }
    uint64_t bits = s->st[s->idx >> 1][s->idx & 1];
    s->idx++;
    double d;
    memcpy(&d, &bits, sizeof d);
    return d - 1.0;
}

/* SchedulerService::reSeed (kpz/schedulerService.cpp:460-470) */
void ko_dsfmt_reseed(ko_dsfmt* s, uint32_t seed)
{
    ko_dsfmt_init(s, seed);
    for (int a = 0; a < 100000; ++a) ko_dsfmt_close_open(s);
}

/* SchedulerCPU::mcs / mcsPQ (kpz/schedulerCPU.inl:21-88, kpz/schedulerCPU.cpp:35-46) */
void ko_rs_mcs(uint32_t* w, int lx, int ly, ko_dsfmt* s, int n, int pq, double p, double q)
{
    ko_rs_mcs_count(w, lx, ly, s, n, pq, p, q, 0, 0);
}

void ko_rs_mcs_count(uint32_t* w, int lx, int ly, ko_dsfmt* s, int n, int pq, double p, double q,
                     int64_t* dep, int64_t* des)
{
    int64_t nd = 0, nr = 0;
    int L = 1 << lx, M = 1 << ly;
    uint64_t N = (uint64_t)1 << (lx + ly);
    int oneone = pq && p == 1.0 && q == 1.0;
    for (; n > 0; --n) {
        for (uint64_t a = 0; a < N; ++a) {
            int x = (int)(ko_dsfmt_close_open(s) * L);
            int y = (int)(ko_dsfmt_close_open(s) * M);
            int c = ko_local_get(w, lx, x, y);
            int r = ko_local_get(w, lx, (x + 1) & (L - 1), y) & 1;
            int l = (ko_local_get(w, lx, x, (y + 1) & (M - 1)) >> 1) & 1;
            int config = c | (r << 2) | (l << 3);
            if (!pq) {
                if (config != 12) continue;
            } else if (oneone) {
                if (config != 12 && config != 3) continue;
            } else {
                if (config == 12) {
                    if (ko_dsfmt_close_open(s) >= p) continue;
                } else if (config == 3) {
                    if (ko_dsfmt_close_open(s) >= q) continue;
                } else continue;
            }
            ko_local_flip(w, lx, x, y, 3);
            ko_local_flip(w, lx, (x + 1) & (L - 1), y, 1);
            ko_local_flip(w, lx, x, (y + 1) & (M - 1), 2);
            if (config == 12) ++nd; else ++nr;
        }
    }
    if (dep) *dep += nd;
    if (des) *des += nr;
}

/* SchedulerService::generateDisorder2 (kpz/schedulerService.cpp:54-71): for every word, bit s
 * (s = 0, 2, ..., 30: the x-slope bit of each of its 16 sites) is set when a dSFMT draw is
 * below `fill`; words in index order. */
void ko_generate_disorder2(uint32_t* dis, int lx, int ly, ko_dsfmt* s, double fill)
{
    const uint64_t nw = ko_size_words(lx, ly);
    for (uint64_t a = 0; a < nw; ++a) {
        uint32_t t = 0;
        for (int b = 0; b < 32; b += 2)
            if (ko_dsfmt_close_open(s) < fill) t |= 1u << b;
        dis[a] = t;
    }
}

/* SchedulerCPU::mcsDisorder2 (kpz/schedulerCPU.cpp:48-80): as mcsPQ, with the rates of the
 * site's disorder class c(m_disorder) (the 2 bits of dis at the site). */
void ko_rs_mcs_dis(uint32_t* w, int lx, int ly, ko_dsfmt* s, int n, const double p[4], const double q[4],
                   const uint32_t* dis, int64_t* dep, int64_t* des)
{
    int64_t nd = 0, nr = 0;
    int L = 1 << lx, M = 1 << ly;
    uint64_t N = (uint64_t)1 << (lx + ly);
    for (; n > 0; --n) {
        for (uint64_t a = 0; a < N; ++a) {
            int x = (int)(ko_dsfmt_close_open(s) * L);
            int y = (int)(ko_dsfmt_close_open(s) * M);
            int c = ko_local_get(w, lx, x, y);
            int r = ko_local_get(w, lx, (x + 1) & (L - 1), y) & 1;
            int l = (ko_local_get(w, lx, x, (y + 1) & (M - 1)) >> 1) & 1;
            int config = c | (r << 2) | (l << 3);
            int cls = ko_local_get(dis, lx, x, y);
            if (config == 12) {
                if (ko_dsfmt_close_open(s) >= p[cls]) continue;
            } else if (config == 3) {
                if (ko_dsfmt_close_open(s) >= q[cls]) continue;
            } else continue;
            ko_local_flip(w, lx, x, y, 3);
            ko_local_flip(w, lx, (x + 1) & (L - 1), y, 1);
            ko_local_flip(w, lx, x, (y + 1) & (M - 1), 2);
            if (config == 12) ++nd; else ++nr;
        }
    }
    if (dep) *dep += nd;
    if (des) *des += nr;
}
