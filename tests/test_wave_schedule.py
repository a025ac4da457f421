"""The register-wavefront pass (cudakpz_b200/csrc/scabit_wave.cu) restated on the CPU, lanes
as numpy vectors, and checked against the oracle's per-site SCABit -- CPU only.

This pins the kernel's schedule, not its code: half-step h updates local row tau - h at tick
tau on a window of rows; within a tick all updates are shifted or none is; the x-carry
crosses lanes like the warp shuffles and crosses warps through a buffer that lane 0
publishes one tick ahead; lane 31's carry flips reach the right warp's lane 0 one tick late;
every half-step runs at every tick (also outside its exact rows); rows [2k, 2k + B) of each
band are stored.  The GPU kernel is compared word for word with the oracle by
tests/test_gpu_sca.py::test_wave_kernel_bit_exact."""
import numpy as np
import pytest

M32 = 0xFFFFFFFF


def wave_pass(oracle, src, lx, ly, K, B, t0, seed, stream, p, q):
    Wr, rows, Q = 1 << (lx - 6), 1 << ly, 1 << (lx + ly - 6)
    nwarps, H, NH, NW = Wr // 32, 2 * K, 2 * K, 2 * K + 5
    Tp, Tq = oracle.threshold(p), oracle.threshold(q)
    ap, aq = (M32 if Tp >= 1 << 32 else 0), (M32 if Tq >= 1 << 32 else 0)
    hp, hq = (M32 if 0 < Tp < 1 << 32 else 0), (M32 if 0 < Tq < 1 << 32 else 0)
    assert Tp in (0, 1 << 31, 1 << 32) and Tq in (0, 1 << 31, 1 << 32)  # DEC_NONE / DEC_ONE
    key = [seed & M32, seed >> 32]
    lane = np.arange(Wr) & 31
    dst = np.zeros_like(src)
    dep = des = 0
    for y0 in range(0, rows, B):
        Bc = min(B, rows - y0)
        R, ylo = Bc + 2 * H, (y0 - H) % rows

        def row(rho):
            gy = (ylo + rho) % rows
            return [src[qd * Q + gy * Wr: qd * Q + (gy + 1) * Wr].astype(np.uint64) for qd in range(4)]

        win = [[np.zeros(Wr, np.uint64) for _ in range(NW)] for _ in range(4)]
        for qd, v in enumerate(row(0)):
            win[qd][H] = v
        xbuf = np.zeros((2, nwarps, NH), np.uint64)
        fbuf = np.zeros((2, nwarps, NH), np.uint64)
        par0 = ylo & 1
        if par0:
            xbuf[0, :, 0] = win[2][H][::32]
        for tau0 in range(0, R, 4):
            for i in range(4):
                tau = tau0 + i
                shifted = (par0 + tau) & 1
                if tau + 1 < R:  # (1) the next row enters the window
                    for qd, v in enumerate(row(tau + 1)):
                        win[qd][H + i + 1] = v
                if tau >= 1 and not shifted:  # (2) lane 0 applies the left warp's carry flips
                    for h in range(NH):
                        win[2 * (1 - (h & 1))][H + i - 1 - h][::32] ^= fbuf[(tau - 1) & 1, (np.arange(nwarps) - 1) % nwarps, h]
                for h in range(NH):  # (3) every half-step, every tick
                    r, sg, s = tau - h, h & 1, H + i - h
                    tX, tY = win[2 * sg][s].copy(), win[2 * sg + 1][s].copy()
                    oX, oY = win[2 * (1 - sg)][s].copy(), win[2 * (1 - sg) + 1][s + 1].copy()
                    xX = oX
                    if shifted:
                        nb = np.roll(oX, -1)  # shuffle down within the warp
                        nb[31::32] = xbuf[tau & 1, (np.arange(nwarps) + 1) % nwarps, h]
                        xX = ((oX >> 1) | ((nb & 1) << 31)) & M32
                    cp = (~(tX | tY) & M32) & xX & oY
                    cq = tX & tY & (~(xX | oY) & M32)
                    if hp or hq:
                        gy, step = (ylo + r) % rows, 2 * (t0 + (h >> 1)) + (h & 1)
                        rw = np.zeros(Wr, np.uint64)
                        for g in range(Wr // 4):
                            rw[4 * g: 4 * g + 4] = oracle.philox([((gy << (lx - 8)) + g) & M32, step, 1 << 8, stream], key)
                        m = (cp & (ap | (hp & ~rw & M32))) | (cq & (aq | (hq & ~rw & M32)))
                    else:
                        m = (cp & ap) | (cq & aq)
                    if H <= r < H + Bc:
                        dep += int(sum(bin(int(v)).count("1") for v in (m & cp)))
                        des += int(sum(bin(int(v)).count("1") for v in (m & cq)))
                    win[2 * sg][s], win[2 * sg + 1][s] = tX ^ m, tY ^ m
                    win[2 * (1 - sg) + 1][s + 1] = oY ^ m
                    if shifted:
                        cin = np.roll(m >> 31, 1)  # shuffle up within the warp
                        win[2 * (1 - sg)][s] = oX ^ ((m << 1) & M32) ^ np.where(lane != 0, cin, 0)
                        fbuf[tau & 1, :, h] = m[31::32] >> 31
                    else:
                        win[2 * (1 - sg)][s] = oX ^ m
                rho = tau - H  # (4) a finished band row leaves the window
                if H <= rho < H + Bc:
                    gy = (ylo + rho) % rows
                    for qd in range(4):
                        dst[qd * Q + gy * Wr: qd * Q + (gy + 1) * Wr] = win[qd][i].astype(np.uint32)
                if not shifted:  # (5) lane 0 publishes the words the left warp reads next tick
                    for h in range(NH):
                        xbuf[(tau + 1) & 1, :, h] = win[2 * (1 - (h & 1))][H + i + 1 - h][::32]
            for qd in range(4):  # the window moves by the unit's 4 ticks
                win[qd][:NW - 4] = win[qd][4:]
    return dst, (dep, des)


@pytest.mark.parametrize("lx,ly,K,B,p,q", [
    (11, 5, 2, 8, 1.0, 0.0),   # one warp per row
    (12, 6, 2, 8, 1.0, 1.0),   # two warps: the cross-warp carry buffers
    (11, 3, 4, 8, 0.5, 0.5),   # 8 rows: every band's halo wraps the lattice; one random plane
    (12, 5, 2, 12, 0.5, 0.0),  # a band length that does not divide the rows
])
def test_wave_schedule_matches_oracle(oracle, lx, ly, K, B, p, q):
    init = oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=17, mcs=2)
    ref = init.copy()
    rc = oracle.sca_mcs(ref, lx, ly, oracle.ENC_CBBIT, 9, 3, 0, K, p, q)
    got, cnt = wave_pass(oracle, init, lx, ly, K, B, 0, 9, 3, p, q)
    d = np.nonzero(got != ref)[0]
    assert d.size == 0, (d.size, int(d[0]))
    assert cnt == rc
