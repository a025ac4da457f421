"""GPU roughness / correlator / invariants against the CPU oracle, through the C ABI.

Reference behaviour: kpz/correlator.cpp:37-106 (height walk), :337-399 and :463-477
(correlate), kpz/roughness.cpp:38-43 (normAndSetW2), kpz/schedulerService.cpp:721-854
(consistency).  S1 and S2 are exact integers on both sides; the higher moments are
FP64 sums on the GPU against long-double sums in the oracle, compared with relative
tolerance 1e-12.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def make(kpzb, oracle, lx, ly, sched="scaBit", seed=4, mcs=5):
    enc = oracle.ENC_CBBIT if sched == "scaBit" else oracle.ENC_LOCAL
    w = oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=seed, mcs=mcs)
    if enc == oracle.ENC_LOCAL:
        w = oracle.cbbit_to_local(w, lx, ly)
    s = kpzb.Scheduler(lx, ly, scheduler=sched)
    s.pushSystem(w)
    return s, w, enc


@pytest.mark.parametrize("sched", ["scaBit", "sca"])
@pytest.mark.parametrize("lx,ly", [(8, 8), (10, 9), (12, 6)])
def test_roughness_matches_oracle(kpzb, oracle, sched, lx, ly):
    s, w, enc = make(kpzb, oracle, lx, ly, sched)
    r = s.roughness()
    ref = oracle.roughness(w, lx, ly, enc)
    np.testing.assert_allclose([r.w2] + r.h, ref, rtol=RTOL, atol=1e-12)
    h = oracle.heights(w, lx, ly, enc)
    ps = oracle.power_sums(h)
    (s1, s2), (hmin, hmax) = s.heightSums()
    assert (s1, s2) == (ps[0], ps[1])
    assert (hmin, hmax) == (int(h.min()), int(h.max()))


def test_flat_start_roughness(kpzb, oracle):
    for sched, enc in (("scaBit", oracle.ENC_CBBIT), ("sca", oracle.ENC_LOCAL)):
        s = kpzb.Scheduler(9, 9, scheduler=sched)
        r = s.roughness()
        ref = oracle.roughness(oracle.homogeneous(9, 9, enc), 9, 9, enc)
        np.testing.assert_allclose([r.w2] + r.h, ref, rtol=RTOL, atol=1e-12)
        s.close()


@pytest.mark.parametrize("sched", ["scaBit", "sca"])
def test_correlate_matches_oracle(kpzb, oracle, sched):
    lx = ly = 10
    s, w, enc = make(kpzb, oracle, lx, ly, sched)
    tag = s.correlateTag()
    snap = w.copy()
    s.setPQ(0.7, 0.3)
    s.supplySeed(99)
    s.mcsPQSyncRng(6)
    r, ch, cs = s.correlate()
    cur = s.popSystem()
    ref = oracle.correlate(cur, snap, lx, ly, enc, tag.h[0])
    np.testing.assert_allclose([r.w2] + r.h, ref[:8], rtol=RTOL, atol=1e-12)
    np.testing.assert_allclose(ch, ref[8], rtol=1e-10, atol=1e-12)
    assert cs == ref[9]


def test_correlate_self_is_w2(kpzb, oracle):
    s, w, enc = make(kpzb, oracle, 10, 10)
    tag = s.correlateTag()
    r, ch, cs = s.correlate()
    assert cs == 1.0
    np.testing.assert_allclose(ch, tag.w2, rtol=1e-12)


def test_correlate_without_tag_is_state_error(kpzb):
    s = kpzb.Scheduler(9, 9)
    with pytest.raises(kpzb.KpzbError) as e:
        s.correlate()
    assert e.value.status == 5


@pytest.mark.parametrize("lx,ly", [(8, 8), (11, 9)])
def test_invariants_valid_and_broken(kpzb, oracle, lx, ly):
    s, w, enc = make(kpzb, oracle, lx, ly)
    ok, rep = s.consitencyCheck()
    assert ok and rep == [0, 0, 0]
    assert oracle.check_invariants(w, lx, ly, enc) == [0, 0, 0]
    # plant a defect on the host: flip one x-slope bit
    bad = w.copy()
    bad[5] ^= 1 << 3
    s.pushSystem(bad)
    ok, rep = s.consitencyCheck()
    assert not ok
    assert rep == oracle.check_invariants(bad, lx, ly, enc)


def test_invariants_local_encoding(kpzb, oracle):
    s, w, enc = make(kpzb, oracle, 9, 9, "sca")
    ok, rep = s.consitencyCheck()
    assert ok
    bad = w.copy()
    bad[17] ^= 2
    s.pushSystem(bad)
    ok, rep = s.consitencyCheck()
    assert rep == oracle.check_invariants(bad, 9, 9, enc)


def sawtooth_lattice(oracle, lx, amp):
    """ENC_CBBIT words of the surface h(x, y) = t(x) + t(y), t a triangle wave rising and falling
    by one per site between -amp/2 and amp/2 (a sum of two +-1 walks, so every plaquette closes):
    heights near zero with steep slopes, i.e. large offsets inside every 64-site chunk."""
    L = 1 << lx
    x = np.arange(L)
    ph = (x + amp // 2) % (2 * amp)  # t(0) = 0: the walk starts at mid height
    t = np.where(ph < amp, ph, 2 * amp - ph) - amp // 2
    h = t[None, :] + t[:, None]  # h[y, x]
    sx = (h > np.roll(h, 1, axis=1)).astype(np.uint32)  # s_x(x, y) = [h(x,y) > h(x-1,y)]
    sy = (h > np.roll(h, 1, axis=0)).astype(np.uint32)  # s_y(x, y) = [h(x,y) > h(x,y-1)]
    yy, xx = np.meshgrid(np.arange(L), x, indexing="ij")
    word = (yy >> 2) * (L >> 2) + (xx >> 2)
    bit = ((xx & 3) << 1) | ((yy & 3) << 3)
    local = np.zeros(L * L // 16, dtype=np.uint64)
    np.add.at(local, word.ravel(), ((sx | (sy << 1)).astype(np.uint64) << bit.astype(np.uint64)).ravel())
    return oracle.local_to_cbbit(local.astype(np.uint32), lx, lx)


@pytest.mark.parametrize("case", ["flat6", "rough300", "sawtooth"])
def test_odd_moments_near_zero_height(kpzb, oracle, case):
    """The roughness walk builds each 64-site chunk's sum of h^k from exact integer power sums of
    the offsets from the chunk's first height, expanded binomially in FP64 once per chunk; where
    heights are near zero while the offsets are large, the expansion's terms cancel.  The odd
    moments <h^3>, <h^5>, <h^7> against the oracle's per-site long-double sums (exact integers
    here): absolute error at most 1e-12 * <|h|^k> + 1e-12, on a flat start after 6 MCS, a rough
    surface after 300 MCS (p = q = 1/2), and a steep sawtooth surface centred on zero."""
    lx = ly = 9
    if case == "sawtooth":
        w = sawtooth_lattice(oracle, lx, 64)
    else:
        w = oracle.homogeneous(lx, ly, oracle.ENC_CBBIT)
        oracle.sca_mcs_words(w, lx, ly, 5, 0, 0, 6 if case == "flat6" else 300, 0.5, 0.5)
    rep = oracle.check_invariants(w, lx, ly, oracle.ENC_CBBIT)
    assert list(rep) == [0, 0, 0], rep  # a valid surface
    s = kpzb.Scheduler(lx, ly)
    s.pushSystem(w)
    r = s.roughness()
    s.close()
    ref = oracle.roughness(w, lx, ly, oracle.ENC_CBBIT)
    h = oracle.heights(w, lx, ly, oracle.ENC_CBBIT).astype(np.float64)
    for k in (3, 5, 7):
        scale = float(np.mean(np.abs(h) ** k))
        assert abs(r.h[k - 1] - ref[k]) <= 1e-12 * scale + 1e-12, (k, r.h[k - 1], ref[k], scale)
