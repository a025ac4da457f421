"""Quenched binary disorder (mcsDisorder2SyncRng) on the GPU against the oracle's restatement
(kpz/kpzSCACores.cu:217-280 for SCA, the DT caller at kpz/kpz.cu:238-246), word for word.
The oracle's disorder generator and rule are pinned to the reference's own
generateDisorder2 / SchedulerCPU::mcsDisorder2 in test_oracle_golden.py."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def disorder_words(oracle, lx, ly, fill, seed, two_bits=False):
    d = oracle.generate_disorder2(lx, ly, oracle.DSFMT(seed), fill)
    if two_bits:  # classes 2 and 3 too: set the odd (y-slope) bit of some sites
        d2 = oracle.generate_disorder2(lx, ly, oracle.DSFMT(seed + 1), 0.5)
        d = d | (d2 << 1)
    return d


CASES = [("scaBit", 9, 9, [0.9, 0.3], [0.1, 0.6], False),
         ("scaBit", 10, 8, [0.5, 1.0], [0.5, 0.0], False),
         ("scaBit", 9, 9, [0.7, 0.2, 1.0, 0.5], [0.2, 0.9, 0.0, 0.5], True),
         ("sca", 9, 9, [0.95, 0.4], [0.05, 0.4], False)]


@pytest.mark.parametrize("sched,lx,ly,p,q,two", CASES)
def test_sca_disorder_bit_exact(kpzb, oracle, sched, lx, ly, p, q, two):
    dis = disorder_words(oracle, lx, ly, 0.3, 5, two)
    enc = oracle.ENC_CBBIT if sched == "scaBit" else oracle.ENC_LOCAL
    n = 5
    s = kpzb.Scheduler(lx, ly, scheduler=sched)
    for c in range(len(p)):
        s.setPQ(p[c], q[c], c)
    s.supplySeed(17)
    s.setDisorder(dis)
    s.enableCounters(True)
    s.mcsDisorder2SyncRng(n)
    got = s.popSystem()
    cnt = s.counters()
    s.close()
    ref = oracle.homogeneous(lx, ly, enc)
    rc = oracle.sca_mcs_dis(ref, lx, ly, enc, 17, 0, 0, n, p, q, dis)
    assert np.array_equal(got, ref)
    assert cnt == rc


def test_dt_disorder_bit_exact(kpzb, oracle):
    lx, ly = 10, 9
    p, q = [0.95, 0.5], [0.05, 0.5]
    dis = disorder_words(oracle, lx, ly, 0.4, 8)
    s = kpzb.Scheduler(lx, ly, scheduler="dt")
    s.setDtInner("dt")  # ko_dt_mcs_dis emulates the DT scheme
    s.setPQ(p[0], q[0])
    s.setPQ(p[1], q[1], 1)
    s.supplySeed(3)
    s.setDisorder(dis)
    s.mcsDisorder2SyncRng(3)
    got = s.popSystem()
    s.close()
    ref = oracle.homogeneous(lx, ly, oracle.ENC_LOCAL)
    oracle.dt_mcs_dis(ref, lx, ly, 3, 0, 0, 3, p, q, dis)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("sched", ["scaBit", "dt"])
def test_equal_class_rates_give_the_plain_run(kpzb, oracle, sched):
    lx, ly = 10, 9
    dis = disorder_words(oracle, lx, ly, 0.5, 2, two_bits=True)
    out = []
    for use_dis in (False, True):
        s = kpzb.Scheduler(lx, ly, scheduler=sched)
        s.setPQ(0.8, 0.15)
        s.supplySeed(6)
        if use_dis:
            s.setDisorder(dis)  # classes 1..3 follow class 0
            s.mcsDisorder2SyncRng(4)
        else:
            s.mcsPQSyncRng(4)
        out.append(s.popSystem())
        s.close()
    assert np.array_equal(out[0], out[1])


def test_disorder_requires_words(kpzb):
    s = kpzb.Scheduler(9, 9)
    with pytest.raises(kpzb.KpzbError):
        s.mcsDisorder2SyncRng(1)
    with pytest.raises(kpzb.KpzbError):
        s.setPQ(0.5, 0.5, 4)
    s.close()
