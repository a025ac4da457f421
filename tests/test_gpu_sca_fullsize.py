"""The timed plans at the timed size: 16384^2 lattices (2^28 sites) advanced by the exact pass
plans the benchmark runs, compared word for word with the CPU oracle, with the deposition /
desorption counters.

The oracle side is ko_sca_mcs_words (32 sites per word operation; pinned to the per-site
restatement in tests/test_oracle_words.py), so a 16384^2 run of 13 MCS takes seconds on the
host.  Each run covers at least two whole passes of the pass kernel plus a remainder of
one-half-step launches.  Reference rule: kpz/kpzSCABit.cu:179-290 with the masks of
kpz/kpzSCABitCores.cu:69-74,139-145; DT: kpz/schedulerDT.cu:38-78, kpz/kpz.cu:126-155.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LX = LY = 14
SEED = 42


def first_diff(a, b):
    d = np.nonzero(a != b)[0]
    return None if d.size == 0 else (int(d[0]), hex(int(a[d[0]])), hex(int(b[d[0]])), int(d.size))


def run_plan(kpzb, p, q, n, fusion):
    s = kpzb.Scheduler(LX, LY, scheduler="scaBit")
    s.setPQ(p, q)
    s.supplySeed(SEED, 0)
    s.setFusion(fusion)
    s.enableCounters(True)
    plan = s.plan()
    s.mcsPQSyncRng(n)
    got = s.popSystem()
    cnt = s.counters()
    s.close()
    return got, cnt, plan


def oracle_run(oracle, p, q, n):
    ref = oracle.homogeneous(LX, LY, oracle.ENC_CBBIT)
    cnt = oracle.sca_mcs_words(ref, LX, LY, SEED, 0, 0, n, p, q)
    return ref, cnt


# (p, q, KPZB_PASS_KERNEL, MCS per pass, MCS run, expected (kind, CTAs per SM))
HEADLINE_PLANS = [
    (1.0, 0.0, "wave2", 6, 13, ("wave", 2)),   # 2 passes + 1 MCS of half-step launches
    (0.5, 0.5, "band1", 4, 9, ("band", 1)),    # 2 passes + 1 MCS
    (1.0, 0.0, "strip64", 6, 13, ("strip", 64)),
    (1.0, 0.0, "strip128", 8, 17, ("strip", 128)),
    (0.5, 0.5, "strip64", 4, 9, ("strip", 64)),
    (0.5, 0.5, "strip32", 6, 13, ("strip", 32)),
]


@pytest.mark.parametrize("p,q,kernel,k,n,expect", HEADLINE_PLANS)
def test_forced_headline_plan_16384_vs_oracle(kpzb, oracle, monkeypatch, p, q, kernel, k, n, expect):
    monkeypatch.setenv("KPZB_PASS_KERNEL", kernel)
    got, cnt, plan = run_plan(kpzb, p, q, n, k)
    assert (plan[0], plan[2], plan[1]) == (k, expect[0], expect[1]), plan
    ref, rc = oracle_run(oracle, p, q, n)
    assert first_diff(got, ref) is None, first_diff(got, ref)
    assert cnt == rc


@pytest.mark.parametrize("p,q", [(1.0, 0.0), (0.5, 0.5)])
def test_tuned_plan_16384_vs_oracle(kpzb, oracle, monkeypatch, p, q):
    """Whatever plan the tuner picks on this GPU (the plan the benchmark times), two whole
    passes and a remainder, word for word."""
    monkeypatch.delenv("KPZB_PASS_KERNEL", raising=False)
    s = kpzb.Scheduler(LX, LY, scheduler="scaBit")
    s.setPQ(p, q)
    s.supplySeed(SEED, 0)
    k = s.plan()[0]
    s.close()
    n = 2 * k + 1
    got, cnt, plan = run_plan(kpzb, p, q, n, 0)
    assert plan[0] == k
    ref, rc = oracle_run(oracle, p, q, n)
    assert first_diff(got, ref) is None, (plan, first_diff(got, ref))
    assert cnt == rc


@pytest.mark.parametrize("inner", ["dbsh", "dt"])
def test_dt_16384_one_mcs_vs_oracle(kpzb, oracle, inner):
    """The DT kernel on a 16384^2 lattice (2^20 blocks per domain set, every launch of an MCS)
    against its CPU emulation, word for word, with counters: "dbsh" the default of a new
    handle (the reference's default build), "dt" the single-hit double tiling."""
    p, q = 0.95, 0.05
    s = kpzb.Scheduler(LX, LY, scheduler="dt")
    if inner != "dbsh":
        s.setDtInner(inner)
    s.setPQ(p, q)
    s.supplySeed(1, 0)
    s.enableCounters(True)
    s.mcsPQSyncRng(1)
    got = s.popSystem()
    cnt = s.counters()
    s.close()
    ref = oracle.homogeneous(LX, LY, oracle.ENC_LOCAL)
    rc = oracle.dt_mcs_inner(ref, LX, LY, 1, 0, 0, 1, p, q, inner)
    assert first_diff(got, ref) is None, first_diff(got, ref)
    assert cnt == rc
