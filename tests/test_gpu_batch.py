"""Batched replicas (kpzb_batch_*) against single runs and the oracle, through the C ABI.

Every replica of a batch must equal, word for word, a single SCABit run with the same
(lx, p, q, seed, stream) -- the batch replaces the reference's per-lattice launch loop
(kpz/schedulerSCABit.cu:46-73 driven per lattice by kpz/kpzScaling.cpp:194-215).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RATES = [(1.0, 0.0), (0.9, 0.1), (0.75, 0.25), (0.5, 0.5)]


def single(kpzb, lx, p, q, seed, stream, n, fusion=1):
    s = kpzb.Scheduler(lx, lx, scheduler="scaBit")
    s.setPQ(p, q)
    s.supplySeed(seed, stream)
    s.setFusion(fusion)
    s.mcsPQSyncRng(n)
    w = s.popSystem()
    s.close()
    return w


def make_batch(kpzb, lxs, seed0=1000):
    rng = np.random.default_rng(0)
    pq = [RATES[i] for i in rng.integers(0, len(RATES), size=len(lxs))]
    seeds = [seed0 + i for i in range(len(lxs))]
    b = kpzb.Batch(lxs, [a for a, _ in pq], [c for _, c in pq], seeds)
    return b, pq, seeds


@pytest.mark.parametrize("k,chunk,n", [(8, 2, 37), (3, 4, 25), (1, 8, 9), (5, 1, 5)])
def test_batch_matches_single_runs(kpzb, k, chunk, n):
    lxs = [8, 9, 10, 8, 11, 9, 12, 8]
    b, pq, seeds = make_batch(kpzb, lxs)
    b.setFusion(k, chunk)
    b.mcs(n)
    assert b.deviceMcs() == n
    for i, lx in enumerate(lxs):
        ref = single(kpzb, lx, pq[i][0], pq[i][1], seeds[i], 0, n)
        got = b.pop(i)
        assert np.array_equal(got, ref), (i, lx, pq[i])
    b.close()


def test_batch_small_replicas_vs_oracle(kpzb, oracle):
    lxs = [8, 8, 9]
    b, pq, seeds = make_batch(kpzb, lxs, seed0=7)
    b.mcs(11)
    for i, lx in enumerate(lxs):
        ref = oracle.homogeneous(lx, lx, oracle.ENC_CBBIT)
        oracle.sca_mcs(ref, lx, lx, oracle.ENC_CBBIT, seeds[i], 0, 0, 11, *pq[i])
        assert np.array_equal(b.pop(i), ref)
    b.close()


def test_batch_split_calls_and_push(kpzb, oracle):
    lxs = [9, 10, 12]
    b, pq, seeds = make_batch(kpzb, lxs)
    init = oracle.random_lattice(10, 10, oracle.ENC_CBBIT, seed=2, mcs=3)
    b.push(1, init)
    for n in (3, 8, 16, 1):
        b.mcs(n)
    s = kpzb.Scheduler(10, 10)
    s.setPQ(*pq[1])
    s.supplySeed(seeds[1])
    s.pushSystem(init)
    s.mcsPQSyncRng(28)
    assert np.array_equal(b.pop(1), s.popSystem())
    w2 = b.roughness()
    assert abs(w2[1] - s.roughness().w2) < 1e-12
    b.close()


def test_batch_rejects_bad_sizes(kpzb):
    with pytest.raises(kpzb.KpzbError):
        kpzb.Batch([17], [1.0], [0.0], [1])
    with pytest.raises(kpzb.KpzbError):
        kpzb.Batch([7], [1.0], [0.0], [1])


@pytest.mark.parametrize("cps,k", [(2, 4), (3, 6), (2, 8)])
def test_batch_ctas_per_sm_matches_single_runs(kpzb, cps, k):
    """The 256-thread pass kernel at two or three persistent CTAs per SM (half or a third of the
    SM's shared memory each, so more lattices are banded) gives the single runs' lattices."""
    lxs = [8, 9, 10, 11, 12, 8, 10]
    b, pq, seeds = make_batch(kpzb, lxs, seed0=300)
    b.setFusion(k)
    b.setCtasPerSm(cps)
    assert b.plan() == (k, cps)
    n = 2 * k + 3
    b.mcs(n)
    for i, lx in enumerate(lxs):
        assert np.array_equal(b.pop(i), single(kpzb, lx, pq[i][0], pq[i][1], seeds[i], 0, n)), (i, lx)
    b.close()


def test_batch_autotune_restores_and_matches(kpzb, monkeypatch):
    """Tuning times passes on the replicas and restores them and the MCS count; the tuned plan
    then gives the single runs' lattices.  A batch without a plan is tuned on its first MCS."""
    monkeypatch.delenv("KPZB_AUTOTUNE", raising=False)
    lxs = [8, 10, 12, 9, 11]
    b, pq, seeds = make_batch(kpzb, lxs, seed0=500)
    b.mcs(3)
    before = [b.pop(i) for i in range(len(lxs))]
    k, cps, ms = b.autotune()
    assert k in (2, 4, 6, 8) and cps in (1, 2, 3) and ms > 0
    assert b.deviceMcs() == 3 and b.plan() == (k, cps)
    for i in range(len(lxs)):
        assert np.array_equal(b.pop(i), before[i])
    b.mcs(2 * k + 1)
    for i, lx in enumerate(lxs):
        assert np.array_equal(b.pop(i), single(kpzb, lx, pq[i][0], pq[i][1], seeds[i], 0, 3 + 2 * k + 1)), (i, lx)
    b.close()
    c, pq2, seeds2 = make_batch(kpzb, [8, 9], seed0=900)  # untuned: tuned (or cached) on first use
    c.mcs(5)
    assert c.plan()[1] in (1, 2, 3)
    for i, lx in enumerate([8, 9]):
        assert np.array_equal(c.pop(i), single(kpzb, lx, pq2[i][0], pq2[i][1], seeds2[i], 0, 5))
    c.close()
