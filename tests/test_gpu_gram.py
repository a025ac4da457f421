"""Exact height autocorrelator (kpzb_gram_*) against the CPU oracle, through the C ABI.

G[s][t] = sum_sites h_s h_t of the path-relative heights (kpz/correlator.cpp:47-96) of every
pair of stored snapshots, and S1[s] = sum h_s.  The tensor-core path (tcgen05 kind::i8 on
three signed int8 limbs, int32 windows, int64 recombination) and the int64 CUDA-core path
must both equal the oracle's exact integer Gram: error exactly 0.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def oracle_gram(oracle, lattices, lx, ly):
    H = np.stack([oracle.heights(w, lx, ly, oracle.ENC_CBBIT).astype(np.int64).ravel() for w in lattices])
    return H @ H.T, H.sum(axis=1)


def snapshots(kpzb, lx, ly, n, p=0.6, q=0.3, step=1, seed=5):
    s = kpzb.Scheduler(lx, ly)
    s.setPQ(p, q)
    s.supplySeed(seed)
    out = []
    for _ in range(n):
        s.mcsPQSyncRng(step)
        out.append(s.popSystem())
    s.close()
    return out


@pytest.mark.parametrize("method", [0, 1])
@pytest.mark.parametrize("lx,ly,n", [(8, 8, 5), (10, 9, 12), (9, 7, 64)])
def test_gram_exact_vs_oracle(kpzb, oracle, method, lx, ly, n):
    snaps = snapshots(kpzb, lx, ly, n)
    g = kpzb.Gram(lx, ly, max_snapshots=max(n, 2))
    for w in snaps:
        g.add_host(w)
    G, S1 = g.compute(method)
    Gr, S1r = oracle_gram(oracle, snaps, lx, ly)
    assert np.array_equal(S1, S1r)
    assert np.array_equal(G, Gr), np.argwhere(G != Gr)[:5]
    g.close()


def test_gram_device_snapshots_and_rough_surfaces(kpzb, oracle):
    """Rough surfaces (large heights, all three limbs non-zero) added from device pointers."""
    lx, ly = 11, 8
    s = kpzb.Scheduler(lx, ly)
    s.setPQ(1.0, 0.0)
    s.supplySeed(1)
    g = kpzb.Gram(lx, ly, max_snapshots=8)
    snaps = []
    for _ in range(8):
        s.mcsPQSyncRng(40)
        g.add_device(s.devicePtr())
        snaps.append(s.popSystem())
    (_, _), (hmin, hmax) = s.heightSums()
    G0, S0 = g.compute(0)
    G1, S1 = g.compute(1)
    Gr, Sr = oracle_gram(oracle, snaps, lx, ly)
    assert np.array_equal(G0, Gr) and np.array_equal(G1, Gr)
    assert np.array_equal(S0, Sr) and np.array_equal(S1, Sr)
    g.close()
    s.close()


@pytest.mark.parametrize("method", [0, 1])
def test_gram_all_three_limbs(kpzb, oracle, method):
    """Biased random words: the path walk drifts to |h| ~ 1e5, so l1 and l2 are non-zero."""
    lx, ly = 11, 8
    rng = np.random.default_rng(11)
    snaps = []
    for i in range(6):
        bits = rng.random((oracle.size_words(lx, ly), 32)) < (0.7 if i % 2 else 0.35)
        snaps.append(np.packbits(bits, axis=1, bitorder="little").view(np.uint32).ravel().copy())
    H = [oracle.heights(w, lx, ly, oracle.ENC_CBBIT) for w in snaps]
    spread = max(int(h.max()) - int(h.min()) for h in H)
    assert spread > 2 * 8256  # the top limb is exercised
    g = kpzb.Gram(lx, ly, max_snapshots=6)
    for w in snaps:
        g.add_host(w)
    G, S1 = g.compute(method)
    Gr, S1r = oracle_gram(oracle, snaps, lx, ly)
    assert np.array_equal(S1, S1r)
    assert np.array_equal(G, Gr)
    g.close()


def test_gram_matches_correlator(kpzb):
    """ch of kpzb_correlate equals G[s][t]/N - <h_s><h_t> from the Gram."""
    lx = ly = 10
    N = 1 << (lx + ly)
    s = kpzb.Scheduler(lx, ly)
    s.setPQ(0.7, 0.2)
    s.supplySeed(3)
    s.mcsPQSyncRng(5)
    s.correlateTag()
    g = kpzb.Gram(lx, ly, max_snapshots=2)
    g.add_device(s.devicePtr())
    s.mcsPQSyncRng(7)
    g.add_device(s.devicePtr())
    r, ch, cs = s.correlate()
    G, S1 = g.compute(0)
    ch_g = G[0, 1] / N - (S1[0] / N) * (S1[1] / N)
    assert abs(ch - ch_g) <= 1e-9 * max(1.0, abs(ch))
    g.close()
    s.close()


def test_gram_capacity(kpzb):
    g = kpzb.Gram(9, 9, max_snapshots=1)
    w = kpzb.Scheduler(9, 9).popSystem()
    g.add_host(w)
    with pytest.raises(kpzb.KpzbError) as e:
        g.add_host(w)
    assert e.value.status == 5
    g.close()


@pytest.mark.parametrize("method", [0, 1])
@pytest.mark.parametrize("lx,ly,n", [(8, 6, 3), (12, 4, 64), (9, 11, 17)])
def test_gram_tile_rows_and_partial_counts(kpzb, oracle, method, lx, ly, n):
    """Row lengths of two to 32 tiles, flat lattices and tall ones, and snapshot counts that
    leave most of the 64 lane quads without a snapshot: the slope walk across tiles, the
    per-CTA tile ranges that start inside a row, and the zero rows of absent snapshots."""
    snaps = snapshots(kpzb, lx, ly, n, p=0.55, q=0.45, step=2, seed=13)
    g = kpzb.Gram(lx, ly, max_snapshots=64)
    for w in snaps:
        g.add_host(w)
    G, S1 = g.compute(method)
    Gr, S1r = oracle_gram(oracle, snaps, lx, ly)
    assert np.array_equal(S1, S1r)
    assert np.array_equal(G, Gr), np.argwhere(G != Gr)[:5]
    g.close()


def test_gram_mixed_limb_paths(kpzb, oracle):
    """Snapshots of small heights (one limb) beside steep ones (all three): a tile's warps take
    the one-limb path only when every value of the warp fits, both paths in one Gram."""
    lx, ly = 10, 8
    snaps = snapshots(kpzb, lx, ly, 4, step=3)
    rng = np.random.default_rng(5)
    for i in range(4):
        bits = rng.random((oracle.size_words(lx, ly), 32)) < (0.8 if i % 2 else 0.25)
        snaps.append(np.packbits(bits, axis=1, bitorder="little").view(np.uint32).ravel().copy())
    g = kpzb.Gram(lx, ly, max_snapshots=8)
    for w in snaps:
        g.add_host(w)
    Gr, S1r = oracle_gram(oracle, snaps, lx, ly)
    for method in (0, 1):
        G, S1 = g.compute(method)
        assert np.array_equal(G, Gr) and np.array_equal(S1, S1r), method
    g.close()
