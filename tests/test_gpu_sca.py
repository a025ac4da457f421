"""GPU parity of the SCA / SCABit path against the CPU oracle, through the C ABI.

Bit-exact: both sides consume the same counter-based stream (Philox4x32-10, see
oracle/kpz_oracle.h), so every lattice word must match.  Reference behaviour:
kpz/kpzSCABit.cu:112-290, kpz/kpzSCABitCores.cu:69-74,139-145, kpz/kpzSCACores.cu:121-144,
kpz/schedulerSCABit.cu:46-73.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PQ = [(1.0, 0.0), (0.5, 0.5), (0.95, 0.05), (0.3, 0.7), (0.5, 0.0), (0.75, 0.25), (1.0, 1.0),
      (0.0, 0.0)]


def first_diff(a, b):
    d = np.nonzero(a != b)[0]
    return None if d.size == 0 else (int(d[0]), hex(int(a[d[0]])), hex(int(b[d[0]])), int(d.size))


def run_gpu(kpzb, lx, ly, sched, p, q, seed, n, init=None, fusion=1, stream=0):
    s = kpzb.Scheduler(lx, ly, scheduler=sched)
    s.setPQ(p, q)
    s.supplySeed(seed, stream)
    s.setFusion(fusion)
    if init is not None:
        s.pushSystem(init)
    s.mcsPQSyncRng(n)
    out = s.popSystem()
    s.close()
    return out


@pytest.mark.parametrize("p,q", PQ)
@pytest.mark.parametrize("lx,ly", [(8, 8), (9, 9), (10, 7)])
def test_scabit_flat_start_bit_exact(kpzb, oracle, lx, ly, p, q):
    n = 6
    ref = oracle.homogeneous(lx, ly, oracle.ENC_CBBIT)
    oracle.sca_mcs(ref, lx, ly, oracle.ENC_CBBIT, 42, 0, 0, n, p, q)
    got = run_gpu(kpzb, lx, ly, "scaBit", p, q, 42, n)
    assert first_diff(got, ref) is None, first_diff(got, ref)


@pytest.mark.parametrize("lx,ly", [(11, 9), (12, 8), (14, 4)])
def test_scabit_wide_rows_segment_carry(kpzb, oracle, lx, ly):
    """Rows longer than one CTA segment (4*256 words) exercise the carried one-bit mask."""
    p, q = 0.6, 0.4
    init = oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=5, mcs=3)
    ref = init.copy()
    oracle.sca_mcs(ref, lx, ly, oracle.ENC_CBBIT, 9, 3, 0, 3, p, q)
    got = run_gpu(kpzb, lx, ly, "scaBit", p, q, 9, 3, init=init, stream=3)
    assert first_diff(got, ref) is None, first_diff(got, ref)


# pass kernels selectable for an explicit fusion depth (KPZB_PASS_KERNEL): the streaming
# wavefront kernel with one or two chunks per SM, and the band kernel
KERNELS = ["stream", "stream2", "band"]


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("fusion", [2, 3, 5])
@pytest.mark.parametrize("lx,ly,p,q", [(9, 9, 0.5, 0.5), (10, 10, 1.0, 0.0), (8, 10, 0.9, 0.1),
                                       (11, 6, 0.5, 0.5)])
def test_fused_bit_exact(kpzb, oracle, monkeypatch, lx, ly, p, q, fusion, kernel):
    monkeypatch.setenv("KPZB_PASS_KERNEL", kernel)
    n = 2 * fusion + 1  # whole fused passes plus a single-step remainder
    init = oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=11, mcs=2)
    ref = init.copy()
    oracle.sca_mcs(ref, lx, ly, oracle.ENC_CBBIT, 77, 0, 0, n, p, q)
    got = run_gpu(kpzb, lx, ly, "scaBit", p, q, 77, n, init=init, fusion=fusion)
    assert first_diff(got, ref) is None, first_diff(got, ref)


@pytest.mark.parametrize("kernel", ["stream", "stream2"])
@pytest.mark.parametrize("lx,ly,k,p,q", [
    (8, 8, 2, 0.5, 0.5),    # one 4-word group per row
    (8, 6, 3, 0.75, 0.25),  # fewer rows than chunks: one row per chunk
    (10, 4, 2, 1.0, 0.0),   # 16 rows: each chunk's halo wraps the lattice
    (12, 2, 8, 0.5, 0.5),   # 4 rows, deepest pass: rows loaded many times over
    (13, 3, 6, 0.3, 0.7),   # wide rows, generic rates
    (9, 11, 8, 1.0, 1.0),   # every candidate flips
])
def test_stream_kernel_edges(kpzb, oracle, monkeypatch, lx, ly, k, p, q, kernel):
    """The streaming pass kernel at chunk, halo and ring corner cases, word for word."""
    monkeypatch.setenv("KPZB_PASS_KERNEL", kernel)
    n = 2 * k
    init = oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=13, mcs=3)
    ref = init.copy()
    oracle.sca_mcs(ref, lx, ly, oracle.ENC_CBBIT, 5, 0, 0, n, p, q)
    got = run_gpu(kpzb, lx, ly, "scaBit", p, q, 5, n, init=init, fusion=k)
    assert first_diff(got, ref) is None, first_diff(got, ref)


@pytest.mark.parametrize("kernel", ["wave1", "wave2", "wave3"])
@pytest.mark.parametrize("lx,ly,k,p,q", [
    (11, 7, 2, 1.0, 0.0),   # one warp per row (the cross-warp carry goes through its own lane 0)
    (11, 3, 8, 0.5, 0.5),   # 8 rows, deepest pass: every band's halo wraps the lattice
    (12, 8, 4, 0.5, 0.5),   # two warps per row
    (12, 6, 6, 1.0, 1.0),   # every candidate flips, maxima too
    (13, 7, 8, 0.5, 0.0),   # one random plane, no maxima
    (13, 5, 4, 0.0, 1.0),   # only maxima
    (14, 6, 2, 1.0, 0.0),   # the headline width: eight warps per row
    (14, 5, 6, 0.5, 0.5),
    (14, 4, 4, 0.9, 0.1),   # generic rates: the wave kernel does not cover them, band fallback
])
def test_wave_kernel_bit_exact(kpzb, oracle, monkeypatch, lx, ly, k, p, q, kernel):
    """The register-wavefront pass kernel, word for word, with counters: bands of few rows,
    halos that wrap, one to eight warps per row, one to three CTAs per SM."""
    monkeypatch.setenv("KPZB_PASS_KERNEL", kernel)
    n = 2 * k + 1
    init = oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=17, mcs=2)
    ref = init.copy()
    rc = oracle.sca_mcs(ref, lx, ly, oracle.ENC_CBBIT, 9, 3, 0, n, p, q)
    s = kpzb.Scheduler(lx, ly)
    s.pushSystem(init)
    s.setPQ(p, q)
    s.supplySeed(9, 3)
    s.setFusion(k)
    s.enableCounters(True)
    s.mcsPQSyncRng(n)
    got = s.popSystem()
    cnt = s.counters()
    kind = s.plan()[2]
    s.close()
    assert kind == ("band" if (p, q) == (0.9, 0.1) else "wave")
    assert first_diff(got, ref) is None, first_diff(got, ref)
    assert cnt == rc


@pytest.mark.parametrize("p,q", [(0.95, 0.0), (0.5, 0.5), (1.0, 0.0)])
def test_sca_local_encoding_bit_exact(kpzb, oracle, p, q):
    """SchedulerSCA: ENC_LOCAL push/pop; dynamics identical to the per-site ENC_LOCAL oracle."""
    lx = ly = 9
    init = oracle.cbbit_to_local(oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=3), lx, ly)
    ref = init.copy()
    oracle.sca_mcs(ref, lx, ly, oracle.ENC_LOCAL, 1234, 0, 0, 4, p, q)
    got = run_gpu(kpzb, lx, ly, "sca", p, q, 1234, 4, init=init)
    assert first_diff(got, ref) is None, first_diff(got, ref)


def test_sca_flat_start_local_words(kpzb, oracle):
    s = kpzb.Scheduler(9, 9, scheduler="sca")
    w = s.popSystem()
    assert np.all(w == 0x33CC33CC)
    s.close()
    s = kpzb.Scheduler(9, 9, scheduler="scaBit")
    w = s.popSystem()
    assert np.all(w[: w.size // 2] == 0) and np.all(w[w.size // 2:] == 0xFFFFFFFF)
    s.close()


def test_mcs_split_equals_single_call(kpzb, oracle):
    lx = ly = 10
    a = kpzb.Scheduler(lx, ly)
    a.setPQ(0.7, 0.2)
    a.supplySeed(5)
    a.mcsPQSyncRng(7)
    b = kpzb.Scheduler(lx, ly)
    b.setPQ(0.7, 0.2)
    b.supplySeed(5)
    for k in (1, 2, 4):
        b.mcsPQSyncRng(k)
    assert np.array_equal(a.popSystem(), b.popSystem())
    assert a.deviceMcs() == b.deviceMcs() == 7


def test_counters_height_balance(kpzb, oracle):
    """sum of relative heights changes by 2*(dep - des) modulo 2N (the reference point moves)."""
    lx = ly = 10
    N = 1 << (lx + ly)
    s = kpzb.Scheduler(lx, ly)
    s.setPQ(0.8, 0.3)
    s.supplySeed(2)
    s.enableCounters(True)
    (s1a, _), _ = s.heightSums()
    s.mcsPQSyncRng(5)
    dep, des = s.counters(reset=True)
    (s1b, _), _ = s.heightSums()
    assert dep > 0 and des > 0
    assert (s1b - s1a - 2 * (dep - des)) % (2 * N) == 0
    ref = oracle.homogeneous(lx, ly, oracle.ENC_CBBIT)
    rdep, rdes = oracle.sca_mcs(ref, lx, ly, oracle.ENC_CBBIT, 2, 0, 0, 5, 0.8, 0.3)
    assert (dep, des) == (rdep, rdes)


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("fusion", [1, 4])
def test_counters_fused(kpzb, oracle, monkeypatch, fusion, kernel):
    monkeypatch.setenv("KPZB_PASS_KERNEL", kernel)
    lx, ly = 10, 9
    s = kpzb.Scheduler(lx, ly)
    s.setPQ(0.6, 0.4)
    s.supplySeed(8)
    s.setFusion(fusion)
    s.enableCounters(True)
    s.mcsPQSyncRng(8)
    ref = oracle.homogeneous(lx, ly, oracle.ENC_CBBIT)
    assert s.counters() == oracle.sca_mcs(ref, lx, ly, oracle.ENC_CBBIT, 8, 0, 0, 8, 0.6, 0.4)


@pytest.mark.parametrize("kernel", ["stream", "band", "wave"])
def test_full_size_16384_properties(kpzb, oracle, monkeypatch, kernel):
    """16384^2 (C2 size): fused == unfused bit for bit, invariants hold, height balance."""
    monkeypatch.setenv("KPZB_PASS_KERNEL", kernel)
    lx = ly = 14
    N = 1 << 28
    res = {}
    for fusion in (1, 0, 4, 6):
        s = kpzb.Scheduler(lx, ly)
        s.setPQ(0.5, 0.5)
        s.supplySeed(42)
        s.setFusion(fusion)
        s.enableCounters(True)
        (s1a, _), _ = s.heightSums()
        s.mcsPQSyncRng(12)
        ok, rep = s.consitencyCheck()
        assert ok, rep
        dep, des = s.counters()
        (s1b, _), _ = s.heightSums()
        assert dep > 0 and des > 0
        assert (s1b - s1a - 2 * (dep - des)) % (2 * N) == 0
        res[fusion] = s.popSystem()
        s.close()
    for f in (0, 4, 6):
        assert first_diff(res[1], res[f]) is None, (f, first_diff(res[1], res[f]))


def test_full_size_first_mcs_vs_oracle(kpzb, oracle):
    """16384^2 at (p,q)=(1,0): the first 2 MCS match the oracle word for word."""
    lx = ly = 14
    ref = oracle.homogeneous(lx, ly, oracle.ENC_CBBIT)
    oracle.sca_mcs(ref, lx, ly, oracle.ENC_CBBIT, 42, 0, 0, 2, 1.0, 0.0)
    got = run_gpu(kpzb, lx, ly, "scaBit", 1.0, 0.0, 42, 2, fusion=0)
    assert first_diff(got, ref) is None, first_diff(got, ref)


@pytest.mark.parametrize("sched", ["scaBit", "sca"])
def test_async_push_pop_equals_sync(kpzb, oracle, sched):
    """kpzb_push_async -> kpzb_mcs_async -> kpzb_pop_async -> kpzb_join == the synchronous path."""
    lx = ly = 10
    enc = oracle.ENC_CBBIT if sched == "scaBit" else oracle.ENC_LOCAL
    init = oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=21, mcs=3)
    if enc == oracle.ENC_LOCAL:
        init = oracle.cbbit_to_local(init, lx, ly)
    ref = init.copy()
    oracle.sca_mcs(ref, lx, ly, enc, 8, 0, 0, 9, 0.5, 0.5)
    s = kpzb.Scheduler(lx, ly, scheduler=sched)
    s.setPQ(0.5, 0.5)
    s.supplySeed(8)
    out = np.empty_like(init)
    s.pushSystemAsync(init)
    s.mcsPQSyncRngAsync(9)
    s.popSystemAsync(out)
    s.join()
    assert np.array_equal(out, ref)
    s.close()


@pytest.mark.parametrize("sched,lx", [("scaBit", 11), ("dt", 10), ("db4", 10)])
def test_pipelined_push_equals_sync(kpzb, oracle, sched, lx):
    """A staged kpzb_push_async (the next lattice copied from page-locked memory while the
    current one's MCS, pop and roughness are still queued) gives, step for step, the lattices
    and roughness of the synchronous push -> mcs -> pop -> roughness sequence on a second
    handle, bit for bit; a second push before the next MCS replaces the first."""
    import torch
    ly = lx
    enc = oracle.ENC_CBBIT if sched == "scaBit" else oracle.ENC_LOCAL
    inputs = []
    for k in range(3):
        a = oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=31 + k, mcs=2 + k)
        if enc == oracle.ENC_LOCAL:
            a = oracle.cbbit_to_local(a, lx, ly)
        t = torch.empty(a.size, dtype=torch.int32).pin_memory()
        t.numpy().view(np.uint32)[:] = a
        inputs.append(t)
    outs = [torch.empty(inputs[0].numel(), dtype=torch.int32).pin_memory() for _ in range(3)]
    n = 5
    sa = kpzb.Scheduler(lx, ly, scheduler=sched)
    sb = kpzb.Scheduler(lx, ly, scheduler=sched)
    for s in (sa, sb):
        s.setPQ(0.75, 0.25)
        s.supplySeed(17)
    got_r = []
    sa.pushSystemAsync(inputs[0].numpy().view(np.uint32))
    for k in range(3):
        sa.mcsPQSyncRngAsync(n)
        sa.popSystemAsync(outs[k].numpy().view(np.uint32))
        sa.roughnessAsync()
        if k + 1 < 3:
            if k == 0:  # replaced by the push below before any MCS reads it
                sa.pushSystemAsync(inputs[2].numpy().view(np.uint32))
            sa.pushSystemAsync(inputs[k + 1].numpy().view(np.uint32))
        got_r.append(sa.joinRoughness())
    sa.join()
    for k in range(3):
        sb.pushSystem(inputs[k].numpy().view(np.uint32))
        sb.mcsPQSyncRng(n)
        ref = sb.popSystem()
        got = outs[k].numpy().view(np.uint32)
        assert first_diff(got, ref) is None, (k, first_diff(got, ref))
        r = sb.roughness()
        assert (got_r[k].w2, got_r[k].h) == (r.w2, r.h), k
    sa.close()
    sb.close()


@pytest.mark.parametrize("p,q,kind", [(1.0, 0.0, "strip"), (0.5, 0.5, "strip"), (0.9, 0.1, "band")])
def test_untuned_default_plan(kpzb, oracle, monkeypatch, p, q, kind):
    """KPZB_AUTOTUNE=0: no measurement; the warp-tile kernel for rates of at most one random
    plane, the band heuristic otherwise -- word for word against the oracle either way."""
    monkeypatch.setenv("KPZB_AUTOTUNE", "0")
    monkeypatch.delenv("KPZB_TUNE_CACHE", raising=False)
    lx, ly, n = 13, 7, 13  # a size no other test tunes (the process caches tuned plans)
    ref = oracle.homogeneous(lx, ly, oracle.ENC_CBBIT)
    oracle.sca_mcs(ref, lx, ly, oracle.ENC_CBBIT, 4, 0, 0, n, p, q)
    s = kpzb.Scheduler(lx, ly)
    s.setPQ(p, q)
    s.supplySeed(4)
    s.mcsPQSyncRng(n)
    assert s.plan()[2] == kind
    got = s.popSystem()
    s.close()
    assert first_diff(got, ref) is None, first_diff(got, ref)


@pytest.mark.parametrize("lx,ly,k,band,p,q", [
    (11, 7, 4, 16, 1.0, 0.0),    # a 32-word row: one periodic strip, shuffles wrap the warp
    (11, 5, 6, 64, 0.5, 0.5),    # fewer rows than a tile: the halo wraps the lattice
    (12, 8, 4, 2, 0.5, 0.5),     # two-row tiles: nearly every row is halo
    (12, 6, 8, 16, 1.0, 1.0),    # the deepest pass; every candidate flips
    (13, 7, 6, 24, 0.5, 0.0),    # one random plane, no maxima
    (13, 5, 4, 32, 0.0, 1.0),    # only maxima
    (13, 6, 4, 16, 0.0, 0.5),
    (14, 6, 6, 32, 1.0, 0.0),    # the headline width: nine strips, the last one partly wrapped
    (14, 5, 4, 16, 0.5, 0.5),    # ten strips of 28 columns
    (14, 6, 6, 64, 1.0, 0.5),    # always deposit, desorb on the MSB plane
    (14, 5, 4, 16, 0.5, 1.0),
    (15, 4, 8, 8, 1.0, 0.0),     # 512-word rows
    (14, 4, 4, 16, 0.0, 0.0),    # nothing flips: the pass copies
    (13, 4, 4, 16, 0.9, 0.1),    # generic rates: the strip kernel does not cover them, band fallback
])
def test_strip_kernel_bit_exact(kpzb, oracle, monkeypatch, lx, ly, k, band, p, q):
    """The warp-tile pass kernel (scabit_strip_kernel), word for word with counters: one or
    many strips per row, strips of 30 or 28 columns, tiles of 2 to 64 rows, halos that wrap."""
    monkeypatch.setenv("KPZB_PASS_KERNEL", f"strip{band}")
    n = 2 * k + 1
    init = oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=19, mcs=2)
    ref = init.copy()
    rc = oracle.sca_mcs_words(ref, lx, ly, 11, 5, 0, n, p, q)
    s = kpzb.Scheduler(lx, ly)
    s.pushSystem(init)
    s.setPQ(p, q)
    s.supplySeed(11, 5)
    s.setFusion(k)
    s.enableCounters(True)
    s.mcsPQSyncRng(n)
    got = s.popSystem()
    cnt = s.counters()
    plan = s.plan()
    s.close()
    assert plan[2] == ("band" if (p, q) == (0.9, 0.1) else "strip"), plan
    assert first_diff(got, ref) is None, first_diff(got, ref)
    assert cnt == rc


@pytest.mark.parametrize("fusion", [1, 0])
def test_random_rates_vs_reference_with_injected_decisions(kpzb, oracle, fusion):
    """At random rates, the GPU lattice against the reference's own per-site update fed the
    counter stream's decisions (tests/golden/ref_inject_cbbit.npz, from oracle/ref_inject.cpp),
    one half-step per launch and the tuned pass plan."""
    from test_oracle_ref_inject import STREAM, SEED, cases
    for name, p, q, lx, n, w, want in cases(oracle):
        s = kpzb.Scheduler(lx, lx)
        s.pushSystem(w)
        s.setPQ(p, q)
        s.supplySeed(SEED, STREAM)
        s.setFusion(fusion)
        s.mcsPQSyncRng(n)
        got = s.popSystem()
        s.close()
        assert first_diff(got, want) is None, (name, first_diff(got, want))
