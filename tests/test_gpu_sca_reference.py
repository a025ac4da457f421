"""SCABit against the reference's own GPU SchedulerSCABit<SLCG64> (kpz/schedulerSCABit.cu,
kpz/kpzSCABit.cu), built from the CudaKpz sources for sm_100a by oracle/build_ref.py into
oracle/_ref/kpz_ref_gpu and run on the same GPU:
  * p = 1, q = 0 is deterministic (its EmptyAnyP core compares randomFloat() < 1, always
    true): the lattices must agree word for word;
  * random rates use different streams: the seed-averaged W^2(t) must agree within the
    standard errors (|z| < 4.5 at every t = 2^k; 4096^2, 16 seeds each)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "kpz_ref_gpu"
needs_ref = pytest.mark.skipif(not REF.exists(), reason="reference GPU schedulers not built (needs the CudaKpz sources)")


@needs_ref
@pytest.mark.parametrize("lx,n", [(11, 7), (12, 20)])
def test_deterministic_rates_bit_exact_vs_reference_gpu(kpzb, tmp_path, lx, n):
    f = tmp_path / "ref.bin"
    subprocess.run([str(REF), "scabitdump", str(lx), "1", "0", str(n), str(f)], check=True, capture_output=True,
                   timeout=600)
    ref = np.fromfile(f, dtype=np.uint32)
    s = kpzb.Scheduler(lx, lx, scheduler="scaBit")
    s.setPQ(1.0, 0.0)
    s.supplySeed(99)
    s.mcsPQSyncRng(n)
    got = s.popSystem()
    s.close()
    assert got.size == ref.size
    assert np.array_equal(got, ref)


@needs_ref
@pytest.mark.parametrize("p,q", [(0.5, 0.5), (0.9, 0.1)])
def test_random_rates_statistics_vs_reference_gpu(kpzb, p, q):
    lx, seeds = 12, 16
    ts = [2 ** i for i in range(11)]
    ref = []
    for sd in range(1, seeds + 1):
        r = subprocess.run([str(REF), "scabitcurve", str(lx), str(p), str(q), str(sd)] + [str(t) for t in ts],
                           capture_output=True, text=True, check=True, timeout=600)
        rows = [ln.split() for ln in r.stdout.splitlines() if ln and not ln.startswith("#")]
        ref.append([float(x[1]) for x in rows])
    ours = []
    for sd in range(1, seeds + 1):
        s = kpzb.Scheduler(lx, lx, scheduler="scaBit")
        s.setPQ(p, q)
        s.supplySeed(500 + sd)
        t, cur = 0, []
        for T in ts:
            s.mcsPQSyncRng(T - t)
            t = T
            cur.append(s.roughness().w2)
        ours.append(cur)
        s.close()
    ref, ours = np.array(ref), np.array(ours)
    se = np.sqrt(ref.var(0, ddof=1) / seeds + ours.var(0, ddof=1) / seeds)
    z = (ours.mean(0) - ref.mean(0)) / se
    assert np.all(np.abs(z) < 4.5), (z, ours.mean(0), ref.mean(0))
