"""The drop-in seam end to end: SchedulerB200 (tests/cpp/scheduler_b200_adapter.cpp), a
Kpz::SchedulerService subclass forwarding to this library's C ABI, built against the
reference's own headers and CPU objects into oracle/_ref/kpz_ref_adapter.  The reference's
host analysis -- SchedulerService::roughness and consitencyCheck -- runs unchanged on the
lattice this library produced and popped into m_system, and agrees with kpzb_roughness."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ADAPTER = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "kpz_ref_adapter"
REF_DEFAULT = ADAPTER.parent / "kpz_ref_gpu"  # the reference's default build (DT with KPZ_INNER_DBSH)


@pytest.mark.skipif(not ADAPTER.exists(), reason="adapter not built (needs the CudaKpz sources)")
@pytest.mark.parametrize("lx,p,q,seed,n", [(9, 0.7, 0.2, 5, 6), (10, 0.5, 0.5, 1, 3), (9, 1.0, 0.0, 2, 4)])
def test_reference_frontend_runs_on_this_library(lx, p, q, seed, n):
    r = subprocess.run([str(ADAPTER), str(lx), str(p), str(q), str(seed), str(n)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-500:]
    # the reference prints set-up chatter on stdout beside the result line
    res = [ln.split()[1:] for ln in r.stdout.splitlines() if ln.startswith("RESULT ")]
    assert len(res) == 1, r.stdout[-800:]
    w2_ref, w2_ours, ok = res[0]
    assert int(ok) == 1
    assert float(w2_ref) == pytest.approx(float(w2_ours), rel=1e-12, abs=1e-12)


def _curve(cmd, lx, p, q, seed, ts):
    r = subprocess.run([str(cmd[0]), *cmd[1:], str(lx), str(p), str(q), str(seed), *map(str, ts)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-500:]
    rows = [ln.split() for ln in r.stdout.splitlines() if ln and ln[0].isdigit()]
    assert [int(x[0]) for x in rows] == list(ts), r.stdout[-500:]
    return [float(x[1]) for x in rows]


@pytest.mark.skipif(not (ADAPTER.exists() and REF_DEFAULT.exists()),
                    reason="adapter or reference GPU build missing (needs the CudaKpz sources)")
def test_dt_through_adapter_matches_reference_default_build():
    """--scheduler dt through the adapter (which sets the reference's default inner scheme,
    DBSH, explicitly) against the reference's own default GPU build of SchedulerDT
    (kpz/schedulerDT.cu:38-78 with KPZ_INNER_DBSH): W^2(t) from the reference's host
    SchedulerService::roughness, seed-averaged, within |z| < 4.5 at every t = 2^k
    (independent random streams, so the comparison is statistical)."""
    lx, p, q, seeds = 11, 0.95, 0.05, 12
    ts = [2 ** i for i in range(9)]
    ours = np.array([_curve([ADAPTER, "dtcurve"], lx, p, q, 2000 + s, ts) for s in range(seeds)])
    ref = np.array([_curve([REF_DEFAULT, "dtcurve"], lx, p, q, s + 1, ts) for s in range(seeds)])
    se = np.sqrt(ours.var(0, ddof=1) / seeds + ref.var(0, ddof=1) / seeds)
    z = (ours.mean(0) - ref.mean(0)) / se
    assert np.all(np.abs(z) < 4.5), (z, ours.mean(0), ref.mean(0))
