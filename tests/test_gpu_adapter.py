"""The drop-in seam end to end: SchedulerB200 (tests/cpp/scheduler_b200_adapter.cpp), a
Kpz::SchedulerService subclass forwarding to this library's C ABI, built against the
reference's own headers and CPU objects into oracle/_ref/kpz_ref_adapter.  The reference's
host analysis -- SchedulerService::roughness and consitencyCheck -- runs unchanged on the
lattice this library produced and popped into m_system, and agrees with kpzb_roughness."""
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ADAPTER = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "kpz_ref_adapter"


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
