"""DT statistics against the reference's own GPU DT scheduler (config C3: W^2(t) and beta
within error bars).  The reference's SchedulerDT<SLCG64, dis> with its single-hit
double-tiling inner scheme (KPZ_INNER_DT, kpz/kpzSimulationPrimitivesTemplates.cu:108-141 --
the scheme the DT kernel here follows) is built from the CudaKpz sources by
oracle/build_ref.py into oracle/_ref/kpz_ref_gpu_innerdt and run on the same GPU; both
implementations use independent random streams, so the comparison is statistical: the
seed-averaged W^2 at t = 2^k and the fitted growth exponent must agree within their
standard errors (|z| < 4.5 at every time, beta within 4 sigma); the default DBSH and the DT
scheme at 4096^2 with 16 seeds each -- statistics fine enough to resolve the 0.5 % difference
between two decompositions, which a separate test checks -- the other schemes at 2048^2."""
import functools
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "kpz_ref_gpu_innerdt"
P, Q = 0.95, 0.05
TS = [2 ** i for i in range(11)]


def beta_of(w2):
    t = np.array(TS, dtype=float)
    sel = t >= 16
    return np.polyfit(np.log(t[sel]), np.log(w2[sel]), 1)[0] / 2


REF_DBSH = REF.parent / "kpz_ref_gpu"


# (lx, seeds): the reference's default DBSH and the single-hit DT scheme at 4096^2 with 16
# seeds; the other schemes at 2048^2 with 12 seeds (every scheme compared, the suite kept short)
FINE, COARSE = (12, 16), (11, 12)


@pytest.mark.parametrize("sched,inner,binary,cmd,size", [
    ("dt", "dt", REF, "dtcurve", FINE),
    ("dt", "dbsh", REF_DBSH, "dtcurve", FINE),
    ("dt", "db", REF.parent / "kpz_ref_gpu_innerdb", "dtcurve", COARSE),
    ("dt", "dtdbsh", REF.parent / "kpz_ref_gpu_innerdtdbsh", "dtcurve", COARSE),
    ("dt", "dbshrep", REF.parent / "kpz_ref_gpu_innerdbshrep", "dtcurve", COARSE),
    ("db4", None, REF_DBSH, "db4curve", COARSE),
])
def test_dt_statistics_match_reference_gpu_dt(kpzb, sched, inner, binary, cmd, size):
    """inner "dt": the reference built with KPZ_INNER_DT; "dbsh": its default build
    (KPZ_INNER_DBSH, kpz/param.h); "db", "dtdbsh", "dbshrep": built with KPZ_INNER_DB,
    KPZ_INNER_DTDBSH, KPZ_INNER_DBSHREP -- each against this library's DT kernel with the same
    inner scheme; "db4": the reference's DB4 scheduler (Scheduler<SLCG64, LocalLayoutDB4>,
    --scheduler db4) against this library's."""
    if not binary.exists():
        pytest.skip("reference GPU DT not built (needs the CudaKpz sources)")
    lx, seeds = size
    ref = np.array(reference_curves(str(binary), cmd, lx, seeds))
    ours = np.array(our_curves(kpzb, sched, inner, lx, seeds))
    m_r, m_o = ref.mean(0), ours.mean(0)
    se = np.sqrt(ref.var(0, ddof=1) / seeds + ours.var(0, ddof=1) / seeds)
    z = (m_o - m_r) / se
    assert np.all(np.abs(z) < 4.5), (z, m_o, m_r)
    b_r = np.array([beta_of(x) for x in ref])
    b_o = np.array([beta_of(x) for x in ours])
    sb = np.sqrt(b_r.var(ddof=1) / seeds + b_o.var(ddof=1) / seeds)
    assert abs(b_o.mean() - b_r.mean()) < 4 * sb + 1e-3, (b_o.mean(), b_r.mean(), sb)


@functools.lru_cache(maxsize=None)
def reference_curves(binary, cmd, lx, seeds):
    out = []
    for s in range(1, seeds + 1):
        r = subprocess.run([binary, cmd, str(lx), str(P), str(Q), str(s)] + [str(t) for t in TS],
                           capture_output=True, text=True, check=True, timeout=600)
        rows = [ln.split() for ln in r.stdout.splitlines() if ln and not ln.startswith("#")]
        assert [int(x[0]) for x in rows] == TS
        out.append(tuple(float(x[1]) for x in rows))
    return tuple(out)


_ours = {}


def our_curves(kpzb, sched, inner, lx, seeds):
    key = (sched, inner, lx, seeds)
    if key not in _ours:
        rows = []
        for s in range(1, seeds + 1):
            h = kpzb.Scheduler(lx, lx, scheduler=sched)
            if inner:
                h.setDtInner(inner)
            h.setPQ(P, Q)
            h.supplySeed(1000 + s)
            t, cur = 0, []
            for T in TS:
                h.mcsPQSyncRng(T - t)
                t = T
                cur.append(h.roughness().w2)
            rows.append(cur)
            h.close()
        _ours[key] = rows
    return _ours[key]


def test_statistics_resolve_the_decomposition_difference(kpzb):
    """The power of the comparison above: this library's single-hit DT scheme against the
    reference's default DBSH build differ by about 0.5 % in W^2 at t = 8..64 MCS (a property of
    the two decompositions, seen the same way between the reference's own builds); at 4096^2
    with 16 seeds that difference must stand out (|z| > 6 at some t of 8..64), so a systematic
    of that size between a scheme here and the reference's build of it would fail the test."""
    if not REF_DBSH.exists():
        pytest.skip("reference GPU DT not built (needs the CudaKpz sources)")
    lx, seeds = FINE
    ref = np.array(reference_curves(str(REF_DBSH), "dtcurve", lx, seeds))
    ours = np.array(our_curves(kpzb, "dt", "dt", lx, seeds))
    se = np.sqrt(ref.var(0, ddof=1) / seeds + ours.var(0, ddof=1) / seeds)
    z = (ours.mean(0) - ref.mean(0)) / se
    sel = [i for i, t in enumerate(TS) if 8 <= t <= 64]
    assert np.max(np.abs(z[sel])) > 6, z
