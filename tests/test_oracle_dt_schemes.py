"""CPU checks of the oracle's emulations of the reference's block-level decompositions
(CPU only): DT, DTDBSH, DB, DBSH, DBSHRep (kpz/kpzConst.h:26-35) and the DB4 scheduler
(kpz/scheduler.cu).  Each keeps the surface a valid height field (the reference's
consitencyCheck invariants), changes the total height by exactly 2 (#dep - #des), does
nothing at p = q = 0, and -- where the schemes differ only in what they leave out -- relates
to its sibling as the reference's code says: DB4 attempts ~5.8% fewer sites than a full MCS
(its dead border), DBSHRep repeats every border hit but those of threads 1..31."""
import numpy as np
import pytest

INNER = ["dt", "dtdbsh", "db", "dbsh", "dbshrep"]


def total_height(oracle, w, lx, ly):
    return int(oracle.heights(w, lx, ly, oracle.ENC_LOCAL).astype(np.int64).sum())


@pytest.mark.parametrize("inner", INNER + ["db4"])
def test_scheme_keeps_invariants_and_height_balance(oracle, inner):
    lx, ly = (9, 8)
    init = oracle.cbbit_to_local(oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=3, mcs=5), lx, ly)
    w = init.copy()
    if inner == "db4":
        dep, des = oracle.db4_mcs(w, lx, ly, 11, 1, 0, 4, 0.7, 0.3)
    else:
        dep, des = oracle.dt_mcs_inner(w, lx, ly, 11, 1, 0, 4, 0.7, 0.3, inner)
    assert dep > 0 and des > 0
    assert oracle.check_invariants(w, lx, ly, oracle.ENC_LOCAL) == [0, 0, 0]
    # heights are relative to site (0, 0): compare through the absolute offset of the walk
    h0 = oracle.heights(init, lx, ly, oracle.ENC_LOCAL).astype(np.int64)
    h1 = oracle.heights(w, lx, ly, oracle.ENC_LOCAL).astype(np.int64)
    d = h1 - h0
    # every site's height changed by an even amount; the sum of changes is 2(dep - des)
    # up to the common offset the relative heights hide
    off = (2 * (dep - des) - int(d.sum())) / d.size
    assert np.all(((d + off) % 2) == 0)


@pytest.mark.parametrize("inner", INNER + ["db4"])
def test_zero_rates_change_nothing(oracle, inner):
    lx, ly = 9, 8
    init = oracle.cbbit_to_local(oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=8, mcs=3), lx, ly)
    w = init.copy()
    if inner == "db4":
        oracle.db4_mcs(w, lx, ly, 2, 0, 0, 2, 0.0, 0.0)
    else:
        oracle.dt_mcs_inner(w, lx, ly, 2, 0, 0, 2, 0.0, 0.0, inner)
    assert np.array_equal(w, init)


def test_db4_dead_border_fraction(oracle):
    """At p = q = 1 every active attempt on a local extremum flips; at the flat start every
    second site of a row is a minimum, so the first launch's flips count its live attempts on
    minima.  Over many MCS the DB4 flip count per MCS stays below the DT count by about the
    dead-border fraction (1 - 251*123/32768 = 5.8%)."""
    lx, ly = 9, 8
    w1 = oracle.homogeneous(lx, ly, oracle.ENC_LOCAL)
    w2 = oracle.homogeneous(lx, ly, oracle.ENC_LOCAL)
    d1 = oracle.db4_mcs(w1, lx, ly, 5, 0, 0, 30, 0.5, 0.5)
    d2 = oracle.dt_mcs_inner(w2, lx, ly, 5, 0, 0, 30, 0.5, 0.5, "dt")
    ratio = sum(d1) / sum(d2)
    assert 0.92 < ratio < 0.97, ratio


def test_dbshrep_loses_the_border_hits_of_threads_1_to_31(oracle):
    """With p = 1, q = 0 from the flat start both DBSH and DBSHRep only deposit; DBSHRep
    deposits slightly fewer (1-5%) because the border hits of threads 1..31 of each block are
    never repeated (the reference's reduction leaves them out)."""
    lx, ly = 9, 8
    a = oracle.homogeneous(lx, ly, oracle.ENC_LOCAL)
    b = oracle.homogeneous(lx, ly, oracle.ENC_LOCAL)
    da = oracle.dt_mcs_inner(a, lx, ly, 3, 0, 0, 20, 1.0, 0.0, "dbsh")
    db = oracle.dt_mcs_inner(b, lx, ly, 3, 0, 0, 20, 1.0, 0.0, "dbshrep")
    assert da[1] == 0 and db[1] == 0
    assert 0.95 < db[0] / da[0] < 1.0, (da, db)
