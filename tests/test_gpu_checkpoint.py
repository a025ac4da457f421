"""Checkpoint / resume (kpzb_save / kpzb_load): saveBit's layout (kpz/schedulerService.cpp:
389-401) plus a trailer with the counter-stream state.  A resumed run equals the uninterrupted
one word for word; a plain saveBit file written by the reference's own code loads as a lattice."""
from pathlib import Path

import numpy as np
import pytest

from test_oracle_golden import read_savebit

pytestmark = pytest.mark.gpu
G = Path(__file__).resolve().parent / "golden"


def make(kpzb, lx, ly, sched, p, q, seed, stream=0, fusion=0):
    s = kpzb.Scheduler(lx, ly, scheduler=sched)
    s.setPQ(p, q)
    s.supplySeed(seed, stream)
    s.setFusion(fusion)
    return s


@pytest.mark.parametrize("sched,lx,ly,p,q", [("scaBit", 9, 9, 0.5, 0.5), ("sca", 9, 8, 0.75, 0.25),
                                             ("dt", 10, 9, 0.95, 0.05), ("scaBit", 10, 8, 1.0, 0.0)])
def test_resume_equals_uninterrupted(kpzb, tmp_path, sched, lx, ly, p, q):
    a = make(kpzb, lx, ly, sched, p, q, 21, stream=3)
    a.mcsPQSyncRng(7)
    a.correlateTag()
    f = tmp_path / "ck.bin"
    a.saveBit(f, "t=7")
    a.mcsPQSyncRng(9)
    ref_words, (ref_r, ref_ch, ref_cs) = a.popSystem(), a.correlate()
    a.close()
    # a fresh handle with other rates and seed: everything comes from the file
    b = make(kpzb, lx, ly, sched, 0.1, 0.9, 999)
    b.loadBit(f)
    assert b.deviceMcs() == 7
    b.mcsPQSyncRng(9)
    assert np.array_equal(b.popSystem(), ref_words)
    r, ch, cs = b.correlate()
    assert (r.w2, ch, cs) == (ref_r.w2, ref_ch, ref_cs)
    b.close()


def test_checkpoint_file_is_a_savebit_file(kpzb, tmp_path):
    s = make(kpzb, 9, 9, "sca", 0.5, 0.5, 4)
    s.mcsPQSyncRng(5)
    f = tmp_path / "ck.bin"
    s.saveBit(f, "meta")
    lx, ly, meta, words, rest = read_savebit(f)
    assert (lx, ly, meta) == (9, 9, "meta")
    assert np.array_equal(words, s.popSystem())  # ENC_LOCAL words, as the reference's m_system
    assert rest[:8] == b"KPZBCKPT"
    s.close()


def test_load_reference_savebit_file(kpzb, oracle):
    """The reference's own saveBit output (RS 256^2 after 16 MCS) loads into an SCA handle."""
    lx, ly, _, words, _ = read_savebit(G / "ref_savebit_rs256.bin")
    s = kpzb.Scheduler(lx, ly, scheduler="sca")
    s.loadBit(G / "ref_savebit_rs256.bin")
    assert np.array_equal(s.popSystem(), words)
    assert s.deviceMcs() == 0  # a plain saveBit file carries no MCS
    ok, rep = s.consitencyCheck()
    assert ok, rep
    s.close()


def test_load_rejects_wrong_size(kpzb, tmp_path):
    s = make(kpzb, 9, 9, "scaBit", 0.5, 0.5, 4)
    f = tmp_path / "ck.bin"
    s.saveBit(f)
    t = kpzb.Scheduler(10, 9, scheduler="scaBit")
    with pytest.raises(kpzb.KpzbError):
        t.loadBit(f)
    d = kpzb.Scheduler(9, 9, scheduler="sca")  # same size, other dynamics: trailer rejected
    with pytest.raises(kpzb.KpzbError):
        d.loadBit(f)
    for x in (s, t, d):
        x.close()


@pytest.mark.parametrize("inner", ["dbsh", "dbshrep"])
def test_dt_checkpoint_keeps_the_inner_scheme(kpzb, tmp_path, inner):
    """A DT checkpoint carries the inner decomposition: a handle left at the default scheme
    resumes with the saved one, bit for bit; DB4 checkpoints resume too."""
    a = make(kpzb, 10, 9, "dt", 0.9, 0.2, 5)
    a.setDtInner(inner)
    a.mcsPQSyncRng(3)
    f = tmp_path / "dt.bin"
    a.saveBit(f)
    a.mcsPQSyncRng(4)
    ref = a.popSystem()
    a.close()
    b = kpzb.Scheduler(10, 9, scheduler="dt")
    b.loadBit(f)
    b.mcsPQSyncRng(4)
    assert np.array_equal(b.popSystem(), ref)
    b.close()
    c = make(kpzb, 9, 8, "db4", 0.9, 0.2, 6)
    c.mcsPQSyncRng(2)
    g = tmp_path / "db4.bin"
    c.saveBit(g)
    c.mcsPQSyncRng(3)
    ref4 = c.popSystem()
    c.close()
    d = kpzb.Scheduler(9, 8, scheduler="db4")
    d.loadBit(g)
    d.mcsPQSyncRng(3)
    assert np.array_equal(d.popSystem(), ref4)
    d.close()
