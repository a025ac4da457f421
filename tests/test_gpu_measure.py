"""kpzb_measure_run (device-side measurements on the reference's sampling schedule) against the
same schedule driven step by step through kpzb_mcs + kpzb_roughness / kpzb_corr_tag /
kpzb_correlate, and against the CPU oracle.  Reference loop: kpz/kpzScaling.cpp:194-215,
SchedulerService::correlate (kpz/schedulerService.cpp:292-297)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def stepwise(kpzb, lx, ly, sched, p, q, seed, times, corr_start=-1, corr_stop=0, fusion=0):
    s = kpzb.Scheduler(lx, ly, scheduler=sched)
    s.setPQ(p, q)
    s.supplySeed(seed)
    s.setFusion(fusion)
    rows = []
    tagged = False
    for t in times:
        s.mcsPQSyncRng(int(t) - s.deviceMcs())
        r = s.roughness()
        row = [float(t), r.w2, *r.h, np.nan, np.nan]
        if corr_start >= 0 and t == corr_start:
            s.correlateTag()
            tagged = True
        elif tagged and t <= corr_stop:
            _, ch, cs = s.correlate()
            row[9], row[10] = ch, cs
        rows.append(row)
    s.close()
    return np.array(rows)


def measured(kpzb, lx, ly, sched, p, q, seed, end, sampling=None, corr_start=-1, corr_stop=0, fusion=0):
    s = kpzb.Scheduler(lx, ly, scheduler=sched)
    s.setPQ(p, q)
    s.supplySeed(seed)
    s.setFusion(fusion)
    rows = s.measureRun(end, sampling, corr_start, corr_stop)
    assert s.deviceMcs() == end
    s.close()
    return rows


@pytest.mark.parametrize("sched,lx,ly,p,q,fusion", [("scaBit", 9, 9, 0.5, 0.5, 0), ("scaBit", 10, 8, 1.0, 0.0, 4),
                                                    ("sca", 9, 9, 0.75, 0.25, 1), ("dt", 10, 9, 0.95, 0.05, 0)])
def test_measure_run_equals_stepwise(kpzb, sched, lx, ly, p, q, fusion):
    end = 300
    smp = kpzb.make_sampling("exp", density=0.1)
    times = kpzb.sample_times(0, end, smp)
    got = measured(kpzb, lx, ly, sched, p, q, 7, end, smp, corr_start=25, corr_stop=200, fusion=fusion)
    assert 25 in times.tolist()
    ref = stepwise(kpzb, lx, ly, sched, p, q, 7, times, corr_start=25, corr_stop=200, fusion=fusion)
    np.testing.assert_array_equal(got, ref)
    assert np.isnan(got[got[:, 0] <= 25, 9]).all() and not np.isnan(got[(got[:, 0] > 25) & (got[:, 0] <= 200), 9]).any()


def test_measure_run_tag_between_samples_and_linear(kpzb):
    end = 60
    smp = kpzb.make_sampling("linear", interval=9)
    got = measured(kpzb, 9, 9, "scaBit", 0.6, 0.3, 3, end, smp, corr_start=20, corr_stop=50)
    times = sorted(set(kpzb.sample_times(0, end, smp).tolist()) | {20})
    assert got[:, 0].tolist() == times  # the tag time is a measurement row of its own
    ref = stepwise(kpzb, 9, 9, "scaBit", 0.6, 0.3, 3, times, corr_start=20, corr_stop=50)
    np.testing.assert_array_equal(got, ref)


def test_measure_run_against_oracle(kpzb, oracle):
    lx = ly = 8
    p, q, seed, end = 0.5, 0.5, 11, 40
    smp = kpzb.make_sampling("exp", density=0.3)
    got = measured(kpzb, lx, ly, "scaBit", p, q, seed, end, smp)
    w = oracle.homogeneous(lx, ly, oracle.ENC_CBBIT)
    t = 0
    for row in got:
        oracle.sca_mcs(w, lx, ly, oracle.ENC_CBBIT, seed, 0, t, int(row[0]) - t, p, q)
        t = int(row[0])
        r = oracle.roughness(w, lx, ly, oracle.ENC_CBBIT)
        assert row[1] == pytest.approx(r[0], rel=1e-12, abs=1e-12)
        np.testing.assert_allclose(row[2:9], r[1:8], rtol=1e-12)


def test_measure_run_small_buffer_and_tag_now(kpzb):
    s = kpzb.Scheduler(9, 9)
    s.setPQ(0.5, 0.5)
    s.supplySeed(2)
    s.mcsPQSyncRng(5)
    rows = s.measureRun(30, kpzb.make_sampling("linear", interval=5), corr_start=5, corr_stop=30)
    assert rows[0, 0] == 5 and np.isnan(rows[0, 9])  # snapshot row at the current time
    assert not np.isnan(rows[1:, 9]).any()
    assert rows[:, 0].tolist() == [5, 10, 15, 20, 25, 30]
    s.close()


@pytest.mark.parametrize("sched", ["scaBit", "sca", "dt"])
def test_roughness_async_equals_sync(kpzb, sched):
    """kpzb_roughness_async / kpzb_roughness_join (SchedulerService::roughnessAsync /
    joinRoughness): the value of the lattice at enqueue time, equal to kpzb_roughness."""
    lx, ly = (10, 9)
    s = kpzb.Scheduler(lx, ly, scheduler=sched)
    s.setPQ(0.7, 0.2)
    s.supplySeed(4)
    with pytest.raises(kpzb.KpzbError):
        s.joinRoughness()  # nothing pending
    s.mcsPQSyncRngAsync(5)
    s.roughnessAsync()
    s.mcsPQSyncRngAsync(3)  # enqueued after: not part of the pending result
    r_async = s.joinRoughness()
    s.close()
    t = kpzb.Scheduler(lx, ly, scheduler=sched)
    t.setPQ(0.7, 0.2)
    t.supplySeed(4)
    t.mcsPQSyncRng(5)
    r = t.roughness()
    t.close()
    assert r_async.w2 == r.w2 and r_async.h == r.h
