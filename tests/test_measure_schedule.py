"""Measurement schedule (kpzb_sample_times) against a restatement of the reference's
SamplingParam::nextEval (kpz/sampling.h:84-100) and the EndEvent that closes every run
(kpz/kpzFrontend.cpp:744-752).  Host code only: runs without a GPU."""
import math

import numpy as np
import pytest


def ref_times(start, end, mode, density=0.1, interval=0):
    """kpz/sampling.h:84-100: linear -> t + interval; exp -> ceil(exp(log(t + 10) + density));
    the frontend advances to min(next, next event), the last event being the end time."""
    out, t = [], start
    while t < end:
        if mode == "linear":
            n = t + interval
        else:
            n = int(math.ceil(math.exp(math.log(t + 10) + density)))
        t = min(n, end)
        out.append(t)
    return out


@pytest.mark.parametrize("start,end,density", [(0, 1000, 0.1), (0, 10**6, 0.1), (37, 5000, 0.05),
                                                (0, 12, 0.1), (0, 5, 0.3)])
def test_exp_sampling_matches_reference_rule(kpzb, start, end, density):
    got = kpzb.sample_times(start, end, kpzb.make_sampling("exp", density=density))
    assert got.tolist() == ref_times(start, end, "exp", density=density)


@pytest.mark.parametrize("start,end,interval", [(0, 100, 7), (10, 11, 5), (0, 64, 64), (3, 1000, 1)])
def test_linear_sampling_matches_reference_rule(kpzb, start, end, interval):
    got = kpzb.sample_times(start, end, kpzb.make_sampling("linear", interval=interval))
    assert got.tolist() == ref_times(start, end, "linear", interval=interval)


def test_random_sampling_spacing(kpzb):
    mean = 20.0
    t = kpzb.sample_times(0, 200000, kpzb.make_sampling("random", random_mean=mean, seed=9))
    d = np.diff(np.concatenate([[0], t]))[:-1]  # the last step is clipped at the end time
    assert d.min() >= mean and d.max() < 2 * mean  # t + floor(u*mean + mean), u in [0, 1)
    assert abs(d.mean() - 1.5 * mean + 0.5) < 0.2
    again = kpzb.sample_times(0, 200000, kpzb.make_sampling("random", random_mean=mean, seed=9))
    assert np.array_equal(t, again)  # seeded counter stream: reproducible


def test_empty_and_invalid(kpzb):
    assert kpzb.sample_times(50, 50).size == 0
    with pytest.raises(kpzb.KpzbError):
        kpzb.sample_times(0, 10, kpzb.make_sampling("linear", interval=0))
    with pytest.raises(kpzb.KpzbError):
        kpzb.sample_times(0, 10, kpzb.make_sampling("exp", density=0.0))
