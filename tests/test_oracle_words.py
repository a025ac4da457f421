"""The oracle's word-parallel SCABit restatement (ko_sca_mcs_words, 32 sites per operation)
against its per-site restatement (ko_sca_mcs, itself pinned to the reference's CPU
checkerboard schedulers at deterministic rates by test_oracle_golden.py): equal lattices and
equal deposition / desorption counts for every kind of rate -- none, one and many random
planes, rates near 0 and 1 -- on square and flat lattices, random starts, streams and start
times.  The word form is what the full-size GPU parity tests compare against."""
import numpy as np
import pytest

RATES = [(1.0, 0.0), (0.5, 0.5), (0.95, 0.05), (0.3, 0.7), (0.5, 0.0), (1.0, 1.0), (0.0, 0.0),
         (0.75, 0.25), (0.123456, 0.987), (1e-9, 0.999999999), (0.0, 1.0), (0.5, 1.0)]


@pytest.mark.parametrize("p,q", RATES)
@pytest.mark.parametrize("lx,ly", [(8, 8), (9, 7), (10, 3)])
def test_word_form_equals_per_site(oracle, lx, ly, p, q):
    a = oracle.random_lattice(lx, ly, oracle.ENC_CBBIT, seed=3, mcs=2)
    b = a.copy()
    ra = oracle.sca_mcs(a, lx, ly, oracle.ENC_CBBIT, 7, 2, 5, 3, p, q)
    rb = oracle.sca_mcs_words(b, lx, ly, 7, 2, 5, 3, p, q)
    assert np.array_equal(a, b)
    assert ra == rb


def test_word_form_flat_start_long_run(oracle):
    lx, ly = 9, 9
    a = oracle.homogeneous(lx, ly, oracle.ENC_CBBIT)
    b = a.copy()
    ra = oracle.sca_mcs(a, lx, ly, oracle.ENC_CBBIT, 42, 0, 0, 20, 0.5, 0.5)
    rb = oracle.sca_mcs_words(b, lx, ly, 42, 0, 0, 20, 0.5, 0.5)
    assert np.array_equal(a, b) and ra == rb
