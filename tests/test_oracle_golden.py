"""Pin the CPU oracle against golden vectors produced by the reference's own code (CPU only).

The fixtures in tests/golden/ were written by tests/golden/make_golden.py, which runs the
CudaKpz CPU schedulers compiled from their sources (oracle/build_ref.py):
  * SchedulerCPU random-sequential 256^2 run with dSFMT (kpz/schedulerCPU.inl:74-88),
  * dSFMT-19937 draws (inc/dSFMT/dSFMT.h:262-264),
  * SchedulerCPUCBBit / SchedulerCPUCB checkerboard runs at deterministic rates
    (kpz/schedulerCPUCBBit_nested.inl:261-295),
  * Correlator roughness / correlate and SchedulerService::consitencyCheck.
Everything here is bit-exact, except the FP moments, which must agree to the last bit too
because both sides accumulate the same integers in the same order.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

G = Path(__file__).resolve().parent / "golden"


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()


def test_philox_known_answers(oracle):
    # Random123 known-answer vectors for Philox4x32-10 (Salmon et al., SC'11)
    assert oracle.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    f = 0xFFFFFFFF
    assert oracle.philox([f, f, f, f], [f, f]) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                         [0xA4093822, 0x299F31D0]) == [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_dsfmt_matches_reference(oracle):
    d = json.loads((G / "ref_dsfmt.json").read_text())
    r = oracle.DSFMT(1234, reseed=False)
    assert [r.close_open() for _ in range(8)] == d["seed1234_first8"]
    r = oracle.DSFMT(1, reseed=True)
    assert [r.close_open() for _ in range(8)] == d["seed1_reseeded_first8"]


def test_random_sequential_256_matches_reference(oracle):
    """Config C1: RS CPU scheduler, 256^2, p=1 q=0, seed 1; W^2 and moments at t=2^k."""
    g = json.loads((G / "ref_rs256_seed1.json").read_text())
    lx = g["lx"]
    w = oracle.homogeneous(lx, lx, oracle.ENC_LOCAL)
    rng = oracle.DSFMT(g["seed"])
    t = 0
    for T, row in zip(g["t"], g["roughness"]):
        oracle.rs_mcs(w, lx, lx, rng, T - t)
        t = T
        assert list(oracle.roughness(w, lx, lx, oracle.ENC_LOCAL)) == row, T
    assert sha(w) == g["final_lattice_sha256"]


def _sca_cases():
    z = np.load(G / "ref_sca_deterministic.npz")
    keys = sorted(k[:-3] for k in z.files if k.endswith("_in"))
    return z, keys


@pytest.mark.parametrize("key", _sca_cases()[1])
def test_sca_deterministic_matches_reference(oracle, key):
    z, _ = _sca_cases()
    cmd, lxs, ps, qs, _init = key.split("_")
    lx, p, q = int(lxs[2:]), float(ps[1:]), float(qs[1:])
    enc = oracle.ENC_CBBIT if cmd == "cbbit" else oracle.ENC_LOCAL
    w = z[key + "_in"].copy()
    oracle.sca_mcs(w, lx, lx, enc, 123, 0, 0, 7, p, q)
    assert np.array_equal(w, z[key + "_out"])


@pytest.mark.parametrize("enc", [0, 1])
@pytest.mark.parametrize("lx", [6, 8, 9])
def test_roughness_and_correlator_match_reference(oracle, enc, lx):
    z = np.load(G / "ref_analysis.npz")
    k = f"enc{enc}_lx{lx}"
    w, s = z[k + "_sys"], z[k + "_snap"]
    assert np.array_equal(oracle.roughness(w, lx, lx, enc), z[k + "_rough"])
    snap_mean = oracle.roughness(s, lx, lx, enc)[1]
    np.testing.assert_array_equal(oracle.correlate(w, s, lx, lx, enc, snap_mean), z[k + "_corr"])


@pytest.mark.parametrize("lx", [6, 8, 9])
def test_consistency_check_matches_reference(oracle, lx):
    z = np.load(G / "ref_analysis.npz")
    k = f"enc0_lx{lx}"
    w = z[k + "_sys"].copy()
    assert (oracle.check_invariants(w, lx, lx, 0) == [0, 0, 0]) == bool(z[k + "_check_valid"])
    w[3] ^= 1 << 4
    assert (oracle.check_invariants(w, lx, lx, 0) == [0, 0, 0]) == bool(z[k + "_check_broken"])


def read_savebit(path):
    """Parse SchedulerService::saveBit's layout (kpz/schedulerService.cpp:389-401):
    "<lx>\\n<ly>\\n" + meta + '\\0' + the lattice words; returns (lx, ly, meta, words, rest)."""
    b = Path(path).read_bytes()
    nl1 = b.index(b"\n")
    nl2 = b.index(b"\n", nl1 + 1)
    lx, ly = int(b[:nl1]), int(b[nl1 + 1:nl2])
    z = b.index(b"\0", nl2 + 1)
    meta = b[nl2 + 1:z].decode()
    nw = 1 << (lx + ly - 4)
    words = np.frombuffer(b[z + 1:z + 1 + 4 * nw], dtype=np.uint32)
    return lx, ly, meta, words, b[z + 1 + 4 * nw:]


def test_savebit_fixture_is_the_rs_lattice(oracle):
    """The reference's saveBit file of the RS run (256^2, seed 1, 16 MCS) holds exactly the
    oracle's lattice after the same 16 MCS."""
    lx, ly, meta, words, rest = read_savebit(G / "ref_savebit_rs256.bin")
    assert (lx, ly, meta, rest) == (8, 8, "CudaKpz saveBit fixture", b"")
    w = oracle.homogeneous(8, 8, oracle.ENC_LOCAL)
    oracle.rs_mcs(w, 8, 8, oracle.DSFMT(1), 16)
    assert np.array_equal(words, w)


def test_disorder_generation_and_rs_dynamics(oracle):
    """SchedulerService::generateDisorder2 and SchedulerCPU::mcsDisorder2 (256^2, seed 3,
    fill 0.3, 20 MCS, class rates (0.9,0.1) and (0.3,0.6)), reproduced bit for bit."""
    z = np.load(G / "ref_disorder.npz")
    rng = oracle.DSFMT(3)
    d = oracle.generate_disorder2(8, 8, rng, 0.3)
    assert np.array_equal(d, z["disorder"])
    w = oracle.homogeneous(8, 8, oracle.ENC_LOCAL)
    oracle.rs_mcs_dis(w, 8, 8, rng, 20, [0.9, 0.3], [0.1, 0.6], d)
    assert np.array_equal(w, z["lattice"])


def test_disorder_with_equal_rates_is_the_plain_dynamics(oracle):
    """The counter-stream disorder restatement with every class at the same rates is the plain
    SCA / DT dynamics (same random stream)."""
    lx = ly = 9
    dis = oracle.random_lattice(lx, ly, oracle.ENC_LOCAL, seed=4)  # arbitrary class bits
    a = oracle.homogeneous(lx, ly, oracle.ENC_CBBIT)
    b = a.copy()
    oracle.sca_mcs(a, lx, ly, oracle.ENC_CBBIT, 5, 0, 0, 3, 0.7, 0.2)
    oracle.sca_mcs_dis(b, lx, ly, oracle.ENC_CBBIT, 5, 0, 0, 3, [0.7] * 4, [0.2] * 4, dis)
    assert np.array_equal(a, b)
