"""The C++ SchedulerService-style header (include/kpzb_scheduler.hpp) over the C ABI.

CPU: the demo client compiles and links against libkpzb200.so.  GPU: it runs and its
lattice equals the oracle's word for word (kpz/kpzScaling.cpp:142-215 is the reference caller
it mirrors).
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "cpp" / "scheduler_demo.cpp"


def build(tmp_path):
    exe = tmp_path / "scheduler_demo"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(SRC), "-o", str(exe),
                    "-L", str(ROOT / "cudakpz_b200"), "-lkpzb200",
                    "-Wl,-rpath," + str(ROOT / "cudakpz_b200")], check=True)
    return exe


def test_cpp_frontend_compiles_and_links(tmp_path):
    assert build(tmp_path).exists()


@pytest.mark.gpu
def test_cpp_frontend_runs_bit_exact(tmp_path, oracle):
    exe = build(tmp_path)
    out = tmp_path / "lat.bin"
    r = subprocess.run([str(exe), "9", "0.7", "0.2", "1234", "6", str(out)], capture_output=True,
                       text=True, check=True)
    w2, h1, ch, cs, ok = r.stdout.split()
    got = np.fromfile(out, dtype=np.uint32)
    ref = oracle.homogeneous(9, 9, oracle.ENC_CBBIT)
    oracle.sca_mcs(ref, 9, 9, oracle.ENC_CBBIT, 1234, 0, 0, 6, 0.7, 0.2)
    assert np.array_equal(got, ref)
    rr = oracle.roughness(ref, 9, 9, oracle.ENC_CBBIT)
    assert abs(float(w2) - rr[0]) < 1e-12 and ok == "1"
