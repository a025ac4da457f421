"""The C-ABI library loads and exports every symbol include/kpzb.h declares (no GPU needed).

No compute calls are made here; the GPU parity tests call through the same ABI.
"""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "kpzb.h"
LIB = ROOT / "cudakpz_b200" / "libkpzb200.so"


def declared_symbols():
    text = HEADER.read_text()
    # strip comments
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(kpzb_[a-z0-9_]+)\s*\(", text)))


def ensure_lib():
    if not LIB.exists():
        # build.py is loaded by path: importing the package itself needs the library
        import importlib.util
        spec = importlib.util.spec_from_file_location("kpzb_build", ROOT / "cudakpz_b200" / "build.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    return LIB


def test_header_declares_api():
    syms = declared_symbols()
    for must in ("kpzb_create", "kpzb_mcs", "kpzb_push", "kpzb_pop", "kpzb_roughness",
                 "kpzb_correlate", "kpzb_batch_mcs", "kpzb_gram_compute", "kpzb_check_invariants"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(ensure_lib()))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"not exported: {missing}"


def test_exports_match_nm():
    out = subprocess.run(["nm", "-D", "--defined-only", str(ensure_lib())], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (kpzb_[a-z0-9_]+)$", out, flags=re.M))
    assert set(declared_symbols()) <= exported


def test_python_binding_covers_header():
    from cudakpz_b200._lib import SIGNATURES
    assert set(declared_symbols()) == set(SIGNATURES)


def test_version_and_errors_without_gpu():
    from cudakpz_b200._lib import lib
    assert b"sm_100a" in lib.kpzb_version()
    # argument validation happens before any device call
    h = ctypes.c_void_p()
    assert lib.kpzb_create(ctypes.byref(h), 31, 8, 1, 0) == 1  # KPZB_EINVAL
    assert b"out of range" in lib.kpzb_last_error()
    assert lib.kpzb_create(ctypes.byref(h), 7, 8, 1, 0) == 1
    assert lib.kpzb_create(ctypes.byref(h), 12, 12, 9, 0) == 1
    assert lib.kpzb_set_pq(None, 0.5, 0.5) == 1
    assert lib.kpzb_mcs(None, 1) == 1


@pytest.mark.parametrize("lx,ly", [(20, 19), (30, 9)])
def test_size_limit_rejected_before_allocation(lx, ly):
    from cudakpz_b200._lib import lib
    h = ctypes.c_void_p()
    assert lib.kpzb_create(ctypes.byref(h), lx, ly, 1, 0) == 1
