"""ctypes binding of libkpzb200.so (the C ABI in include/kpzb.h).

The shared library is built in tree by ``cudakpz_b200.build``.  There is no
fallback: if the library is missing or fails to load, importing this module
raises ``ImportError`` with the reason.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libkpzb200.so"

KPZB_OK = 0
STATUS_NAMES = {0: "KPZB_OK", 1: "KPZB_EINVAL", 2: "KPZB_ENOMEM", 3: "KPZB_ECUDA",
                4: "KPZB_ETIMEOUT", 5: "KPZB_ESTATE", 6: "KPZB_EUNSUPPORTED"}

ENC_LOCAL, ENC_CBBIT = 0, 1
DYN_SCA, DYN_SCABIT, DYN_DT, DYN_DB4 = 0, 1, 2, 3


class KpzbError(RuntimeError):
    """A kpzb_* call returned a non-zero status."""

    def __init__(self, status: int, func: str, msg: str):
        super().__init__(f"{func} -> {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_i64p = C.POINTER(C.c_int64)
_dblp = C.POINTER(C.c_double)
_intp = C.POINTER(C.c_int)
_vp = C.c_void_p

class Sampling(C.Structure):
    """kpzb_sampling (include/kpzb.h)."""
    _fields_ = [("mode", C.c_int), ("density", C.c_double), ("interval", C.c_uint32),
                ("random_mean", C.c_double), ("seed", C.c_uint64)]


SAMPLE_EXP, SAMPLE_LINEAR, SAMPLE_RANDOM = 0, 1, 2

# name -> (restype, argtypes); every symbol declared in include/kpzb.h
SIGNATURES = {
    "kpzb_last_error": (C.c_char_p, []),
    "kpzb_version": (C.c_char_p, []),
    "kpzb_probe_alu_peak": (C.c_int, [C.c_int, _dblp, _dblp]),
    "kpzb_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.c_int, C.c_int, C.c_int]),
    "kpzb_destroy": (C.c_int, [_vp]),
    "kpzb_init_homogeneous": (C.c_int, [_vp]),
    "kpzb_set_pq": (C.c_int, [_vp, C.c_double, C.c_double]),
    "kpzb_seed": (C.c_int, [_vp, C.c_uint64, C.c_uint32]),
    "kpzb_mcs": (C.c_int, [_vp, C.c_int]),
    "kpzb_set_dt_inner": (C.c_int, [_vp, C.c_int]),
    "kpzb_mcs_scale": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "kpzb_set_pq_class": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double]),
    "kpzb_set_disorder": (C.c_int, [_vp, _vp]),
    "kpzb_mcs_disorder": (C.c_int, [_vp, C.c_int]),
    "kpzb_mcs_disorder_async": (C.c_int, [_vp, C.c_int]),
    "kpzb_mcs_async": (C.c_int, [_vp, C.c_int]),
    "kpzb_join": (C.c_int, [_vp]),
    "kpzb_set_fusion": (C.c_int, [_vp, C.c_int]),
    "kpzb_get_fusion": (C.c_int, [_vp, _intp]),
    "kpzb_get_plan": (C.c_int, [_vp, _intp, _intp, _intp]),
    "kpzb_save": (C.c_int, [_vp, C.c_char_p, C.c_char_p]),
    "kpzb_load": (C.c_int, [_vp, C.c_char_p]),
    "kpzb_sample_times": (C.c_int, [C.POINTER(Sampling), C.c_uint64, C.c_uint64, _u64p, C.c_int, _intp]),
    "kpzb_measure_run": (C.c_int, [_vp, C.POINTER(Sampling), C.c_uint64, C.c_int64, C.c_uint64, _dblp,
                                   C.c_int, _intp]),
    "kpzb_autotune": (C.c_int, [_vp, _intp, _intp, C.POINTER(C.c_float)]),
    "kpzb_push": (C.c_int, [_vp, _vp]),
    "kpzb_pop": (C.c_int, [_vp, _vp]),
    "kpzb_push_async": (C.c_int, [_vp, _vp]),
    "kpzb_pop_async": (C.c_int, [_vp, _vp]),
    "kpzb_push_device": (C.c_int, [_vp, _vp]),
    "kpzb_pop_device": (C.c_int, [_vp, _vp]),
    "kpzb_size_words": (C.c_size_t, [_vp]),
    "kpzb_encoding": (C.c_int, [_vp]),
    "kpzb_roughness": (C.c_int, [_vp, _dblp]),
    "kpzb_roughness_async": (C.c_int, [_vp]),
    "kpzb_roughness_join": (C.c_int, [_vp, _dblp]),
    "kpzb_roughness_noalloc": (C.c_int, [_vp, C.c_int, C.c_int, _dblp, _vp]),
    "kpzb_height_sums": (C.c_int, [_vp, _i64p, _i64p]),
    "kpzb_corr_tag": (C.c_int, [_vp, _dblp]),
    "kpzb_correlate": (C.c_int, [_vp, _dblp]),
    "kpzb_get_mcs": (C.c_int, [_vp, _u64p]),
    "kpzb_set_mcs": (C.c_int, [_vp, C.c_uint64]),
    "kpzb_counters": (C.c_int, [_vp, _i64p, C.c_int]),
    "kpzb_enable_counters": (C.c_int, [_vp, C.c_int]),
    "kpzb_check_invariants": (C.c_int, [_vp, _i64p]),
    "kpzb_device_ptr": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(C.c_size_t)]),
    "kpzb_stream": (_vp, [_vp]),
    "kpzb_set_stream": (C.c_int, [_vp, _vp]),
    "kpzb_batch_create": (C.c_int, [C.POINTER(_vp), C.c_int, _intp, _dblp, _dblp, _u64p,
                                    C.POINTER(C.c_uint32), C.c_int]),
    "kpzb_batch_destroy": (C.c_int, [_vp]),
    "kpzb_batch_init_homogeneous": (C.c_int, [_vp]),
    "kpzb_batch_mcs": (C.c_int, [_vp, C.c_int]),
    "kpzb_batch_set_fusion": (C.c_int, [_vp, C.c_int, C.c_int]),
    "kpzb_batch_set_ctas_per_sm": (C.c_int, [_vp, C.c_int]),
    "kpzb_batch_get_plan": (C.c_int, [_vp, _intp, _intp]),
    "kpzb_batch_autotune": (C.c_int, [_vp, _intp, _intp, C.POINTER(C.c_float)]),
    "kpzb_batch_get_mcs": (C.c_int, [_vp, _u64p]),
    "kpzb_batch_push": (C.c_int, [_vp, C.c_int, _vp]),
    "kpzb_batch_pop": (C.c_int, [_vp, C.c_int, _vp]),
    "kpzb_batch_roughness": (C.c_int, [_vp, _dblp]),
    "kpzb_gram_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.c_int, C.c_int, C.c_int]),
    "kpzb_gram_destroy": (C.c_int, [_vp]),
    "kpzb_gram_add_device": (C.c_int, [_vp, _vp]),
    "kpzb_gram_add_host": (C.c_int, [_vp, _vp]),
    "kpzb_gram_compute": (C.c_int, [_vp, C.c_int, _i64p, _i64p]),
    "kpzb_gram_count": (C.c_int, [_vp]),
}


def _load():
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing; build it with `python -m cudakpz_b200.build` "
            "(the CUDA path has no fallback)")
    try:
        lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
    except OSError as e:  # pragma: no cover - depends on the machine
        raise ImportError(f"cannot load {LIB_PATH}: {e}") from e
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int, func: str) -> None:
    if status != KPZB_OK:
        raise KpzbError(status, func, lib.kpzb_last_error().decode(errors="replace"))
