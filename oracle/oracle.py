"""ctypes wrapper of the CPU oracle (oracle/libkpz_oracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs
use this module.  The C sources (kpz_oracle.c) restate the reference's algorithm
with file:line citations; see kpz_oracle.h for the random-stream specification.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SO = HERE / "libkpz_oracle.so"
SRC = HERE / "kpz_oracle.c"


def build() -> Path:
    if not SO.exists() or SO.stat().st_mtime < max(SRC.stat().st_mtime,
                                                    (HERE / "kpz_oracle.h").stat().st_mtime):
        subprocess.run(["sh", str(HERE / "build.sh")], check=True)
    return SO


def _load():
    build()
    lib = C.CDLL(str(SO))
    u32p, i64p, dblp = C.POINTER(C.c_uint32), C.POINTER(C.c_int64), C.POINTER(C.c_double)
    sig = {
        "ko_philox4x32_10": (None, [u32p, u32p, u32p]),
        "ko_plane_word": (C.c_uint32, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                       C.c_uint64]),
        "ko_site_u": (C.c_uint32, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                   C.c_int]),
        "ko_threshold": (C.c_uint64, [C.c_double]),
        "ko_size_words": (C.c_uint64, [C.c_int, C.c_int]),
        "ko_init_homogeneous": (None, [u32p, C.c_int, C.c_int, C.c_int]),
        "ko_local_to_cbbit": (None, [u32p, u32p, C.c_int, C.c_int]),
        "ko_cbbit_to_local": (None, [u32p, u32p, C.c_int, C.c_int]),
        "ko_sca_halfstep": (None, [u32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64,
                                   C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, i64p, i64p]),
        "ko_sca_mcs": (None, [u32p, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint64,
                              C.c_int, C.c_double, C.c_double, i64p, i64p]),
        "ko_sca_mcs_words": (None, [u32p, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint64, C.c_int,
                                    C.c_double, C.c_double, i64p, i64p]),
        "ko_heights": (None, [u32p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int32)]),
        "ko_power_sums": (None, [C.POINTER(C.c_int32), C.c_uint64, i64p, i64p]),
        "ko_roughness": (None, [u32p, C.c_int, C.c_int, C.c_int, dblp]),
        "ko_correlate": (None, [u32p, u32p, C.c_int, C.c_int, C.c_int, C.c_double, dblp]),
        "ko_check_invariants": (None, [u32p, C.c_int, C.c_int, C.c_int, i64p]),
        "ko_dt_mcs": (None, [u32p, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint64, C.c_int,
                             C.c_double, C.c_double, i64p, i64p]),
        "ko_dt_plan": (None, [C.c_uint64, C.c_uint32, C.c_uint64, C.POINTER(C.c_int),
                              C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "ko_dsfmt_size": (C.c_size_t, []),
        "ko_dsfmt_init": (None, [C.c_void_p, C.c_uint32]),
        "ko_dsfmt_reseed": (None, [C.c_void_p, C.c_uint32]),
        "ko_dsfmt_close_open": (C.c_double, [C.c_void_p]),
        "ko_rs_mcs": (None, [u32p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_double,
                             C.c_double]),
        "ko_rs_mcs_count": (None, [u32p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                   C.c_double, C.c_double, i64p, i64p]),
        "ko_sca_mcs_dis": (None, [u32p, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint64,
                                  C.c_int, dblp, dblp, u32p, i64p, i64p]),
        "ko_dt_mcs_dis": (None, [u32p, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint64, C.c_int,
                                 dblp, dblp, u32p, i64p, i64p]),
        "ko_dt_mcs_dbsh": (None, [u32p, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint64, C.c_int,
                                  dblp, dblp, u32p, i64p, i64p]),
        "ko_dt_mcs_db": (None, [u32p, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint64, C.c_int,
                                dblp, dblp, u32p, i64p, i64p]),
        "ko_dt_mcs_dtdbsh": (None, [u32p, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint64, C.c_int,
                                    dblp, dblp, u32p, i64p, i64p]),
        "ko_dt_mcs_dbshrep": (None, [u32p, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint64, C.c_int,
                                     dblp, dblp, u32p, i64p, i64p]),
        "ko_db4_mcs": (None, [u32p, C.c_int, C.c_int, C.c_uint64, C.c_uint32, C.c_uint64, C.c_int,
                              C.c_double, C.c_double, i64p, i64p]),
        "ko_generate_disorder2": (None, [u32p, C.c_int, C.c_int, C.c_void_p, C.c_double]),
        "ko_rs_mcs_dis": (None, [u32p, C.c_int, C.c_int, C.c_void_p, C.c_int, dblp, dblp, u32p, i64p,
                                 i64p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()
ENC_LOCAL, ENC_CBBIT = 0, 1


def _u32(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib.ko_philox4x32_10(c, k, o)
    return [int(v) for v in o]


def threshold(p: float) -> int:
    return int(lib.ko_threshold(p))


def size_words(lx: int, ly: int) -> int:
    return 1 << (lx + ly - 4)


def homogeneous(lx: int, ly: int, encoding: int) -> np.ndarray:
    w = np.empty(size_words(lx, ly), dtype=np.uint32)
    lib.ko_init_homogeneous(_u32(w), lx, ly, encoding)
    return w


def local_to_cbbit(local: np.ndarray, lx: int, ly: int) -> np.ndarray:
    out = np.empty_like(local)
    lib.ko_local_to_cbbit(_u32(local), _u32(out), lx, ly)
    return out


def cbbit_to_local(cb: np.ndarray, lx: int, ly: int) -> np.ndarray:
    out = np.empty_like(cb)
    lib.ko_cbbit_to_local(_u32(cb), _u32(out), lx, ly)
    return out


def sca_mcs(w: np.ndarray, lx: int, ly: int, encoding: int, seed: int, stream: int, t0: int,
            n: int, p: float, q: float):
    """In place; returns (#deposits, #desorptions)."""
    dep, des = C.c_int64(0), C.c_int64(0)
    lib.ko_sca_mcs(_u32(w), lx, ly, encoding, seed, stream, t0, n, p, q, C.byref(dep), C.byref(des))
    return dep.value, des.value


def sca_mcs_words(w: np.ndarray, lx: int, ly: int, seed: int, stream: int, t0: int, n: int, p: float,
                  q: float):
    """ko_sca_mcs on ENC_CBBIT words, 32 sites per operation (equal results, fast at 16384^2).
    In place; returns (#deposits, #desorptions)."""
    dep, des = C.c_int64(0), C.c_int64(0)
    lib.ko_sca_mcs_words(_u32(w), lx, ly, seed, stream, t0, n, p, q, C.byref(dep), C.byref(des))
    return dep.value, des.value


def dt_mcs(w: np.ndarray, lx: int, ly: int, seed: int, stream: int, t0: int, n: int,
           p: float, q: float):
    """Double-tiling RS emulation (ENC_LOCAL, in place); returns (#deposits, #desorptions)."""
    dep, des = C.c_int64(0), C.c_int64(0)
    lib.ko_dt_mcs(_u32(w), lx, ly, seed, stream, t0, n, p, q, C.byref(dep), C.byref(des))
    return dep.value, des.value


def _rates4(r):
    r = list(r) + [r[-1]] * (4 - len(r))
    return (C.c_double * 4)(*r[:4])


def sca_mcs_dis(w: np.ndarray, lx: int, ly: int, encoding: int, seed: int, stream: int, t0: int,
                n: int, p, q, dis: np.ndarray):
    """Quenched disorder: rate class = the 2 bits of `dis` (ENC_LOCAL) at each site picks
    p[c], q[c] (lists of up to 4; missing classes repeat the last).  In place; (#dep, #des)."""
    dep, des = C.c_int64(0), C.c_int64(0)
    lib.ko_sca_mcs_dis(_u32(w), lx, ly, encoding, seed, stream, t0, n, _rates4(p), _rates4(q), _u32(dis),
                       C.byref(dep), C.byref(des))
    return dep.value, des.value


def dt_mcs_dis(w: np.ndarray, lx: int, ly: int, seed: int, stream: int, t0: int, n: int, p, q,
               dis: np.ndarray):
    dep, des = C.c_int64(0), C.c_int64(0)
    lib.ko_dt_mcs_dis(_u32(w), lx, ly, seed, stream, t0, n, _rates4(p), _rates4(q), _u32(dis),
                      C.byref(dep), C.byref(des))
    return dep.value, des.value


def dt_mcs_dbsh(w: np.ndarray, lx: int, ly: int, seed: int, stream: int, t0: int, n: int, p, q,
                dis: np.ndarray = None, shift: bool = True):
    """DT with the reference's default DBSH inner scheme (shift=False: DB, no per-round cell
    offset), ENC_LOCAL, in place; returns (#dep, #des)."""
    dep, des = C.c_int64(0), C.c_int64(0)
    d = None if dis is None else _u32(dis)
    pp = p if isinstance(p, (list, tuple)) else [p]
    qq = q if isinstance(q, (list, tuple)) else [q]
    fn = lib.ko_dt_mcs_dbsh if shift else lib.ko_dt_mcs_db
    fn(_u32(w), lx, ly, seed, stream, t0, n, _rates4(pp), _rates4(qq), d, C.byref(dep), C.byref(des))
    return dep.value, des.value


def dt_mcs_inner(w: np.ndarray, lx: int, ly: int, seed: int, stream: int, t0: int, n: int, p, q,
                 inner: str, dis: np.ndarray = None):
    """DT with inner scheme "dt", "dbsh", "db", "dtdbsh" or "dbshrep", ENC_LOCAL, in place;
    returns (#dep, #des)."""
    fn = {"dt": lib.ko_dt_mcs_dis, "dbsh": lib.ko_dt_mcs_dbsh, "db": lib.ko_dt_mcs_db,
          "dtdbsh": lib.ko_dt_mcs_dtdbsh, "dbshrep": lib.ko_dt_mcs_dbshrep}[inner]
    dep, des = C.c_int64(0), C.c_int64(0)
    d = None if dis is None else _u32(dis)
    pp = p if isinstance(p, (list, tuple)) else [p]
    qq = q if isinstance(q, (list, tuple)) else [q]
    fn(_u32(w), lx, ly, seed, stream, t0, n, _rates4(pp), _rates4(qq), d, C.byref(dep), C.byref(des))
    return dep.value, des.value


def db4_mcs(w: np.ndarray, lx: int, ly: int, seed: int, stream: int, t0: int, n: int, p: float, q: float):
    """The DB4 scheduler's MCS, ENC_LOCAL, in place; returns (#dep, #des)."""
    dep, des = C.c_int64(0), C.c_int64(0)
    lib.ko_db4_mcs(_u32(w), lx, ly, seed, stream, t0, n, p, q, C.byref(dep), C.byref(des))
    return dep.value, des.value


def generate_disorder2(lx: int, ly: int, rng: "DSFMT", fill: float) -> np.ndarray:
    """SchedulerService::generateDisorder2 (ENC_LOCAL words, one class bit per site)."""
    d = np.empty(size_words(lx, ly), dtype=np.uint32)
    lib.ko_generate_disorder2(_u32(d), lx, ly, rng.ptr, fill)
    return d


def rs_mcs_dis(w: np.ndarray, lx: int, ly: int, rng: "DSFMT", n: int, p, q, dis: np.ndarray):
    """SchedulerCPU::mcsDisorder2 in place; returns (#dep, #des)."""
    dep, des = C.c_int64(0), C.c_int64(0)
    lib.ko_rs_mcs_dis(_u32(w), lx, ly, rng.ptr, n, _rates4(p), _rates4(q), _u32(dis), C.byref(dep),
                      C.byref(des))
    return dep.value, des.value


def dt_plan(seed: int, stream: int, t: int):
    ox, oy = C.c_int(), C.c_int()
    order = (C.c_int * 4)()
    lib.ko_dt_plan(seed, stream, t, C.byref(ox), C.byref(oy), order)
    return ox.value, oy.value, list(order)


def heights(w: np.ndarray, lx: int, ly: int, encoding: int) -> np.ndarray:
    h = np.empty((1 << ly, 1 << lx), dtype=np.int32)
    lib.ko_heights(_u32(w), lx, ly, encoding, h.ctypes.data_as(C.POINTER(C.c_int32)))
    return h


def power_sums(h: np.ndarray):
    """Exact sum h^k, k=1..7, as Python ints."""
    h = np.ascontiguousarray(h, dtype=np.int32)
    lo = (C.c_int64 * 7)()
    hi = (C.c_int64 * 7)()
    lib.ko_power_sums(h.ctypes.data_as(C.POINTER(C.c_int32)), h.size, lo, hi)
    out = []
    for k in range(7):
        v = (int(hi[k]) << 64) | (int(lo[k]) & ((1 << 64) - 1))
        if v >= 1 << 127:
            v -= 1 << 128
        out.append(v)
    return out


def roughness(w: np.ndarray, lx: int, ly: int, encoding: int) -> np.ndarray:
    out = np.empty(8, dtype=np.float64)
    lib.ko_roughness(_u32(w), lx, ly, encoding, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def correlate(sys: np.ndarray, snap: np.ndarray, lx: int, ly: int, encoding: int,
              snap_mean: float) -> np.ndarray:
    out = np.empty(10, dtype=np.float64)
    lib.ko_correlate(_u32(sys), _u32(snap), lx, ly, encoding, snap_mean,
                     out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def check_invariants(w: np.ndarray, lx: int, ly: int, encoding: int):
    rep = (C.c_int64 * 3)()
    lib.ko_check_invariants(_u32(w), lx, ly, encoding, rep)
    return [int(v) for v in rep]


class DSFMT:
    """dSFMT-19937 restatement (bit-identical to the reference's vendored dSFMT)."""

    def __init__(self, seed: int, reseed: bool = True):
        self._buf = C.create_string_buffer(int(lib.ko_dsfmt_size()))
        if reseed:
            lib.ko_dsfmt_reseed(self._buf, seed)
        else:
            lib.ko_dsfmt_init(self._buf, seed)

    def close_open(self) -> float:
        return float(lib.ko_dsfmt_close_open(self._buf))

    @property
    def ptr(self):
        return self._buf


def rs_mcs(w: np.ndarray, lx: int, ly: int, rng: DSFMT, n: int, pq: bool = False,
           p: float = 1.0, q: float = 0.0):
    """SchedulerCPU::mcs (pq False) / mcsPQ (pq True) in place; returns (#dep, #des)."""
    dep, des = C.c_int64(0), C.c_int64(0)
    lib.ko_rs_mcs_count(_u32(w), lx, ly, rng.ptr, n, int(pq), p, q, C.byref(dep), C.byref(des))
    return dep.value, des.value


def random_lattice(lx: int, ly: int, encoding: int, seed: int, mcs: int = 4,
                   p: float = 0.5, q: float = 0.5) -> np.ndarray:
    """A valid (consistent) rough lattice: flat start evolved by the oracle SCA."""
    w = homogeneous(lx, ly, encoding)
    sca_mcs(w, lx, ly, encoding, seed, 7, 0, mcs, p, q)
    return w
