"""SchedulerService-style host front end over the kpzb C ABI.

Mirrors the public surface of ``Kpz::SchedulerService`` (kpz/schedulerService.h:73-255)
and the GPU schedulers it fronts (``SchedulerSCA``, ``SchedulerSCABit``,
``SchedulerDT``; kpz/schedulerSCA.h, kpz/schedulerSCABit.h, kpz/schedulerDT.h):
same method names, same argument meaning, same default rates per scheduler, and
host lattices in the reference's word layouts.  All compute goes through
libkpzb200.so; nothing here computes on the host.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _lib
from ._lib import check, lib

ENC_LOCAL = _lib.ENC_LOCAL
ENC_CBBIT = _lib.ENC_CBBIT

# --scheduler names of kpz/kpzFrontend.cpp:355-403
_DYN = {"sca": _lib.DYN_SCA, "scaBit": _lib.DYN_SCABIT, "dt": _lib.DYN_DT, "db4": _lib.DYN_DB4}
# setPQDefault of each scheduler (kpz/schedulerSCA.h:37-39, kpz/schedulerSCABit.h:35-37);
# the DT and DB4 schedulers' mcs() run the p=1, q=0 SyncRng core (kpz/kpz.cu:157-162,208-216)
_DEFAULT_PQ = {_lib.DYN_SCA: (0.95, 0.0), _lib.DYN_SCABIT: (0.5, 0.0), _lib.DYN_DT: (1.0, 0.0),
               _lib.DYN_DB4: (1.0, 0.0)}
# KPZ_INNER_DD of the reference (kpz/kpzConst.h:26-35) -> kpzb_set_dt_inner
_DT_INNER = {"dt": 0, "dbsh": 1, "db": 2, "dtdbsh": 3, "dbshrep": 4}


@dataclass
class Roughness:
    """Kpz::Roughness (kpz/schedulerService.h:52-66): W^2 and raw moments <h^k>, k=1..7."""

    w2: float
    h: List[float] = field(default_factory=list)

    @classmethod
    def from_array(cls, a) -> "Roughness":
        return cls(float(a[0]), [float(v) for v in a[1:8]])

    def __str__(self) -> str:  # operator<< (kpz/schedulerService.cpp:73-79)
        return "\t".join([repr(self.w2)] + [repr(v) for v in self.h])


class Scheduler:
    """One lattice on one GPU.  ``scheduler`` is one of ``"sca"``, ``"scaBit"``, ``"dt"``,
    ``"db4"``."""

    def __init__(self, lx: int, ly: Optional[int] = None, scheduler: str = "scaBit",
                 device: int = 0):
        if scheduler not in _DYN:
            raise ValueError(f"unknown scheduler {scheduler!r}; expected one of {sorted(_DYN)}")
        ly = lx if ly is None else ly
        self._dyn = _DYN[scheduler]
        self.lx, self.ly = lx, ly
        h = C.c_void_p()
        check(lib.kpzb_create(C.byref(h), lx, ly, self._dyn, device), "kpzb_create")
        self._h = h
        self._p, self._q = _DEFAULT_PQ[self._dyn]
        check(lib.kpzb_set_pq(h, self._p, self._q), "kpzb_set_pq")
        self._mcs = 0

    # ---- lifecycle -------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.kpzb_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # ---- geometry --------------------------------------------------------------
    def encoding(self) -> int:
        return lib.kpzb_encoding(self._h)

    def size_words(self) -> int:
        return int(lib.kpzb_size_words(self._h))

    def size(self) -> int:
        return 1 << (self.lx + self.ly)

    # ---- state -----------------------------------------------------------------
    def initHomogeneous(self) -> None:
        check(lib.kpzb_init_homogeneous(self._h), "kpzb_init_homogeneous")

    def setPQ(self, p: float, q: float, n: int = 0) -> bool:
        """SchedulerService::setPQ(p, q, n): rates of disorder class n (0 = the plain rates)."""
        if n == 0:
            check(lib.kpzb_set_pq(self._h, p, q), "kpzb_set_pq")
            self._p, self._q = float(p), float(q)
        else:
            check(lib.kpzb_set_pq_class(self._h, n, p, q), "kpzb_set_pq_class")
        return True

    def setDtInner(self, inner: str) -> None:
        """DT handles: "dbsh" (single-hit dead border: the reference's default build,
        kpz/param.h:36, and the default of a new handle), "dt" (single-hit double tiling,
        about twice as fast), "db" (dead border, no offset), "dtdbsh" (double tiling with a
        per-round cell offset) or "dbshrep" (DBSH with the border hits replaced after the
        rounds)."""
        if inner not in _DT_INNER:
            raise ValueError(f"unknown DT inner scheme {inner!r}; expected one of {sorted(_DT_INNER)}")
        check(lib.kpzb_set_dt_inner(self._h, _DT_INNER[inner]), "kpzb_set_dt_inner")

    def mcsScale(self) -> float:
        """SchedulerService::mcsScale (kpz/schedulerService.h:241)."""
        s = C.c_double()
        check(lib.kpzb_mcs_scale(self._h, C.byref(s)), "kpzb_mcs_scale")
        return s.value

    def setDisorder(self, words: np.ndarray) -> None:
        """Quenched disorder classes, ENC_LOCAL words (SchedulerService::m_disorder)."""
        w = np.ascontiguousarray(words, dtype=np.uint32)
        if w.size != self.size_words():
            raise ValueError("disorder needs one word per lattice word (ENC_LOCAL layout)")
        check(lib.kpzb_set_disorder(self._h, w.ctypes.data), "kpzb_set_disorder")

    def mcsDisorder2SyncRng(self, n: int) -> None:
        check(lib.kpzb_mcs_disorder(self._h, int(n)), "kpzb_mcs_disorder")
        self._mcs += int(n)

    def mcsDisorder2SyncRngAsync(self, n: int) -> None:
        check(lib.kpzb_mcs_disorder_async(self._h, int(n)), "kpzb_mcs_disorder_async")
        self._mcs += int(n)

    def rateP(self) -> float:
        return self._p

    def rateQ(self) -> float:
        return self._q

    def supplySeed(self, seed: int, stream: int = 0) -> None:
        """Seed the counter stream (resets the device MCS counter)."""
        check(lib.kpzb_seed(self._h, C.c_uint64(seed), C.c_uint32(stream)), "kpzb_seed")

    def setFusion(self, mcs_per_pass: int) -> None:
        check(lib.kpzb_set_fusion(self._h, mcs_per_pass), "kpzb_set_fusion")

    def fusion(self) -> int:
        v = C.c_int()
        check(lib.kpzb_get_fusion(self._h, C.byref(v)), "kpzb_get_fusion")
        return int(v.value)

    def plan(self):
        """(mcs_per_pass, ctas_per_sm, pass_kernel) used for the current rates; pass_kernel is
        "half-steps", "band", "stream", "wave" or "strip" (kpzb_get_plan; for "strip" the middle
        entry is the output rows of a tile)."""
        k, c, kind = C.c_int(), C.c_int(), C.c_int()
        check(lib.kpzb_get_plan(self._h, C.byref(k), C.byref(c), C.byref(kind)), "kpzb_get_plan")
        return int(k.value), int(c.value), ("half-steps", "band", "stream", "wave", "strip")[kind.value]

    def saveBit(self, path: str, meta: Optional[str] = None) -> None:
        """SchedulerService::saveBit's file (kpz/schedulerService.cpp:389-401) plus the resume
        trailer (kpzb_save)."""
        check(lib.kpzb_save(self._h, str(path).encode(), None if meta is None else meta.encode()), "kpzb_save")

    def loadBit(self, path: str) -> None:
        """Restore a kpzb_save checkpoint (lattice, MCS, seed, rates, correlator tag) or the
        lattice of a plain saveBit file (kpzb_load)."""
        check(lib.kpzb_load(self._h, str(path).encode()), "kpzb_load")
        v = C.c_uint64()
        check(lib.kpzb_get_mcs(self._h, C.byref(v)), "kpzb_get_mcs")
        self._mcs = int(v.value)

    def measureRun(self, end: int, sampling=None, corr_start: int = -1, corr_stop: int = 0):
        """The frontend's measurement loop (kpz/kpzScaling.cpp:194-215) with the analysis on the
        device: advance to `end`, measuring at every sample time of `sampling` (default: the
        reference's exp sampling with density 0.1).  Returns an (n, 11) array of rows
        {t, W^2, <h^1..7>, ch, cs} (kpzb_measure_run)."""
        smp = sampling if sampling is not None else make_sampling()
        n = C.c_int()
        st = lib.kpzb_measure_run(self._h, C.byref(smp), end, corr_start, corr_stop, None, 0, C.byref(n))
        if st != _lib.KPZB_OK and n.value == 0:
            check(st, "kpzb_measure_run")
        rows = np.zeros((max(n.value, 1), 11), dtype=np.float64)
        check(lib.kpzb_measure_run(self._h, C.byref(smp), end, corr_start, corr_stop,
                                   rows.ctypes.data_as(C.POINTER(C.c_double)), rows.shape[0], C.byref(n)),
              "kpzb_measure_run")
        return rows[: n.value]

    def autotune(self):
        """Measure the pass shapes for the current rates; returns (mcs_per_pass, ctas_per_sm,
        ms_per_mcs) of the fastest."""
        k, c, ms = C.c_int(), C.c_int(), C.c_float()
        check(lib.kpzb_autotune(self._h, C.byref(k), C.byref(c), C.byref(ms)), "kpzb_autotune")
        return int(k.value), int(c.value), float(ms.value)

    def enableCounters(self, on: bool = True) -> None:
        check(lib.kpzb_enable_counters(self._h, int(on)), "kpzb_enable_counters")

    def counters(self, reset: bool = False):
        out = (C.c_int64 * 2)()
        check(lib.kpzb_counters(self._h, out, int(reset)), "kpzb_counters")
        return int(out[0]), int(out[1])

    # ---- dynamics (kpz/schedulerService.h:199-215) ---------------------------------
    def mcsPQSyncRng(self, n: int) -> None:
        check(lib.kpzb_mcs(self._h, int(n)), "kpzb_mcs")
        self._mcs += int(n)

    def mcsPQ(self, n: int) -> None:
        self.mcsPQSyncRng(n)

    def mcsSyncRng(self, n: int) -> None:
        p, q = _DEFAULT_PQ[self._dyn]
        self.setPQ(p, q)
        self.mcsPQSyncRng(n)

    def mcs(self, n: int) -> None:
        self.mcsSyncRng(n)

    def mcsPQSyncRngAsync(self, n: int) -> None:
        check(lib.kpzb_mcs_async(self._h, int(n)), "kpzb_mcs_async")
        self._mcs += int(n)

    def mcsPQAsync(self, n: int) -> None:
        self.mcsPQSyncRngAsync(n)

    def join(self) -> None:
        check(lib.kpzb_join(self._h), "kpzb_join")

    def deviceMcs(self) -> int:
        v = C.c_uint64()
        check(lib.kpzb_get_mcs(self._h, C.byref(v)), "kpzb_get_mcs")
        return int(v.value)

    def setDeviceMcs(self, t: int) -> None:
        check(lib.kpzb_set_mcs(self._h, C.c_uint64(t)), "kpzb_set_mcs")

    def mcs_count(self) -> int:
        return self._mcs

    def setMcs(self, mcs: int) -> None:
        self._mcs = int(mcs)

    # ---- host <-> device (kpz/schedulerBase.cu:35-52) -------------------------------
    def pushSystem(self, words: np.ndarray) -> None:
        w = np.ascontiguousarray(words, dtype=np.uint32)
        if w.size != self.size_words():
            raise ValueError(f"expected {self.size_words()} words, got {w.size}")
        check(lib.kpzb_push(self._h, w.ctypes.data), "kpzb_push")

    def pushSystemAsync(self, words: np.ndarray) -> None:
        """Enqueue the host->device copy; `words` must stay alive (and should be page-locked)
        until join().  For scaBit, dt and db4 the copy runs on the handle's copy stream into a
        stage buffer, overlapping work already queued (which still sees the previous lattice);
        work queued afterwards sees the pushed one."""
        if words.dtype != np.uint32 or not words.flags.c_contiguous or words.size != self.size_words():
            raise ValueError("expected a contiguous uint32 array of size_words() words")
        check(lib.kpzb_push_async(self._h, words.ctypes.data), "kpzb_push_async")

    def popSystemAsync(self, out: np.ndarray) -> np.ndarray:
        if out.dtype != np.uint32 or not out.flags.c_contiguous or out.size != self.size_words():
            raise ValueError("expected a contiguous uint32 array of size_words() words")
        check(lib.kpzb_pop_async(self._h, out.ctypes.data), "kpzb_pop_async")
        return out

    def popSystem(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.size_words(), dtype=np.uint32)
        check(lib.kpzb_pop(self._h, out.ctypes.data), "kpzb_pop")
        return out

    def stream(self) -> int:
        return int(lib.kpzb_stream(self._h) or 0)

    def setStream(self, stream_ptr: int) -> None:
        check(lib.kpzb_set_stream(self._h, C.c_void_p(stream_ptr)), "kpzb_set_stream")

    def devicePtr(self) -> int:
        p = C.c_void_p()
        n = C.c_size_t()
        check(lib.kpzb_device_ptr(self._h, C.byref(p), C.byref(n)), "kpzb_device_ptr")
        return int(p.value or 0)

    # ---- measurement -------------------------------------------------------------
    def roughness(self) -> Roughness:
        out = (C.c_double * 8)()
        check(lib.kpzb_roughness(self._h, out), "kpzb_roughness")
        return Roughness.from_array(out)

    def roughnessAsync(self) -> None:
        """SchedulerService::roughnessAsync: enqueue the roughness behind the enqueued work."""
        check(lib.kpzb_roughness_async(self._h), "kpzb_roughness_async")

    def joinRoughness(self) -> Roughness:
        """Wait for the handle's stream and return the roughness enqueued by roughnessAsync."""
        out = (C.c_double * 8)()
        check(lib.kpzb_roughness_join(self._h, out), "kpzb_roughness_join")
        return Roughness.from_array(out)

    def heightSums(self):
        s = (C.c_int64 * 2)()
        mm = (C.c_int64 * 2)()
        check(lib.kpzb_height_sums(self._h, s, mm), "kpzb_height_sums")
        return (int(s[0]), int(s[1])), (int(mm[0]), int(mm[1]))

    def correlateTag(self) -> Roughness:
        out = (C.c_double * 8)()
        check(lib.kpzb_corr_tag(self._h, out), "kpzb_corr_tag")
        return Roughness.from_array(out)

    def correlate(self):
        """Returns (Roughness of the current lattice, ch, cs) against the tagged snapshot."""
        out = (C.c_double * 10)()
        check(lib.kpzb_correlate(self._h, out), "kpzb_correlate")
        return Roughness.from_array(out), float(out[8]), float(out[9])

    def consitencyCheck(self):
        """Returns (ok, [bad rows, bad columns, bad plaquettes])."""
        rep = (C.c_int64 * 3)()
        check(lib.kpzb_check_invariants(self._h, rep), "kpzb_check_invariants")
        r = [int(v) for v in rep]
        return all(v == 0 for v in r), r

    consistencyCheck = consitencyCheck


class Batch:
    """Many independent SCABit lattices advanced together (kpzb_batch_*)."""

    def __init__(self, lx, p, q, seed, stream=None, device: int = 0):
        n = len(lx)
        self.n = n
        self.lx = [int(v) for v in lx]
        arr_lx = (C.c_int * n)(*self.lx)
        arr_p = (C.c_double * n)(*[float(v) for v in p])
        arr_q = (C.c_double * n)(*[float(v) for v in q])
        arr_s = (C.c_uint64 * n)(*[int(v) for v in seed])
        arr_st = (C.c_uint32 * n)(*([0] * n if stream is None else [int(v) for v in stream]))
        h = C.c_void_p()
        check(lib.kpzb_batch_create(C.byref(h), n, arr_lx, arr_p, arr_q, arr_s, arr_st, device),
              "kpzb_batch_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.kpzb_batch_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def initHomogeneous(self):
        check(lib.kpzb_batch_init_homogeneous(self._h), "kpzb_batch_init_homogeneous")

    def mcs(self, n: int):
        check(lib.kpzb_batch_mcs(self._h, int(n)), "kpzb_batch_mcs")

    def setFusion(self, mcs_per_pass: int, passes_per_graph: int = 8):
        check(lib.kpzb_batch_set_fusion(self._h, mcs_per_pass, passes_per_graph),
              "kpzb_batch_set_fusion")

    def setCtasPerSm(self, ctas_per_sm: int):
        check(lib.kpzb_batch_set_ctas_per_sm(self._h, ctas_per_sm), "kpzb_batch_set_ctas_per_sm")

    def plan(self):
        """(MCS per pass, CTAs per SM) of the pass kernel (kpzb_batch_get_plan)."""
        k, c = C.c_int(), C.c_int()
        check(lib.kpzb_batch_get_plan(self._h, C.byref(k), C.byref(c)), "kpzb_batch_get_plan")
        return int(k.value), int(c.value)

    def autotune(self):
        """Time every pass shape on the replicas, keep the fastest, restore the replicas
        (kpzb_batch_autotune); returns (MCS per pass, CTAs per SM, ms per MCS)."""
        k, c, ms = C.c_int(), C.c_int(), C.c_float()
        check(lib.kpzb_batch_autotune(self._h, C.byref(k), C.byref(c), C.byref(ms)), "kpzb_batch_autotune")
        return int(k.value), int(c.value), float(ms.value)

    def deviceMcs(self) -> int:
        v = C.c_uint64()
        check(lib.kpzb_batch_get_mcs(self._h, C.byref(v)), "kpzb_batch_get_mcs")
        return int(v.value)

    def push(self, i: int, words: np.ndarray):
        w = np.ascontiguousarray(words, dtype=np.uint32)
        check(lib.kpzb_batch_push(self._h, i, w.ctypes.data), "kpzb_batch_push")

    def pop(self, i: int) -> np.ndarray:
        out = np.empty(1 << (2 * self.lx[i] - 4), dtype=np.uint32)
        check(lib.kpzb_batch_pop(self._h, i, out.ctypes.data), "kpzb_batch_pop")
        return out

    def roughness(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        check(lib.kpzb_batch_roughness(self._h, out.ctypes.data_as(C.POINTER(C.c_double))),
              "kpzb_batch_roughness")
        return out


class Gram:
    """Exact height autocorrelator over stored snapshots (kpzb_gram_*)."""

    TENSOR, INT64 = 0, 1

    def __init__(self, lx: int, ly: int, max_snapshots: int, device: int = 0):
        h = C.c_void_p()
        check(lib.kpzb_gram_create(C.byref(h), lx, ly, max_snapshots, device), "kpzb_gram_create")
        self._h = h
        self.lx, self.ly = lx, ly

    def close(self):
        if getattr(self, "_h", None):
            lib.kpzb_gram_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def add_device(self, ptr: int):
        check(lib.kpzb_gram_add_device(self._h, C.c_void_p(ptr)), "kpzb_gram_add_device")

    def add_host(self, words: np.ndarray):
        w = np.ascontiguousarray(words, dtype=np.uint32)
        check(lib.kpzb_gram_add_host(self._h, w.ctypes.data), "kpzb_gram_add_host")

    def count(self) -> int:
        return int(lib.kpzb_gram_count(self._h))

    def compute(self, method: int = TENSOR):
        n = self.count()
        G = np.zeros((n, n), dtype=np.int64)
        S1 = np.zeros(n, dtype=np.int64)
        check(lib.kpzb_gram_compute(self._h, method, G.ctypes.data_as(C.POINTER(C.c_int64)),
                                    S1.ctypes.data_as(C.POINTER(C.c_int64))), "kpzb_gram_compute")
        return G, S1


def probe_alu_peak(device: int = -1):
    """Measured integer-ALU throughput (LOP3 chain ops/s, 3-input add chain ops/s) of a GPU:
    the denominator of the INT roofline of the bitwise SCA update (kpzb_probe_alu_peak)."""
    a, b = C.c_double(0.0), C.c_double(0.0)
    check(lib.kpzb_probe_alu_peak(device, C.byref(a), C.byref(b)), "kpzb_probe_alu_peak")
    return a.value, b.value


def make_sampling(mode: str = "exp", density: float = 0.1, interval: int = 0, random_mean: float = 0.0,
                  seed: int = 0):
    """kpzb_sampling for SamplingParam's modes (kpz/sampling.h:66-100): "exp" (density),
    "linear" (interval) or "random" (mean)."""
    m = {"exp": _lib.SAMPLE_EXP, "linear": _lib.SAMPLE_LINEAR, "random": _lib.SAMPLE_RANDOM}[mode]
    return _lib.Sampling(m, density, interval, random_mean, seed)


def sample_times(start: int, end: int, sampling=None):
    """Measurement times after `start` up to and including `end` (kpzb_sample_times)."""
    smp = sampling if sampling is not None else make_sampling()
    n = C.c_int()
    check(lib.kpzb_sample_times(C.byref(smp), start, end, None, 0, C.byref(n)), "kpzb_sample_times")
    out = np.zeros(max(n.value, 1), dtype=np.uint64)
    check(lib.kpzb_sample_times(C.byref(smp), start, end, out.ctypes.data_as(C.POINTER(C.c_uint64)),
                                out.size, C.byref(n)), "kpzb_sample_times")
    return out[: n.value]
