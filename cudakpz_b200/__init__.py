"""cudakpz_b200 -- B200-native (sm_100a) octahedron-model KPZ hot path.

The compute lives in libkpzb200.so (C ABI: include/kpzb.h); this package is the
SchedulerService-style host front end.  Importing it fails loudly when the
library has not been built: there is no CPU fallback.
"""
from ._lib import KpzbError, lib  # noqa: F401  (raises ImportError if the .so is missing)
from .scheduler import (ENC_CBBIT, ENC_LOCAL, Batch, Gram, Roughness, Scheduler,  # noqa: F401
                        make_sampling, probe_alu_peak, sample_times)

__all__ = ["Scheduler", "Batch", "Gram", "Roughness", "KpzbError", "ENC_LOCAL", "ENC_CBBIT",
           "probe_alu_peak", "make_sampling", "sample_times"]
