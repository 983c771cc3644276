"""FP64 peak of the current GPU, measured with a DFMA burst kernel.

The driver-written peaks cover HBM copy bandwidth and bf16 tensor GEMMs only;
the HDG element path computes in FP64 on the CUDA cores, so its compute roof
is measured here: every thread runs a long chain of independent FP64 FMAs and
the elapsed time is taken with CUDA events.
"""
from __future__ import annotations

import ctypes as C

from .core import load_library


def fp64_peak_tflops(device: int = 0) -> float:
    lib = load_library()
    lib.hfem_fp64_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
    out = C.c_double(0.0)
    rc = lib.hfem_fp64_peak(device, C.byref(out))
    if rc != 0:
        raise RuntimeError(f"hfem_fp64_peak failed ({rc})")
    return out.value
