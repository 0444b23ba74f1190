"""Measured roofline denominators of the current GPU (libcrp_peaks.so):
L2 read bandwidth, FP32 and FP64 FMA throughput and the hardware cosine
throughput, from the microbenchmarks in csrc/peaks.cu.  The HBM copy
bandwidth is the pool's own measurement (MEASURED_PEAKS.json)."""
from __future__ import annotations

import ctypes as C
import os

_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libcrp_peaks.so")


class Peaks(C.Structure):
    _fields_ = [("l2_gbs", C.c_double), ("fp32_tflops", C.c_double), ("fp64_tflops", C.c_double),
                ("cos_gops", C.c_double), ("sm_count", C.c_int32), ("_pad", C.c_int32)]


def measure() -> dict:
    if not os.path.exists(_LIB):
        raise RuntimeError(f"{_LIB} is not built (python crpropa3_b200/build.py)")
    lib = C.CDLL(_LIB)
    lib.crp_peaks_measure.argtypes = [C.POINTER(Peaks)]
    lib.crp_peaks_measure.restype = C.c_int
    p = Peaks()
    r = lib.crp_peaks_measure(C.byref(p))
    if r != 0:
        raise RuntimeError(f"crp_peaks_measure failed with CUDA error {r}")
    return {"l2_gbs": p.l2_gbs, "fp32_tflops": p.fp32_tflops, "fp64_tflops": p.fp64_tflops,
            "cos_gops": p.cos_gops, "sm_count": p.sm_count}
