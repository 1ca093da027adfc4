"""rcwa_b200 -- B200-native RCWA solve path behind a C ABI.

The compute path lives in ``librcwa_b200.so`` (CUDA kernels for sm_100a plus
the ``extern "C"`` boundary declared in ``include/rcwa_b200.h``).  This Python
package only loads that library through ctypes and mirrors the reference's
step-function API for tests, benchmarks and Python callers.
"""
from .configs import (ParamSpec, Problem, SourceSpec, StackSpec, c1_pillars,
                      c2_sweep, c3_batch, c3_request, c4_trapezoid,
                      demo_triangle, ref_eps)

__all__ = [
    "ParamSpec", "Problem", "SourceSpec", "StackSpec", "c1_pillars", "c2_sweep",
    "c3_batch", "c3_request", "c4_trapezoid", "demo_triangle", "ref_eps",
]
