"""B200-native (sm_100a) FDTD time-step engine for the MGALIKE/special-topics
inverted-F-antenna solver.

Host-side mirror of the reference's backend interface (js_fdtd/src/backends):
``build_problem_from_scenario`` (scenario.js), the ``b200`` backend object
(registry contract) and the post-loop S11 / far-field products, all over the
C ABI of ``libfdtd_b200.so`` (include/fdtd_b200.h).
"""
from ._native import FdtdError, build, device_count, lib
from .backend import B200Backend, Engine
from .registry import list_backends, load_backend, select_backend
from .scenario import Problem, build_problem_from_scenario

__all__ = ["FdtdError", "build", "device_count", "lib", "B200Backend", "Engine", "Problem",
           "build_problem_from_scenario", "list_backends", "load_backend", "select_backend"]
