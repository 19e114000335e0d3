"""shaderous_b200: a B200-native compressible-hydro step behind the reference's simulation API.

The compute path is the in-tree CUDA library ``libshaderous_b200.so`` (sm_100a) reached through
its C ABI (``include/shaderous_b200.h``); :mod:`shaderous_b200.sim` is the Python host mirror.
"""
from .sim import Config, Diagnostics, Problem, RunResult, ShaderousError, Sim, prims_to_state, problem_prims

__all__ = ["Config", "Diagnostics", "Problem", "RunResult", "ShaderousError", "Sim", "prims_to_state", "problem_prims"]
