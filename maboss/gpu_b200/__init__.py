"""B200 (sm_100a) trajectory engine for stochastic Boolean networks (MaBoSS semantics).

The engine is the C-ABI library libmaboss_b200.so (include/maboss_b200.h); this package is a
thin ctypes binding over it. Nothing here computes trajectories: without the library every
entry point raises.
"""
from ._lib import EngineError, build, lib
from .engine import (Batch, Context, Model, Module, Result, RunConfig, Stats, gradient, merge_results,
                     mutant_sweep, rand_state_size)

__all__ = ["EngineError", "build", "lib", "Batch", "Context", "Model", "Module", "Result", "RunConfig", "Stats",
           "gradient", "merge_results", "mutant_sweep", "rand_state_size"]
