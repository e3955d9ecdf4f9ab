"""B200-native heads-up Discounted-CFR range-vs-range postflop solver.

`poker_trainer_b200.solver.Solver` mirrors the reference solver crate's API
(AhanDatta/Poker-Trainer, crates/solver/src/lib.rs) over libdcfr.so, a C-ABI
library whose hot path is hand-written sm_100a CUDA (csrc/kernels.cu).
"""
from . import abi  # noqa: F401

__all__ = ["abi", "solver", "workloads", "build"]
