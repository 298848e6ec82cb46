"""bbfmm_b200: the bbFMM M2L / P2P / pass hot path on B200 (sm_100a)."""
from .fmm import AdaptiveBatch, AdaptiveSolver, Batch, Solver, batch_depth, bbfmm, reference_depth, set_cost, shard_sets  # noqa: F401
from . import operators  # noqa: F401
