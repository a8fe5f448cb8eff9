"""B200 tabu-search engine for the Maximum Diversity Problem and Max Bisection.

Python mirror of the C-ABI in include/ts_b200.h; the compute path is the
hand-written sm_100a CUDA in libts_b200.so (no CPU fallback).
"""
from ._capi import (EXPORTS, LIB_PATH, PASS_AUTO, PASS_ROWS, PASS_TILE, PROBLEM_MAXBS, PROBLEM_MDP,
                    STRUCT_NAMES, TENURE_FIXED, TENURE_REF, TRACE_DTYPE, TsError, lib)
from .engine import (Batch, BatchJobSpec, Graph, Served, Server, Solver, SolveResult, batch_solve,
                     default_params,
                     perturb_draws,
                     perturbation_based_tabu_search, random_start, struct_id, tabu_search)
from . import gen

__all__ = [
    "EXPORTS", "LIB_PATH", "PASS_AUTO", "PASS_ROWS", "PASS_TILE", "PROBLEM_MAXBS", "PROBLEM_MDP", "STRUCT_NAMES", "TENURE_FIXED", "TENURE_REF",
    "TRACE_DTYPE", "TsError", "lib", "Graph", "Solver", "SolveResult", "default_params",
    "perturbation_based_tabu_search", "struct_id", "tabu_search", "gen", "random_start",
    "perturb_draws", "Batch", "BatchJobSpec", "batch_solve", "Server", "Served",
]
