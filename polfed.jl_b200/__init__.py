"""polfed_b200 -- the POLFED filter-and-Lanczos path on NVIDIA B200 (sm_100a).

A drop-in for Polfed.jl's hot path: matrix-free models, the KPM target
mapping and ``polfed(...)`` with its report, all executed by the CUDA
library ``libpolfed_b200.so`` through its C ABI (``include/polfed_b200.h``).

This directory is loaded as the Python package ``polfed_b200`` (its folder
name carries a dot, so it is imported by path; see ``load_package``).
"""
from . import _lib
from .core import (autotune, set_step_width, step_variant, step_profile, tune_block_size, set_filter_slab, set_launch_overlap, BenchmarkReport, DoSConfig, FactorizationConfig, FactorizationReport, MappingConfig,
                   Report, SpectralTransformReport, TransformConfig, apply, basis_index, basis_states,
                   chebyshev_filter, clenshaw_finalsum, clenshaw_recurrence, col_major, display_report,
                   expectedkrylovdim, kpm_moments, lanczos_extrema, normalize_target_spec, polfed,
                   polfed_batch, worker_handles, SolverPool, PoolStats, solver_pool)
from .models import (BoundOperator, QSunOperator, QSunSpinOperator, SparseOperator, SpinChainOperator, as_operator, chain_bonds,
                     goe_matrix, j1j2_hamiltonian, qsun_hamiltonian, qsun_parameters, qsun_spin_grain,
                     qsun_spin_parameters, spin_sector_count, xxz_hamiltonian)

__all__ = [
    "polfed", "lanczos_extrema", "MappingConfig", "TransformConfig", "FactorizationConfig", "DoSConfig",
    "Report", "SpectralTransformReport", "FactorizationReport", "BenchmarkReport", "display_report",
    "xxz_hamiltonian", "j1j2_hamiltonian", "qsun_hamiltonian", "qsun_parameters", "qsun_spin_parameters", "qsun_spin_grain",
    "spin_sector_count", "QSunSpinOperator", "chain_bonds",
    "goe_matrix", "SpinChainOperator", "QSunOperator", "SparseOperator", "as_operator", "apply", "clenshaw_recurrence",
    "clenshaw_finalsum", "chebyshev_filter", "kpm_moments", "basis_states", "basis_index", "col_major",
    "normalize_target_spec", "expectedkrylovdim", "load_library", "autotune", "set_step_width", "step_variant", "step_profile", "tune_block_size", "set_filter_slab", "set_launch_overlap", "polfed_batch", "worker_handles", "SolverPool", "PoolStats", "solver_pool", "BoundOperator",
]


def load_library():
    """Load libpolfed_b200.so (raises when it is missing)."""
    return _lib.load()
