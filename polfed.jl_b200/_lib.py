"""ctypes binding of libpolfed_b200.so (the C ABI declared in include/polfed_b200.h).

The library is the only compute path: if it is missing or fails to load, every
call raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpolfed_b200.so")

PF_OK = 0
PF_ERR_INVALID = 1
PF_ERR_CUDA = 2
PF_ERR_NOMEM = 3
PF_ERR_NUMERIC = 4
PF_ERR_UNSUPPORTED = 5

PF_F64, PF_F32 = 0, 1
PF_MEM_HOST, PF_MEM_DEVICE = 0, 1
PF_TARGET_MAXDOS, PF_TARGET_MIDDLE, PF_TARGET_OFFSET, PF_TARGET_UNRESCALED, PF_TARGET_RESCALED = range(5)
PF_WHICH_SR, PF_WHICH_LR = 0, 1
KERNEL_IDS = {"Jackson": 0, "Lorentz": 1, "Fejer": 2, "LanczosK": 3, "WangZunger": 4, "Dirichlet": 5}
PF_PROBE_GAUSSIAN, PF_PROBE_RADEMACHER = 0, 1
PF_PREC_FP64, PF_PREC_MIXED = 0, 1
PF_REPORT_MAX_CHECKS = 128
PF_WIDTH_COOP = 0

EXPORTED = [
    "pf_abi_version", "pf_abi_sizes", "pf_last_error", "pf_handle_create", "pf_handle_destroy", "pf_handle_stream",
    "pf_handle_synchronize", "pf_handle_set_overlap", "pf_op_spin_chain_create", "pf_op_qsun_create", "pf_op_qsun_spin_create", "pf_op_destroy",
    "pf_op_dim", "pf_basis_unrank", "pf_basis_rank", "pf_apply", "pf_clenshaw_recurrence",
    "pf_clenshaw_finalsum", "pf_filter", "pf_kpm_moments", "pf_params_default", "pf_solve", "pf_solve_hermitian",
    "pf_lanczos_extrema", "pf_autotune", "pf_apply_noalloc", "pf_op_bind", "pf_set_step_width",
    "pf_op_csr_create", "pf_op_csr_create_hermitian",
    "pf_pool_create", "pf_pool_destroy", "pf_solve_footprint", "pf_pool_solve_batch", "pf_pool_submit",
    "pf_pool_poll", "pf_pool_fetch", "pf_pool_cancel", "pf_pool_get_stats", "pf_pool_stream",
    "pf_pool_set_priority_dim", "pf_pool_set_admission", "pf_pool_request_times",
    "pf_pool_wait", "pf_pool_shutdown", "pf_pool_set_batching", "pf_step_variant", "pf_step_profile", "pf_set_step_variant",
    "pf_gather_peak", "pf_set_filter_slab", "pf_gram_bf16x3",
]
PF_REQ_QUEUED, PF_REQ_RUNNING, PF_REQ_DONE, PF_REQ_FAILED, PF_REQ_REJECTED = 0, 1, 2, 3, 4
PF_ADMIT_FIFO, PF_ADMIT_SHORTEST = 0, 1


class PolfedError(RuntimeError):
    """A non-zero status returned by the library (message from pf_last_error)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[pf status {code}] {msg}")
        self.code = code


class PolfedArgumentError(PolfedError, ValueError):
    """PF_ERR_INVALID: the reference raises ArgumentError / DimensionMismatch here."""


class PolfedRejected(PolfedError):
    """A served request that cannot be met: fewer than ``howmany`` states lie
    within reach of its target (the reference's bisection error)."""


class pf_params(ctypes.Structure):
    _fields_ = [
        ("target_kind", ctypes.c_int), ("target_value", ctypes.c_double),
        ("has_Emin", ctypes.c_int), ("has_Emax", ctypes.c_int),
        ("Emin", ctypes.c_double), ("Emax", ctypes.c_double),
        ("has_left", ctypes.c_int), ("has_right", ctypes.c_int),
        ("left", ctypes.c_double), ("right", ctypes.c_double),
        ("order", ctypes.c_int), ("cutoff", ctypes.c_double), ("normalization", ctypes.c_double),
        ("order_safety_factor", ctypes.c_double), ("tol", ctypes.c_double),
        ("eigentol", ctypes.c_double), ("overestimate_iters", ctypes.c_double),
        ("which", ctypes.c_int), ("dos_N", ctypes.c_int), ("dos_R", ctypes.c_int),
        ("dos_kernel", ctypes.c_int), ("probe_kind", ctypes.c_int), ("seed", ctypes.c_uint64),
        ("probes", ctypes.c_void_p), ("precision", ctypes.c_int), ("reorth_passes", ctypes.c_int),
        ("extrema_maxdim", ctypes.c_int), ("refine", ctypes.c_int), ("autotune", ctypes.c_int),
        ("host_qr", ctypes.c_int),
    ]


class pf_report(ctypes.Structure):
    _fields_ = [
        ("Emin", ctypes.c_double), ("Emax", ctypes.c_double), ("a", ctypes.c_double), ("b", ctypes.c_double),
        ("target", ctypes.c_double), ("left", ctypes.c_double), ("right", ctypes.c_double),
        ("order", ctypes.c_int), ("order_safety_factor", ctypes.c_double),
        ("matvecs", ctypes.c_int64), ("kpm_block_matvecs", ctypes.c_int64),
        ("blocksize", ctypes.c_int), ("howmany", ctypes.c_int),
        ("iters_needed", ctypes.c_int), ("iters_reserved", ctypes.c_int), ("krylovdim", ctypes.c_int),
        ("tol", ctypes.c_double), ("residual", ctypes.c_double), ("converged_tol", ctypes.c_int),
        ("eigentol", ctypes.c_double), ("eigenresidual", ctypes.c_double),
        ("converged_eigentol", ctypes.c_int), ("refined", ctypes.c_int), ("numofchecks", ctypes.c_int),
        ("converged_history", ctypes.c_int * PF_REPORT_MAX_CHECKS),
        ("krylovdim_history", ctypes.c_int * PF_REPORT_MAX_CHECKS),
        ("maxresidual_history", ctypes.c_double * PF_REPORT_MAX_CHECKS),
        ("stage_seconds", ctypes.c_double * 10),
        ("basis_bytes_reserved", ctypes.c_double), ("basis_bytes_used", ctypes.c_double),
        ("kernel_launches", ctypes.c_int64), ("qr_restarts", ctypes.c_int),
    ]


class pf_pool_stats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
        ("queued", ctypes.c_int64), ("running", ctypes.c_int64), ("eigenpairs", ctypes.c_int64),
        ("bytes_budget", ctypes.c_double), ("bytes_in_use", ctypes.c_double), ("bytes_peak", ctypes.c_double),
        ("p50_latency", ctypes.c_double), ("p99_latency", ctypes.c_double), ("mean_latency", ctypes.c_double),
        ("busy_seconds", ctypes.c_double), ("rejected", ctypes.c_int64),
        ("filter_launches", ctypes.c_double), ("filter_seconds", ctypes.c_double),
        ("filter_bytes", ctypes.c_double), ("filter_instance_steps", ctypes.c_double),
    ]


_LIB = None


def load():
    """Load libpolfed_b200.so; raises if it is absent (no fallback path exists)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libpolfed_b200.so not built ({LIB_PATH}); run polfed.jl_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, f64, u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_uint64
    sig = {
        "pf_abi_version": (i32, []),
        "pf_abi_sizes": (None, [ctypes.POINTER(ctypes.c_size_t)] * 3),
        "pf_last_error": (ctypes.c_char_p, []),
        "pf_handle_create": (i32, [i32, ctypes.POINTER(vp)]),
        "pf_handle_destroy": (i32, [vp]),
        "pf_handle_stream": (i32, [vp, ctypes.POINTER(vp)]),
        "pf_handle_synchronize": (i32, [vp]),
        "pf_handle_set_overlap": (i32, [vp, i32]),
        "pf_op_spin_chain_create": (i32, [vp, i32, i32, i32, vp, vp, vp, vp, ctypes.POINTER(vp)]),
        "pf_op_qsun_create": (i32, [vp, i32, i32, f64, vp, vp, vp, vp, ctypes.POINTER(vp)]),
        "pf_op_qsun_spin_create": (i32, [vp, i32, i32, i32, i32, i32, f64, vp, vp, vp, vp, ctypes.POINTER(vp)]),
        "pf_op_destroy": (i32, [vp]),
        "pf_op_csr_create": (i32, [vp, i64, i64, vp, vp, vp, ctypes.POINTER(vp)]),
        "pf_op_csr_create_hermitian": (i32, [vp, i64, i64, vp, vp, vp, ctypes.POINTER(vp)]),
        "pf_op_bind": (i32, [vp, vp, ctypes.POINTER(vp)]),
        "pf_op_dim": (i64, [vp]),
        "pf_basis_unrank": (i32, [vp, i64, vp, vp]),
        "pf_basis_rank": (i32, [vp, i64, vp, vp]),
        "pf_apply": (i32, [vp, i32, f64, f64, i32, vp, i64, vp, i64]),
        "pf_apply_noalloc": (i32, [vp, i32, f64, f64, i32, vp, i64, vp, i64]),
        "pf_clenshaw_recurrence": (i32, [vp, i32, f64, f64, f64, i32, vp, vp, vp, vp, i64]),
        "pf_clenshaw_finalsum": (i32, [vp, i32, f64, f64, f64, i32, vp, vp, vp, vp, i64]),
        "pf_filter": (i32, [vp, i32, f64, f64, i32, vp, i32, vp, i64, vp, i64]),
        "pf_kpm_moments": (i32, [vp, i32, f64, f64, i32, i32, vp, i64, i32, u64, vp]),
        "pf_params_default": (None, [ctypes.POINTER(pf_params)]),
        "pf_solve": (i32, [vp, ctypes.POINTER(pf_params), i32, i32, vp, i32, vp, vp, i32,
                           ctypes.POINTER(pf_report), ctypes.POINTER(i32)]),
        "pf_solve_hermitian": (i32, [vp, ctypes.POINTER(pf_params), i32, i32, vp, i32, vp, vp, i32,
                                     ctypes.POINTER(pf_report), ctypes.POINTER(i32)]),
        "pf_lanczos_extrema": (i32, [vp, vp, i32, f64, f64, ctypes.POINTER(f64), ctypes.POINTER(f64)]),
        "pf_autotune": (i32, [vp, i32, i32, ctypes.POINTER(i32), vp]),
        "pf_set_step_width": (i32, [vp, i32, i32, i32]),
        "pf_set_step_variant": (i32, [vp, i32, i32, i32, i32]),
        "pf_gather_peak": (i32, [vp, i32, ctypes.POINTER(f64)]),
        "pf_set_filter_slab": (i32, [vp, i32]),
        "pf_gram_bf16x3": (i32, [vp, i64, i32, vp, i64, vp, i32, vp]),
        "pf_step_variant": (i32, [vp, i32, i32, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i32)]),
        "pf_step_profile": (i32, [vp, i32, i32, ctypes.POINTER(i32)]),
        "pf_pool_create": (i32, [i32, i32, f64, ctypes.POINTER(vp)]),
        "pf_pool_destroy": (i32, [vp]),
        "pf_pool_stream": (i32, [vp, i32, ctypes.POINTER(vp)]),
        "pf_pool_set_priority_dim": (i32, [vp, i64]),
        "pf_pool_set_admission": (i32, [vp, i32, f64]),
        "pf_solve_footprint": (f64, [vp, ctypes.POINTER(pf_params), i32, i32]),
        "pf_pool_solve_batch": (i32, [vp, i32, vp, vp, vp, vp, vp, i32, vp, vp, i32, vp, vp]),
        "pf_pool_submit": (i32, [vp, vp, ctypes.POINTER(pf_params), i32, i32, vp, vp, i32, ctypes.POINTER(i64)]),
        "pf_pool_poll": (i32, [vp, i64, ctypes.POINTER(i32)]),
        "pf_pool_fetch": (i32, [vp, i64, f64, vp, ctypes.POINTER(pf_report), ctypes.POINTER(i32)]),
        "pf_pool_cancel": (i32, [vp, i64]),
        "pf_pool_get_stats": (i32, [vp, ctypes.POINTER(pf_pool_stats)]),
        "pf_pool_request_times": (i32, [vp, i64, vp]),
        "pf_pool_wait": (i32, [vp, i64, f64, ctypes.POINTER(i32)]),
        "pf_pool_shutdown": (i32, [vp]),
        "pf_pool_set_batching": (i32, [vp, i32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if L.pf_abi_version() != 1:
        raise RuntimeError("libpolfed_b200.so ABI version mismatch")
    _LIB = L
    return L


def check(status: int) -> None:
    if status != PF_OK:
        msg = load().pf_last_error().decode(errors="replace")
        if status == PF_ERR_INVALID:
            raise PolfedArgumentError(status, msg)
        raise PolfedError(status, msg)


_HANDLES: dict[int, int] = {}


def handle(device: int = 0) -> int:
    """The process-wide default handle of a device (created on first use)."""
    if device not in _HANDLES:
        h = ctypes.c_void_p()
        check(load().pf_handle_create(device, ctypes.byref(h)))
        _HANDLES[device] = h.value
    return _HANDLES[device]


def new_handle(device: int = 0) -> int:
    """A fresh handle (own stream, cuBLAS / cuSOLVER handles, workspaces)."""
    h = ctypes.c_void_p()
    check(load().pf_handle_create(device, ctypes.byref(h)))
    return h.value


def stream_of(h: int) -> int:
    s = ctypes.c_void_p()
    check(load().pf_handle_stream(h, ctypes.byref(s)))
    return s.value or 0


def gather_peak(device: int = 0, log2_rows: int = 17) -> float:
    """Measured bytes/s of random row gathers from an L2-resident block
    (pf_gather_peak): the ceiling of an L2-resident step kernel."""
    v = ctypes.c_double()
    check(load().pf_gather_peak(handle(device), int(log2_rows), ctypes.byref(v)))
    return v.value


def synchronize(h: int) -> None:
    check(load().pf_handle_synchronize(h))
