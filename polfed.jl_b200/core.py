"""``polfed`` and its configuration / report types, mirroring Polfed.jl's API.

* ``polfed(op, x0, howmany, target; mapping, transform, fact, dos, produce_report)``
  -- PolfedCore.jl:194-263 (operator-callback overload; the operator is a
  matrix-free model from :mod:`models`).
* ``MappingConfig``, ``TransformConfig``, ``FactorizationConfig``,
  ``DoSConfig`` -- Polfed/Structs/*.jl with the PolfedDefaults.jl defaults.
* target specs -- Polfed/Structs/TargetSpec.jl:26-58.
* ``Report`` -- Report.jl:16-62 (SpectralTransformReport, FactorizationReport,
  BenchmarkReport fields).
* ``lanczos_extrema`` -- Lanczos.jl:183-212.
* operator-level drop-ins ``apply`` / ``clenshaw_recurrence`` /
  ``clenshaw_finalsum`` / ``chebyshev_filter`` / ``kpm_moments`` -- the
  ``MappingConfig`` callbacks (MappingConfig.jl:28-45) and ``dos_moments``
  (Moments.jl:42-46), on CUDA tensors.

Everything runs in libpolfed_b200.so; this module only marshals arguments.
"""
from __future__ import annotations

import ctypes
import math
import threading
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from .models import Operator, as_operator

# ------------------------------------------------------------------ configs


@dataclass
class MappingConfig:
    """MappingConfig.jl:82-103.  On the GPU the strategy is always NoParallel
    (Plan.jl:64-67); ``Emin``/``Emax`` skip the Lanczos probes when given."""
    Emin: Optional[float] = None
    Emax: Optional[float] = None
    parallel_strategy: Optional[str] = None
    optimize_mapping: bool = False


@dataclass
class TransformConfig:
    """TransformConfig.jl:77-100 (PolfedDefaults.jl:104-133)."""
    normalization: float = 1.0
    cutoff: float = 0.17
    left: Optional[float] = None
    right: Optional[float] = None
    order: Optional[int] = None
    order_safety_factor: float = 0.97
    polynomialtype: str = "Chebyshev"


@dataclass
class FactorizationConfig:
    """FactorizationConfig.jl:49-70 (PolfedDefaults.jl:151-191).
    ``reorth_passes`` 1 is the reference's FullRO; 2 is CGS2 in FP64; 3 is CGS2
    with its first Gram product on the tensor cores in split BF16.  ``refine_passes``:
    FP64 refinement passes of a ``precision="mixed"`` solve (0: none).
    ``host_qr``: factor every iteration's Gram matrices on the host instead of
    the device (the same results; the device form restarts with it when a
    block breaks down)."""
    which: str = "LR"
    tol: float = 1e-14
    eigentol: float = 1e-9
    overestimate_iters: float = 1.25
    reorth_passes: int = 1
    refine_passes: int = 4
    host_qr: bool = False


@dataclass
class DoSConfig:
    """DensitiesOfStatesConfig.jl:39-51 (PolfedDefaults.jl:203-217).
    ``probes`` (D x R, normalised columns) pins the otherwise random KPM probes."""
    N: int = 250
    R: int = 300
    kernel: str = "Jackson"
    probe_kind: str = "gaussian"
    seed: Optional[int] = None
    probes: Optional[np.ndarray] = None


def normalize_target_spec(target):
    """TargetSpec.jl:26-58 -> (kind id, value)."""
    if isinstance(target, str):
        if target == "maxdos":
            return _lib.PF_TARGET_MAXDOS, 0.0
        if target == "middle":
            return _lib.PF_TARGET_MIDDLE, 0.0
        raise ValueError(f"Unknown target symbol: {target}")
    if isinstance(target, tuple) and len(target) == 2 and isinstance(target[0], str):
        tag, val = target
        if isinstance(val, bool) or not isinstance(val, (int, float, np.integer, np.floating)):
            raise ValueError(f"Target tuple value must be Real, got {type(val)}")
        if tag == "absolute":
            raise ValueError("`(:absolute, value)` is no longer supported. Use `(:unrescaled, value)` instead.")
        if tag == "quantile":
            raise ValueError("`(:quantile, q)` is no longer supported.")
        if tag == "offset":
            if not (-1 <= val <= 1):
                raise ValueError(f"Offset target requires `eta in [-1, 1]`, got {val}")
            return _lib.PF_TARGET_OFFSET, float(val)
        if tag == "unrescaled":
            return _lib.PF_TARGET_UNRESCALED, float(val)
        if tag == "rescaled":
            return _lib.PF_TARGET_RESCALED, float(val)
        raise ValueError(f"Unknown target tuple tag: {tag}")
    if isinstance(target, (int, float, np.integer, np.floating)) and not isinstance(target, bool):
        return _lib.PF_TARGET_UNRESCALED, float(target)
    raise ValueError(f"Unsupported target specification: {target}")


def expectedkrylovdim(howmany: int, blocksize: int, eta: float) -> int:
    """PolfedDefaults.jl:61-62."""
    return int(math.ceil((20.427 * blocksize + 1.696 * howmany) * eta))


# ------------------------------------------------------------------ reports

STAGES = ("tridiagonalization", "mapping", "overlap", "orthogonalization", "reorthogonalization",
          "convergence", "extrema", "dos", "bounds_order", "total")


@dataclass
class SpectralTransformReport:
    target: float
    target_strategy: str
    left: float
    right: float
    polynomialtype: str
    order: int
    order_safety_factor: float
    howmany: int
    matrixvec_muls: int
    Emin: float
    Emax: float
    a: float
    b: float


@dataclass
class FactorizationReport:
    factorizationtype: str
    blocksize: int
    howmany: int
    itersneeded: int
    itersreserved: int
    krylovdim: int
    tol: float
    residual: float
    converged_tol: int
    eigentol: float
    eigenresidual: float
    converged_eigentol: int
    refined: int
    numofchecks: int
    converged_history: list
    krylovbasisdim_history: list
    maxresidual_history: list


@dataclass
class BenchmarkReport:
    stage_seconds: dict
    basis_bytes_reserved: float
    basis_bytes_used: float
    kpm_block_matvecs: int
    kernel_launches: int
    qr_restarts: int = 0


@dataclass
class Report:
    spectral: SpectralTransformReport
    factorization: FactorizationReport
    benchmark: BenchmarkReport


def _target_strategy(kind: int, value: float) -> str:
    return {0: ":maxdos", 1: ":middle", 2: f"(:offset, {value:.6g})", 3: f"(:unrescaled, {value:.6g})",
            4: f"(:rescaled, {value:.6g})"}[kind]


def _make_report(r: _lib.pf_report, kind: int, value: float) -> Report:
    n = r.numofchecks
    spec = SpectralTransformReport(r.target, _target_strategy(kind, value), r.left, r.right, "Chebyshev", r.order,
                                   r.order_safety_factor, r.howmany, int(r.matvecs), r.Emin, r.Emax, r.a, r.b)
    fac = FactorizationReport("LanczosFactorization" if r.blocksize == 1 else "BlockLanczosFactorization",
                              r.blocksize, r.howmany, r.iters_needed, r.iters_reserved, r.krylovdim, r.tol,
                              r.residual, r.converged_tol, r.eigentol, r.eigenresidual, r.converged_eigentol,
                              r.refined, r.numofchecks, list(r.converged_history[:n]), list(r.krylovdim_history[:n]),
                              list(r.maxresidual_history[:n]))
    bench = BenchmarkReport({k: r.stage_seconds[i] for i, k in enumerate(STAGES)}, r.basis_bytes_reserved,
                            r.basis_bytes_used, int(r.kpm_block_matvecs), int(r.kernel_launches),
                            int(r.qr_restarts))
    return Report(spec, fac, bench)


def display_report(report: Report) -> str:
    """Plain-text summary in the layout of Report.jl:47-62 (no colours)."""
    s, f, b = report.spectral, report.factorization, report.benchmark
    lines = [
        "Spectral Transformation Report:",
        f"- Targeted {s.howmany} eigenpairs with strategy {s.target_strategy} at rescaled energy {s.target:.6f}",
        f"- Exposing ev's in the rescaled interval [{s.left:.2e}, {s.right:.2e}], with width "
        f"δ = {s.right - s.left:.2e}",
        f"- Performing '{s.polynomialtype}' spectral transformation of order K = {s.order} "
        f"(and order safety factor {s.order_safety_factor})",
        f"- Matrix multiplication performed {s.matrixvec_muls} times!",
        f"Factorization Report: ({f.factorizationtype} with blocksize {f.blocksize})",
        f"- Number of converged eigenpairs:   {min(f.converged_tol, f.converged_eigentol)} (out of {f.howmany} requested)",
        f"- Lanczos convergence satisfied by: {f.converged_tol} (with tolerance {f.tol:.2e}, max residual {f.residual:.2e})",
        f"- Eigen convergence satisfied by:   {f.converged_eigentol} (with tolerance {f.eigentol:.2e}, "
        f"max residual {f.eigenresidual:.2e})",
        f"- Iterations needed: {f.itersneeded} (out of {f.itersreserved} reserved)",
        "Timings (CUDA events, seconds): " + ", ".join(f"{k}={v:.4f}" for k, v in b.stage_seconds.items()),
    ]
    text = "\n".join(lines)
    print(text)
    return text


# ------------------------------------------------------------------ solving

def _params(op: Operator, howmany: int, target, mapping: MappingConfig, transform: TransformConfig,
            fact: FactorizationConfig, dos: DoSConfig, precision: str):
    p = _lib.pf_params()
    _lib.load().pf_params_default(ctypes.byref(p))
    kind, val = normalize_target_spec(target)
    p.target_kind, p.target_value = kind, val
    if mapping.Emin is not None:
        p.has_Emin, p.Emin = 1, float(mapping.Emin)
    if mapping.Emax is not None:
        p.has_Emax, p.Emax = 1, float(mapping.Emax)
    if transform.polynomialtype != "Chebyshev":
        raise NotImplementedError("only the Chebyshev filter is implemented")
    if transform.left is not None:
        p.has_left, p.left = 1, float(transform.left)
    if transform.right is not None:
        p.has_right, p.right = 1, float(transform.right)
    p.order = 0 if transform.order is None else int(transform.order)
    if transform.order is not None and transform.order <= 0:
        raise ValueError("order must be positive")
    p.cutoff = transform.cutoff
    p.normalization = transform.normalization
    p.order_safety_factor = transform.order_safety_factor
    if fact.which not in ("LR", "SR"):
        raise ValueError(f"Unknown sorting mode: {fact.which}")
    p.which = _lib.PF_WHICH_LR if fact.which == "LR" else _lib.PF_WHICH_SR
    p.tol = fact.tol
    p.eigentol = fact.eigentol
    p.overestimate_iters = fact.overestimate_iters
    p.reorth_passes = int(fact.reorth_passes)
    p.host_qr = 1 if fact.host_qr else 0
    p.refine = int(fact.refine_passes)
    p.dos_N, p.dos_R = int(dos.N), int(dos.R)
    if dos.kernel not in _lib.KERNEL_IDS:
        raise ValueError(f"Unknown kernel: {dos.kernel}. Available: {list(_lib.KERNEL_IDS)}")
    p.dos_kernel = _lib.KERNEL_IDS[dos.kernel]
    p.probe_kind = {"gaussian": _lib.PF_PROBE_GAUSSIAN, "rademacher": _lib.PF_PROBE_RADEMACHER}[dos.probe_kind]
    p.seed = int(dos.seed) if dos.seed is not None else int(np.random.default_rng().integers(0, 2 ** 63))
    p.precision = {"fp64": _lib.PF_PREC_FP64, "mixed": _lib.PF_PREC_MIXED}[precision]
    keep = None
    if dos.probes is not None:
        keep = np.asfortranarray(dos.probes, dtype=np.float64)
        if keep.shape != (op.dim, dos.R):
            raise ValueError(f"probes must be D x R = {op.dim} x {dos.R}")
        p.probes = keep.ctypes.data
    return p, keep, kind, val


def polfed(op: Operator, x0, howmany: int, target, *, produce_report: bool = False,
           mapping: Optional[MappingConfig] = None, transform: Optional[TransformConfig] = None,
           fact: Optional[FactorizationConfig] = None, dos: Optional[DoSConfig] = None,
           precision: str = "fp64", vecs: bool = True):
    """POLFED on the B200 (PolfedCore.jl:194-263).

    ``op`` is a model operator or a real symmetric / complex Hermitian
    matrix (scipy.sparse, a CSR triple or dense; PolfedCore.jl:153-184).  ``x0`` is D (scalar
    Lanczos) or D x s (block Lanczos): a host array, or a
    column-major float64 CUDA tensor (then the eigenvectors are returned as a
    column-major CUDA tensor and never leave HBM).  A non-normalised /
    non-orthonormal start is replaced by a normalised copy, as the reference
    does.  Returns ``(vals, vecs)`` or ``(vals, vecs, report)``: the converged
    eigenpairs, ascending."""
    mapping = mapping or MappingConfig()
    transform = transform or TransformConfig()
    fact = fact or FactorizationConfig()
    dos = dos or DoSConfig()
    if howmany < 1:
        raise ValueError("howmany must be positive")
    op = as_operator(op)   # polfed(mat, ...): a sparse or dense matrix runs as a CSR operator
    if getattr(op, "is_complex", False):
        return _polfed_hermitian(op, x0, howmany, target, produce_report, mapping, transform, fact, dos,
                                 precision, vecs)
    D = op.dim
    on_device = _is_cuda_tensor(x0)
    if on_device:
        # device path: x0 and the eigenvectors stay in HBM (column-major CUDA tensors)
        import torch
        if x0.dtype != torch.float64:
            raise ValueError("x0 must be float64")
        if x0.dim() == 1:
            s = 1
            if x0.shape[0] != D or x0.stride(0) != 1:
                raise ValueError(f"x0 must be a contiguous vector of length {D}")
        elif x0.dim() == 2:
            s = x0.shape[1]
            if x0.shape[0] != D or x0.stride(0) != 1 or x0.stride(1) != D:
                raise ValueError(f"x0 must be a column-major {D} x s CUDA tensor")
        else:
            raise ValueError("x0 must be a vector or a matrix")
        x_ptr, x_mem = x0.data_ptr(), _lib.PF_MEM_DEVICE
        V = col_major(D, howmany, device=x0.device.index or 0) if vecs else None
        v_ptr, v_mem = (V.data_ptr() if vecs else None), _lib.PF_MEM_DEVICE
        keep_x = x0
    else:
        x = np.asarray(x0, dtype=np.float64)
        if x.ndim not in (1, 2):
            raise ValueError("x0 must be a vector or a matrix")
        if x.shape[0] != D:
            raise ValueError(f"x0 has {x.shape[0]} rows; the operator dimension is {D}")
        if x.size == 0:
            raise ValueError("POLFED initial vector must not be empty.")
        s = 1 if x.ndim == 1 else x.shape[1]
        keep_x = np.asfortranarray(x.reshape(D, s))
        x_ptr, x_mem = keep_x.ctypes.data, _lib.PF_MEM_HOST
        V = _host_out(D, howmany, device=op.device) if vecs else None
        v_ptr, v_mem = (V.ctypes.data if vecs else None), _lib.PF_MEM_HOST
    p, keep, kind, val = _params(op, howmany, target, mapping, transform, fact, dos, precision)
    vals = np.zeros(howmany)
    rep = _lib.pf_report()
    n = ctypes.c_int(0)
    _lib.check(_lib.load().pf_solve(op.op, ctypes.byref(p), s, howmany, x_ptr, x_mem, vals.ctypes.data, v_ptr,
                                    v_mem, ctypes.byref(rep), ctypes.byref(n)))
    del keep, keep_x
    k = n.value
    out_vals = vals[:k].copy()
    if vecs:
        out_vecs = V[:, :k]   # the first k columns: contiguous, no second pass over D x k
    else:
        out_vecs = None
    if produce_report:
        return out_vals, out_vecs, _make_report(rep, kind, val)
    return out_vals, out_vecs


def _polfed_hermitian(op, x0, howmany, target, produce_report, mapping, transform, fact, dos, precision, vecs):
    """polfed on a complex Hermitian matrix (``pf_solve_hermitian``): x0 is
    D or D x s complex (host, or a column-major complex128 CUDA tensor); the
    eigenvectors come back complex, unit norm, arbitrary phase.  KPM probes, if
    given (D x R, real or complex), act on the real embedding as [Re; Im]."""
    D = op.complex_dim
    on_device = _is_cuda_tensor(x0)
    if on_device:
        import torch
        if x0.dtype != torch.complex128:
            raise ValueError("x0 must be complex128")
        s = 1 if x0.dim() == 1 else x0.shape[1]
        if x0.shape[0] != D or x0.stride(0) != 1 or (x0.dim() == 2 and x0.stride(1) != D):
            raise ValueError(f"x0 must be a column-major {D} x s complex CUDA tensor")
        keep_x = x0
        x_ptr, x_mem = x0.data_ptr(), _lib.PF_MEM_DEVICE
        V = torch.empty((howmany, D), dtype=torch.complex128, device=x0.device).t() if vecs else None
        v_ptr, v_mem = (V.data_ptr() if vecs else None), _lib.PF_MEM_DEVICE
    else:
        x = np.asarray(x0, dtype=np.complex128)
        if x.ndim not in (1, 2) or x.shape[0] != D or x.size == 0:
            raise ValueError(f"x0 must be a non-empty vector or matrix with {D} rows")
        s = 1 if x.ndim == 1 else x.shape[1]
        keep_x = np.asfortranarray(x.reshape(D, s))
        x_ptr, x_mem = keep_x.ctypes.data, _lib.PF_MEM_HOST
        V = _host_out(D, howmany, np.complex128, device=op.device) if vecs else None
        v_ptr, v_mem = (V.ctypes.data if vecs else None), _lib.PF_MEM_HOST
    if dos.probes is not None:
        pr = np.asarray(dos.probes)
        if pr.shape != (D, dos.R):
            raise ValueError(f"probes must be D x R = {D} x {dos.R}")
        dos = DoSConfig(N=dos.N, R=dos.R, kernel=dos.kernel, probe_kind=dos.probe_kind, seed=dos.seed,
                        probes=np.vstack([pr.real, pr.imag]) if np.iscomplexobj(pr) else np.vstack([pr, 0 * pr]))
    p, keep, kind, val = _params(op, howmany, target, mapping, transform, fact, dos, precision)
    vals = np.zeros(howmany)
    rep = _lib.pf_report()
    n = ctypes.c_int(0)
    _lib.check(_lib.load().pf_solve_hermitian(op.op, ctypes.byref(p), s, howmany, x_ptr, x_mem, vals.ctypes.data,
                                              v_ptr, v_mem, ctypes.byref(rep), ctypes.byref(n)))
    del keep, keep_x
    k = n.value
    out_vecs = V[:, :k] if vecs else None
    if produce_report:
        return vals[:k].copy(), out_vecs, _make_report(rep, kind, val)
    return vals[:k].copy(), out_vecs


_WORKERS: dict = {}


def worker_handles(n: int, device: int = 0):
    """n process-wide worker handles of a device (each its own stream)."""
    hs = _WORKERS.setdefault(device, [])
    while len(hs) < n:
        hs.append(_lib.new_handle(device))
    return hs[:n]


def _host_out(D: int, m: int, dtype=np.float64, device: int = 0):
    """A column-major D x m host array for eigenvectors, in page-locked
    memory from torch's caching host allocator when CUDA is available (made
    with the operator's device current, so no other device gets a context),
    so the device-to-host copy of the results runs at the link's speed and
    the buffers of earlier results are reused; plain memory otherwise.  Only
    the returned columns are written."""
    try:
        import torch
        if torch.cuda.is_available():
            tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.complex128
            with torch.cuda.device(device):
                return torch.empty((m, D), dtype=tdt, pin_memory=True).numpy().T
    except (ImportError, RuntimeError):
        pass
    return np.zeros((D, m), dtype=dtype, order="F")


def _host_x0(op: Operator, x0):
    x = np.asarray(x0, dtype=np.float64)
    if x.ndim not in (1, 2):
        raise ValueError("x0 must be a vector or a matrix")
    if x.shape[0] != op.dim:
        raise ValueError(f"x0 has {x.shape[0]} rows; the operator dimension is {op.dim}")
    if x.size == 0:
        raise ValueError("POLFED initial vector must not be empty.")
    s = 1 if x.ndim == 1 else x.shape[1]
    return np.asfortranarray(x.reshape(op.dim, s)), s


def _device_x0(op: Operator, x0):
    import torch
    D = op.dim
    if x0.dtype != torch.float64:
        raise ValueError("x0 must be float64")
    if x0.dim() == 1:
        if x0.shape[0] != D or x0.stride(0) != 1:
            raise ValueError(f"x0 must be a contiguous vector of length {D}")
    elif x0.dim() == 2:
        if x0.shape[0] != D or x0.stride(0) != 1 or x0.stride(1) != D:
            raise ValueError(f"x0 must be a column-major {D} x s CUDA tensor")
    else:
        raise ValueError("x0 must be a vector or a matrix")
    return x0


def _solve_kwargs(kwargs):
    allowed = {"mapping", "transform", "fact", "dos", "precision", "produce_report", "vecs"}
    bad = set(kwargs) - allowed
    if bad:
        raise TypeError(f"unexpected keyword arguments {sorted(bad)}")
    return (kwargs.get("mapping") or MappingConfig(), kwargs.get("transform") or TransformConfig(),
            kwargs.get("fact") or FactorizationConfig(), kwargs.get("dos") or DoSConfig(),
            kwargs.get("precision", "fp64"), bool(kwargs.get("produce_report", False)), bool(kwargs.get("vecs", True)))


@dataclass
class PoolStats:
    """Counters and latency percentiles of a SolverPool (seconds, bytes)."""
    submitted: int
    completed: int
    failed: int
    queued: int
    running: int
    eigenpairs: int
    bytes_budget: float
    bytes_in_use: float
    bytes_peak: float
    p50_latency: float
    p99_latency: float
    mean_latency: float
    busy_seconds: float
    rejected: int
    filter_launches: float
    filter_seconds: float
    filter_bytes: float
    filter_instance_steps: float


class SolverPool:
    """Many POLFED solves on one device through the native request pool.

    ``workers`` solves run at once, each on its own handle and stream, so their
    latency-bound launches and host round trips overlap.  A request starts when
    a worker is free and its device footprint (``footprint``) fits in
    ``hbm_budget`` bytes (``None``: 90 % of the free memory at creation);
    otherwise it waits, first in first out.  ``solve_batch`` runs a list of
    problems to completion; ``submit`` / ``poll`` / ``result`` serve a stream
    of requests.  Every request runs the same solve as ``polfed`` and gives
    the same result whether it runs alone or among others."""

    def __init__(self, workers: int = 4, device: int = 0, hbm_budget: Optional[float] = None,
                 priority_dim: Optional[int] = None):
        self.device = device
        h = ctypes.c_void_p()
        _lib.check(_lib.load().pf_pool_create(device, int(workers), float(hbm_budget or 0.0), ctypes.byref(h)))
        self._pool = h
        self._pending: dict = {}
        self._cancelled: list = []   # result arrays of cancelled requests a worker may still write
        # native calls in flight from any Python thread; close() frees the pool
        # only after the last of them has returned
        self._cv = threading.Condition()
        self._active = 0
        self._closed = False
        if priority_dim is not None:
            self.set_priority_dim(priority_dim)

    def _native(self, name, *args):
        """Call pf_pool_<name>(pool, *args) so that close() cannot free the
        pool under it; returns the status."""
        with self._cv:
            if self._closed or self._pool is None:
                raise _lib.PolfedArgumentError(_lib.PF_ERR_INVALID, "pool is closed")
            self._active += 1
            pool = self._pool
        try:
            return getattr(_lib.load(), "pf_pool_" + name)(pool, *args)
        finally:
            with self._cv:
                self._active -= 1
                self._cv.notify_all()

    def set_admission(self, policy: str = "fifo", max_wait: float = 30.0):
        """Admission order: "fifo" (arrival order, the default) or "shortest"
        (least expected work first; a request queued ``max_wait`` seconds goes
        first and is not overtaken)."""
        pol = {"fifo": _lib.PF_ADMIT_FIFO, "shortest": _lib.PF_ADMIT_SHORTEST}[policy]
        _lib.check(self._native("set_admission", pol, float(max_wait)))

    def set_batching(self, on: bool = True):
        """Batched filtering (default off): the Clenshaw steps of all requests
        in flight share one multi-instance launch per step.  Off: each request
        runs its own graph-captured filter.  Results are the same either way."""
        _lib.check(self._native("set_batching", 1 if on else 0))

    def set_priority_dim(self, dim: int):
        """Requests with operator dimension <= ``dim`` (default 65536; 0: none)
        run on high-priority streams; results are unchanged."""
        _lib.check(self._native("set_priority_dim", int(dim)))

    def close(self):
        """Stop the pool: queued requests fail ("pool destroyed"), threads
        waiting for them return, running requests finish; then free it."""
        with self._cv:
            if self._closed or self._pool is None or not self._pool.value:
                self._closed = True
                return
            self._closed = True
            pool = self._pool
        _lib.check(_lib.load().pf_pool_shutdown(pool))
        with self._cv:
            self._cv.wait_for(lambda: self._active == 0)
        _lib.check(_lib.load().pf_pool_destroy(pool))
        self._pool = None
        self._pending.clear()
        self._cancelled.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover - interpreter shutdown
            pass

    @staticmethod
    def footprint(op: Operator, howmany: int, target, s: int, **kwargs) -> float:
        """Estimated device bytes of one solve (what admission charges)."""
        mapping, transform, fact, dos, precision, _, _ = _solve_kwargs(kwargs)
        p, keep, _, _ = _params(op, howmany, target, mapping, transform, fact, dos, precision)
        return _lib.load().pf_solve_footprint(op.op, ctypes.byref(p), int(s), int(howmany))

    def streams(self):
        """The pool's CUDA stream handles (integers): each worker's default-
        and high-priority stream."""
        out, w = [], 0
        while True:
            st = ctypes.c_void_p()
            if self._native("stream", w, ctypes.byref(st)) != _lib.PF_OK:
                return out
            out.append(st.value or 0)
            w += 1

    def solve_batch(self, ops, x0s, howmany: int, target, **kwargs):
        """Solve ``ops[i]`` from ``x0s[i]`` for all i; returns one ``polfed``
        result tuple per problem, in order.  ``x0s`` are all host arrays, or
        all column-major float64 CUDA tensors (then the eigenvectors come back
        as CUDA tensors and never leave HBM)."""
        if len(ops) != len(x0s):
            raise ValueError("one x0 per operator is required")
        n = len(ops)
        if n == 0:
            return []
        ops = [as_operator(o, self.device) for o in ops]
        mapping, transform, fact, dos, precision, want_rep, want_vecs = _solve_kwargs(kwargs)
        on_device = _is_cuda_tensor(x0s[0])
        if any(_is_cuda_tensor(x) != on_device for x in x0s):
            raise ValueError("x0s must be all host arrays or all CUDA tensors")
        keep = []
        params, xptr, ss, vals, vecs = [], [], [], [], []
        for op, x0 in zip(ops, x0s):
            if op.device != self.device:
                raise ValueError("operator and pool are on different devices")
            if on_device:
                x, s = _device_x0(op, x0), (1 if x0.dim() == 1 else x0.shape[1])
                xptr.append(x.data_ptr())
                V = col_major(op.dim, howmany, device=self.device) if want_vecs else None
            else:
                x, s = _host_x0(op, x0)
                xptr.append(x.ctypes.data)
                V = _host_out(op.dim, howmany, device=op.device) if want_vecs else None
            p, kp, kind, val = _params(op, howmany, target, mapping, transform, fact, dos, precision)
            keep += [x, kp]
            params.append(p)
            ss.append(s)
            vals.append(np.zeros(howmany))
            vecs.append(V)
        P = ctypes.c_void_p
        mem = _lib.PF_MEM_DEVICE if on_device else _lib.PF_MEM_HOST
        vptr = [(V.data_ptr() if on_device else V.ctypes.data) for V in vecs] if want_vecs else None
        a_ops = (P * n)(*[op.op for op in ops])
        a_par = (P * n)(*[ctypes.addressof(p) for p in params])
        a_s = (ctypes.c_int * n)(*ss)
        a_nev = (ctypes.c_int * n)(*([int(howmany)] * n))
        a_x = (P * n)(*xptr)
        a_v = (P * n)(*[v.ctypes.data for v in vals])
        a_V = (P * n)(*vptr) if want_vecs else None
        reps = (_lib.pf_report * n)()
        nconv = (ctypes.c_int * n)()
        _lib.check(self._native("solve_batch", n, a_ops, a_par, a_s, a_nev, a_x, mem, a_v, a_V, mem, reps, nconv))
        del keep
        out = []
        for i in range(n):
            k = nconv[i]
            V = vecs[i][:, :k] if want_vecs else None   # a view: no second pass over D x nev
            res = (vals[i][:k].copy(), V)
            if want_rep:
                res = res + (_make_report(reps[i], kind, val),)
            out.append(res)
        return out

    def submit(self, op: Operator, x0, howmany: int, target, **kwargs) -> int:
        """Queue one solve; returns its request id.  ``x0`` is copied."""
        op = as_operator(op, self.device)
        mapping, transform, fact, dos, precision, want_rep, want_vecs = _solve_kwargs(kwargs)
        if op.device != self.device:
            raise ValueError("operator and pool are on different devices")
        if dos.probes is not None:
            raise ValueError("served requests draw their KPM probes from dos.seed")
        x, s = _host_x0(op, x0)
        p, _, kind, val = _params(op, howmany, target, mapping, transform, fact, dos, precision)
        V = _host_out(op.dim, howmany, device=op.device) if want_vecs else None
        rid = ctypes.c_int64()
        _lib.check(self._native("submit", op.op, ctypes.byref(p), s, int(howmany), x.ctypes.data,
                                V.ctypes.data if want_vecs else None, _lib.PF_MEM_HOST, ctypes.byref(rid)))
        # the operator stays referenced until the result is collected: the
        # worker binds it when the request starts and updates its tuning after
        self._pending[rid.value] = (V, int(howmany), want_rep, kind, val, op)
        return rid.value

    def poll(self, request: int) -> str:
        """"queued", "running", "done", "failed" or "rejected" (the target
        cannot hold ``howmany`` states; ``result`` raises the reference's
        bisection error)."""
        st = ctypes.c_int()
        _lib.check(self._native("poll", int(request), ctypes.byref(st)))
        return ("queued", "running", "done", "failed", "rejected")[st.value]

    def wait(self, request: int, timeout: Optional[float] = None) -> str:
        """Wait until the request has finished (or ``timeout`` seconds pass)
        without collecting it; returns its state as ``poll`` does."""
        state = ctypes.c_int()
        _lib.check(self._native("wait", int(request), -1.0 if timeout is None else float(timeout),
                                ctypes.byref(state)))
        return ("queued", "running", "done", "failed", "rejected")[state.value]

    def times(self, request: int):
        """(submitted, started, finished) in seconds since the pool was
        created; -1 for what has not happened yet.  Valid until ``result``."""
        t = (ctypes.c_double * 3)()
        _lib.check(self._native("request_times", int(request), t))
        return tuple(t)

    def result(self, request: int, timeout: Optional[float] = None):
        """Wait for a request and return its ``polfed`` result tuple; raises the
        request's error if it failed (the request is released either way)."""
        V, howmany, want_rep, kind, val, _op = self._pending[request]
        vals = np.zeros(howmany)
        rep = _lib.pf_report()
        n = ctypes.c_int()
        st = self._native("fetch", int(request), -1.0 if timeout is None else float(timeout), vals.ctypes.data,
                          ctypes.byref(rep), ctypes.byref(n))
        if not (st == _lib.PF_ERR_NUMERIC and b"timeout" in _lib.load().pf_last_error()):
            self._pending.pop(request, None)
        if st != _lib.PF_OK and n.value == -_lib.PF_REQ_REJECTED:
            raise _lib.PolfedRejected(st, _lib.load().pf_last_error().decode(errors="replace"))
        _lib.check(st)
        k = n.value
        res = (vals[:k].copy(), V[:, :k] if V is not None else None)
        if want_rep:
            res = res + (_make_report(rep, kind, val),)
        return res

    def cancel(self, request: int):
        """Drop a queued request.  A request that has already started runs to
        the end and is then discarded; its worker still writes the result
        arrays, so they stay referenced until the pool is closed."""
        _lib.check(self._native("cancel", int(request)))
        held = self._pending.pop(request, None)
        if held is not None:
            self._cancelled.append(held)

    def stats(self) -> PoolStats:
        st = _lib.pf_pool_stats()
        _lib.check(self._native("get_stats", ctypes.byref(st)))
        return PoolStats(**{f: getattr(st, f) for f, _ in st._fields_})


_POOLS: dict = {}


def solver_pool(workers: int = 4, device: int = 0) -> SolverPool:
    """A process-wide SolverPool per (device, workers), created on first use."""
    key = (device, int(workers))
    if key not in _POOLS:
        _POOLS[key] = SolverPool(workers=workers, device=device)
    return _POOLS[key]


def polfed_batch(ops, x0s, howmany: int, target, *, workers: int = 4, **kwargs):
    """Solve many independent problems (e.g. disorder realisations) with
    ``workers`` solves in flight at once through the native request pool.
    ``x0s`` are host arrays or column-major CUDA tensors.  Returns one
    ``polfed`` result tuple per problem, in order."""
    if len(ops) != len(x0s):
        raise ValueError("one x0 per operator is required")
    if not ops:
        return []
    ops = [as_operator(o) for o in ops]
    return solver_pool(max(1, workers), ops[0].device).solve_batch(ops, x0s, howmany, target, **kwargs)


def tune_block_size(op: Operator, howmany: int, target, candidates=(4, 8, 16), seed: int = 7, **kwargs):
    """The block size for solves of this operator and request: one complete
    ``polfed`` solve at each candidate s (after an untimed one that also tunes
    the step kernel for that s), from the same seeded random start, timed on
    the host around a device synchronisation.  Returns ``(best_s, {s:
    converged pairs per second})``; ``kwargs`` are ``polfed``'s (``vecs`` is
    forced off).  Solves in flight together (a pool) share the device, so a
    batch's best s is that of one solve only approximately."""
    import time
    import torch
    op = as_operator(op)
    kwargs = dict(kwargs, vecs=False)
    kwargs.pop("produce_report", None)
    rates = {}
    for s in candidates:
        if s < 1 or s > op.dim:
            continue
        x0 = np.random.default_rng(seed).random((op.dim, s))
        polfed(op, x0, howmany, target, **kwargs)
        torch.cuda.synchronize(op.device)
        t = time.perf_counter()
        vals, _ = polfed(op, x0, howmany, target, **kwargs)
        torch.cuda.synchronize(op.device)
        rates[s] = len(vals) / (time.perf_counter() - t)
    if not rates:
        raise ValueError("no candidate block size fits the operator")
    return max(rates, key=rates.get), rates


def _is_cuda_tensor(x) -> bool:
    try:
        import torch
    except ImportError:  # pragma: no cover
        return False
    return isinstance(x, torch.Tensor) and x.is_cuda


def lanczos_extrema(op: Operator, x0, maxdim: int = 1000, tol: float = 1e-14, eigentol: float = 1e-8):
    """(Emin, Emax) by two Lanczos probes (Lanczos.jl:183-212)."""
    x = np.ascontiguousarray(x0, dtype=np.float64).ravel()
    if len(x) != op.dim:
        raise ValueError("x0 length must match the matrix dimension.")
    lo, hi = ctypes.c_double(), ctypes.c_double()
    _lib.check(_lib.load().pf_lanczos_extrema(op.op, x.ctypes.data, maxdim, tol, eigentol,
                                              ctypes.byref(lo), ctypes.byref(hi)))
    return lo.value, hi.value


# ---------------------------------------------------- operator-level drop-ins

def _cm(t, D):
    """(pointer, s, ld, dtype id) of a CUDA tensor holding a column-major D x s block."""
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise ValueError("operator-level calls take CUDA tensors")
    if t.dtype == torch.float64:
        dt = _lib.PF_F64
    elif t.dtype == torch.float32:
        dt = _lib.PF_F32
    else:
        raise ValueError("dtype must be float64 or float32")
    if t.dim() == 1:
        if t.shape[0] != D or t.stride(0) != 1:
            raise ValueError("vector length must equal the operator dimension and be contiguous")
        return t.data_ptr(), 1, D, dt
    if t.dim() != 2 or t.shape[0] != D or t.stride(0) != 1:
        raise ValueError("blocks must be column-major D x s (stride(0) == 1)")
    return t.data_ptr(), t.shape[1], max(t.stride(1), D), dt


def col_major(D: int, s: int, dtype=None, device: int = 0):
    """An uninitialised column-major D x s CUDA tensor."""
    import torch
    dtype = torch.float64 if dtype is None else dtype
    return torch.empty((s, D), dtype=dtype, device=f"cuda:{device}").t()


def _sync_in(op):
    import torch
    torch.cuda.synchronize(op.device)


def _sync_out(op):
    _lib.synchronize(op.handle)


def apply(op: Operator, Y, X, a: float = 1.0, b: float = 0.0):
    """Y = (H X - b X)/a  (f!_rescaled of Plan.jl:173-177; a=1, b=0: f!)."""
    D = op.dim
    px, s, ldx, dt = _cm(X, D)
    py, s2, ldy, dt2 = _cm(Y, D)
    if s != s2 or dt != dt2:
        raise ValueError("X and Y must have the same shape and dtype")
    _sync_in(op)
    _lib.check(_lib.load().pf_apply(op.op, dt, a, b, s, px, ldx, py, ldy))
    _sync_out(op)
    return Y


def clenshaw_recurrence(op: Operator, b1, b2, b3, c: float, X, a: float = 1.0, b: float = 0.0):
    """b1 = c X + 2 Htilde b2 - b3 (vector_dispatch.jl:113-125)."""
    D = op.dim
    p1, s, ld, dt = _cm(b1, D)
    ptrs = [_cm(t, D) for t in (b2, b3, X)]
    if any(q[1] != s or q[2] != ld or q[3] != dt for q in ptrs):
        raise ValueError("all blocks must share shape, leading dimension and dtype")
    _sync_in(op)
    _lib.check(_lib.load().pf_clenshaw_recurrence(op.op, dt, a, b, c, s, p1, ptrs[0][0], ptrs[1][0], ptrs[2][0], ld))
    _sync_out(op)
    return b1


def clenshaw_finalsum(op: Operator, b1, b2, c0: float, Y, X, a: float = 1.0, b: float = 0.0):
    """Y = c0 X + Htilde b1 - b2 (vector_dispatch.jl:127-139)."""
    D = op.dim
    py, s, ld, dt = _cm(Y, D)
    ptrs = [_cm(t, D) for t in (b1, b2, X)]
    if any(q[1] != s or q[2] != ld or q[3] != dt for q in ptrs):
        raise ValueError("all blocks must share shape, leading dimension and dtype")
    _sync_in(op)
    _lib.check(_lib.load().pf_clenshaw_finalsum(op.op, dt, a, b, c0, s, ptrs[0][0], ptrs[1][0], py, ptrs[2][0], ld))
    _sync_out(op)
    return Y


def chebyshev_filter(op: Operator, Y, X, coeffs, a: float = 1.0, b: float = 0.0):
    """Y = sum_k coeffs[k] T_k(Htilde) X (ClenshawAlgorithm.jl:12-29)."""
    D = op.dim
    px, s, ldx, dt = _cm(X, D)
    py, s2, ldy, dt2 = _cm(Y, D)
    if s != s2 or dt != dt2:
        raise ValueError("X and Y must have the same shape and dtype")
    c = np.ascontiguousarray(coeffs, dtype=np.float64)
    _sync_in(op)
    _lib.check(_lib.load().pf_filter(op.op, dt, a, b, len(c) - 1, c.ctypes.data, s, px, ldx, py, ldy))
    _sync_out(op)
    return Y


def kpm_moments(op: Operator, N: int, R: int, a: float = 1.0, b: float = 0.0, probes=None,
                probe_kind: str = "gaussian", seed: int = 0, dtype: str = "fp64"):
    """KPM moments (Moments.jl:42-140); ``probes`` a column-major D x R CUDA tensor."""
    mu = np.zeros(N)
    if probes is not None:
        pp, R2, ldp, dt = _cm(probes, op.dim)
        if R2 != R:
            raise ValueError("probes must have R columns")
    else:
        pp, ldp = None, op.dim
        dt = _lib.PF_F64 if dtype == "fp64" else _lib.PF_F32
    kind = {"gaussian": _lib.PF_PROBE_GAUSSIAN, "rademacher": _lib.PF_PROBE_RADEMACHER}[probe_kind]
    _sync_in(op)
    _lib.check(_lib.load().pf_kpm_moments(op.op, dt, a, b, N, R, pp, ldp, kind, seed, mu.ctypes.data))
    _sync_out(op)
    return mu


def autotune(op: Operator, s: int, dtype: str = "fp64"):
    """Time every variant of the step kernel for block width ``s`` (1..16
    columns per thread, and width 0 = the warp-cooperative chain step where
    offered); the fastest is kept on the operator.  Returns
    (width, {width: ms})."""
    w = ctypes.c_int(0)
    t = (ctypes.c_float * 6)()
    dt = _lib.PF_F64 if dtype == "fp64" else _lib.PF_F32
    _lib.check(_lib.load().pf_autotune(op.op, dt, int(s), ctypes.byref(w), ctypes.addressof(t)))
    widths = [1, 2, 4, 8, 16, _lib.PF_WIDTH_COOP]
    return w.value, {widths[i]: t[i] for i in range(6) if t[i] > 0}


def set_filter_slab(op: Operator, cols: int = 0):
    """Filter column slabs: ``cols`` > 0 filters in slabs of that many columns
    (a divisor of s); <= 0 whole blocks (the default).  Results are unchanged."""
    _lib.check(_lib.load().pf_set_filter_slab(op.op, int(cols)))


def set_launch_overlap(on: bool = True, device: int = 0):
    """Programmatic dependent launch of the step kernels on the device's
    default handle (on by default): each step's launch and table set-up
    overlap the previous step's tail.  Results are identical either way."""
    _lib.check(_lib.load().pf_handle_set_overlap(_lib.handle(device), 1 if on else 0))


def step_variant(op: Operator, s: int, dtype: str = "fp64"):
    """The step-kernel variant in use for block width ``s``: (columns per
    thread, gathers per batch, resident CTAs per SM); width 0 is the
    warp-cooperative chain step."""
    w, u, mb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    dt = _lib.PF_F64 if dtype == "fp64" else _lib.PF_F32
    _lib.check(_lib.load().pf_step_variant(op.op, dt, int(s), ctypes.byref(w), ctypes.byref(u), ctypes.byref(mb)))
    return w.value, u.value, mb.value


def step_profile(op: Operator, s: int, dtype: str = "fp64") -> int:
    """The profile (0..9, as for ``set_step_width``) of the step-kernel
    variant in use for block width ``s``."""
    pr = ctypes.c_int()
    dt = _lib.PF_F64 if dtype == "fp64" else _lib.PF_F32
    _lib.check(_lib.load().pf_step_profile(op.op, dt, int(s), ctypes.byref(pr)))
    return pr.value


def set_step_width(op: Operator, s: int, width: int, dtype: str = "fp64", profile: int = 0):
    """Pin the step-kernel variant for block width ``s`` (see ``autotune``):
    ``width`` columns per thread (0: the warp-cooperative chain step) and a
    (gather batch, register cap) ``profile`` 0..4; 5 (Quantum Sun only: all
    of a row's gathers as asynchronous global-to-shared copies); 6, 8, 9
    (Quantum Sun only: shared-memory row tiles of 1, 2 or 4 rows per thread);
    7 (spin chains on an Sz sector: local flip-rank updates)."""
    dt = _lib.PF_F64 if dtype == "fp64" else _lib.PF_F32
    _lib.check(_lib.load().pf_set_step_variant(op.op, dt, int(s), int(width), int(profile)))


def basis_states(op: Operator, idx):
    """Basis states of indices ``idx`` (CUDA int64 tensor) -> CUDA uint64-as-int64 tensor."""
    import torch
    out = torch.empty_like(idx)
    _sync_in(op)
    _lib.check(_lib.load().pf_basis_unrank(op.op, idx.numel(), idx.data_ptr(), out.data_ptr()))
    _sync_out(op)
    return out


def basis_index(op: Operator, states):
    """Indices of basis ``states`` (CUDA int64 tensor), -1 when outside the sector."""
    import torch
    out = torch.empty_like(states)
    _sync_in(op)
    _lib.check(_lib.load().pf_basis_rank(op.op, states.numel(), states.data_ptr(), out.data_ptr()))
    _sync_out(op)
    return out
