"""Model constructors mirroring ``Polfed.Models`` (SpinHalfChains.jl, QSun/).

The reference constructors return a ``SparseMatrixCSC``; here they return a
matrix-free operator descriptor whose device form (``pf_op``) the CUDA kernels
apply directly.  Arguments, defaults and validation follow the reference:

* ``xxz_hamiltonian``  -- SpinHalfChains.jl:74-99
* ``j1j2_hamiltonian`` -- SpinHalfChains.jl:189-220
* ``qsun_hamiltonian`` -- Models/Models.jl:97-115 -> QSun/QSun.jl:277-324 ->
  QSun/QuantumSun.jl:1-102 (full space, matrix-free for S = 1/2, device-built
  CSR for S > 1/2) and QSun/QuantumSun_U1_conserving.jl:1-212 (total-S_z
  sector, any S, device-built CSR)

Random draws use a numpy ``Generator`` (``rng``); Julia's MersenneTwister
streams are not reproducible outside Julia, so a realisation is identified by
its explicit parameter arrays (``fields``, ``couplings``, ...), which every
operator exposes.
"""
from __future__ import annotations

import ctypes
import math
from typing import Optional, Sequence

import numpy as np

from . import _lib

_SUPPORTED_BOUNDARIES = ("periodic", "open")


def chain_bonds(L: int, distance: int, boundary: str = "periodic"):
    """0-based bonds of ``_chain_bonds`` (SpinHalfChains.jl:227-243)."""
    if boundary not in _SUPPORTED_BOUNDARIES:
        raise ValueError(f"boundary must be one of (:periodic, :open); got {boundary}.")
    if boundary == "open":
        if distance >= L:
            return []
        return [(i, i + distance) for i in range(L - distance)]
    bonds = []
    for i in range(1, L + 1):
        j = (i + distance - 1) % L + 1  # mod1(i + distance, L)
        if i == j:
            continue
        bonds.append((i - 1, j - 1))
    return bonds


def _validate_chain_length(L: int) -> None:
    if L < 2:
        raise ValueError(f"L must be at least 2; got L={L}.")


def _resolve_fields(L: int, field: float, W: float, fields, rng) -> np.ndarray:
    """``_resolve_fields`` (SpinHalfChains.jl:245-257): h_i = field + W (2u - 1)."""
    if fields is not None:
        fields = np.asarray(fields, dtype=np.float64).ravel()
        if len(fields) != L:
            raise ValueError(f"fields must have length L={L}; got length {len(fields)}.")
        return fields.copy()
    W = float(W)
    if W < 0:
        raise ValueError(f"W must be non-negative; got {W}.")
    if W == 0:
        return np.full(L, float(field))
    rng = np.random.default_rng() if rng is None else rng
    return float(field) + W * (2 * rng.random(L) - 1)


class Operator:
    """Base of the matrix-free operators: owns the device descriptor."""

    kind = "operator"

    def __init__(self, device: int = 0):
        self.device = device
        self._op: Optional[int] = None

    @property
    def handle(self) -> int:
        return _lib.handle(self.device)

    @property
    def op(self) -> int:
        if self._op is None:
            self._op = self._create()
        return self._op

    def _create(self) -> int:  # pragma: no cover - abstract
        raise NotImplementedError

    @property
    def dim(self) -> int:
        return int(_lib.load().pf_op_dim(self.op))

    @property
    def shape(self):
        return (self.dim, self.dim)

    def bind(self, handle: int) -> "BoundOperator":
        """A view of this operator that runs on another handle (stream) of the
        same device; it shares the device tables (pf_op_bind)."""
        return BoundOperator(self, handle)

    def close(self) -> None:
        if self._op is not None:
            _lib.load().pf_op_destroy(self._op)
            self._op = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BoundOperator(Operator):
    """An operator view bound to a specific handle (see Operator.bind)."""

    def __init__(self, base: Operator, handle: int):
        super().__init__(base.device)
        self.base = base
        self.kind = base.kind
        self._handle = handle
        out = ctypes.c_void_p()
        _lib.check(_lib.load().pf_op_bind(base.op, handle, ctypes.byref(out)))
        self._op = out.value

    @property
    def handle(self) -> int:
        return self._handle


class SpinChainOperator(Operator):
    """Spin-1/2 chain H = sum_b J_b[(S+S- + h.c.)/2 + Delta_b SzSz] + sum_i h_i Sz_i
    on the sector with ``Lup`` up spins (``Lup=-1``: full 2^L space)."""

    kind = "spin_chain"

    def __init__(self, L: int, Lup: int, bonds: Sequence, couplings, anisotropies, fields, device: int = 0):
        super().__init__(device)
        if not (0 <= Lup <= L or Lup == -1):
            raise ValueError(f"Lup must satisfy 0 <= Lup <= L; got Lup={Lup} for L={L}.")
        self.L = int(L)
        self.Lup = int(Lup)
        self.bonds = [(int(i), int(j)) for i, j in bonds]
        self.couplings = np.asarray(couplings, dtype=np.float64).reshape(-1)
        self.anisotropies = np.asarray(anisotropies, dtype=np.float64).reshape(-1)
        self.fields = np.asarray(fields, dtype=np.float64).reshape(-1)
        if len(self.couplings) != len(self.bonds) or len(self.anisotropies) != len(self.bonds):
            raise ValueError("one coupling and one anisotropy per bond are required")
        if len(self.fields) != self.L:
            raise ValueError(f"fields must have length L={self.L}; got length {len(self.fields)}.")

    def _create(self) -> int:
        nb = len(self.bonds)
        bonds = np.ascontiguousarray(np.array(self.bonds, dtype=np.int32).reshape(-1) if nb else np.zeros(2, np.int32))
        J = np.ascontiguousarray(self.couplings if nb else np.zeros(1))
        Dl = np.ascontiguousarray(self.anisotropies if nb else np.zeros(1))
        f = np.ascontiguousarray(self.fields)
        out = ctypes.c_void_p()
        _lib.check(_lib.load().pf_op_spin_chain_create(
            self.handle, self.L, self.Lup, nb, bonds.ctypes.data, J.ctypes.data, Dl.ctypes.data,
            f.ctypes.data, ctypes.byref(out)))
        return out.value

    def expected_dim(self) -> int:
        return 2 ** self.L if self.Lup < 0 else math.comb(self.L, self.Lup)


class QSunOperator(Operator):
    """Spin-1/2 Quantum Sun in the full space (QuantumSun.jl:1-102)."""

    kind = "qsun"

    def __init__(self, L_loc: int, L_grain: int, g0: float, couplings, neighbors, fields, grain,
                 device: int = 0):
        super().__init__(device)
        self.L_loc = int(L_loc)
        self.L_grain = int(L_grain)
        self.g0 = float(g0)
        self.couplings = np.asarray(couplings, dtype=np.float64).reshape(-1)
        self.neighbors = np.asarray(neighbors, dtype=np.int32).reshape(-1)
        self.fields = np.asarray(fields, dtype=np.float64).reshape(-1)
        dg = 2 ** self.L_grain
        self.grain = np.asarray(grain, dtype=np.float64).reshape(dg, dg)
        for arr, name in ((self.couplings, "couplings"), (self.neighbors, "neighbors"), (self.fields, "fields")):
            if len(arr) != self.L_loc:
                raise ValueError(f"{name} must have length L_loc={self.L_loc}")

    def _create(self) -> int:
        c = np.ascontiguousarray(self.couplings)
        n = np.ascontiguousarray(self.neighbors, dtype=np.int32)
        f = np.ascontiguousarray(self.fields)
        g = np.ascontiguousarray(self.grain)
        out = ctypes.c_void_p()
        _lib.check(_lib.load().pf_op_qsun_create(
            self.handle, self.L_loc, self.L_grain, self.g0, c.ctypes.data, n.ctypes.data, f.ctypes.data,
            g.ctypes.data, ctypes.byref(out)))
        return out.value


def spin_sector_count(n_sites: int, d: int, total: int) -> int:
    """Number of strings of ``n_sites`` digits in 0..d-1 with digit sum
    ``total`` (the states of a total-S_z sector: digit = m + S)."""
    if total < 0 or total > n_sites * (d - 1):
        return 0
    cnt = [1] + [0] * total
    for _ in range(n_sites):
        nxt = [0] * (total + 1)
        for t in range(total + 1):
            nxt[t] = sum(cnt[t - c] for c in range(min(d - 1, t) + 1))
        cnt = nxt
    return cnt[total]


def _spin_sector(L: int, S: float, S_z: float):
    """(d, digit-sum target) of the sector S_z for L spins S, with the
    reference's check (QuantumSun_U1_conserving.jl:17-20)."""
    sector_index = S_z + L * S
    if abs(S_z) > L * S or not float(sector_index).is_integer():
        raise ValueError(f"Wrong total value of spin to given spin-S particles. You chose S = {S} and S_z = {S_z}.")
    return int(round(2 * S)) + 1, int(round(sector_index))


def qsun_spin_grain(goe, L_loc: int, L_grain: int, S: float, *, gamma: float = 1.0, use_U1: bool = False,
                    S_z: float = 0.0) -> np.ndarray:
    """The grain block as the reference builds it from the GOE draw: the full
    space takes gamma GOE / sqrt(dg + 1) (QuantumSun.jl:29-30); the sector masks
    the GOE to equal grain magnetisation and scales it by gamma / sqrt(tr(R^2) /
    dim) with R = kron(I, masked) restricted to the sector
    (QuantumSun_U1_conserving.jl:34-90); tr(R^2) = sum over grain states g of
    (localized completions of g) * sum_g' masked[g, g']^2."""
    d = int(round(2 * S)) + 1
    dg = d ** L_grain
    goe = np.asarray(goe, dtype=np.float64).reshape(dg, dg)
    if not use_U1:
        return gamma * goe / math.sqrt(dg + 1)
    _, T = _spin_sector(L_loc + L_grain, S, S_z)
    gsum = np.array([sum((g // d ** i) % d for i in range(L_grain)) for g in range(dg)])
    masked = np.where(gsum[:, None] == gsum[None, :], goe, 0.0)
    dim = spin_sector_count(L_loc + L_grain, d, T)
    mult = np.array([spin_sector_count(L_loc, d, T - int(gs)) for gs in gsum], dtype=np.float64)
    tr = float(np.sum(mult * np.sum(masked * masked, axis=1)))
    return gamma * masked / math.sqrt(tr / dim)


class QSunSpinOperator(Operator):
    """The Quantum Sun for spin S (QuantumSun.jl:1-102) or in the total-S_z
    sector (``use_U1``; QuantumSun_U1_conserving.jl:1-212), assembled as a CSR
    matrix on the device (``pf_op_qsun_spin_create``).  ``grain`` is the final
    (2S+1)^L_grain block (``qsun_spin_grain``)."""

    kind = "qsun_spin"

    def __init__(self, L_loc: int, L_grain: int, S: float, g0: float, couplings, neighbors, fields, grain,
                 use_U1: bool = False, S_z: float = 0.0, device: int = 0):
        super().__init__(device)
        if not float(2 * S).is_integer() or S <= 0:
            raise ValueError(f"Wrong value of spin. Only integer spins or half-integer spins are possible. You chose S = {S}")
        self.L_loc, self.L_grain, self.S = int(L_loc), int(L_grain), float(S)
        self.g0, self.use_U1, self.S_z = float(g0), bool(use_U1), float(S_z)
        if self.use_U1:
            _spin_sector(self.L_loc + self.L_grain, self.S, self.S_z)
        self.couplings = np.asarray(couplings, dtype=np.float64).reshape(-1)
        self.neighbors = np.asarray(neighbors, dtype=np.int32).reshape(-1)
        self.fields = np.asarray(fields, dtype=np.float64).reshape(-1)
        dg = (int(round(2 * S)) + 1) ** self.L_grain
        self.grain = np.asarray(grain, dtype=np.float64).reshape(dg, dg)
        for arr, name in ((self.couplings, "couplings"), (self.neighbors, "neighbors"), (self.fields, "fields")):
            if len(arr) != self.L_loc:
                raise ValueError(f"{name} must have length L_loc={self.L_loc}")

    def _create(self) -> int:
        c = np.ascontiguousarray(self.couplings)
        n = np.ascontiguousarray(self.neighbors, dtype=np.int32)
        f = np.ascontiguousarray(self.fields)
        g = np.ascontiguousarray(self.grain)
        out = ctypes.c_void_p()
        _lib.check(_lib.load().pf_op_qsun_spin_create(
            self.handle, self.L_loc, self.L_grain, int(round(2 * self.S)), 1 if self.use_U1 else 0,
            int(round(2 * self.S_z)), self.g0, c.ctypes.data, n.ctypes.data, f.ctypes.data, g.ctypes.data,
            ctypes.byref(out)))
        return out.value


class SparseOperator(Operator):
    """A real symmetric or complex Hermitian sparse matrix as the operator of
    ``polfed(mat, ...)`` (PolfedCore.jl:153-184, whose operator is
    ``mul!(Y, mat, X)``).  ``mat`` is anything with ``tocsr()`` (a
    scipy.sparse matrix), a CSR triple ``(indptr, indices, values)`` of a
    square matrix, or a dense 2-D array.  Symmetry (Hermiticity) is the
    caller's contract, as in the reference.  Complex values give a Hermitian
    operator (``is_complex``): the device holds its real embedding
    [[A, -B], [B, A]] of twice the dimension and ``polfed`` solves it in the
    complex problem's terms (``pf_solve_hermitian``); the reference's CPU path
    takes such matrices, its GPU path refuses them (PolfedCore.jl:160-162)."""

    kind = "csr"

    def __init__(self, mat, device: int = 0):
        super().__init__(device)
        if hasattr(mat, "tocsr"):
            m = mat.tocsr()
            if m.shape[0] != m.shape[1]:
                raise ValueError(f"the matrix must be square; got {m.shape}")
            indptr, indices, values = m.indptr, m.indices, m.data
        elif isinstance(mat, tuple) and len(mat) == 3:
            indptr, indices, values = mat
        else:
            a = np.asarray(mat)
            if a.ndim != 2 or a.shape[0] != a.shape[1]:
                raise ValueError(f"the matrix must be square; got shape {a.shape}")
            rows, cols = np.nonzero(a)
            indptr = np.searchsorted(rows, np.arange(a.shape[0] + 1))
            indices, values = cols, a[rows, cols]
        self.is_complex = bool(np.iscomplexobj(values))
        self.indptr = np.ascontiguousarray(indptr, dtype=np.int64)
        self.indices = np.ascontiguousarray(indices, dtype=np.int32)
        self.values = np.ascontiguousarray(values, dtype=np.complex128 if self.is_complex else np.float64)
        if self.is_complex:
            D = len(self.indptr) - 1
            rows = np.repeat(np.arange(D), np.diff(self.indptr)) if D > 0 else np.zeros(0, np.int64)
            if np.any(self.values.imag[rows == self.indices] != 0.0):
                raise ValueError("a Hermitian matrix has a real diagonal")
        if self.indptr.ndim != 1 or len(self.indptr) < 2:
            raise ValueError("indptr must hold D + 1 row pointers")
        if len(self.indices) != len(self.values) or self.indptr[-1] != len(self.values):
            raise ValueError("indices and values must hold indptr[-1] entries")

    def _create(self) -> int:
        D = len(self.indptr) - 1
        nnz = len(self.values)
        idx = self.indices if nnz else np.zeros(1, np.int32)
        val = self.values if nnz else np.zeros(1)
        out = ctypes.c_void_p()
        create = _lib.load().pf_op_csr_create_hermitian if self.is_complex else _lib.load().pf_op_csr_create
        if self.is_complex and not nnz:
            val = np.zeros(1, np.complex128)
        _lib.check(create(self.handle, D, nnz, self.indptr.ctypes.data, idx.ctypes.data, val.ctypes.data,
                          ctypes.byref(out)))
        return out.value

    @property
    def complex_dim(self) -> int:
        """H's dimension for a Hermitian operator (its device embedding has twice it)."""
        return len(self.indptr) - 1


def as_operator(mat, device: int = 0) -> Operator:
    """An Operator as is; a matrix (sparse, CSR triple or dense) as a SparseOperator."""
    return mat if isinstance(mat, Operator) else SparseOperator(mat, device=device)


def xxz_hamiltonian(L: int, Lup: int, J: float, Delta: float, W: float, *, boundary: str = "periodic",
                    field: float = 0.0, fields=None, rng=None, device: int = 0) -> SpinChainOperator:
    """XXZ chain (SpinHalfChains.jl:74-99)."""
    _validate_chain_length(L)
    bonds = chain_bonds(int(L), 1, boundary)
    local_fields = _resolve_fields(int(L), field, W, fields, rng)
    return SpinChainOperator(L, Lup, bonds, [float(J)] * len(bonds), [float(Delta)] * len(bonds),
                             local_fields, device=device)


def j1j2_hamiltonian(L: int, Lup: int, J1: float, J2: float, Delta1: float, Delta2: float, W: float, *,
                     boundary: str = "periodic", field: float = 0.0, fields=None, rng=None,
                     device: int = 0) -> SpinChainOperator:
    """J1-J2 XXZ chain (SpinHalfChains.jl:189-220)."""
    _validate_chain_length(L)
    nn = chain_bonds(int(L), 1, boundary)
    nnn = chain_bonds(int(L), 2, boundary)
    local_fields = _resolve_fields(int(L), field, W, fields, rng)
    return SpinChainOperator(L, Lup, nn + nnn, [float(J1)] * len(nn) + [float(J2)] * len(nnn),
                             [float(Delta1)] * len(nn) + [float(Delta2)] * len(nnn), local_fields,
                             device=device)


def goe_matrix(n: int, rng) -> np.ndarray:
    """(X + X^T)/sqrt(2), X ~ randn (RandomUtils.jl:5-8)."""
    X = rng.standard_normal((n, n))
    return (X + X.T) / math.sqrt(2)


def qsun_parameters(L_loc: int, L_grain: int, alpha: float, *, gamma: float = 1.0, w: float = 0.5,
                    hz: float = 1.0, zeta: float = 0.2, rng=None):
    """Random draws of build_hamiltonian (QuantumSun.jl:21-30) in the same order:
    fields ~ U[hz-w, hz+w], neighbours ~ U{0..L_grain-1}, couplings c_1 = 1,
    c_j = alpha^(j-1+U(-zeta,zeta)), grain = gamma * GOE / sqrt(dg + 1)."""
    rng = np.random.default_rng() if rng is None else rng
    fields = rng.random(L_loc) * ((hz + w) - (hz - w)) + (hz - w)
    neighbors = rng.integers(0, L_grain, size=L_loc)
    couplings = np.zeros(L_loc)
    if alpha > 0:
        couplings[0] = 1.0
        for j in range(2, L_loc + 1):
            u = j - 1 + rng.random() * 2 * zeta - zeta
            couplings[j - 1] = alpha ** u
    dg = 2 ** L_grain
    grain = gamma * goe_matrix(dg, rng) / math.sqrt(dg + 1)
    return fields, neighbors, couplings, grain


def qsun_spin_parameters(L_loc: int, L_grain: int, alpha: float, S: float = 0.5, *, w: float = 0.5,
                         hz: float = 1.0, zeta: float = 0.2, rng=None):
    """The draws of build_hamiltonian / build_hamiltonian_cons in their order
    (QuantumSun.jl:21-30, QuantumSun_U1_conserving.jl:28-36): fields, grain
    neighbours, couplings, then the raw GOE of dimension (2S+1)^L_grain (its
    scaling depends on the model: ``qsun_spin_grain``)."""
    rng = np.random.default_rng() if rng is None else rng
    fields = rng.random(L_loc) * ((hz + w) - (hz - w)) + (hz - w)
    neighbors = rng.integers(0, L_grain, size=L_loc)
    couplings = np.zeros(L_loc)
    if alpha > 0:
        couplings[0] = 1.0
        for j in range(2, L_loc + 1):
            u = j - 1 + rng.random() * 2 * zeta - zeta
            couplings[j - 1] = alpha ** u
    dg = (int(round(2 * S)) + 1) ** L_grain
    return fields, neighbors, couplings, goe_matrix(dg, rng)


def qsun_hamiltonian(L_loc: int, L_grain: int, g0: float, alpha: float, *, gamma: float = 1.0, w: float = 0.5,
                     hz: float = 1.0, zeta: float = 0.2, S: float = 0.5, rng=None, use_U1: bool = False,
                     S_z: float = 0.0, couplings=None, neighbors=None, fields=None, grain=None,
                     device: int = 0) -> QSunOperator:
    """Quantum Sun model (QSun.jl:277-324).  The spin-1/2 full space
    (QuantumSun.jl:1-102) is the matrix-free ``QSunOperator``; spin S > 1/2 and
    the total-S_z sector (``use_U1``, QuantumSun_U1_conserving.jl:1-212) are a
    ``QSunSpinOperator`` assembled on the device.  Explicit ``couplings`` /
    ``neighbors`` / ``fields`` / ``grain`` override the draws (``grain`` is the
    final block; for S > 1/2 or the sector see ``qsun_spin_grain``)."""
    if not float(2 * S).is_integer():
        raise ValueError(f"Wrong value of spin. Only integer spins or half-integer spins are possible. You chose S = {S}")
    if S != 0.5 or use_U1:
        if use_U1:
            _spin_sector(L_loc + L_grain, S, S_z)
        f, n, c, goe = qsun_spin_parameters(L_loc, L_grain, alpha, S, w=w, hz=hz, zeta=zeta, rng=rng)
        g = qsun_spin_grain(goe, L_loc, L_grain, S, gamma=gamma, use_U1=use_U1, S_z=S_z) if grain is None else grain
        return QSunSpinOperator(L_loc, L_grain, S, g0, c if couplings is None else couplings,
                                n if neighbors is None else neighbors, f if fields is None else fields, g,
                                use_U1=use_U1, S_z=S_z, device=device)
    f, n, c, g = qsun_parameters(L_loc, L_grain, alpha, gamma=gamma, w=w, hz=hz, zeta=zeta, rng=rng)
    return QSunOperator(L_loc, L_grain, g0, c if couplings is None else couplings,
                        n if neighbors is None else neighbors, f if fields is None else fields,
                        g if grain is None else grain, device=device)
