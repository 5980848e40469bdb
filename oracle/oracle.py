"""CPU oracle for the POLFED filter-and-Lanczos path -- TEST INFRASTRUCTURE ONLY.

This module is the checker for the CUDA library.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm
may import it; the product never does.  It restates, in FP64 numpy plus the C
kernels of ``polfed_oracle.c``, the reference algorithm of Polfed.jl (Julia):

* models -- ``Models/SpinHalfChains.jl:227-315``, ``QSun/QuantumSun.jl:1-102``,
  ``QSun/QuantumSun_U1_conserving.jl:1-212``, ``QSun/SpinOperators.jl:5-69``,
  ``QSun/HilbertSpace.jl:9-41``
* rescaling -- ``Polfed/Plan/Plan.jl:128-191``
* target spec -- ``Polfed/Structs/TargetSpec.jl:26-58``, ``Plan.jl:203-281``
* DoS / KPM -- ``DensetiesOfStates/DensitiesOfStates.jl:14-43``,
  ``Moments.jl:42-140``, ``Kernels.jl:33-86``
* bounds / order -- ``SpectralTransformation/GetBounds.jl:1-118``,
  ``GetOrderOfExpansion.jl:1-70``, ``Bisection.jl:18-40``
* transform -- ``DefineTransformation.jl:11-48``, ``Clenshaw/*``
* Lanczos -- ``Lanczos/Lanczos.jl:119-143``, ``LanczosMethod.jl:55-117``,
  ``LanczosAlgorithm.jl:11-54``, ``Factorization/*``, ``Convergence/*``
* driver -- ``Polfed/PolfedCore.jl:43-263``, ``polfed_algorithm.jl:15-37``

Parity pins: the model matrices are checked against the reference's own
known-answer tests (``test/test_models.jl``), the spectral helpers against
``test/test_spectral_helpers.jl`` and the end-to-end driver against
``test/test_polfed.jl:29-61,166-176`` (see ``tests/test_oracle_golden.py``).
Julia's RNG streams cannot be reproduced, so random inputs are passed as
explicit arrays (fields, couplings, GOE block, KPM probes, x0).

Un-vendored dependencies restated here: QuadGK.jl 2.11 (``quadgk``: adaptive
Gauss-Kronrod 7/15, restated from the published rule) and Julia's
LinearAlgebra (``qr`` -> LAPACK Householder via numpy, ``eigen`` -> LAPACK
via numpy ``eigh``).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np
import scipy.sparse as sp

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    """Load (building if needed) the oracle's C kernels."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "_build", "liborc.so")
    if not os.path.exists(path):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    L = ctypes.CDLL(path)
    i64, i32, f64 = ctypes.c_int64, ctypes.c_int, ctypes.c_double
    vp = ctypes.c_void_p
    L.orc_sector_basis.restype = i64
    L.orc_sector_basis.argtypes = [i32, i32, vp]
    L.orc_sector_rank.restype = None
    L.orc_sector_rank.argtypes = [i64, vp, i64, vp, vp]
    L.orc_spin_chain_coo.restype = i64
    L.orc_spin_chain_coo.argtypes = [i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp]
    L.orc_qsun_coo.restype = i64
    L.orc_qsun_coo.argtypes = [i32, i32, f64, vp, vp, vp, vp, vp, vp, vp]
    L.orc_csr_apply.restype = None
    L.orc_csr_apply.argtypes = [i64, vp, vp, vp, i32, vp, i64, vp, i64]
    L.orc_csr_rescaled.restype = None
    L.orc_csr_rescaled.argtypes = [i64, vp, vp, vp, f64, f64, i32, vp, i64, vp, i64]
    L.orc_clenshaw_filter.restype = None
    L.orc_clenshaw_filter.argtypes = [i64, vp, vp, vp, f64, f64, i32, vp, i32, vp, vp, vp]
    L.orc_kpm_trace.restype = None
    L.orc_kpm_trace.argtypes = [i64, vp, vp, vp, f64, f64, i32, i32, vp, vp]
    L.orc_bucket_apply.restype = None
    L.orc_bucket_apply.argtypes = [i64, i32, vp, vp, vp, vp, vp, i32, vp, vp]
    L.orc_bucket_filter.restype = None
    L.orc_bucket_filter.argtypes = [i64, i32, vp, vp, vp, vp, vp, i32, vp, i32, vp, vp, vp]
    L.orc_bucket_kpm_trace.restype = None
    L.orc_bucket_kpm_trace.argtypes = [i64, i32, vp, vp, vp, vp, vp, i32, i32, vp, vp]
    L.orc_num_threads.restype = i32
    L.orc_set_num_threads.argtypes = [i32]
    _LIB = L
    return L


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


# ----------------------------------------------------------------- models

def chain_bonds(L: int, distance: int, boundary: str = "periodic"):
    """0-based bonds of ``_chain_bonds`` (SpinHalfChains.jl:227-243)."""
    if boundary not in ("periodic", "open"):
        raise ValueError(f"boundary must be one of (:periodic, :open); got {boundary}")
    if boundary == "open":
        if distance >= L:
            return []
        return [(i, i + distance) for i in range(L - distance)]
    bonds = []
    for i in range(1, L + 1):
        j = (i + distance - 1) % L + 1  # mod1
        if i == j:
            continue
        bonds.append((i - 1, j - 1))
    return bonds


def sector_basis(L: int, Lup: int) -> np.ndarray:
    n = lib().orc_sector_basis(L, Lup, None)
    out = np.empty(max(n, 1), dtype=np.uint64)
    lib().orc_sector_basis(L, Lup, _p(out))
    return out[:n]


def sector_rank(basis: np.ndarray, states: np.ndarray) -> np.ndarray:
    basis = np.ascontiguousarray(basis, dtype=np.uint64)
    states = np.ascontiguousarray(states, dtype=np.uint64)
    out = np.empty(len(states), dtype=np.int64)
    lib().orc_sector_rank(len(basis), _p(basis), len(states), _p(states), _p(out))
    return out


def _coo_to_csr(rows, cols, vals, D) -> sp.csr_matrix:
    # scipy sums duplicates like Julia's `sparse(I, J, V, m, n)`.
    M = sp.coo_matrix((vals, (rows, cols)), shape=(D, D)).tocsr()
    M.sum_duplicates()
    M.sort_indices()
    return M


def spin_chain_matrix(L, Lup, bonds, J, Delta, fields) -> sp.csr_matrix:
    """Sparse H of ``_spin_half_hamiltonian`` (SpinHalfChains.jl:267-315)."""
    nb = len(bonds)
    bi = np.array([b[0] for b in bonds] or [0], dtype=np.int32)
    bj = np.array([b[1] for b in bonds] or [0], dtype=np.int32)
    J = np.ascontiguousarray(np.broadcast_to(np.asarray(J, dtype=np.float64), (max(nb, 1),)))
    Dl = np.ascontiguousarray(np.broadcast_to(np.asarray(Delta, dtype=np.float64), (max(nb, 1),)))
    fields = np.ascontiguousarray(fields, dtype=np.float64)
    n = lib().orc_spin_chain_coo(L, Lup, nb, _p(bi), _p(bj), _p(J), _p(Dl), _p(fields),
                                 None, None, None)
    rows = np.empty(n, np.int64)
    cols = np.empty(n, np.int64)
    vals = np.empty(n, np.float64)
    lib().orc_spin_chain_coo(L, Lup, nb, _p(bi), _p(bj), _p(J), _p(Dl), _p(fields),
                             _p(rows), _p(cols), _p(vals))
    D = lib().orc_sector_basis(L, Lup, None)
    return _coo_to_csr(rows, cols, vals, D)


def xxz_matrix(L, Lup, J, Delta, fields, boundary="periodic"):
    """``xxz_hamiltonian`` with explicit fields (SpinHalfChains.jl:74-99)."""
    if L < 2:
        raise ValueError(f"L must be at least 2; got L={L}.")
    bonds = chain_bonds(L, 1, boundary)
    return spin_chain_matrix(L, Lup, bonds, [J] * len(bonds), [Delta] * len(bonds), fields)


def j1j2_matrix(L, Lup, J1, J2, D1, D2, fields, boundary="periodic"):
    """``j1j2_hamiltonian`` with explicit fields (SpinHalfChains.jl:189-220)."""
    if L < 2:
        raise ValueError(f"L must be at least 2; got L={L}.")
    nn = chain_bonds(L, 1, boundary)
    nnn = chain_bonds(L, 2, boundary)
    bonds = nn + nnn
    J = [J1] * len(nn) + [J2] * len(nnn)
    Dl = [D1] * len(nn) + [D2] * len(nnn)
    return spin_chain_matrix(L, Lup, bonds, J, Dl, fields)


def qsun_matrix(L_loc, L_grain, g0, coup, nbr, fields, Hg) -> sp.csr_matrix:
    """Sparse H of ``build_hamiltonian`` (QuantumSun.jl:1-102), S = 1/2."""
    coup = np.ascontiguousarray(coup, dtype=np.float64)
    nbr = np.ascontiguousarray(nbr, dtype=np.int32)
    fields = np.ascontiguousarray(fields, dtype=np.float64)
    Hg = np.ascontiguousarray(Hg, dtype=np.float64)
    n = lib().orc_qsun_coo(L_loc, L_grain, g0, _p(coup), _p(nbr), _p(fields), _p(Hg),
                           None, None, None)
    rows = np.empty(n, np.int64)
    cols = np.empty(n, np.int64)
    vals = np.empty(n, np.float64)
    lib().orc_qsun_coo(L_loc, L_grain, g0, _p(coup), _p(nbr), _p(fields), _p(Hg),
                       _p(rows), _p(cols), _p(vals))
    return _coo_to_csr(rows, cols, vals, 1 << (L_loc + L_grain))


# ------------------------------------------------ spin-S Quantum Sun family
class _SpinBasis:
    """``SpinBasis`` (SpinOperators.jl:5-21): d = 2S + 1 levels per site,
    ceil(log2 d) bits per site in a packed state code."""

    def __init__(self, S):
        self.S = float(S)
        self.d = int(round(2 * S)) + 1
        self.bits = int(math.ceil(math.log2(self.d)))
        self.mask = (1 << self.bits) - 1

    def get_spin(self, state, site):                     # SpinOperators.jl:23-27
        return float((state >> (site * self.bits)) & self.mask) - self.S

    def set_spin(self, state, site, m_new):              # SpinOperators.jl:29-34
        shift = site * self.bits
        state &= ~(self.mask << shift)
        return state | (int(round(m_new + self.S)) << shift)

    def sigma_z(self, state, site):                      # SpinOperators.jl:38-41
        return self.get_spin(state, site), state

    def _ladder(self, state, site, cu, cd):
        m = self.get_spin(state, site)
        S = self.S
        has_up, has_down = m < S, m > -S
        c_up = cu * math.sqrt(S * (S + 1) - m * (m + 1)) if has_up else 0.0
        c_down = cd * math.sqrt(S * (S + 1) - m * (m - 1)) if has_down else 0.0
        s_up = self.set_spin(state, site, m + 1) if has_up else 0
        s_down = self.set_spin(state, site, m - 1) if has_down else 0
        return has_up, c_up, s_up, has_down, c_down, s_down

    def sigma_x(self, state, site):                      # SpinOperators.jl:43-53
        return self._ladder(state, site, 0.5, 0.5)

    def sigma_y(self, state, site):                      # SpinOperators.jl:55-69
        return self._ladder(state, site, 1 / 2j, -(1 / 2j))


def _spin_states(L, B):
    """``build_hilbert`` (HilbertSpace.jl:9-32): every packed code, sorted."""
    states = [0]
    for site in range(L):
        shift = site * B.bits
        states = [st | (si << shift) for st in states for si in range(B.d)]
    return sorted(states)


def _qsun_spin_terms(states, index, L_loc, L_grain, g0, coup, nbr, fields, B, keep, use_y):
    """The fields and S^x S^x (and S^y S^y) entries in the reference's push
    order (QuantumSun.jl:35-95, QuantumSun_U1_conserving.jl:92-207); keep(i)
    says whether state index i belongs to the basis."""
    rows, cols, vals = [], [], []
    for k, state in enumerate(states):
        if not keep(k):
            continue
        for j in range(L_loc):
            val_z, _ = B.sigma_z(state, L_grain + j)
            rows.append(k), cols.append(k), vals.append(fields[j] * val_z)
        for j in range(L_loc):
            site_loc, site_grain = L_grain + j, int(nbr[j])
            for op in ((B.sigma_x, B.sigma_y) if use_y else (B.sigma_x,)):
                has1, c1, s1, has2, c2, s2 = op(state, site_loc)
                for has, c, s in ((has1, c1, s1), (has2, c2, s2)):
                    if not has:
                        continue
                    hg1, cg1, sg1, hg2, cg2, sg2 = op(s, site_grain)
                    for hg, cg, sg in ((hg1, cg1, sg1), (hg2, cg2, sg2)):
                        if not hg:
                            continue
                        new = index.get(sg, -1)
                        if new >= 0 and keep(new):
                            v = g0 * coup[j] * c * cg
                            rows.append(new), cols.append(k), vals.append(float(np.real(v)))
    return rows, cols, vals


def qsun_spin_matrix(L_loc, L_grain, g0, coup, nbr, fields, goe, S=0.5, gamma=1.0, use_U1=False,
                     S_z=0.0) -> sp.csr_matrix:
    """Sparse H of ``build_hamiltonian`` (QuantumSun.jl:1-102) for spin S, or of
    ``build_hamiltonian_cons`` (QuantumSun_U1_conserving.jl:1-212) for the
    total-S_z sector, from the raw GOE draw ``goe`` (the reference scales it
    per model).  Pure Python: small sizes only."""
    B = _SpinBasis(S)
    L = L_loc + L_grain
    if use_U1:
        sector_index = S_z + L * S
        if abs(S_z) > L * S or not float(sector_index).is_integer():
            raise ValueError(f"Wrong total value of spin to given spin-S particles. You chose S = {S} and S_z = {S_z}.")
    states = _spin_states(L, B)
    index = {st: i for i, st in enumerate(states)}
    dim = len(states)
    d = B.d
    dim_loc, dim_grain = d ** L_loc, d ** L_grain
    goe = np.asarray(goe, dtype=np.float64).reshape(dim_grain, dim_grain)
    coup = np.asarray(coup, dtype=np.float64)
    fields = np.asarray(fields, dtype=np.float64)
    if not use_U1:
        H_grain = gamma * goe / math.sqrt(dim_grain + 1)
        rows, cols, vals = _qsun_spin_terms(states, index, L_loc, L_grain, g0, coup, nbr, fields, B,
                                            lambda k: True, False)
        H = sp.coo_matrix((vals, (rows, cols)), shape=(dim, dim)).tocsr()
        return (H + sp.kron(sp.identity(dim_loc), sp.csr_matrix(H_grain))).tocsr()
    # QuantumSun_U1_conserving.jl:37-90: grain mask, sector rows, restricted and normalised R
    H_grain = goe.copy()
    gstates = states[:dim_grain]          # codes of the grain sites alone (the lowest codes)
    for II in range(dim_grain):
        for JJ in range(dim_grain):
            sI = sum(B.get_spin(gstates[II], j) for j in range(L_grain))
            sJ = sum(B.get_spin(gstates[JJ], j) for j in range(L_grain))
            if sJ != sI:
                H_grain[II, JJ] = 0.0
    mag = np.array([sum(B.sigma_z(st, j)[0] for j in range(L)) for st in states])
    rows_mag = np.full(dim, -1, dtype=np.int64)
    counter = 0
    for k in range(dim):
        if mag[k] == S_z:
            rows_mag[k] = counter
            counter += 1
    dim_red = counter
    R = sp.kron(sp.identity(dim_loc), sp.csr_matrix(H_grain)).tocoo()
    sel = (mag[R.row] == S_z) & (mag[R.col] == S_z)
    R_cons = sp.coo_matrix((R.data[sel], (rows_mag[R.row[sel]], rows_mag[R.col[sel]])),
                           shape=(dim_red, dim_red)).tocsr()
    R_cons = gamma * R_cons / math.sqrt((R_cons @ R_cons).diagonal().sum() / dim_red)
    rows, cols, vals = _qsun_spin_terms(states, index, L_loc, L_grain, g0, coup, nbr, fields, B,
                                        lambda k: mag[k] == S_z, True)
    H = sp.coo_matrix((vals, (rows_mag[rows], rows_mag[cols])), shape=(dim_red, dim_red)).tocsr()
    return (H + R_cons).tocsr()


class CSROperator:
    """FP64 CSR operator with the reference's apply / rescaled / Clenshaw /
    KPM-trace routines (C kernels of polfed_oracle.c)."""

    def __init__(self, M):
        M = sp.csr_matrix(M, dtype=np.float64)
        M.sort_indices()
        self.M = M
        self.D = M.shape[0]
        self.rowptr = np.ascontiguousarray(M.indptr, dtype=np.int64)
        self.colidx = np.ascontiguousarray(M.indices, dtype=np.int64)
        self.vals = np.ascontiguousarray(M.data, dtype=np.float64)

    def _cm(self, X):
        X = np.asarray(X, dtype=np.float64)
        return np.asfortranarray(X.reshape(self.D, -1))

    def apply(self, X):
        Xc = self._cm(X)
        s = Xc.shape[1]
        Y = np.zeros_like(Xc, order="F")
        lib().orc_csr_apply(self.D, _p(self.rowptr), _p(self.colidx), _p(self.vals), s,
                            _p(Xc), self.D, _p(Y), self.D)
        return Y.reshape(np.shape(X))

    def rescaled(self, X, a, b):
        Xc = self._cm(X)
        s = Xc.shape[1]
        Y = np.zeros_like(Xc, order="F")
        lib().orc_csr_rescaled(self.D, _p(self.rowptr), _p(self.colidx), _p(self.vals),
                               a, b, s, _p(Xc), self.D, _p(Y), self.D)
        return Y.reshape(np.shape(X))

    def filter(self, X, a, b, coeffs):
        Xc = self._cm(X)
        s = Xc.shape[1]
        coeffs = np.ascontiguousarray(coeffs, dtype=np.float64)
        K = len(coeffs) - 1
        Y = np.zeros_like(Xc, order="F")
        work = np.empty(3 * self.D * s, dtype=np.float64)
        lib().orc_clenshaw_filter(self.D, _p(self.rowptr), _p(self.colidx), _p(self.vals),
                                  a, b, K, _p(coeffs), s, _p(Xc), _p(Y), _p(work))
        return Y.reshape(np.shape(X))

    def kpm_trace(self, a, b, N, probes):
        P = np.asfortranarray(probes, dtype=np.float64).reshape(self.D, -1, order="F")
        R = P.shape[1]
        mu = np.zeros(N, dtype=np.float64)
        lib().orc_kpm_trace(self.D, _p(self.rowptr), _p(self.colidx), _p(self.vals),
                            a, b, N, R, _p(P), _p(mu))
        return mu


class BucketOperator:
    """The reference's CPU "optimized mapping" (the CPU baseline's operator):
    the diagonal and the off-diagonal entries grouped into buckets of equal
    value, both rounded to 15 digits (get_diags_and_offdiagonals_by_value,
    optimization.jl:134-182; entries below 1e-13 dropped), buckets in
    ascending value, each row's columns in ascending order (allocate / pack,
    optimization.jl:229-265).  Htilde uses the rescaled diagonal (d - b)/a and
    values v/a (optimize_spectral_transform, optimization.jl:101-104).  Same
    interface as CSROperator; the C kernels follow cpu/mapping.jl,
    cpu/clenshaw_recurrence_relation.jl, cpu/clenshaw_final_sum.jl and the
    threaded KPM of Moments.jl:87-109."""

    def __init__(self, M, tol=1e-13, digits=15):
        M = sp.csr_matrix(M, dtype=np.float64)
        M.sort_indices()
        self.D = M.shape[0]
        D = self.D
        self.diag = np.ascontiguousarray(np.round(M.diagonal(), digits))
        coo = M.tocoo()
        keep = (coo.row != coo.col) & (np.abs(coo.data) >= tol)
        rows, cols = coo.row[keep].astype(np.int64), coo.col[keep].astype(np.int64)
        keys = np.round(coo.data[keep], digits)
        vals, inv = np.unique(keys, return_inverse=True)
        self.bval = np.ascontiguousarray(vals)
        self.nb = len(vals)
        starts, flats, offs, off = [], [], [], 0
        for k in range(self.nb):
            sel = inv == k
            r, c = rows[sel], cols[sel]
            order = np.lexsort((c, r))
            r, c = r[order], c[order]
            starts.append(np.searchsorted(r, np.arange(D + 1)).astype(np.int64))
            flats.append(c)
            offs.append(off)
            off += len(c)
        self.bstart = np.ascontiguousarray(np.concatenate(starts) if starts else np.zeros(D + 1, np.int64))
        self.bflat = np.ascontiguousarray(np.concatenate(flats) if flats else np.zeros(1, np.int64))
        self.boff = np.ascontiguousarray(np.array(offs if offs else [0], dtype=np.int64))
        self._scaled = {}

    def _tables(self, a, b):
        key = (a, b)
        if key not in self._scaled:
            self._scaled = {key: (np.ascontiguousarray((self.diag - b) / a), np.ascontiguousarray(self.bval / a))}
        return self._scaled[key]

    def _cm(self, X):
        X = np.asarray(X, dtype=np.float64)
        return np.asfortranarray(X.reshape(self.D, -1))

    def _apply(self, X, a, b):
        Xc = self._cm(X)
        dg, bv = self._tables(a, b)
        Y = np.zeros_like(Xc, order="F")
        lib().orc_bucket_apply(self.D, self.nb, _p(dg), _p(bv), _p(self.bstart), _p(self.boff), _p(self.bflat),
                               Xc.shape[1], _p(Xc), _p(Y))
        return Y.reshape(np.shape(X))

    def apply(self, X):
        return self._apply(X, 1.0, 0.0)

    def rescaled(self, X, a, b):
        return self._apply(X, a, b)

    def filter(self, X, a, b, coeffs):
        Xc = self._cm(X)
        dg, bv = self._tables(a, b)
        coeffs = np.ascontiguousarray(coeffs, dtype=np.float64)
        Y = np.zeros_like(Xc, order="F")
        work = np.empty(3 * self.D, dtype=np.float64)
        lib().orc_bucket_filter(self.D, self.nb, _p(dg), _p(bv), _p(self.bstart), _p(self.boff), _p(self.bflat),
                                len(coeffs) - 1, _p(coeffs), Xc.shape[1], _p(Xc), _p(Y), _p(work))
        return Y.reshape(np.shape(X))

    def kpm_trace(self, a, b, N, probes):
        P = np.asfortranarray(probes, dtype=np.float64).reshape(self.D, -1, order="F")
        dg, bv = self._tables(a, b)
        mu = np.zeros(N, dtype=np.float64)
        lib().orc_bucket_kpm_trace(self.D, self.nb, _p(dg), _p(bv), _p(self.bstart), _p(self.boff),
                                   _p(self.bflat), N, P.shape[1], _p(P), _p(mu))
        return mu


# ------------------------------------------------------- spectral helpers

def Jackson(n, N):
    return ((N - n + 1) * math.cos(math.pi * n / (N + 1))
            + math.sin(math.pi * n / (N + 1)) / math.tan(math.pi / (N + 1))) / (N + 1)


def Lorentz(n, N, lam=1.0):
    return math.sinh(lam * (1 - n / N)) / math.sinh(lam)


def Fejer(n, N):
    return 1 - n / N


def LanczosK(n, N, M=3):
    if n == 0:
        return 1
    return (math.sin(math.pi * n / N) / (math.pi * n / N)) ** M


def WangZunger(n, N, alpha=1.0, beta=1.0):
    return math.exp(-((alpha * n / N) ** beta))


def Dirichlet(n, N):
    return 1


KERNELS = {"Jackson": Jackson, "Lorentz": Lorentz, "Fejer": Fejer, "LanczosK": LanczosK,
           "WangZunger": WangZunger, "Dirichlet": Dirichlet}


def get_kernel(name):
    """``get_kernel`` (Kernels.jl:82-86)."""
    if name not in KERNELS:
        raise ValueError(f"Unknown kernel: {name}. Available: {list(KERNELS)}")
    return KERNELS[name]


def coefficients(lam, n):
    """Default Chebyshev filter coefficients (PolfedDefaults.jl:104): c_0 = 1."""
    return (2 - (n == 0)) * math.cos(n * math.acos(lam))


def clenshaw_scalar(coef: Callable[[int], float], order: int, x):
    """Scalar Chebyshev Clenshaw (ClenshawAlgorithm.jl:35-54, FinalSum.jl:26-30),
    vectorised over an array of points ``x``."""
    x = np.asarray(x, dtype=np.float64)
    b2 = np.zeros_like(x)  # b[2]
    b3 = np.zeros_like(x)  # b[3]
    for k in range(order, 0, -1):
        b1 = coef(k) + 2.0 * x * b2 + (-1.0) * b3
        b3 = b2
        b2 = b1
    return coef(0) * 1.0 + 1.0 * x * b2 + (-1.0) * 1.0 * b3


def clenshaw_coeffs_scalar(c: np.ndarray, x):
    return clenshaw_scalar(lambda k: c[k], len(c) - 1, x)


def bisection(f, x1, x2, tol=1e-8, max_iter=500):
    """Bisection.jl:18-40."""
    if f(x1) * f(x2) > 0:
        raise RuntimeError("The function must have opposite signs at a and b")
    it = 0
    while (x2 - x1) / 2 >= tol and it < max_iter:
        x = (x1 + x2) / 2
        fc = f(x)
        if fc == 0 or (x2 - x1) / 2 <= tol:
            return x
        elif f(x1) * fc < 0:
            x2 = x
        else:
            x1 = x
        it += 1
    return (x1 + x2) / 2


# Gauss-Kronrod 7/15 nodes and weights (the published QUADPACK qk15 rule).
_XGK = np.array([0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
                 0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
                 0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
                 0.207784955007898467600689403773245, 0.0])
_WGK = np.array([0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
                 0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
                 0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
                 0.204432940075298892414161999234649, 0.209482141084727828012999174891714])
_WG = np.array([0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
                0.381830050505118944950369775488975, 0.417959183673469387755102040816327])


def _gk_rule(f, a, b):
    c = 0.5 * (a + b)
    h = 0.5 * (b - a)
    xs = np.concatenate([c - h * _XGK[:7], [c], c + h * _XGK[:7][::-1]])
    fx = np.asarray(f(xs), dtype=np.float64)
    fl = fx[:7]
    fc = fx[7]
    fr = fx[8:][::-1]
    Ik = _WGK[7] * fc + np.sum(_WGK[:7] * (fl + fr))
    Ig = _WG[3] * fc + np.sum(_WG[:3] * (fl[1::2] + fr[1::2]))
    Ik *= h
    Ig *= h
    return Ik, abs(Ik - Ig)


def quadgk(f, a, b, atol=1e-12, rtol=1e-12, maxevals=10 ** 7):
    """Adaptive Gauss-Kronrod (7,15) quadrature in the manner of QuadGK.jl 2.x:
    start from [a, b]; while the summed error exceeds max(atol, rtol |I|),
    bisect the segment with the largest error estimate."""
    import heapq
    if a == b:
        return 0.0, 0.0
    I, E = _gk_rule(f, a, b)
    segs = [(-E, a, b, I, E)]
    nev = 15
    while E > max(atol, rtol * abs(I)) and nev < maxevals:
        _, sa, sb, sI, sE = heapq.heappop(segs)
        mid = 0.5 * (sa + sb)
        if not (sa < mid < sb):
            heapq.heappush(segs, (-sE, sa, sb, sI, sE))
            break
        I1, E1 = _gk_rule(f, sa, mid)
        I2, E2 = _gk_rule(f, mid, sb)
        nev += 30
        I = (I - sI) + I1 + I2
        E = (E - sE) + E1 + E2
        heapq.heappush(segs, (-E1, sa, mid, I1, E1))
        heapq.heappush(segs, (-E2, mid, sb, I2, E2))
    I = sum(s[3] for s in segs)
    E = sum(s[4] for s in segs)
    return I, E


def analytical_orderofexpansion(lam, delta):
    """GetOrderOfExpansion.jl:8-10."""
    return 2.65499 * math.sqrt(1 - lam ** 2) / delta


_BOUNDS = {
    "mean": (lambda t, d: t - d, lambda t, d: t + d),
    "left": (lambda t, d: t, lambda t, d: t + 2 * d),
    "right": (lambda t, d: t - 2 * d, lambda t, d: t),
}


@dataclass
class TransformPlan:
    """TransformPlan of Plan.jl:32-44 (rescaled units)."""
    target_spec: tuple
    howmany: int
    target: Optional[float] = None
    left: Optional[float] = None
    right: Optional[float] = None
    order: Optional[int] = None
    cutoff: float = 0.17
    normalization: float = 1.0
    order_safety_factor: float = 0.97
    coefficients: Callable = coefficients


def normalize_target_spec(target):
    """TargetSpec.jl:26-58, returning a (kind, value) tuple."""
    if isinstance(target, str):
        if target == "maxdos":
            return ("maxdos", None)
        if target == "middle":
            return ("middle", None)
        raise ValueError(f"Unknown target symbol: {target}")
    if isinstance(target, tuple) and len(target) == 2 and isinstance(target[0], str):
        tag, val = target
        if isinstance(val, bool) or not isinstance(val, (int, float, np.floating, np.integer)):
            raise ValueError(f"Target tuple value must be Real, got {type(val)}")
        if tag == "absolute":
            raise ValueError("`(:absolute, value)` is no longer supported. Use `(:unrescaled, value)` instead.")
        if tag == "quantile":
            raise ValueError("`(:quantile, q)` is no longer supported.")
        if tag == "offset":
            if not (-1 <= val <= 1):
                raise ValueError(f"Offset target requires `eta in [-1, 1]`, got {val}")
            return ("offset", float(val))
        if tag == "unrescaled":
            return ("unrescaled", float(val))
        if tag == "rescaled":
            return ("rescaled", float(val))
        raise ValueError(f"Unknown target tuple tag: {tag}")
    if isinstance(target, (int, float, np.floating, np.integer)) and not isinstance(target, bool):
        return ("unrescaled", float(target))
    raise ValueError(f"Unsupported target specification: {target}")


def findmaximaldensity(rho):
    """Plan.jl:243-249."""
    x = np.linspace(-0.99, 0.99, 5000)
    vals = rho(x)
    return float(x[int(np.argmax(vals))])


def resolve_target(plan: TransformPlan, a, b, rho):
    """Plan.jl:260-281."""
    if plan.target is not None:
        return
    kind, val = plan.target_spec
    if kind == "maxdos":
        plan.target = findmaximaldensity(rho)
    elif kind == "offset":
        peak = findmaximaldensity(rho)
        plan.target = peak + val * (1.0 - peak) if val >= 0 else peak + val * (1.0 + peak)
    elif kind == "middle":
        plan.target = 0.0
    elif kind == "rescaled":
        plan.target = val
    elif kind == "unrescaled":
        plan.target = (val - b) / a
    else:
        raise ValueError(f"Unsupported target specification: {plan.target_spec}")


def build_transform_plan(target, howmany, a, b, left=None, right=None, order=None,
                         cutoff=0.17, normalization=1.0, osf=0.97):
    """Plan.jl:203-236."""
    spec = normalize_target_spec(target)
    plan = TransformPlan(spec, howmany, cutoff=cutoff, normalization=normalization,
                         order_safety_factor=osf, order=order)
    plan.left = None if left is None else (left - b) / a
    plan.right = None if right is None else (right - b) / a
    kind, val = spec
    if kind == "unrescaled":
        plan.target = (val - b) / a
    elif kind == "rescaled":
        plan.target = val
    elif kind == "middle":
        plan.target = 0.0
    return plan


def _filter_poly(plan, order, target):
    c = np.array([plan.coefficients(target, n) for n in range(order + 1)])
    norm_ = clenshaw_coeffs_scalar(c, target)
    return lambda x: clenshaw_coeffs_scalar(c, x) / norm_ * plan.normalization


def getbounds_from_dos(plan: TransformPlan, rho, position="mean"):
    """GetBounds.jl:57-81."""
    ahat, bhat = _BOUNDS[position]
    t = plan.target

    def fun(d):
        lo = max(ahat(t, d), -1.0)
        hi = min(bhat(t, d), 1.0)
        howmany_dos, _ = quadgk(rho, lo, hi, atol=1e-12, rtol=1e-12)
        return -1 if howmany_dos >= plan.howmany else +1

    d = bisection(fun, 0.0, 1.0, tol=1e-8)
    plan.left = max(ahat(t, d), -1.0)
    plan.right = min(bhat(t, d), 1.0)


def getbounds_from_K(plan: TransformPlan, position="mean"):
    """GetBounds.jl:90-118."""
    ahat, bhat = _BOUNDS[position]
    t = plan.target
    p = _filter_poly(plan, plan.order, t)

    def fun(d):
        lo = max(ahat(t, d), -1.0)
        hi = min(bhat(t, d), 1.0)
        m = max(float(p(lo)), float(p(hi)))
        return -1 if m >= plan.cutoff else +1

    d = bisection(fun, 0.0, 1.0, tol=1e-8)
    plan.left = max(ahat(t, d), -1.0)
    plan.right = min(bhat(t, d), 1.0)


def getorderofexpansion_in_interval(plan: TransformPlan):
    """GetOrderOfExpansion.jl:36-70."""
    target = (plan.left + plan.right) / 2
    halfwidth = (plan.right - plan.left) / 2

    def fun(order):
        order = int(math.floor(order))
        p = _filter_poly(plan, order, target)
        m = max(float(p(plan.left)), float(p(plan.right)))
        return -1 if m >= plan.cutoff else +1

    Kmax = math.ceil(analytical_orderofexpansion(target, halfwidth) * 2)
    K = bisection(fun, 10, Kmax, tol=1)
    plan.order = int(math.floor(K * plan.order_safety_factor))
    if plan.order_safety_factor < 1.0:
        getbounds_from_K(plan, "mean")


def getbounds(plan: TransformPlan, a, b, rho, position="mean"):
    """GetBounds.jl:19-48."""
    bounds_set = plan.left is not None and plan.right is not None
    order_set = plan.order is not None
    if plan.target is None:
        resolve_target(plan, a, b, rho)
    if bounds_set and order_set:
        raise RuntimeError("Both interval bounds and polynomial order are specified. "
                           "Please set only one or neither.")
    elif bounds_set:
        pass
    elif order_set:
        getbounds_from_K(plan, position)
    else:
        getbounds_from_dos(plan, rho, position)


def getorderofexpansion(plan: TransformPlan):
    if plan.order is None:
        getorderofexpansion_in_interval(plan)


def filter_coefficients(plan: TransformPlan):
    """Normalised coefficients of definetransformation! (DefineTransformation.jl:18-30)."""
    K = plan.order
    c = np.array([plan.coefficients(plan.target, n) for n in range(K + 1)])
    norm_ = 1.0 / clenshaw_coeffs_scalar(c, plan.target) * plan.normalization
    return c * norm_


def normalized_gaussian_probes(D, R, rng):
    """randn probes normalised per column (Moments.jl:101-102)."""
    P = rng.standard_normal((D, R))
    P /= np.linalg.norm(P, axis=0, keepdims=True)
    return np.asfortranarray(P)


def dos_moments(op, a, b, N, probes):
    """dos_moments (Moments.jl:42-109): mu *= D/R."""
    R = probes.shape[1]
    mu = op.kpm_trace(a, b, N, probes)
    return mu * (op.D / R)


def make_rho(mu, N, kernel="Jackson"):
    """getdos! (DensitiesOfStates.jl:27-34)."""
    kf = get_kernel(kernel)
    coeffs = np.array([kf(i, N) * mu[i] * (2 - (i == 0)) for i in range(N)])

    # The quadrature of getbounds_from_dos integrates up to x = +-1 exactly,
    # where 1/sqrt(1 - x^2) is infinite; nodes that round onto +-1 are moved
    # to the nearest double inside (-1, 1), as the library's rho does, so the
    # integrand stays finite.
    xm = np.nextafter(1.0, 0.0)

    def rho(x):
        x = np.clip(np.asarray(x, dtype=np.float64), -xm, xm)
        return clenshaw_coeffs_scalar(coeffs, x) / (np.pi * np.sqrt(1 - x ** 2))
    return rho


def expectedkrylovdim(howmany, blocksize, eta):
    """PolfedDefaults.jl:61-62."""
    return int(math.ceil((20.427 * blocksize + 1.696 * howmany) * eta))


# ------------------------------------------------------------------ Lanczos

@dataclass
class LanczosInfo:
    converged: int = 0
    eigenconverged: int = 0
    residual: float = 1.0
    eigenresidual: float = 1.0
    numiter: int = 0
    maxiter: int = 0
    numofchecks: int = 0
    converged_history: list = field(default_factory=list)
    krylovdim_history: list = field(default_factory=list)
    maxresidual_history: list = field(default_factory=list)
    krylovdim: int = 0


def _sortvals(lam, which):
    """EigSorter.jl:41-57 (stable sort like Julia's sortperm)."""
    if which == "SR":
        return np.argsort(lam, kind="stable")
    if which == "LR":
        return np.argsort(-lam, kind="stable")
    if which == "LM":
        return np.argsort(-np.abs(lam), kind="stable")
    if which == "SM":
        return np.argsort(np.abs(lam), kind="stable")
    raise ValueError(f"Unknown sorting mode: {which}")


def lanczos(f, x0, howmany, which="SR", maxdim=None, tol=1e-14, eigentol=1e-8, mapvals=None,
            reorth_passes=1):
    """Scalar (x0 1-D) or block (x0 2-D) Lanczos with FullRO, as in
    Lanczos.jl:119-143 / LanczosMethod.jl:55-83 / LanczosAlgorithm.jl:11-54.

    Returns (vals ascending, vecs, info)."""
    mapvals = f if mapvals is None else mapvals
    block = np.ndim(x0) == 2
    X0 = np.asarray(x0, dtype=np.float64).reshape(len(x0), -1)
    D, s = X0.shape
    if maxdim is None:
        maxdim = 500 * howmany
    maxiter = int(math.ceil(maxdim / s))
    maxdim = maxiter * s
    info = LanczosInfo(maxiter=maxiter)
    nextcheck = max(howmany // s + 1, 2)

    basis = np.zeros((D, maxdim), dtype=np.float64, order="F")
    T = np.zeros((maxdim, maxdim), dtype=np.float64)
    alphas = np.zeros(maxdim)
    betas = np.zeros(maxdim)
    vals = np.zeros(howmany)
    vecs = np.zeros((D, howmany), order="F")

    def fmap(V):
        Y = f(V if block else V[:, 0])
        return np.asarray(Y, dtype=np.float64).reshape(D, -1)

    # lanczositer (Factorization.jl:50-67)
    k = 0
    basis[:, 0:s] = X0
    k = s
    v_last = X0.copy()
    v_prev = np.zeros_like(X0)
    r = fmap(v_last)
    if block:
        A = v_last.T @ r
        A = np.triu(A) + np.triu(A, 1).T  # Hermitian(alpha_k): upper triangle
        T[k - s:k, k - s:k] = A
        r = r - X0 @ A
    else:
        alphas[0] = float(v_last[:, 0] @ r[:, 0])
        r = r - X0 * alphas[0]
    info.numiter = 1

    while True:
        # 1 tridiagonalization (BlockLanczosFactorization.jl:115-131 / LanczosFactorization.jl:61-67)
        if block:
            Q, Rm = np.linalg.qr(r, mode="reduced")
            T[k:k + s, k - s:k] = Rm
            T[k - s:k, k:k + s] = Rm.T
            beta_last = Rm
            newv = Q
        else:
            beta = float(np.linalg.norm(r))
            newv = r / beta
            betas[k - 1] = beta
            beta_last = beta
        basis[:, k:k + s] = newv
        v_prev = v_last
        v_last = newv.copy()
        k += s
        # 2 mapping
        r = fmap(v_last)
        # 3 overlap, 4 orthogonalization
        if block:
            A = v_last.T @ r
            A = np.triu(A) + np.triu(A, 1).T
            T[k - s:k, k - s:k] = A
            r = r - (v_last @ A + v_prev @ beta_last.T)
        else:
            alphas[k - 1] = float(v_last[:, 0] @ r[:, 0])
            r = r - (alphas[k - 1] * v_last + beta_last * v_prev)
        # 5 reorthogonalization (FullRO: all but the last two blocks)
        nB = k - 2 * s
        if nB > 0:
            B = basis[:, :nB]
            for _ in range(reorth_passes):
                r = r - B @ (B.T @ r)

        # convergence (ConvergenceInfo.jl:63-130)
        info.numiter += 1
        if nextcheck == info.numiter or info.numiter >= maxiter:
            if block:
                Tm = T[:k, :k]
                Tm = np.triu(Tm) + np.triu(Tm, 1).T
            else:
                Tm = np.diag(alphas[:k]) + np.diag(betas[:k - 1], 1) + np.diag(betas[:k - 1], -1)
            lam, phi = np.linalg.eigh(Tm)
            idxs = _sortvals(lam, which)
            conv = 0
            maxres = 0.0
            for i in range(howmany):
                pos = idxs[i]
                if block:
                    res = float(np.linalg.norm(beta_last @ phi[k - s:k, pos]))
                else:
                    res = abs(beta_last * phi[k - 1, pos])
                if res > maxres:
                    maxres = res
                if maxres < tol:
                    conv += 1
            info.numofchecks += 1
            info.converged = conv
            info.residual = maxres
            info.converged_history.append(conv)
            info.krylovdim_history.append(k)
            info.maxresidual_history.append(maxres)
            if conv == howmany or info.numiter >= maxiter:
                sel = idxs[:conv]
                vecs[:, :conv] = basis[:, :k] @ phi[:, sel]
                for i in range(conv):
                    v = vecs[:, i]
                    Hv = np.asarray(mapvals(v), dtype=np.float64).reshape(D)
                    vals[i] = float(v @ Hv)
                ec = 0
                do_count = True
                maxe = 0.0
                for i in range(conv):
                    v = vecs[:, i]
                    rr = np.asarray(mapvals(v), dtype=np.float64).reshape(D) - vals[i] * v
                    res = float(np.linalg.norm(rr))
                    if do_count and res < eigentol:
                        ec += 1
                    else:
                        do_count = False
                    maxe = max(maxe, res)
                info.eigenconverged = ec
                info.eigenresidual = maxe
            # next_checking! (NextChecking.jl:23-42)
            if info.residual > 1e-2:
                nextcheck = info.numiter + 20
            elif info.residual > 1e-3:
                nextcheck = info.numiter + 10
            else:
                nextcheck = info.numiter + 5
        if info.converged == howmany or info.numiter >= maxiter:
            break

    info.krylovdim = k
    conv = min(info.converged, info.eigenconverged)
    order = np.argsort(vals[:conv], kind="stable")
    return vals[:conv][order].copy(), vecs[:, :conv][:, order].copy(), info


def lanczos_extrema(apply, x0, maxdim=1000, tol=1e-14, eigentol=1e-8):
    """lanczos_extrema (Lanczos.jl:183-212) for an operator callback."""
    x0 = np.asarray(x0, dtype=np.float64)
    n = np.linalg.norm(x0)
    if n == 0:
        raise ValueError("lanczos_extrema requires a nonzero starting vector.")
    seed = x0 / n
    lo = lanczos(apply, seed, 1, which="SR", maxdim=maxdim, tol=tol, eigentol=eigentol)[0]
    hi = lanczos(apply, seed, 1, which="LR", maxdim=maxdim, tol=tol, eigentol=eigentol)[0]
    if len(lo) == 0 or len(hi) == 0:
        raise RuntimeError("Failed to estimate extremal eigenvalue with Lanczos.")
    return float(lo[0]), float(hi[-1])


def prepare_initial_state(x0):
    """_prepare_polfed_initial_state (PolfedCore.jl:43-95)."""
    x0 = np.asarray(x0, dtype=np.float64)
    tol = max(1e-10, 10 * np.finfo(np.float64).eps)
    if x0.ndim == 1:
        if x0.size == 0:
            raise ValueError("POLFED initial vector must not be empty.")
        nrm = np.linalg.norm(x0)
        if not np.isfinite(nrm):
            raise ValueError("POLFED initial vector must contain finite values.")
        if nrm == 0:
            raise ValueError("POLFED initial vector must be nonzero.")
        if abs(nrm - 1.0) <= max(tol, tol * max(abs(nrm), 1.0)):
            return x0
        return x0 / nrm
    D, s = x0.shape
    if D == 0:
        raise ValueError("POLFED initial matrix must have at least one row.")
    if s == 0:
        raise ValueError("POLFED initial matrix must have at least one column.")
    if s > D:
        raise ValueError("POLFED initial matrix cannot have orthonormal columns when it has more columns than rows.")
    G = x0.T @ x0
    if not np.all(np.isfinite(G)):
        raise ValueError("POLFED initial matrix must contain finite values.")
    I = np.eye(s)
    if np.linalg.norm(G - I) <= max(tol, tol * max(np.linalg.norm(G), np.linalg.norm(I))):
        return x0
    Q, _ = np.linalg.qr(x0, mode="reduced")
    return Q


@dataclass
class PolfedResult:
    vals: np.ndarray
    vecs: np.ndarray
    Emin: float
    Emax: float
    a: float
    b: float
    target: float
    left: float
    right: float
    order: int
    coeffs: np.ndarray
    mu: np.ndarray
    info: LanczosInfo
    matvecs: int


def plan_only(op, x0, howmany, target, *, Emin=None, Emax=None, order=None, left=None, right=None,
              cutoff=0.17, normalization=1.0, order_safety_factor=0.97, N=250, kernel="Jackson",
              probes=None):
    """The planning stage of ``polfed`` alone (PolfedCore.jl:194-263 up to
    definetransformation!): Emin / Emax probes, KPM DoS, interval and order.
    Returns a PolfedResult without eigenpairs (vals, vecs, info empty)."""
    x0 = prepare_initial_state(x0)
    v0 = x0 if x0.ndim == 1 else x0[:, 0]
    if Emin is None:
        Emin = float(lanczos(op.apply, v0, 1, which="SR", maxdim=1000)[0][0])
    if Emax is None:
        Emax = float(lanczos(op.apply, v0, 1, which="LR", maxdim=1000)[0][-1])
    a = (Emax - Emin) / 2
    b = (Emax + Emin) / 2
    plan = build_transform_plan(target, howmany, a, b, left=left, right=right, order=order,
                                cutoff=cutoff, normalization=normalization, osf=order_safety_factor)
    mu = dos_moments(op, a, b, N, probes)
    rho = make_rho(mu, N, kernel)
    getbounds(plan, a, b, rho, "mean")
    getorderofexpansion(plan)
    coeffs = filter_coefficients(plan)
    return PolfedResult(np.zeros(0), np.zeros((op.D, 0)), Emin, Emax, a, b, plan.target, plan.left,
                        plan.right, plan.order, coeffs, mu, LanczosInfo(), 0)


def polfed(op, x0, howmany, target, *, Emin=None, Emax=None, order=None, left=None,
           right=None, cutoff=0.17, normalization=1.0, order_safety_factor=0.97,
           N=250, R=300, kernel="Jackson", probes=None, probe_rng=None, tol=1e-14,
           eigentol=1e-9, which="LR", overestimate_iters=1.25, reorth_passes=1):
    """The POLFED driver (PolfedCore.jl:194-263, polfed_algorithm.jl:15-37)
    on an oracle operator (``op.apply``, ``op.rescaled``, ``op.filter``,
    ``op.kpm_trace``).  ``probes`` (D x R, normalised columns) replaces the
    reference's unseeded randn probes."""
    x0 = prepare_initial_state(x0)
    v0 = x0 if x0.ndim == 1 else x0[:, 0]
    if Emin is None:
        Emin = float(lanczos(op.apply, v0, 1, which="SR", maxdim=1000)[0][0])
    if Emax is None:
        Emax = float(lanczos(op.apply, v0, 1, which="LR", maxdim=1000)[0][-1])
    a = (Emax - Emin) / 2
    b = (Emax + Emin) / 2
    plan = build_transform_plan(target, howmany, a, b, left=left, right=right, order=order,
                                cutoff=cutoff, normalization=normalization, osf=order_safety_factor)
    s = 1 if x0.ndim == 1 else x0.shape[1]
    maxdim = expectedkrylovdim(howmany, s, overestimate_iters)
    if probes is None:
        rng = probe_rng if probe_rng is not None else np.random.default_rng()
        probes = normalized_gaussian_probes(op.D, R, rng)
    mu = dos_moments(op, a, b, N, probes)
    rho = make_rho(mu, N, kernel)
    getbounds(plan, a, b, rho, "mean")
    getorderofexpansion(plan)
    coeffs = filter_coefficients(plan)

    def ftrans(V):
        return op.filter(V, a, b, coeffs)

    vals, vecs, info = lanczos(ftrans, x0, howmany, which=which, maxdim=maxdim, tol=tol,
                               eigentol=eigentol, mapvals=op.apply, reorth_passes=reorth_passes)
    matvecs = plan.order * s * info.numiter + howmany
    return PolfedResult(vals, vecs, Emin, Emax, a, b, plan.target, plan.left, plan.right,
                        plan.order, coeffs, mu, info, matvecs)
