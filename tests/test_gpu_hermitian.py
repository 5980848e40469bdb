"""Complex Hermitian input on the B200 (the reference's CPU path takes it,
its GPU path refuses it: PolfedCore.jl:160-162).

The device holds the real embedding M = [[A, -B], [B, A]] of H = A + iB; the
solve runs the complex block Lanczos as the real block Lanczos from [v, i v]
and returns complex eigenvectors.  Checked against dense complex ``eigh``:
the eigenvalues nearest the target (1e-10), FP64 residuals ||H psi - E psi||
below the eigen tolerance, an orthonormal set, and whole eigenspaces of
degenerate eigenvalues.
"""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _hermitian(D, per_row, seed):
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(D), per_row)
    cols = rng.integers(0, D, size=D * per_row)
    vals = rng.standard_normal(D * per_row) + 1j * rng.standard_normal(D * per_row)
    A = sp.coo_matrix((vals, (rows, cols)), shape=(D, D)).tocsr()
    H = (A + A.conj().T) * 0.5 + sp.diags(rng.standard_normal(D))
    H.sum_duplicates()
    return H.tocsr()


def _check(H, vals, vecs, rep, nev, tol=1e-10):
    """nev eigenpairs of H: each value an eigenvalue of the dense spectrum
    (1e-10) inside the filter's window [left, right] (every pair POLFED keeps
    has a filter value above the cutoff there), FP64 residuals below tol, an
    orthonormal set, ascending."""
    ev = np.linalg.eigvalsh(H.toarray())
    a, b = rep.spectral.a, rep.spectral.b
    lo, hi = a * rep.spectral.left + b, a * rep.spectral.right + b
    assert len(vals) == nev
    assert np.all(np.diff(vals) >= 0)
    for v in vals:
        assert np.min(np.abs(ev - v)) < 1e-10 * max(1, abs(v))
        assert lo - 1e-9 <= v <= hi + 1e-9
    # as many copies of each eigenvalue as H has (a degenerate one counts its multiplicity)
    for v in np.unique(np.round(vals, 8)):
        assert np.sum(np.abs(vals - v) < 1e-8) <= np.sum(np.abs(ev - v) < 1e-8)
    for j in range(nev):
        v = vecs[:, j]
        assert abs(np.linalg.norm(v) - 1) < 1e-9
        assert np.linalg.norm(H @ v - vals[j] * v) < tol
    G = vecs.conj().T @ vecs
    np.testing.assert_allclose(G, np.eye(nev), atol=1e-8)


def test_embedding_apply(pkg, cuda):
    H = _hermitian(200, 6, 1)
    op = pkg.SparseOperator(H)
    assert op.is_complex and op.dim == 400
    rng = np.random.default_rng(2)
    Z = rng.standard_normal((200, 3)) + 1j * rng.standard_normal((200, 3))
    X = np.vstack([Z.real, Z.imag])
    Xd = cuda.tensor(np.ascontiguousarray(X.T), dtype=cuda.float64, device="cuda:0").t()
    Y = pkg.col_major(400, 3)
    pkg.apply(op, Y, Xd)
    got = Y.t().contiguous().cpu().numpy().T
    HZ = H @ Z
    ref = np.vstack([HZ.real, HZ.imag])
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12


@pytest.mark.parametrize("s", [1, 2])
def test_hermitian_solve_matches_dense(pkg, cuda, s):
    H = _hermitian(300, 5, 10 + s)
    rng = np.random.default_rng(3)
    x0 = rng.standard_normal((300, s)) + 1j * rng.standard_normal((300, s))
    x0 = x0[:, 0] if s == 1 else x0
    nev = 10
    vals, vecs, rep = pkg.polfed(H, x0, nev, ("rescaled", 0.4), produce_report=True,
                                 dos=pkg.DoSConfig(N=96, R=24, seed=4),
                                 fact=pkg.FactorizationConfig(eigentol=1e-10, overestimate_iters=2.0))
    _check(H, vals, vecs, rep, nev)
    assert rep.factorization.blocksize == s


def test_degenerate_spectrum_keeps_whole_eigenspaces(pkg, cuda):
    """H = I_2 (x) H0: every eigenvalue twice; the solve returns both
    orthonormal eigenvectors of each."""
    H0 = _hermitian(150, 5, 21)
    H = sp.kron(sp.identity(2), H0).tocsr()
    rng = np.random.default_rng(5)
    x0 = rng.standard_normal((300, 2)) + 1j * rng.standard_normal((300, 2))
    nev = 8
    vals, vecs, rep = pkg.polfed(H, x0, nev, ("rescaled", 0.3), produce_report=True,
                                 dos=pkg.DoSConfig(N=96, R=24, seed=6),
                                 fact=pkg.FactorizationConfig(eigentol=1e-10, overestimate_iters=2.0))
    _check(H, vals, vecs, rep, nev)
    # pairs of equal eigenvalues
    np.testing.assert_allclose(vals[0::2], vals[1::2], rtol=1e-10, atol=1e-10)


def test_real_matrix_as_complex_and_device_start(pkg, orc, cuda):
    """A real symmetric matrix given as complex returns the real path's
    eigenvalues (the same KPM probes, so the same plan); a complex128 CUDA
    start keeps the vectors on the device."""
    rng = np.random.default_rng(7)
    Hr = _hermitian(250, 5, 31).real.tocsr()
    Hr = ((Hr + Hr.T) * 0.5).tocsr()
    x0 = rng.standard_normal(250)
    probes = orc.normalized_gaussian_probes(250, 24, np.random.default_rng(9))
    dos = pkg.DoSConfig(N=96, R=24, probes=probes)
    vr, _, rr = pkg.polfed(Hr, x0, 6, ("rescaled", 0.5), produce_report=True, dos=dos,
                           fact=pkg.FactorizationConfig(eigentol=1e-10))
    Hc = Hr.astype(np.complex128)
    xd = cuda.tensor(x0.astype(np.complex128), device="cuda:0")
    vc, wc, rep = pkg.polfed(Hc, xd, 6, ("rescaled", 0.5), produce_report=True, dos=dos,
                             fact=pkg.FactorizationConfig(eigentol=1e-10))
    assert wc.is_cuda and wc.dtype == cuda.complex128
    assert rep.spectral.order == rr.spectral.order
    np.testing.assert_allclose(vc, vr, rtol=1e-10, atol=1e-10)
    _check(Hc, vc, wc.cpu().numpy(), rep, 6)


def test_real_solve_refuses_a_hermitian_operator(pkg, cuda):
    import ctypes
    from polfed_b200 import _lib
    op = pkg.SparseOperator(_hermitian(50, 3, 41))
    p = _lib.pf_params()
    _lib.load().pf_params_default(ctypes.byref(p))
    x = np.ones(100)
    vals = np.zeros(2)
    n = ctypes.c_int(0)
    st = _lib.load().pf_solve(op.op, ctypes.byref(p), 1, 2, x.ctypes.data, _lib.PF_MEM_HOST, vals.ctypes.data,
                              None, _lib.PF_MEM_HOST, None, ctypes.byref(n))
    assert st == _lib.PF_ERR_INVALID
    assert "pf_solve_hermitian" in _lib.load().pf_last_error().decode()
