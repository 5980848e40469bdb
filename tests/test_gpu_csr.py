"""User matrices: ``polfed(mat, ...)`` (PolfedCore.jl:153-184) through the CSR
operator (pf_op_csr_create).

The CSR step must give the matrix-free operators' results when fed the same
Hamiltonian (the oracle's CSR of a spin chain and of a Quantum Sun), agree
with scipy on a random sparse symmetric matrix (FP64 to 1e-12, FP32 to 2e-5
relative), drive the filter and KPM, and solve to the oracle's eigenvalues
(1e-10 relative) with FP64 residuals below the eigen tolerance.
"""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

RTOL64, RTOL32 = 1e-12, 2e-5


def _dev(cuda, A, dtype):
    A = np.asarray(A).reshape(A.shape[0], -1)
    return cuda.tensor(np.ascontiguousarray(A.T), dtype=dtype, device="cuda:0").t()


def _host(t):
    return t.t().contiguous().cpu().numpy().T


def _random_symmetric(D, per_row, seed):
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(D), per_row)
    cols = rng.integers(0, D, size=D * per_row)
    vals = rng.standard_normal(D * per_row)
    A = sp.coo_matrix((vals, (rows, cols)), shape=(D, D)).tocsr()
    A = (A + A.T) * 0.5 + sp.diags(rng.standard_normal(D))
    A.sum_duplicates()
    return A.tocsr()


def test_csr_matches_matrix_free_operators(pkg, orc, cuda):
    rng = np.random.default_rng(8)
    f = 5 * (2 * rng.random(12) - 1)
    chain = pkg.xxz_hamiltonian(12, 6, 1.0, 1.0, 0.0, fields=f)
    Hc = orc.xxz_matrix(12, 6, 1.0, 1.0, f)
    fq, nq, cq, gq = pkg.qsun_parameters(7, 3, 0.75, rng=rng)
    qsun = pkg.QSunOperator(7, 3, 1.0, cq, nq, fq, gq)
    Hq = orc.qsun_matrix(7, 3, 1.0, cq, nq, fq, gq)
    for mf, H in ((chain, Hc), (qsun, Hq)):
        csr = pkg.SparseOperator(H)
        D = H.shape[0]
        assert csr.dim == D
        for s in (1, 8):
            X = rng.standard_normal((D, s))
            Y1, Y2 = pkg.col_major(D, s), pkg.col_major(D, s)
            pkg.apply(mf, Y1, _dev(cuda, X, cuda.float64), a=2.5, b=-0.3)
            pkg.apply(csr, Y2, _dev(cuda, X, cuda.float64), a=2.5, b=-0.3)
            a, b = _host(Y1), _host(Y2)
            assert np.linalg.norm(a - b) / np.linalg.norm(a) < RTOL64
        # filter and KPM through the CSR step
        Emax = float(np.abs(H).sum(axis=1).max()) * 1.01
        plan = orc.build_transform_plan(("rescaled", 0.31), 10, 1.0, 0.0, order=40)
        coeffs = orc.filter_coefficients(plan)[:41]
        X = rng.standard_normal((D, 8))
        Y = pkg.col_major(D, 8)
        pkg.chebyshev_filter(csr, Y, _dev(cuda, X, cuda.float64), coeffs, a=Emax, b=0.0)
        ref = orc.CSROperator(H).filter(X, Emax, 0.0, coeffs)
        assert np.linalg.norm(_host(Y) - ref) / np.linalg.norm(ref) < 10 * RTOL64
        probes = orc.normalized_gaussian_probes(D, 16, np.random.default_rng(2))
        mu = pkg.kpm_moments(csr, 32, 16, a=Emax, b=0.0, probes=_dev(cuda, probes, cuda.float64))
        mu_ref = orc.dos_moments(orc.CSROperator(H), Emax, 0.0, 32, probes)
        assert np.max(np.abs(mu - mu_ref)) < 1e-10 * D


@pytest.mark.parametrize("dtype", ["fp64", "fp32"])
def test_csr_apply_random_matrix(pkg, cuda, dtype):
    A = _random_symmetric(3000, 9, 11)
    op = pkg.SparseOperator(A)
    D = A.shape[0]
    dt, tol = (cuda.float64, RTOL64) if dtype == "fp64" else (cuda.float32, RTOL32)
    for s in (1, 4, 16):
        X = np.random.default_rng(s).standard_normal((D, s))
        Xr = X if dtype == "fp64" else X.astype(np.float32).astype(np.float64)
        Y = pkg.col_major(D, s, dtype=dt)
        pkg.apply(op, Y, _dev(cuda, X, dt))
        ref = A @ Xr
        assert np.linalg.norm(_host(Y).astype(np.float64) - ref) / np.linalg.norm(ref) < tol, (s, dtype)


def test_polfed_on_a_matrix_matches_oracle(pkg, orc, cuda):
    A = _random_symmetric(2000, 6, 5)
    D = A.shape[0]
    x0 = np.random.default_rng(3).random((D, 4))
    probes = orc.normalized_gaussian_probes(D, 24, np.random.default_rng(4))
    ref = orc.polfed(orc.CSROperator(A), x0, 12, ("rescaled", 0.2), N=96, R=24, probes=probes,
                     overestimate_iters=2.0)
    for mat in (A, A.toarray()):                       # sparse and dense input
        vals, vecs = pkg.polfed(mat, x0, 12, ("rescaled", 0.2),
                                fact=pkg.FactorizationConfig(overestimate_iters=2.0),
                                dos=pkg.DoSConfig(N=96, R=24, probes=probes))
        assert len(vals) == len(ref.vals) and len(vals) >= 1
        assert np.max(np.abs(vals - ref.vals) / np.maximum(1, np.abs(ref.vals))) < 1e-10
        for j in range(len(vals)):
            v = vecs[:, j]
            assert np.linalg.norm(A @ v - vals[j] * v) < 1e-9


def test_served_request_outlives_its_matrix_operator(pkg, cuda):
    A = _random_symmetric(1500, 6, 9)
    x0 = np.random.default_rng(1).random(A.shape[0])
    with pkg.SolverPool(workers=2) as pool:
        alone, _ = pkg.polfed(A, x0, 8, ("rescaled", 0.3), dos=pkg.DoSConfig(N=64, R=16, seed=3))
        rid = pool.submit(A, x0, 8, ("rescaled", 0.3), dos=pkg.DoSConfig(N=64, R=16, seed=3))
        vals, vecs = pool.result(rid)
    assert np.max(np.abs(vals - alone) / np.maximum(1, np.abs(alone))) < 1e-10


def test_csr_rejects_bad_input(pkg, cuda):
    from polfed_b200 import _lib
    with pytest.raises(ValueError):                     # indptr ends at 1, three entries
        pkg.SparseOperator((np.array([0, 2, 1]), np.array([0, 1, 0]), np.array([1.0, 2.0, 3.0])))
    decreasing = pkg.SparseOperator((np.array([0, 2, 1, 3]), np.array([0, 1, 2]), np.array([1.0, 2.0, 3.0])))
    with pytest.raises(_lib.PolfedArgumentError, match="non-decreasing"):
        decreasing.op
    out_of_range = pkg.SparseOperator((np.array([0, 1, 2]), np.array([0, 5]), np.array([1.0, 2.0])))
    with pytest.raises(_lib.PolfedArgumentError, match="column index"):
        out_of_range.op
