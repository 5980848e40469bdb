"""The Quantum Sun beyond the spin-1/2 full space on the B200: spin S > 1/2
(QuantumSun.jl:1-102) and the total-S_z sector of any spin
(QuantumSun_U1_conserving.jl:1-212), assembled as CSR on the device.

The device matrix must equal the oracle's restatement of the reference's
builder applied to the same draws (FP64 to 1e-12, FP32 to 2e-5 relative), in
the reference's state order, and solves must return FP64 eigenpairs of it
nearest the target.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL64, RTOL32 = 1e-12, 2e-5

# (L_loc, L_grain, S, use_U1, S_z)
CASES = [
    (6, 2, 0.5, True, 0.0),    # D = 70
    (7, 2, 0.5, True, 0.5),    # odd L, half-integer S_z: D = 126
    (4, 2, 1.0, False, 0.0),   # D = 3^6 = 729
    (4, 2, 1.0, True, 0.0),    # D = 141
    (3, 2, 1.5, True, 0.5),    # D = 4^5 strings with digit sum 8
    (3, 1, 1.5, False, 0.0),   # D = 4^4 = 256
    (3, 2, 2.0, True, -1.0),   # spin 2
]


def _dev(cuda, A, dtype):
    A = np.asarray(A).reshape(A.shape[0], -1)
    return cuda.tensor(np.ascontiguousarray(A.T), dtype=dtype, device="cuda:0").t()


def _host(t):
    return t.t().contiguous().cpu().numpy().T


def _build(pkg, orc, case, seed, gamma=1.0):
    L_loc, L_grain, S, u1, S_z = case
    rng = np.random.default_rng(seed)
    f, n, c, goe = pkg.qsun_spin_parameters(L_loc, L_grain, 0.75, S, rng=rng)
    grain = pkg.qsun_spin_grain(goe, L_loc, L_grain, S, gamma=gamma, use_U1=u1, S_z=S_z)
    op = pkg.QSunSpinOperator(L_loc, L_grain, S, 1.0, c, n, f, grain, use_U1=u1, S_z=S_z)
    H = orc.qsun_spin_matrix(L_loc, L_grain, 1.0, c, n, f, goe, S=S, gamma=gamma, use_U1=u1, S_z=S_z)
    return op, H


@pytest.mark.parametrize("case", CASES)
def test_device_built_matrix_equals_the_reference_builder(pkg, orc, cuda, case):
    op, H = _build(pkg, orc, case, seed=11)
    D = H.shape[0]
    assert op.dim == D
    rng = np.random.default_rng(12)
    X = rng.standard_normal((D, 3))
    ref = H @ X
    for dt, tol in ((cuda.float64, RTOL64), (cuda.float32, RTOL32)):
        Y = pkg.col_major(D, 3, dtype=dt)
        pkg.apply(op, Y, _dev(cuda, X, dt))
        got = _host(Y)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < tol, (case, dt)
    # every column: the device operator applied to a unit vector is that column
    E = np.eye(D)[:, :min(D, 24)]
    Y = pkg.col_major(D, E.shape[1])
    pkg.apply(op, Y, _dev(cuda, E, cuda.float64))
    np.testing.assert_allclose(_host(Y), H.toarray()[:, :E.shape[1]], rtol=1e-13, atol=1e-14)


@pytest.mark.parametrize("case", [CASES[1], CASES[3], CASES[4]])
def test_solves_on_device_built_operators(pkg, orc, cuda, case):
    """The GPU solve and the oracle's POLFED on identical inputs (the same
    matrix, KPM probes and x0): same plan, same eigenvalues to 1e-10, and
    every returned pair an FP64 eigenpair of the device-built matrix."""
    op, H = _build(pkg, orc, case, seed=21)
    D = H.shape[0]
    nev, N, R = 8, 96, 24
    rng = np.random.default_rng(22)
    x0 = rng.random(D)
    probes = orc.normalized_gaussian_probes(D, R, np.random.default_rng(23))
    ref = orc.polfed(orc.CSROperator(H), x0, nev, ("rescaled", 0.5), N=N, R=R, probes=probes,
                     overestimate_iters=2.0, eigentol=1e-10)
    vals, vecs, rep = pkg.polfed(op, x0, nev, ("rescaled", 0.5), produce_report=True,
                                 dos=pkg.DoSConfig(N=N, R=R, probes=probes),
                                 fact=pkg.FactorizationConfig(eigentol=1e-10, overestimate_iters=2.0))
    assert rep.spectral.order == ref.order
    assert abs(rep.spectral.Emin - ref.Emin) < 1e-9 * max(1, abs(ref.Emin))
    assert len(vals) == len(ref.vals) == nev
    np.testing.assert_allclose(vals, ref.vals, rtol=1e-10, atol=1e-10)
    for j in range(nev):
        v = vecs[:, j]
        assert abs(np.linalg.norm(v) - 1) < 1e-9
        assert np.linalg.norm(H @ v - vals[j] * v) < 1e-10


def test_sector_dimensions_and_errors_on_device(pkg, cuda):
    """The device sector count matches the reference's sizes (test_qsun.jl:20-76)
    and an invalid sector fails with the reference's message."""
    for (L_loc, L_grain, S, S_z, dim) in ((2, 2, 0.5, 0.0, 6), (2, 1, 0.5, 0.5, 3), (1, 1, 1.5, 1.0, 3)):
        op = pkg.qsun_hamiltonian(L_loc, L_grain, 1.0, 0.5, S=S, use_U1=True, S_z=S_z, rng=np.random.default_rng(1))
        assert op.dim == dim
    op = pkg.qsun_hamiltonian(2, 2, 1.0, 0.5, S=1.0, rng=np.random.default_rng(1))
    assert op.dim == 81
    from polfed_b200 import _lib
    op = pkg.QSunSpinOperator(2, 2, 0.5, 1.0, [1.0, 0.5], [0, 1], [1.0, 1.0], np.eye(4))
    op.use_U1, op.S_z = True, 0.5   # bypass the host check: the library refuses it too
    with pytest.raises(_lib.PolfedError, match="Wrong total value of spin"):
        op.op
