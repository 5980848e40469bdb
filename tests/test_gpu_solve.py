"""End-to-end POLFED solves on the B200 against the CPU oracle and dense eigh.

Shared inputs pin what the reference leaves random: explicit fields,
couplings and grain blocks, explicit KPM probe vectors and x0.  With those
fixed, the GPU and the oracle resolve the same target, interval and order,
and return the same eigenvalues to 1e-10 relative, each with an FP64
residual ||H psi - E psi|| below the eigen tolerance.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check_pairs(H, vals, vecs, tol):
    assert np.all(np.diff(vals) >= 0), "eigenvalues must be ascending (LanczosMethod.jl:76)"
    for j in range(len(vals)):
        v = vecs[:, j]
        assert abs(np.linalg.norm(v) - 1) < 1e-9
        r = np.linalg.norm(H @ v - vals[j] * v)
        assert r < tol, (j, r)


def _vs_exact(H, vals):
    ev = np.linalg.eigvalsh(H.toarray())
    return float(np.max(np.min(np.abs(ev[:, None] - vals[None, :]), axis=0) / np.maximum(1, np.abs(vals))))


def _solve_both(pkg, orc, op, H, x0, nev, target, *, N=96, R=24, seed=0, overestimate_iters=2.0, **kw):
    """Oracle and GPU solves on identical inputs.  The Krylov budget is doubled
    (overestimate_iters = 2) so that neither run stops at the last allowed
    iteration: there the reference's tol = 1e-14 sits at the rounding floor and
    whether the last pair passes depends on rounding, not on the algorithm."""
    D = H.shape[0]
    probes = orc.normalized_gaussian_probes(D, R, np.random.default_rng(seed))
    okw = {k: v for k, v in kw.items() if k in ("Emin", "Emax", "order", "tol", "eigentol")}
    ref = orc.polfed(orc.CSROperator(H), x0, nev, target, N=N, R=R, probes=probes,
                     overestimate_iters=overestimate_iters, **okw)
    mapping = pkg.MappingConfig(Emin=kw.get("Emin"), Emax=kw.get("Emax"))
    transform = pkg.TransformConfig(order=kw.get("order"))
    fact = pkg.FactorizationConfig(tol=kw.get("tol", 1e-14), eigentol=kw.get("eigentol", 1e-9),
                                   overestimate_iters=overestimate_iters)
    vals, vecs, rep = pkg.polfed(op, x0, nev, target, produce_report=True, mapping=mapping,
                                 transform=transform, fact=fact, dos=pkg.DoSConfig(N=N, R=R, probes=probes))
    return ref, vals, vecs, rep


def test_xxz_scalar_lanczos_matches_oracle(pkg, orc, cuda):
    # C1 shape at L = 12: random-field XXZ, Sz = 0, s = 1, target eps = 0.5
    L = 12
    rng = np.random.default_rng(1)
    f = 5 * (2 * rng.random(L) - 1)
    op = pkg.xxz_hamiltonian(L, L // 2, 1.0, 1.0, 0.0, fields=f)
    H = orc.xxz_matrix(L, L // 2, 1.0, 1.0, f)
    x0 = rng.random(H.shape[0])
    ref, vals, vecs, rep = _solve_both(pkg, orc, op, H, x0, 10, ("rescaled", 0.5))
    s = rep.spectral
    assert abs(s.Emin - ref.Emin) < 1e-9 * abs(ref.Emin) and abs(s.Emax - ref.Emax) < 1e-9 * abs(ref.Emax)
    assert s.order == ref.order
    assert abs(s.left - ref.left) < 1e-7 and abs(s.right - ref.right) < 1e-7
    assert len(vals) == len(ref.vals) == 10
    np.testing.assert_allclose(vals, ref.vals, rtol=1e-10, atol=1e-10)
    _check_pairs(H, vals, vecs, 1e-9)
    assert _vs_exact(H, vals) < 1e-10
    assert rep.factorization.blocksize == 1 and rep.factorization.converged_tol == 10
    assert rep.spectral.matrixvec_muls == s.order * rep.factorization.itersneeded + 10


@pytest.mark.parametrize("s", [2, 3, 4, 8, 20])
def test_qsun_block_lanczos_matches_oracle(pkg, orc, cuda, s):
    rng = np.random.default_rng(10 + s)
    f, n, c, g = pkg.qsun_parameters(7, 3, 0.75, rng=rng)
    op = pkg.QSunOperator(7, 3, 1.0, c, n, f, g)
    H = orc.qsun_matrix(7, 3, 1.0, c, n, f, g)
    D = H.shape[0]
    x0, _ = np.linalg.qr(rng.standard_normal((D, s)))
    ref, vals, vecs, rep = _solve_both(pkg, orc, op, H, x0, 24, ("rescaled", 0.5), seed=s)
    assert rep.spectral.order == ref.order
    assert len(vals) == len(ref.vals) == 24
    np.testing.assert_allclose(vals, ref.vals, rtol=1e-10, atol=1e-10)
    _check_pairs(H, vals, vecs, 1e-9)
    assert _vs_exact(H, vals) < 1e-10


@pytest.mark.parametrize("target", ["maxdos", "middle", ("offset", 0.3), ("offset", -0.4), ("unrescaled", 1.5)])
def test_j1j2_targets(pkg, orc, cuda, target):
    rng = np.random.default_rng(5)
    L = 14
    f = 2 * rng.random(L) - 1
    op = pkg.j1j2_hamiltonian(L, 7, 1.0, 0.5, 1.0, 1.0, 0.0, fields=f)
    H = orc.j1j2_matrix(L, 7, 1.0, 0.5, 1.0, 1.0, f)
    D = H.shape[0]
    x0, _ = np.linalg.qr(rng.standard_normal((D, 4)))
    ref, vals, vecs, rep = _solve_both(pkg, orc, op, H, x0, 16, target, N=128, R=32)
    assert abs(rep.spectral.target - ref.target) < 1e-9
    assert rep.spectral.order == ref.order
    np.testing.assert_allclose(vals, ref.vals, rtol=1e-10, atol=1e-10)
    _check_pairs(H, vals, vecs, 1e-9)


def test_explicit_extrema_and_order(pkg, orc, cuda):
    rng = np.random.default_rng(8)
    L = 12
    f = 3 * (2 * rng.random(L) - 1)
    op = pkg.xxz_hamiltonian(L, 6, 1.0, 0.5, 0.0, fields=f)
    H = orc.xxz_matrix(L, 6, 1.0, 0.5, f)
    ev = np.linalg.eigvalsh(H.toarray())
    x0, _ = np.linalg.qr(rng.standard_normal((H.shape[0], 3)))
    ref, vals, vecs, rep = _solve_both(pkg, orc, op, H, x0, 9, 0.0, Emin=ev[0] - 0.1, Emax=ev[-1] + 0.1,
                                       order=150)
    assert rep.spectral.order == 150 == ref.order
    assert rep.spectral.Emin == ev[0] - 0.1
    np.testing.assert_allclose(vals, ref.vals, rtol=1e-10, atol=1e-10)
    _check_pairs(H, vals, vecs, 1e-9)


def test_cgs2_and_tolerances(pkg, orc, cuda):
    # two reorthogonalisation passes (CGS2) give the same eigenpairs
    rng = np.random.default_rng(9)
    L = 12
    f = 5 * (2 * rng.random(L) - 1)
    op = pkg.xxz_hamiltonian(L, 6, 1.0, 1.0, 0.0, fields=f)
    H = orc.xxz_matrix(L, 6, 1.0, 1.0, f)
    x0, _ = np.linalg.qr(rng.standard_normal((H.shape[0], 4)))
    probes = orc.normalized_gaussian_probes(H.shape[0], 16, rng)
    dos = pkg.DoSConfig(N=64, R=16, probes=probes)
    v1, _ = pkg.polfed(op, x0, 12, ("rescaled", -0.2), dos=dos, vecs=False)
    v2, w2 = pkg.polfed(op, x0, 12, ("rescaled", -0.2), dos=dos,
                        fact=pkg.FactorizationConfig(reorth_passes=2))
    np.testing.assert_allclose(v1, v2, rtol=1e-11, atol=1e-11)
    _check_pairs(H, v2, w2, 1e-9)


def test_device_probes_and_repeatability(pkg, orc, cuda):
    # the default path draws probes on the device; a fixed seed repeats bit for bit
    rng = np.random.default_rng(12)
    L = 12
    f = 4 * (2 * rng.random(L) - 1)
    op = pkg.xxz_hamiltonian(L, 6, 1.0, 1.0, 0.0, fields=f)
    H = orc.xxz_matrix(L, 6, 1.0, 1.0, f)
    x0 = rng.random(H.shape[0])
    dos = pkg.DoSConfig(seed=1234)
    a = pkg.polfed(op, x0, 8, ("rescaled", 0.2), dos=dos, produce_report=True)
    b = pkg.polfed(op, x0, 8, ("rescaled", 0.2), dos=dos, produce_report=True)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert a[2].spectral.order == b[2].spectral.order
    _check_pairs(H, a[0], a[1], 1e-9)
    assert _vs_exact(H, a[0]) < 1e-10


def test_input_validation(pkg, cuda):
    from polfed_b200 import _lib
    op = pkg.xxz_hamiltonian(8, 4, 1.0, 1.0, 0.0, fields=[0.1] * 8)
    D = op.dim
    with pytest.raises(ValueError):
        pkg.polfed(op, np.ones(D + 1), 2, "middle")
    with pytest.raises(ValueError):
        pkg.polfed(op, np.ones(D), 2, ("offset", 2.0))
    with pytest.raises(_lib.PolfedArgumentError):
        pkg.polfed(op, np.zeros(D), 2, "middle")
    with pytest.raises(_lib.PolfedArgumentError):
        pkg.polfed(op, np.full(D, np.nan), 2, "middle")
    with pytest.raises(_lib.PolfedArgumentError):
        pkg.polfed(op, np.ones(D), 2, "middle",
                   transform=pkg.TransformConfig(left=-1.0, right=1.0, order=20),
                   mapping=pkg.MappingConfig(Emin=-5.0, Emax=5.0))


def test_unnormalised_start_is_normalised(pkg, orc, cuda):
    # PolfedCore.jl:43-95: a non-orthonormal x0 is replaced by an orthonormal copy
    rng = np.random.default_rng(4)
    L = 10
    f = 2 * rng.random(L) - 1
    op = pkg.xxz_hamiltonian(L, 5, 1.0, 1.0, 0.0, fields=f)
    H = orc.xxz_matrix(L, 5, 1.0, 1.0, f)
    x0 = rng.random((H.shape[0], 2)) * 7.0
    x0c = x0.copy()
    vals, vecs = pkg.polfed(op, x0, 6, ("rescaled", 0.1), dos=pkg.DoSConfig(N=64, R=8, seed=5))
    np.testing.assert_array_equal(x0, x0c)
    assert len(vals) == 6
    _check_pairs(H, vals, vecs, 1e-9)


def test_config_c1_full_size(pkg, orc, cuda):
    # The reference's CPU-runnable configuration: XXZ L=14, PBC, J=1, Delta=1,
    # h ~ U[-5,5], Sz=0 (D=3432), eps=0.5, nev=20, s=1, automatic order, DoS
    # defaults (N=250, R=300) and the reference's Krylov budget (eta = 1.25,
    # 68 iterations).  GPU and oracle see the same probes and x0; both return
    # the converged prefix, every returned pair is an exact eigenpair.
    rng = np.random.default_rng(2024)
    L = 14
    op = pkg.xxz_hamiltonian(L, 7, 1.0, 1.0, 5.0, rng=rng)
    H = orc.xxz_matrix(L, 7, 1.0, 1.0, op.fields)
    D = H.shape[0]
    x0 = rng.random(D)
    probes = orc.normalized_gaussian_probes(D, 300, rng)
    ref = orc.polfed(orc.CSROperator(H), x0, 20, ("rescaled", 0.5), probes=probes, eigentol=1e-10)
    vals, vecs, rep = pkg.polfed(op, x0, 20, ("rescaled", 0.5), produce_report=True,
                                 dos=pkg.DoSConfig(probes=probes), fact=pkg.FactorizationConfig(eigentol=1e-10))
    assert rep.spectral.order == ref.order
    assert abs(len(vals) - len(ref.vals)) <= 1, (len(vals), len(ref.vals), rep.factorization)
    assert len(vals) >= 12
    _check_pairs(H, vals, vecs, 1e-10)
    assert _vs_exact(H, vals) < 1e-10
    n = min(len(vals), len(ref.vals))
    common = np.intersect1d(np.round(vals, 8), np.round(ref.vals, 8))
    assert len(common) >= n - 1


def test_mixed_precision_refinement(pkg, orc, cuda):
    """PF_PREC_MIXED: the FP32 filter alone leaves every Ritz vector near
    1e-6..1e-5 in FP64 residual, so with refinement off the solve returns no
    pair at eigentol = 1e-10.  The FP64 refinement passes (filter, then
    Rayleigh-Ritz with the FP64 H) bring pairs to 1e-10: every pair returned is
    an FP64 eigenpair to 1e-10 with the FP64 solve's eigenvalue.  With 8
    passes this problem returns 26 of the FP64 solve's 32 pairs (the last
    targets converge at the rate of the filter's side lobes, ~0.8 per pass)."""
    rng = np.random.default_rng(33)
    f, n, c, g = pkg.qsun_parameters(8, 3, 0.75, rng=rng)
    op = pkg.QSunOperator(8, 3, 1.0, c, n, f, g)
    H = orc.qsun_matrix(8, 3, 1.0, c, n, f, g)
    D = H.shape[0]
    x0, _ = np.linalg.qr(rng.standard_normal((D, 4)))
    probes = orc.normalized_gaussian_probes(D, 32, rng)
    kw = dict(dos=pkg.DoSConfig(N=128, R=32, probes=probes), produce_report=True)
    v64, V64, r64 = pkg.polfed(op, x0, 32, ("rescaled", 0.4), fact=pkg.FactorizationConfig(eigentol=1e-10), **kw)
    assert len(v64) == 32
    v0, _, r0 = pkg.polfed(op, x0, 32, ("rescaled", 0.4), precision="mixed",
                           fact=pkg.FactorizationConfig(eigentol=1e-10, refine_passes=0), **kw)
    assert len(v0) == 0 and r0.factorization.refined == 0
    res = {}
    for passes in (4, 8):
        vm, Vm, rm = pkg.polfed(op, x0, 32, ("rescaled", 0.4), precision="mixed",
                                fact=pkg.FactorizationConfig(eigentol=1e-10, refine_passes=passes), **kw)
        assert rm.spectral.order == r64.spectral.order
        assert rm.factorization.refined == len(vm)
        _check_pairs(H, vm, Vm, 1e-10)
        d = np.abs(vm[:, None] - v64[None, :]).min(axis=1) / np.maximum(1, np.abs(vm))
        assert np.all(d < 1e-10), d.max()
        res[passes] = (len(vm), rm.factorization.eigenresidual)
    assert res[8][0] >= 24 and res[8][0] >= res[4][0]
    assert res[8][1] < res[4][1] < 1e-6


def test_cgs2_with_tensor_core_first_pass(pkg, orc, cuda):
    """reorth_passes = 3: CGS2 whose first Gram product runs on the tensor
    cores in split BF16 gives the eigenpairs of the FP64 reorthogonalisation."""
    rng = np.random.default_rng(21)
    f, n, c, g = pkg.qsun_parameters(8, 3, 0.75, rng=rng)
    op = pkg.QSunOperator(8, 3, 1.0, c, n, f, g)
    H = orc.qsun_matrix(8, 3, 1.0, c, n, f, g)
    D = H.shape[0]
    x0, _ = np.linalg.qr(rng.standard_normal((D, 8)))
    probes = orc.normalized_gaussian_probes(D, 32, rng)
    dos = pkg.DoSConfig(N=128, R=32, probes=probes)
    v1, _ = pkg.polfed(op, x0, 40, ("rescaled", 0.3), dos=dos, vecs=False,
                       fact=pkg.FactorizationConfig(eigentol=1e-10, overestimate_iters=2.0))
    v3, w3 = pkg.polfed(op, x0, 40, ("rescaled", 0.3), dos=dos,
                        fact=pkg.FactorizationConfig(eigentol=1e-10, overestimate_iters=2.0, reorth_passes=3))
    assert len(v3) == len(v1) >= 38
    np.testing.assert_allclose(v3, v1, rtol=1e-11, atol=1e-11)
    _check_pairs(H, v3, w3, 1e-10)


@pytest.mark.parametrize("s", [1, 3, 4, 20, 40])
def test_device_lanczos_algebra_equals_the_host_qr(pkg, orc, cuda, s):
    """The s x s algebra of an iteration (alpha, the CholQR passes, the
    projected matrix) runs on the device; its Cholesky repeats the host
    factorisation's rounded operations in order, so a solve gives bit for bit
    what the host QR (Gram matrices read back every iteration) gives.  Blocks
    of up to 32 columns take the fused block passes in both forms (s = 20:
    64-row tiles), wider ones the library products (s = 40)."""
    rng = np.random.default_rng(30 + s)
    f, n, c, g = pkg.qsun_parameters(8, 3, 0.75, rng=rng)
    op = pkg.QSunOperator(8, 3, 1.0, c, n, f, g)
    H = orc.qsun_matrix(8, 3, 1.0, c, n, f, g)
    x0, _ = np.linalg.qr(rng.standard_normal((H.shape[0], s)))
    x0 = x0[:, 0] if s == 1 else x0
    dos = pkg.DoSConfig(N=96, R=24, seed=7)
    out = []
    for host_qr in (False, True):
        fact = pkg.FactorizationConfig(eigentol=1e-10, host_qr=host_qr)
        out.append(pkg.polfed(op, x0, 16, ("rescaled", 0.4), produce_report=True, dos=dos, fact=fact))
    (v0, w0, r0), (v1, w1, r1) = out
    assert r0.benchmark.qr_restarts == 0 and r1.benchmark.qr_restarts == 0
    assert len(v0) == 16
    np.testing.assert_array_equal(v0, v1)
    np.testing.assert_array_equal(w0, w1)
    assert r0.spectral.Emin == r1.spectral.Emin and r0.spectral.Emax == r1.spectral.Emax
    _check_pairs(H, v0, w0, 1e-10)


def test_block_breakdown_restarts_with_the_host_qr(pkg, orc, cuda):
    """A starting block holding an eigenvector makes that column of the first
    residual block vanish, so the device CholQR flags a breakdown; the run
    restarts with the host QR (Householder on the broken block, as the
    reference's qr) and returns exactly what the host QR gives from the
    start.  Returned pairs are FP64 eigenpairs."""
    L = 10
    rng = np.random.default_rng(5)
    f = 3 * (2 * rng.random(L) - 1)
    op = pkg.xxz_hamiltonian(L, L // 2, 1.0, 1.0, 0.0, fields=f)
    H = orc.xxz_matrix(L, L // 2, 1.0, 1.0, f)
    ev, U = np.linalg.eigh(H.toarray())
    D = H.shape[0]
    mid = int(np.argmin(np.abs(ev - 0.5 * (ev[0] + ev[-1]))))
    w = rng.standard_normal(D)
    w -= U[:, mid] * (U[:, mid] @ w)
    x0 = np.stack([U[:, mid], w / np.linalg.norm(w)], axis=1)
    mapping = pkg.MappingConfig(Emin=float(ev[0]), Emax=float(ev[-1]))
    dos = pkg.DoSConfig(N=96, R=24, seed=3)
    res = []
    for host_qr in (False, True):
        fact = pkg.FactorizationConfig(host_qr=host_qr)
        try:
            res.append(pkg.polfed(op, x0, 6, ("rescaled", 0.5), produce_report=True, dos=dos, mapping=mapping,
                                  fact=fact))
        except Exception as e:   # the host QR's own outcome, whatever it is, must be reproduced
            res.append(repr(e))
    dev, host = res
    if isinstance(host, str):
        assert dev == host
        return
    (v0, w0, r0), (v1, w1, r1) = dev, host
    assert r0.benchmark.qr_restarts == 1 and r1.benchmark.qr_restarts == 0
    np.testing.assert_array_equal(v0, v1)
    np.testing.assert_array_equal(w0, w1)
    _check_pairs(H, v0, w0, 1e-9)


def test_block_size_tuner(pkg, orc, cuda):
    """tune_block_size times one complete solve per candidate block size and
    returns the fastest; solves at every candidate return eigenvalues of H
    (to 1e-10 against the dense spectrum)."""
    rng = np.random.default_rng(41)
    f, n, c, g = pkg.qsun_parameters(7, 3, 0.75, rng=rng)
    op = pkg.QSunOperator(7, 3, 1.0, c, n, f, g)
    kw = dict(dos=pkg.DoSConfig(N=96, R=24, seed=3), fact=pkg.FactorizationConfig(eigentol=1e-10))
    best, rates = pkg.tune_block_size(op, 12, ("rescaled", 0.4), (2, 4), **kw)
    assert best in (2, 4) and set(rates) == {2, 4} and all(r > 0 for r in rates.values())
    assert rates[best] == max(rates.values())
    H = orc.qsun_matrix(7, 3, 1.0, c, n, f, g)
    vals = {}
    for s in (2, 4):
        x0 = np.random.default_rng(7).random((H.shape[0], s))
        vals[s], _ = pkg.polfed(op, x0, 12, ("rescaled", 0.4), vecs=False, **kw)
    for s in (2, 4):
        assert len(vals[s]) >= 10
        assert _vs_exact(H, vals[s]) < 1e-10
