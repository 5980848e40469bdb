"""GPU solves against the oracle at the benchmarked configurations.

Each test runs the CUDA solve and the CPU oracle on identical inputs (the
realisation's explicit parameters, the same x0 and the same KPM probe
vectors), at the configuration's own sizes and with the reference's Krylov
budget (overestimate_iters = 1.25), and requires:

* the same spectral plan: Emin / Emax within 1e-9 relative, the same filter
  order K, the same interval [left, right] to 1e-7;
* every returned pair an eigenpair of the FP64 Hamiltonian: unit norm and
  ||H psi - E psi|| <= 1e-10 (eigentol, LanczosMethod.jl:74-82 and
  CalculatingResiduals.jl:8-42);
* the same eigenvalues as the oracle to 1e-10 relative.  The returned set is
  the converged prefix of the Ritz values ordered by filter value; at the
  reference's last allowed iteration the tol = 1e-14 test of the last pair sits
  at the rounding floor, so the two counts may differ by one and one pair at
  the end of the prefix may differ (rounding slack, asserted explicitly).

Configurations: the Quantum Sun benchmark (L_loc = 13, L_grain = 3,
D = 65536, s = 8, nev = 200, eps = 0.5); one disorder realisation of each
size of the disorder batch (XXZ L = 16 and L = 18, Sz = 0, W = 3, nev = 50);
two small members of the served stream (Quantum Sun L_loc = 10, XXZ L = 15);
and the largest XXZ member of the served stream (L = 20, D = 184,756, nev =
200, s = 16), where the oracle's Lanczos is too slow: there the plan is
compared with the oracle's, every pair is checked against the oracle's FP64
CSR matrix, and two solves from independent starts must return the same set.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EIGENTOL = 1e-10


def _pairs_ok(H, vals, vecs, tol=EIGENTOL):
    assert np.all(np.diff(vals) >= 0), "eigenvalues must be ascending (LanczosMethod.jl:76)"
    R = H @ vecs - vecs * vals[None, :]
    res = np.linalg.norm(R, axis=0)
    nrm = np.linalg.norm(vecs, axis=0)
    assert np.all(np.abs(nrm - 1) < 1e-9), nrm
    assert np.all(res <= tol), (int(np.argmax(res)), float(res.max()))


def _same_set(vals, ref, slack=1):
    """GPU and oracle prefixes agree up to the documented rounding slack."""
    assert abs(len(vals) - len(ref)) <= slack, (len(vals), len(ref))
    if len(ref) == 0:
        return 0
    d = np.abs(vals[:, None] - ref[None, :]) / np.maximum(1.0, np.abs(ref[None, :]))
    nearest = d.min(axis=1)
    matched = int(np.sum(nearest < 1e-10))
    assert matched >= min(len(vals), len(ref)) - slack, (matched, len(vals), len(ref))
    return matched


def _plan_matches(rep, ref):
    s = rep.spectral
    assert abs(s.Emin - ref.Emin) <= 1e-9 * abs(ref.Emin), (s.Emin, ref.Emin)
    assert abs(s.Emax - ref.Emax) <= 1e-9 * abs(ref.Emax), (s.Emax, ref.Emax)
    assert s.order == ref.order, (s.order, ref.order)
    assert abs(s.left - ref.left) < 1e-7 and abs(s.right - ref.right) < 1e-7


def _solve_both(pkg, orc, op, H, x0, nev, target, probes):
    ref = orc.polfed(orc.CSROperator(H), x0, nev, target, probes=probes, eigentol=EIGENTOL)
    vals, vecs, rep = pkg.polfed(op, x0, nev, target, produce_report=True, dos=pkg.DoSConfig(probes=probes),
                                 fact=pkg.FactorizationConfig(eigentol=EIGENTOL))
    return ref, vals, vecs, rep


def test_qsun_benchmark_configuration(pkg, orc, cuda):
    """Quantum Sun L_loc = 13, L_grain = 3 (D = 65536), alpha = 0.75,
    zeta = 0.2, fields U[0.5, 1.5], gamma = 1, g0 = 1; s = 8, nev = 200,
    (:rescaled, 0.5); DoS N = 250, R = 300 (Jackson)."""
    rng = np.random.default_rng(4242)
    f, n, c, g = pkg.qsun_parameters(13, 3, 0.75, gamma=1.0, w=0.5, hz=1.0, zeta=0.2, rng=rng)
    op = pkg.QSunOperator(13, 3, 1.0, c, n, f, g)
    H = orc.qsun_matrix(13, 3, 1.0, c, n, f, g)
    D = H.shape[0]
    assert D == 65536
    x0, _ = np.linalg.qr(rng.standard_normal((D, 8)))
    probes = orc.normalized_gaussian_probes(D, 300, rng)
    ref, vals, vecs, rep = _solve_both(pkg, orc, op, H, x0, 200, ("rescaled", 0.5), probes)
    _plan_matches(rep, ref)
    assert len(ref.vals) >= 190 and len(vals) >= 190
    _pairs_ok(H, vals, vecs)
    _same_set(vals, ref.vals)


@pytest.mark.parametrize("L,eps,seed", [(16, 0.3, 31337), (18, 0.7, 31337 + 256)])
def test_disorder_batch_realisations(pkg, orc, cuda, L, eps, seed):
    """One realisation of each size of the disorder batch: XXZ, Sz = 0,
    Delta = 1, W = 3, nev = 50, s = 8."""
    rng = np.random.default_rng(seed)
    op = pkg.xxz_hamiltonian(L, L // 2, 1.0, 1.0, 3.0, rng=rng)
    H = orc.xxz_matrix(L, L // 2, 1.0, 1.0, op.fields)
    D = H.shape[0]
    x0 = np.asfortranarray(rng.random((D, 8)))
    probes = orc.normalized_gaussian_probes(D, 300, rng)
    ref, vals, vecs, rep = _solve_both(pkg, orc, op, H, x0, 50, ("rescaled", eps), probes)
    _plan_matches(rep, ref)
    assert len(vals) >= 45
    _pairs_ok(H, vals, vecs)
    _same_set(vals, ref.vals)


def test_served_stream_small_members(pkg, orc, cuda):
    """Two members of the served stream: Quantum Sun L_loc = 10 (D = 8192,
    nev = 20, s = 4, eps = 0.25) and XXZ L = 15 in the Sz = -1/2 sector
    (D = 6435, W = 5, nev = 50, s = 16, eps = 0.8)."""
    rng = np.random.default_rng(2025)
    f, n, c, g = pkg.qsun_parameters(10, 3, 0.75, rng=rng)
    q = pkg.QSunOperator(10, 3, 1.0, c, n, f, g)
    Hq = orc.qsun_matrix(10, 3, 1.0, c, n, f, g)
    x = pkg.xxz_hamiltonian(15, 7, 1.0, 1.0, 5.0, rng=rng)
    Hx = orc.xxz_matrix(15, 7, 1.0, 1.0, x.fields)
    for op, H, s, nev, eps in ((q, Hq, 4, 20, 0.25), (x, Hx, 16, 50, 0.8)):
        D = H.shape[0]
        x0 = np.asfortranarray(rng.random((D, s)))
        probes = orc.normalized_gaussian_probes(D, 300, rng)
        ref, vals, vecs, rep = _solve_both(pkg, orc, op, H, x0, nev, ("rescaled", eps), probes)
        _plan_matches(rep, ref)
        _pairs_ok(H, vals, vecs)
        _same_set(vals, ref.vals)


def test_served_stream_largest_xxz_member(pkg, orc, cuda):
    """XXZ L = 20, Sz = 0 (D = 184,756), W = 5, nev = 200, s = 16,
    eps = 0.5: the plan (extrema, interval, order) equals the oracle's on
    the same probes; every returned pair is an eigenpair of the oracle's FP64
    CSR matrix; two solves from independent starts return the same set."""
    rng = np.random.default_rng(77)
    op = pkg.xxz_hamiltonian(20, 10, 1.0, 1.0, 5.0, rng=rng)
    H = orc.xxz_matrix(20, 10, 1.0, 1.0, op.fields)
    D = H.shape[0]
    assert D == 184756
    R = 32
    probes = orc.normalized_gaussian_probes(D, R, rng)
    x0a = np.asfortranarray(rng.random((D, 16)))
    x0b = np.asfortranarray(rng.random((D, 16)))
    ref = orc.plan_only(orc.CSROperator(H), x0a, 200, ("rescaled", 0.5), probes=probes, N=250)
    dos = pkg.DoSConfig(R=R, probes=probes)
    fact = pkg.FactorizationConfig(eigentol=EIGENTOL)
    va, Va, ra = pkg.polfed(op, x0a, 200, ("rescaled", 0.5), produce_report=True, dos=dos, fact=fact)
    _plan_matches(ra, ref)
    assert len(va) >= 190
    _pairs_ok(H, va, Va)
    vb, Vb, rb = pkg.polfed(op, x0b, 200, ("rescaled", 0.5), produce_report=True, dos=dos, fact=fact)
    _pairs_ok(H, vb, Vb)
    _same_set(va, vb)
