"""Parity of the CUDA kernels with the CPU oracle (needs a B200).

Integer work (basis enumeration and ranking) must be bit-exact; FP64 operator
work must agree to ~1e-13 relative; FP32 work within single-precision
roundoff.  Every call goes through the C ABI of libpolfed_b200.so.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL64 = 1e-12   # FP64 operator / filter parity, relative to the block norm
RTOL32 = 2e-5    # FP32 operator parity, relative to the block norm


def _models(pkg, orc, rng):
    """(name, product operator, oracle CSR matrix) for small seeded models."""
    out = []
    L = 12
    f = 5 * (2 * rng.random(L) - 1)
    out.append(("xxz_L12_pbc", pkg.xxz_hamiltonian(L, 6, 1.0, 1.0, 0.0, fields=f),
                orc.xxz_matrix(L, 6, 1.0, 1.0, f)))
    f = 2 * rng.random(11) - 1
    out.append(("xxz_L11_open_Lup4", pkg.xxz_hamiltonian(11, 4, 0.7, 1.3, 0.0, fields=f, boundary="open"),
                orc.xxz_matrix(11, 4, 0.7, 1.3, f, boundary="open")))
    f = 2 * rng.random(14) - 1
    out.append(("j1j2_L14", pkg.j1j2_hamiltonian(14, 7, 1.0, 0.5, 1.0, 0.8, 0.0, fields=f),
                orc.j1j2_matrix(14, 7, 1.0, 0.5, 1.0, 0.8, f)))
    f = rng.random(9)
    bonds = pkg.chain_bonds(9, 1, "periodic")
    out.append(("chain_full_L9", pkg.SpinChainOperator(9, -1, bonds, [1.0] * 9, [0.6] * 9, f),
                orc.spin_chain_matrix(9, -1, bonds, [1.0] * 9, [0.6] * 9, f)))
    fq, nq, cq, gq = pkg.qsun_parameters(7, 3, 0.75, rng=rng)
    out.append(("qsun_7_3", pkg.QSunOperator(7, 3, 1.0, cq, nq, fq, gq),
                orc.qsun_matrix(7, 3, 1.0, cq, nq, fq, gq)))
    fq, nq, cq, gq = pkg.qsun_parameters(6, 2, 0.5, rng=rng)
    out.append(("qsun_6_2", pkg.QSunOperator(6, 2, 0.8, cq, nq, fq, gq),
                orc.qsun_matrix(6, 2, 0.8, cq, nq, fq, gq)))
    return out


@pytest.fixture(scope="module")
def models(pkg, orc, cuda):
    return _models(pkg, orc, np.random.default_rng(42))


def _dev(cuda, A, dtype):
    """Column-major CUDA copy of a host D x s array."""
    A = np.asarray(A).reshape(A.shape[0], -1)
    t = cuda.tensor(np.ascontiguousarray(A.T), dtype=dtype, device="cuda:0")
    return t.t()


def _host(t):
    return t.t().contiguous().cpu().numpy().T


@pytest.mark.parametrize("L,Lup", [(4, 2), (10, 5), (12, 3), (14, 7), (16, 8), (17, 5), (20, 10), (24, 12)])
def test_basis_unrank_rank_bit_exact(pkg, orc, cuda, L, Lup):
    op = pkg.xxz_hamiltonian(L, Lup, 1.0, 1.0, 0.0, fields=[0.0] * L)
    basis = orc.sector_basis(L, Lup)
    D = len(basis)
    assert op.dim == D == math.comb(L, Lup)
    idx = cuda.arange(D, dtype=cuda.int64, device="cuda:0")
    states = pkg.basis_states(op, idx).cpu().numpy().astype(np.uint64)
    np.testing.assert_array_equal(states, basis)
    back = pkg.basis_index(op, cuda.tensor(basis.astype(np.int64), device="cuda:0")).cpu().numpy()
    np.testing.assert_array_equal(back, np.arange(D))
    # every single-bond flip of every basis state ranks exactly like the oracle's lookup
    rng = np.random.default_rng(L * 100 + Lup)
    sample = basis if D <= 20000 else basis[rng.choice(D, 20000, replace=False)]
    flips = []
    for i in range(L):
        for j in range(i + 1, L):
            m = np.uint64((1 << i) | (1 << j))
            s = sample[((sample & m) != 0) & ((sample & m) != m)]
            flips.append(s ^ m)
    flips = np.concatenate(flips) if flips else np.zeros(0, np.uint64)
    if flips.size:
        got = pkg.basis_index(op, cuda.tensor(flips.astype(np.int64), device="cuda:0")).cpu().numpy()
        np.testing.assert_array_equal(got, orc.sector_rank(basis, flips))
    # states outside the sector map to -1
    bad = np.array([0, (1 << L) - 1, 1 << L], dtype=np.int64)
    got = pkg.basis_index(op, cuda.tensor(bad, device="cuda:0")).cpu().numpy()
    exp = [(0 if Lup == 0 else -1), (0 if Lup == L else -1), -1]
    np.testing.assert_array_equal(got, exp)


def test_full_space_rank_is_identity(pkg, cuda):
    L = 9
    op = pkg.SpinChainOperator(L, -1, pkg.chain_bonds(L, 1), [1.0] * L, [1.0] * L, [0.0] * L)
    idx = cuda.arange(2 ** L, dtype=cuda.int64, device="cuda:0")
    np.testing.assert_array_equal(pkg.basis_states(op, idx).cpu().numpy(), np.arange(2 ** L))


@pytest.mark.parametrize("s", [1, 3, 8, 16])
def test_apply_fp64(pkg, orc, cuda, models, s):
    rng = np.random.default_rng(s)
    for name, op, H in models:
        D = H.shape[0]
        X = rng.standard_normal((D, s))
        Y = pkg.col_major(D, s)
        pkg.apply(op, Y, _dev(cuda, X, cuda.float64))
        ref = H @ X
        err = np.linalg.norm(_host(Y) - ref) / np.linalg.norm(ref)
        assert err < RTOL64, (name, err)
        # rescaled operator (H - b)/a, Plan.jl:173-177
        a, b = 3.7, -0.4
        pkg.apply(op, Y, _dev(cuda, X, cuda.float64), a=a, b=b)
        ref = orc.CSROperator(H).rescaled(X, a, b)
        err = np.linalg.norm(_host(Y) - ref) / np.linalg.norm(ref)
        assert err < RTOL64, (name, err)


def test_diagonal_bit_exact_fp64(pkg, orc, cuda, models):
    # the diagonal is summed in the reference's order (fields, then bonds): H e_i hits it exactly
    for name, op, H in models:
        if op.kind != "spin_chain":
            continue
        D = H.shape[0]
        E = np.zeros((D, 4))
        cols = np.random.default_rng(1).choice(D, 4, replace=False)
        # columns that have no self-flip contribution except the diagonal
        E[cols, np.arange(4)] = 1.0
        Y = pkg.col_major(D, 4)
        pkg.apply(op, Y, _dev(cuda, E, cuda.float64))
        got = _host(Y)[cols, np.arange(4)]
        exp = H.diagonal()[cols]
        np.testing.assert_array_equal(got, exp, err_msg=name)


@pytest.mark.parametrize("s", [1, 4, 16])
def test_apply_fp32(pkg, orc, cuda, models, s):
    rng = np.random.default_rng(10 + s)
    for name, op, H in models:
        D = H.shape[0]
        X = rng.standard_normal((D, s)).astype(np.float32)
        Y = pkg.col_major(D, s, dtype=cuda.float32)
        pkg.apply(op, Y, _dev(cuda, X, cuda.float32), a=2.0, b=0.5)
        ref = orc.CSROperator(H).rescaled(X.astype(np.float64), 2.0, 0.5)
        err = np.linalg.norm(_host(Y) - ref) / np.linalg.norm(ref)
        assert err < RTOL32, (name, err)


@pytest.mark.parametrize("s", [4, 8, 16, 32])
def test_coop_step_matches_per_thread_and_oracle(pkg, orc, cuda, models, s):
    """The warp-cooperative chain step (width 0) against the per-thread step
    and the oracle: apply, the rescaled apply, the diagonal (bit-exact) and a
    K = 40 filter, in FP64 and FP32."""
    rng = np.random.default_rng(100 + s)
    for name, op, H in models:
        if op.kind != "spin_chain":
            continue
        D = H.shape[0]
        Ht = orc.CSROperator(H)
        for dt, dts, tol in ((cuda.float64, "fp64", RTOL64), (cuda.float32, "fp32", RTOL32)):
            per_thread = min(s, 64 // (8 if dts == "fp64" else 4))
            X = rng.standard_normal((D, s))
            out = {}
            for width in (per_thread, 0):
                pkg.set_step_width(op, s, width, dts)
                Y = pkg.col_major(D, s, dtype=dt)
                pkg.apply(op, Y, _dev(cuda, X, dt), a=2.5, b=-0.3)
                out[width] = _host(Y).astype(np.float64)
                ref = Ht.rescaled(X.astype(np.float64) if dts == "fp64" else X.astype(np.float32).astype(np.float64),
                                  2.5, -0.3)
                err = np.linalg.norm(out[width] - ref) / np.linalg.norm(ref)
                assert err < tol, (name, s, dts, width, err)
            diff = np.linalg.norm(out[0] - out[per_thread]) / np.linalg.norm(out[per_thread])
            assert diff <= (1e-14 if dts == "fp64" else 1e-6), (name, s, dts, diff)
            if dts == "fp64":
                # diagonal from the stored array: exact
                E = np.zeros((D, s))
                cols = np.random.default_rng(s).choice(D, min(s, D), replace=False)
                E[cols, np.arange(len(cols))] = 1.0
                Y = pkg.col_major(D, s)
                pkg.apply(op, Y, _dev(cuda, E, cuda.float64))
                np.testing.assert_array_equal(_host(Y)[cols, np.arange(len(cols))], H.diagonal()[cols],
                                              err_msg=name)
                # a filter through the cooperative step
                Emax = float(np.abs(H).sum(axis=1).max())
                plan = orc.build_transform_plan(("rescaled", 0.31), 10, 1.0, 0.0, order=40)
                coeffs = orc.filter_coefficients(plan)[:41]
                Y = pkg.col_major(D, s)
                pkg.chebyshev_filter(op, Y, _dev(cuda, X, cuda.float64), coeffs, a=1.01 * Emax, b=0.0)
                ref = Ht.filter(X, 1.01 * Emax, 0.0, coeffs)
                assert np.linalg.norm(_host(Y) - ref) / np.linalg.norm(ref) < RTOL64 * 10, name
            pkg.set_step_width(op, s, per_thread, dts)   # leave the default variant for later tests


def test_set_step_width_rejects_invalid_widths(pkg, cuda, models):
    from polfed_b200 import _lib
    chain = next(op for name, op, H in models if op.kind == "spin_chain")
    qsun = next(op for name, op, H in models if op.kind != "spin_chain")
    with pytest.raises(_lib.PolfedArgumentError):
        pkg.set_step_width(qsun, 8, 0)          # cooperative step is for chain operators
    with pytest.raises(_lib.PolfedArgumentError):
        pkg.set_step_width(chain, 6, 0)         # s must be 4, 8, 16 or 32
    with pytest.raises(_lib.PolfedArgumentError):
        pkg.set_step_width(chain, 8, 3)         # not a power of two
    with pytest.raises(_lib.PolfedArgumentError):
        pkg.set_step_width(chain, 16, 16)       # 128 bytes of FP64 columns per thread
    w, times = pkg.autotune(chain, 8, "fp64")
    assert w in times and 0 in times            # the cooperative step was timed


def test_clenshaw_step_formulas(pkg, orc, cuda, models):
    # vector_dispatch.jl:113-139 and optimization.jl:307-325:
    #   b1 = c X + 2 Ht b2 - b3,   Y = c0 X + Ht b1 - b2
    rng = np.random.default_rng(7)
    a, b, c = 2.5, 0.3, 0.7
    for name, op, H in models:
        D = H.shape[0]
        Ht = orc.CSROperator(H)
        for s in (1, 6):
            X, B2, B3 = (rng.standard_normal((D, s)) for _ in range(3))
            b1 = pkg.col_major(D, s)
            pkg.clenshaw_recurrence(op, b1, _dev(cuda, B2, cuda.float64), _dev(cuda, B3, cuda.float64), c,
                                    _dev(cuda, X, cuda.float64), a=a, b=b)
            ref = c * X + 2 * Ht.rescaled(B2, a, b) - B3
            assert np.linalg.norm(_host(b1) - ref) / np.linalg.norm(ref) < RTOL64, name
            Y = pkg.col_major(D, s)
            pkg.clenshaw_finalsum(op, _dev(cuda, B2, cuda.float64), _dev(cuda, B3, cuda.float64), c, Y,
                                  _dev(cuda, X, cuda.float64), a=a, b=b)
            ref = c * X + Ht.rescaled(B2, a, b) - B3
            assert np.linalg.norm(_host(Y) - ref) / np.linalg.norm(ref) < RTOL64, name


@pytest.mark.parametrize("K", [0, 1, 2, 3, 40, 257])
def test_filter_matches_oracle(pkg, orc, cuda, models, K):
    rng = np.random.default_rng(K)
    plan = orc.build_transform_plan(("rescaled", 0.31), 10, 1.0, 0.0, order=max(K, 1))
    coeffs = orc.filter_coefficients(plan)[:K + 1] if K >= 1 else np.array([0.8])
    for name, op, H in models:
        D = H.shape[0]
        Ht = orc.CSROperator(H)
        Emax = float(np.abs(H).sum(axis=1).max())   # Gershgorin: |H| <= Emax, so |Ht| < 1
        a, b = Emax * 1.01, 0.0
        for s, dt, tol in ((1, cuda.float64, RTOL64 * 10), (8, cuda.float64, RTOL64 * 10),
                           (8, cuda.float32, 2e-4)):
            X = rng.standard_normal((D, s))
            Y = pkg.col_major(D, s, dtype=dt)
            pkg.chebyshev_filter(op, Y, _dev(cuda, X, dt), coeffs, a=a, b=b)
            ref = Ht.filter(X, a, b, coeffs)
            err = np.linalg.norm(_host(Y) - ref) / max(np.linalg.norm(ref), 1e-300)
            assert err < tol, (name, K, s, dt, err)


def test_kpm_moments_match_oracle(pkg, orc, cuda, models):
    rng = np.random.default_rng(3)
    for name, op, H in models:
        D = H.shape[0]
        Emax = float(np.abs(H).sum(axis=1).max())
        a, b = Emax * 1.05, 0.0
        for N, R in ((1, 1), (2, 3), (5, 3), (64, 37), (128, 70)):
            probes = orc.normalized_gaussian_probes(D, R, rng)
            ref = orc.dos_moments(orc.CSROperator(H), a, b, N, probes)
            got = pkg.kpm_moments(op, N, R, a=a, b=b, probes=_dev(cuda, probes, cuda.float64))
            np.testing.assert_allclose(got, ref, rtol=0, atol=1e-10 * D, err_msg=f"{name} N={N} R={R}")
            got32 = pkg.kpm_moments(op, N, R, a=a, b=b, probes=_dev(cuda, probes, cuda.float32))
            np.testing.assert_allclose(got32, ref, rtol=0, atol=2e-4 * D, err_msg=f"{name} fp32 N={N} R={R}")


def test_kpm_generated_probes(pkg, cuda, models):
    # device-drawn probes are normalised: mu_0 = D exactly; a repeat is bit-identical
    for name, op, H in models:
        D = H.shape[0]
        Emax = float(np.abs(H).sum(axis=1).max())
        for kind in ("gaussian", "rademacher"):
            m1 = pkg.kpm_moments(op, 32, 40, a=Emax, b=0.0, probe_kind=kind, seed=99)
            m2 = pkg.kpm_moments(op, 32, 40, a=Emax, b=0.0, probe_kind=kind, seed=99)
            np.testing.assert_array_equal(m1, m2)
            assert abs(m1[0] - D) < 1e-9 * D, (name, kind)
            # trace of H/a: mu_1 estimates tr(Ht) = tr(H)/Emax
            tr = H.diagonal().sum() / Emax
            assert abs(m1[1] - tr) < 0.5 * D, (name, kind, m1[1], tr)


def test_step_deterministic(pkg, cuda, models):
    rng = np.random.default_rng(0)
    for name, op, H in models:
        D = H.shape[0]
        X = _dev(cuda, rng.standard_normal((D, 8)), cuda.float64)
        Y1, Y2 = pkg.col_major(D, 8), pkg.col_major(D, 8)
        pkg.apply(op, Y1, X)
        pkg.apply(op, Y2, X)
        assert cuda.equal(Y1, Y2), name


def test_operator_errors(pkg, cuda):
    from polfed_b200 import _lib
    op = pkg.xxz_hamiltonian(8, 4, 1.0, 1.0, 0.0, fields=[0.0] * 8)
    D = op.dim
    X = pkg.col_major(D, 2)
    with pytest.raises(ValueError):
        pkg.apply(op, pkg.col_major(D + 1, 2), X)
    with pytest.raises(_lib.PolfedArgumentError):
        pkg.apply(op, pkg.col_major(D, 2), X, a=0.0)
    with pytest.raises(_lib.PolfedError):
        pkg.SpinChainOperator(33, -1, [], [], [], [0.0] * 33).op
    with pytest.raises(_lib.PolfedError):
        pkg.QSunOperator(4, 2, 1.0, [1.0] * 4, [0, 1, 2, 0], [1.0] * 4, np.eye(4)).op


def _tile_ok(op, s, width, elem, ipt):
    """The tiled Quantum Sun step's rule: s / width column groups (a power of
    two), tiles of ipt * 256 / groups rows within the operator and at least
    one grain block, at most 64 KB of tile."""
    groups = s // width
    if s % width or groups & (groups - 1):
        return False
    rows = ipt * 256 // groups
    return 2 ** op.L_grain <= rows <= op.dim and rows * s * elem <= 64 * 1024


@pytest.mark.parametrize("dts", ["fp64", "fp32"])
def test_every_step_variant_gives_identical_results(pkg, orc, cuda, models, dts):
    """The autotuner picks among columns-per-thread widths and (gather batch,
    register cap) profiles; all of them compute the same sums in the same
    order, so a K = 24 filter is bit-identical across variants."""
    dt = cuda.float64 if dts == "fp64" else cuda.float32
    elem = 8 if dts == "fp64" else 4
    s = 8
    rng = np.random.default_rng(9)
    plan = orc.build_transform_plan(("rescaled", 0.2), 10, 1.0, 0.0, order=24)
    coeffs = orc.filter_coefficients(plan)
    for name, op, H in models:
        D = H.shape[0]
        X = _dev(cuda, rng.standard_normal((D, s)), dt)
        Emax = float(np.abs(H).sum(axis=1).max())
        ref = None
        for width in (1, 2, 4, 8):
            if width * elem > 64:
                continue
            profiles = list(range(5))
            if op.kind == "qsun" and width * elem in (16, 32):
                profiles.append(5)                # asynchronous gathers
            for profile, ipt in ((6, 1), (8, 2), (9, 4)):   # shared-memory row tiles
                if op.kind == "qsun" and _tile_ok(op, s, width, elem, ipt):
                    profiles.append(profile)
            if op.kind == "spin_chain" and op.Lup >= 0:
                profiles.append(7)                # local flip-rank updates
            for profile in profiles:
                pkg.set_step_width(op, s, width, dts, profile=profile)
                assert pkg.step_variant(op, s, dts)[0] == width
                Y = pkg.col_major(D, s, dtype=dt)
                pkg.chebyshev_filter(op, Y, X, coeffs, a=1.01 * Emax, b=0.0)
                got = _host(Y)
                if ref is None:
                    ref = got
                else:
                    np.testing.assert_array_equal(got, ref, err_msg=f"{name} width={width} profile={profile}")
        pkg.set_step_width(op, s, min(8, 64 // elem), dts)


@pytest.mark.parametrize("dts", ["fp64", "fp32"])
def test_tiled_qsun_step_large(pkg, cuda, dts):
    """At D = 2^19 the tiled Quantum Sun steps have more tiles than CTAs (the
    persistent loop over tiles) and out-of-tile flips to every high bit; a
    K = 6 filter equals the default kernel's bit for bit."""
    dt = cuda.float64 if dts == "fp64" else cuda.float32
    elem = 8 if dts == "fp64" else 4
    s = 8
    rng = np.random.default_rng(19)
    fq, nq, cq, gq = pkg.qsun_parameters(16, 3, 0.75, rng=rng)
    op = pkg.QSunOperator(16, 3, 1.0, cq, nq, fq, gq)
    D = op.dim
    X = cuda.randn(s, D, dtype=dt, device="cuda:0", generator=cuda.Generator("cuda:0").manual_seed(3)).t()
    coeffs = np.array([0.3, -0.2, 0.15, 0.1, -0.05, 0.02, 0.01])
    width = 4 if elem == 8 else 8
    outs = {}
    for profile in (0, 6, 8, 9):
        pkg.set_step_width(op, s, width, dts, profile=profile)
        Y = pkg.col_major(D, s, dtype=dt)
        pkg.chebyshev_filter(op, Y, X, coeffs, a=40.0, b=0.0)
        outs[profile] = Y.cpu()
    for profile in (6, 8, 9):
        assert cuda.equal(outs[profile], outs[0]), f"profile {profile}"
    assert cuda.isfinite(outs[0]).all()


@pytest.mark.parametrize("dts", ["fp64", "fp32"])
def test_column_slabs_give_identical_filters(pkg, orc, cuda, models, dts):
    """Large blocks are filtered in column slabs (each step gathers from a
    slab that fits in L2); every column's arithmetic is unchanged, so forced
    slabs of 2 and 4 columns reproduce the whole-block filter bit for bit."""
    dt = cuda.float64 if dts == "fp64" else cuda.float32
    s = 8
    rng = np.random.default_rng(19)
    plan = orc.build_transform_plan(("rescaled", 0.1), 10, 1.0, 0.0, order=30)
    coeffs = orc.filter_coefficients(plan)
    for name, op, H in models:
        D = H.shape[0]
        X = _dev(cuda, rng.standard_normal((D, s)), dt)
        Emax = float(np.abs(H).sum(axis=1).max())
        out = {}
        for cols in (-1, 4, 2):
            pkg.set_filter_slab(op, cols)
            Y = pkg.col_major(D, s, dtype=dt)
            pkg.chebyshev_filter(op, Y, X, coeffs, a=1.01 * Emax, b=0.0)
            out[cols] = _host(Y)
        pkg.set_filter_slab(op, 0)
        np.testing.assert_array_equal(out[4], out[-1], err_msg=name)
        np.testing.assert_array_equal(out[2], out[-1], err_msg=name)


@pytest.mark.parametrize("D,nB,s", [(4099, 37, 5), (5000, 300, 8), (70000, 632, 16), (2048, 129, 32)])
def test_tensor_core_gram_split_bf16(pkg, cuda, D, nB, s):
    """pf_gram_bf16x3: G = B^T r on the tcgen05 tensor cores in split BF16
    (three BF16 products, FP32 accumulation, chunk sums in FP64) against the
    FP64 product; every entry within 1e-4 of |B[:, i]| |r[:, c]| (the split
    keeps ~16 mantissa bits of each factor), far better than one BF16 product."""
    from polfed_b200 import _lib
    rng = np.random.default_rng(D + nB + s)
    ldb = nB + 3                                     # a basis with spare columns, as in the solver
    Bh = rng.standard_normal((D, ldb)) / np.sqrt(D)
    rh = rng.standard_normal((D, s)) / np.sqrt(D)
    B = cuda.tensor(Bh, dtype=cuda.float64, device="cuda:0")        # row-major D x ldb
    r = cuda.tensor(rh, dtype=cuda.float64, device="cuda:0")        # row-major D x s
    G = cuda.zeros((s, nB), dtype=cuda.float64, device="cuda:0")    # column-major nB x s
    _lib.check(_lib.load().pf_gram_bf16x3(_lib.handle(0), D, nB, B.data_ptr(), ldb, r.data_ptr(), s, G.data_ptr()))
    got = G.cpu().numpy().T
    ref = Bh[:, :nB].T @ rh
    scale = np.outer(np.linalg.norm(Bh[:, :nB], axis=0), np.linalg.norm(rh, axis=0))
    err = np.abs(got - ref) / scale
    assert err.max() < 1e-4, err.max()
    # one rounding of each factor to BF16 alone is much worse
    bf = lambda x: cuda.tensor(x).to(cuda.bfloat16).to(cuda.float64).numpy()
    single = np.abs(bf(Bh[:, :nB]).T @ bf(rh) - ref) / scale
    assert err.max() < 0.2 * single.max()


def test_launch_overlap_leaves_results_unchanged(pkg, orc, cuda, models):
    """Step kernels launch with programmatic dependent launch (each waits for
    its predecessor's writes before reading a block); plain stream order
    gives the same filters and KPM moments bit for bit."""
    rng = np.random.default_rng(23)
    plan = orc.build_transform_plan(("rescaled", 0.3), 10, 1.0, 0.0, order=30)
    coeffs = orc.filter_coefficients(plan)
    try:
        for name, op, H in models:
            D = H.shape[0]
            Emax = float(np.abs(H).sum(axis=1).max())
            X = _dev(cuda, rng.standard_normal((D, 4)), cuda.float64)
            probes = rng.standard_normal((D, 8))
            probes /= np.linalg.norm(probes, axis=0)
            out = []
            for on in (True, False):
                pkg.set_launch_overlap(on)
                Y = pkg.col_major(D, 4)
                pkg.chebyshev_filter(op, Y, X, coeffs, a=1.01 * Emax, b=0.0)
                mu = pkg.kpm_moments(op, 40, 8, a=1.01 * Emax, b=0.0, probes=_dev(cuda, probes, cuda.float64))
                out.append((_host(Y), np.asarray(mu)))
            np.testing.assert_array_equal(out[0][0], out[1][0], err_msg=name)
            np.testing.assert_array_equal(out[0][1], out[1][1], err_msg=name)
    finally:
        pkg.set_launch_overlap(True)
