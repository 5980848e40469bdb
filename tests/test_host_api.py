"""Host-side logic and the C-ABI library's presence (CPU only, no compute calls)."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "polfed_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(pf_[a-z_0-9]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.load_library()
    declared = _declared_symbols()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/polfed_b200.h but not exported"
    assert lib.pf_abi_version() == 1


def test_struct_mirrors_match_the_library(pkg):
    """The ctypes mirrors of pf_params, pf_report and pf_pool_stats have the
    library's own sizes (a field added on one side only shows here)."""
    from polfed_b200 import _lib
    sz = [ctypes.c_size_t() for _ in range(3)]
    _lib.load().pf_abi_sizes(*[ctypes.byref(x) for x in sz])
    assert sz[0].value == ctypes.sizeof(_lib.pf_params)
    assert sz[1].value == ctypes.sizeof(_lib.pf_report)
    assert sz[2].value == ctypes.sizeof(_lib.pf_pool_stats)


def test_params_defaults_match_reference(pkg):
    from polfed_b200 import _lib
    p = _lib.pf_params()
    _lib.load().pf_params_default(ctypes.byref(p))
    # PolfedDefaults.jl:119-217, Plan.jl:143
    assert p.cutoff == 0.17 and p.normalization == 1.0 and p.order_safety_factor == 0.97
    assert p.tol == 1e-14 and p.eigentol == 1e-9 and p.overestimate_iters == 1.25
    assert p.which == _lib.PF_WHICH_LR and p.dos_N == 250 and p.dos_R == 300
    assert p.dos_kernel == _lib.KERNEL_IDS["Jackson"] and p.extrema_maxdim == 1000
    assert p.precision == _lib.PF_PREC_FP64 and p.reorth_passes == 1
    assert p.refine == 4          # FP64 refinement passes of a mixed-precision solve


def test_target_spec(pkg):
    from polfed_b200 import _lib
    n = pkg.normalize_target_spec
    assert n("maxdos") == (_lib.PF_TARGET_MAXDOS, 0.0)
    assert n("middle") == (_lib.PF_TARGET_MIDDLE, 0.0)
    assert n(("offset", 0.25)) == (_lib.PF_TARGET_OFFSET, 0.25)
    assert n(("unrescaled", -1.2)) == (_lib.PF_TARGET_UNRESCALED, -1.2)
    assert n(0.7) == (_lib.PF_TARGET_UNRESCALED, 0.7)
    assert n(("rescaled", 0.4)) == (_lib.PF_TARGET_RESCALED, 0.4)
    for bad in ["unknown", ("offset", 1.5), ("offset", "0.2"), ("absolute", 0.0), ("quantile", 0.5),
                ("other", 0.0), True]:
        with pytest.raises(ValueError):
            n(bad)


def test_krylov_dim(pkg):
    # PolfedDefaults.jl:61-62 and the shapes quoted for the benchmark configurations
    assert pkg.expectedkrylovdim(20, 1, 1.25) == 68
    assert pkg.expectedkrylovdim(200, 8, 1.25) == 629
    assert pkg.expectedkrylovdim(100, 16, 1.25) == 621
    assert pkg.expectedkrylovdim(3, 2, 1.0) == 46


def test_chain_bonds_and_models(pkg, orc):
    for L in (2, 3, 4, 7):
        for d in (1, 2):
            for bc in ("open", "periodic"):
                assert pkg.chain_bonds(L, d, bc) == orc.chain_bonds(L, d, bc)
    op = pkg.xxz_hamiltonian(6, 3, 1.0, 0.8, 0.0, fields=[0.1] * 6)
    assert op.expected_dim() == 20 and len(op.bonds) == 6
    op = pkg.j1j2_hamiltonian(6, 3, 1.0, 0.5, 1.0, 1.0, 0.0, fields=[0.0] * 6)
    assert len(op.bonds) == 12
    assert op.couplings.tolist() == [1.0] * 6 + [0.5] * 6
    rng = np.random.default_rng(0)
    op = pkg.xxz_hamiltonian(8, 4, 1.0, 1.0, 3.0, rng=rng)
    assert np.all(np.abs(op.fields) <= 3.0)
    for bad in [dict(L=1, Lup=0), dict(L=4, Lup=-2), dict(L=4, Lup=5)]:
        with pytest.raises(ValueError):
            pkg.xxz_hamiltonian(bad["L"], bad["Lup"], 1.0, 1.0, 0.0)
    with pytest.raises(ValueError):
        pkg.xxz_hamiltonian(4, 2, 1.0, 1.0, 0.0, boundary="twisted")
    with pytest.raises(ValueError):
        pkg.xxz_hamiltonian(4, 2, 1.0, 1.0, 0.0, fields=[0.0, 1.0])
    with pytest.raises(ValueError):
        pkg.xxz_hamiltonian(4, 2, 1.0, 1.0, -1.0)
    with pytest.raises(ValueError):
        pkg.j1j2_hamiltonian(4, 2, 1.0, 0.5, 1.0, 0.8, -1.0)


def test_qsun_parameters(pkg):
    rng = np.random.default_rng(11)
    f, n, c, g = pkg.qsun_parameters(13, 3, 0.75, zeta=0.2, hz=1.0, w=0.5, gamma=1.0, rng=rng)
    assert f.shape == (13,) and np.all((f >= 0.5) & (f <= 1.5))
    assert n.shape == (13,) and np.all((n >= 0) & (n < 3))
    assert c[0] == 1.0
    for j in range(2, 14):
        u = math.log(c[j - 1]) / math.log(0.75)
        assert (j - 1) - 0.2 <= u <= (j - 1) + 0.2
    assert g.shape == (8, 8) and np.allclose(g, g.T)
    op = pkg.qsun_hamiltonian(13, 3, 1.0, 0.75, rng=np.random.default_rng(1))
    assert op.L_loc == 13 and op.grain.shape == (8, 8)
    # spin S > 1/2 and the total-S_z sector: device-built CSR operators
    op1 = pkg.qsun_hamiltonian(4, 2, 1.0, 0.5, S=1.0, rng=np.random.default_rng(2))
    assert isinstance(op1, pkg.QSunSpinOperator) and op1.grain.shape == (9, 9)
    op2 = pkg.qsun_hamiltonian(4, 2, 1.0, 0.5, use_U1=True, S_z=1.0, rng=np.random.default_rng(2))
    assert isinstance(op2, pkg.QSunSpinOperator) and op2.use_U1 and op2.grain.shape == (4, 4)
    with pytest.raises(ValueError):
        pkg.qsun_hamiltonian(4, 2, 1.0, 0.5, S=0.3)
    with pytest.raises(ValueError, match="Wrong total value of spin"):
        pkg.qsun_hamiltonian(4, 2, 1.0, 0.5, use_U1=True, S_z=0.5)


def test_pool_refuses_without_a_device_and_footprint_guards(pkg):
    """With no CUDA device the pool is refused with a status (no host fallback),
    and the footprint query rejects null arguments."""
    import ctypes
    import torch
    from polfed_b200 import _lib
    lib = pkg.load_library()
    assert lib.pf_solve_footprint(None, None, 1, 1) == -1.0
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(_lib.PolfedError):
        pkg.SolverPool(workers=2)
    out = ctypes.c_void_p()
    assert lib.pf_pool_create(0, 0, 0.0, ctypes.byref(out)) == _lib.PF_ERR_INVALID   # 0 workers
    assert not out.value


def test_sparse_operator_host_validation(pkg):
    """Matrix input is checked on the host before any device work: square,
    a complex matrix Hermitian on its diagonal, consistent CSR arrays; a dense
    matrix becomes the same CSR as scipy's."""
    import scipy.sparse as sp
    with pytest.raises(ValueError, match="square"):
        pkg.SparseOperator(np.zeros((3, 4)))
    # complex input is a Hermitian operator (real diagonal checked on the host)
    herm = pkg.SparseOperator(sp.csr_matrix(np.array([[1.0, 2j], [-2j, 3.0]])))
    assert herm.is_complex and herm.complex_dim == 2
    with pytest.raises(ValueError, match="real diagonal"):
        pkg.SparseOperator(sp.csr_matrix(np.eye(3) * 1j))
    with pytest.raises(ValueError):
        pkg.SparseOperator((np.array([0, 1]), np.array([0, 0]), np.array([1.0])))
    A = sp.random(40, 40, density=0.2, random_state=3)
    A = (A + A.T).tocsr()
    A.sort_indices()
    d = pkg.SparseOperator(A.toarray())
    np.testing.assert_array_equal(d.indptr, A.indptr)
    np.testing.assert_array_equal(d.indices, A.indices)
    np.testing.assert_array_equal(d.values, A.data)


@pytest.mark.parametrize("S,L_loc,L_grain,S_z", [(0.5, 4, 2, 0.0), (1.0, 3, 2, 1.0), (1.5, 2, 2, 1.0)])
def test_qsun_spin_grain_normalisation(pkg, orc, S, L_loc, L_grain, S_z):
    """The sector's grain block is the GOE masked to equal grain magnetisation
    and scaled so that tr(R^2) / dim = gamma^2 for its embedding R in the
    sector (QuantumSun_U1_conserving.jl:34-90): the oracle's R (fields and
    couplings zero) has exactly the host-side block's entries."""
    rng = np.random.default_rng(4)
    f, n, c, goe = pkg.qsun_spin_parameters(L_loc, L_grain, 0.75, S, rng=rng)
    g = pkg.qsun_spin_grain(goe, L_loc, L_grain, S, gamma=1.3, use_U1=True, S_z=S_z)
    R = orc.qsun_spin_matrix(L_loc, L_grain, 0.0, c, n, np.zeros(L_loc), goe, S=S, gamma=1.3, use_U1=True,
                             S_z=S_z).toarray()
    assert abs(np.trace(R @ R) / R.shape[0] - 1.3 ** 2) < 1e-12
    d = int(round(2 * S)) + 1
    B = orc._SpinBasis(S)
    states = orc._spin_states(L_loc + L_grain, B)
    mag = np.array([sum(B.get_spin(st, j) for j in range(L_loc + L_grain)) for st in states])
    sector = np.nonzero(mag == S_z)[0]
    K = np.kron(np.eye(d ** L_loc), g)[np.ix_(sector, sector)]
    np.testing.assert_allclose(R, K, rtol=1e-13, atol=1e-15)
    assert pkg.spin_sector_count(L_loc + L_grain, d, int(round(S_z + (L_loc + L_grain) * S))) == R.shape[0]


def test_host_result_buffers_are_column_major(pkg):
    """Eigenvector buffers for host results: column-major D x m, real or
    complex (page-locked through torch's caching host allocator when CUDA is
    present, plain memory otherwise); a leading-column view stays contiguous."""
    from polfed_b200 import core
    for dt in (np.float64, np.complex128):
        V = core._host_out(37, 5, dt)
        assert V.shape == (37, 5) and V.dtype == dt and V.flags["F_CONTIGUOUS"]
        assert V[:, :3].flags["F_CONTIGUOUS"]
