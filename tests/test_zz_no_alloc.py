"""pf_apply_noalloc: the operator apply for callers that cannot let the library allocate.

Callers whose device memory is owned by a pool allocator (a CuArray pool, a
caching allocator holding the whole HBM budget) or that cannot absorb
cudaMalloc's implicit synchronisation use this entry point instead of
pf_apply.  It must give pf_apply's result, call after call (the fixed scratch
array it stages blocks in keeps the previous call's data), without changing
the device's free memory, and it must refuse blocks that do not fit its
16 MiB array.  Every call goes through the C ABI.  This file is collected last
so that a run stopping at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = {"fp64": 1e-12, "fp32": 2e-5}   # the operator-parity tolerances of the other GPU tests


def _abi(pkg):
    from polfed_b200 import _lib
    return _lib, _lib.load()


def _call(lib, name, op, dt, a, b, X, Y):
    D, s = X.shape
    return getattr(lib, name)(op.op, dt, a, b, s, X.data_ptr(), max(X.stride(1), D) if s > 1 else D,
                              Y.data_ptr(), max(Y.stride(1), D) if s > 1 else D)


def _models(pkg):
    rng = np.random.default_rng(77)
    f = 4 * (2 * rng.random(14) - 1)
    chain = pkg.j1j2_hamiltonian(14, 7, 1.0, 0.5, 1.0, 0.8, 0.0, fields=f)
    fq, nq, cq, gq = pkg.qsun_parameters(9, 3, 0.75, rng=rng)
    qsun = pkg.QSunOperator(9, 3, 1.0, cq, nq, fq, gq)
    return [("j1j2_L14", chain), ("qsun_9_3", qsun)]


@pytest.mark.parametrize("dtype", ["fp64", "fp32"])
@pytest.mark.parametrize("s", [1, 8])
def test_noalloc_matches_pf_apply_twice(pkg, cuda, dtype, s):
    _lib, lib = _abi(pkg)
    tdt = cuda.float64 if dtype == "fp64" else cuda.float32
    dt = _lib.PF_F64 if dtype == "fp64" else _lib.PF_F32
    for name, op in _models(pkg):
        D = op.dim
        a, b = 2.5, -0.3
        for call in range(2):   # two calls in a row: the second must not see the first's leftovers
            X = pkg.col_major(D, s, dtype=tdt)
            X.copy_(cuda.randn(D, s, dtype=tdt, device="cuda:0", generator=cuda.Generator("cuda:0").manual_seed(call)))
            ref = pkg.col_major(D, s, dtype=tdt)
            got = pkg.col_major(D, s, dtype=tdt)
            got.fill_(float("nan"))
            cuda.cuda.synchronize()
            _lib.check(_call(lib, "pf_apply", op, dt, a, b, X, ref))
            _lib.check(_call(lib, "pf_apply_noalloc", op, dt, a, b, X, got))
            _lib.synchronize(op.handle)
            err = (got - ref).norm().item() / ref.norm().item()
            assert err < RTOL[dtype], (name, s, dtype, call, err)


def test_noalloc_leaves_free_memory_unchanged(pkg, cuda):
    _lib, lib = _abi(pkg)
    name, op = _models(pkg)[1]
    D, s = op.dim, 8
    X = pkg.col_major(D, s)
    X.copy_(cuda.randn(D, s, dtype=cuda.float64, device="cuda:0"))
    Y = pkg.col_major(D, s)
    _lib.check(_call(lib, "pf_apply_noalloc", op, _lib.PF_F64, 1.0, 0.0, X, Y))   # per-device set-up
    _lib.synchronize(op.handle)
    free0, _ = cuda.cuda.mem_get_info(0)
    for _ in range(3):
        _lib.check(_call(lib, "pf_apply_noalloc", op, _lib.PF_F64, 1.0, 0.0, X, Y))
    _lib.synchronize(op.handle)
    free1, _ = cuda.cuda.mem_get_info(0)
    assert free1 == free0


def test_noalloc_rejects_blocks_beyond_its_scratch(pkg, cuda):
    _lib, lib = _abi(pkg)
    name, op = _models(pkg)[1]               # D = 4096
    D = op.dim
    s = (16 << 20) // (2 * D * 8) * 2        # twice the largest FP64 block that fits
    X = pkg.col_major(D, s)
    Y = pkg.col_major(D, s)
    st = _call(lib, "pf_apply_noalloc", op, _lib.PF_F64, 1.0, 0.0, X, Y)
    assert st == _lib.PF_ERR_INVALID
    assert b"16 MiB" in lib.pf_last_error()
    # the largest block that fits is accepted
    s_ok = (16 << 20) // (2 * D * 8)
    X2 = pkg.col_major(D, s_ok)
    X2.zero_()
    Y2 = pkg.col_major(D, s_ok)
    _lib.check(_call(lib, "pf_apply_noalloc", op, _lib.PF_F64, 1.0, 0.0, X2, Y2))
    _lib.synchronize(op.handle)
    assert float(Y2.abs().max()) == 0.0
