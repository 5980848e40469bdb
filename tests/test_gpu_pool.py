"""The native request pool (pf_pool_*): batched and served solves.

Every request in a pool runs the same solve as pf_solve on its own worker
handle, so a problem must give the same eigenpairs whether it is solved
alone or among others running at the same time: eigenvalues equal to 1e-10
relative, each vector with an FP64 residual below the eigen tolerance.  The
served path (submit / poll / result) must admit requests only while their
footprints fit the HBM budget, keep FIFO order, release failed and cancelled
requests, and report latency percentiles.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NEV = 8
TARGET = ("rescaled", 0.5)
EIGENTOL = 1e-9


def _kw(pkg, seed):
    return dict(fact=pkg.FactorizationConfig(eigentol=EIGENTOL, overestimate_iters=2.0),
                dos=pkg.DoSConfig(N=64, R=16, seed=seed))


def _problems(pkg, orc):
    """Three operators of different kinds and sizes; two share one operator."""
    rng = np.random.default_rng(5)
    out = []
    f = 5 * (2 * rng.random(12) - 1)
    xxz = pkg.xxz_hamiltonian(12, 6, 1.0, 1.0, 0.0, fields=f)
    out.append((xxz, orc.xxz_matrix(12, 6, 1.0, 1.0, f), 1))
    f2 = 4 * (2 * rng.random(12) - 1)
    j1j2 = pkg.j1j2_hamiltonian(12, 6, 1.0, 0.5, 1.0, 0.8, 0.0, fields=f2)
    out.append((j1j2, orc.j1j2_matrix(12, 6, 1.0, 0.5, 1.0, 0.8, f2), 2))
    fq, nq, cq, gq = pkg.qsun_parameters(7, 3, 0.75, rng=rng)
    qsun = pkg.QSunOperator(7, 3, 1.0, cq, nq, fq, gq)
    out.append((qsun, orc.qsun_matrix(7, 3, 1.0, cq, nq, fq, gq), 4))
    out.append((xxz, out[0][1], 2))   # the XXZ operator again, with a block start
    return out, rng


def _x0(rng, D, s):
    return rng.random(D) if s == 1 else rng.random((D, s))


def _residuals_ok(H, vals, vecs):
    for j in range(len(vals)):
        v = vecs[:, j]
        assert np.linalg.norm(H @ v - vals[j] * v) < EIGENTOL * 10


def test_batch_matches_each_problem_alone(pkg, orc, cuda):
    probs, rng = _problems(pkg, orc)
    x0s = [_x0(rng, H.shape[0], s) for _, H, s in probs]
    for op, _, s in probs:   # same step width alone and in the mix
        pkg.autotune(op, s, "fp64")
    alone = [pkg.polfed(op, x0, NEV, TARGET, **_kw(pkg, 11 + i)) for i, ((op, _, _), x0) in enumerate(zip(probs, x0s))]
    with pkg.SolverPool(workers=4) as pool:
        # solve_batch takes one parameter set; run the problems one seed at a time in a mix with the others
        mixed = []
        for i in range(len(probs)):
            order = [i] + [j for j in range(len(probs)) if j != i]
            res = pool.solve_batch([probs[j][0] for j in order], [x0s[j] for j in order], NEV, TARGET,
                                   **_kw(pkg, 11 + i))
            mixed.append(res[0])
        st = pool.stats()
    for (op, H, s), (va, Va), (vm, Vm) in zip(probs, alone, mixed):
        assert len(va) == len(vm) and len(va) >= 1
        assert np.max(np.abs(va - vm) / np.maximum(1, np.abs(va))) < 1e-10
        _residuals_ok(H, vm, Vm)
    assert st.completed == 4 * len(probs) and st.failed == 0
    assert st.eigenpairs >= sum(len(v) for v, _ in mixed)


def test_batch_with_device_inputs(pkg, orc, cuda):
    probs, rng = _problems(pkg, orc)
    hx = [_x0(rng, H.shape[0], s) for _, H, s in probs]
    dx = []
    for x in hx:
        x2 = x.reshape(x.shape[0], -1)
        t = pkg.col_major(x2.shape[0], x2.shape[1])
        t.copy_(cuda.from_numpy(np.ascontiguousarray(x2)).to("cuda:0"))
        dx.append(t if x.ndim == 2 else t[:, 0].contiguous())
    ops = [p[0] for p in probs]
    pool = pkg.solver_pool(3)
    host = pool.solve_batch(ops, hx, NEV, TARGET, **_kw(pkg, 3))
    dev = pool.solve_batch(ops, dx, NEV, TARGET, **_kw(pkg, 3))
    for (op, H, s), (vh, _), (vd, Vd) in zip(probs, host, dev):
        assert Vd.is_cuda
        assert np.max(np.abs(vh - vd) / np.maximum(1, np.abs(vh))) < 1e-10
        _residuals_ok(H, vd, Vd.cpu().numpy())


def test_served_stream_respects_budget_and_order(pkg, orc, cuda):
    probs, rng = _problems(pkg, orc)
    op, H, s = probs[2]
    fp = pkg.SolverPool.footprint(op, NEV, TARGET, s, **_kw(pkg, 0))
    assert fp > 8 * H.shape[0] * NEV
    # room for one request at a time although three workers are free
    with pkg.SolverPool(workers=3, hbm_budget=1.5 * fp) as pool:
        ids = [pool.submit(op, _x0(rng, H.shape[0], s), NEV, TARGET, **_kw(pkg, 20 + k)) for k in range(4)]
        states = [pool.poll(r) for r in ids]
        assert states[-1] == "queued"
        res = [pool.result(r) for r in ids]
        st = pool.stats()
    for vals, vecs in res:
        assert len(vals) >= 1
        _residuals_ok(H, vals, vecs)
    assert st.completed == 4 and st.queued == 0 and st.running == 0
    assert st.bytes_peak <= 1.5 * fp + 1
    assert st.bytes_in_use == 0
    assert 0 < st.p50_latency <= st.p99_latency
    assert st.busy_seconds > 0


def test_failed_and_cancelled_requests_are_released(pkg, orc, cuda):
    probs, rng = _problems(pkg, orc)
    op, H, s = probs[0]
    D = H.shape[0]
    with pkg.SolverPool(workers=1) as pool:
        bad = pool.submit(op, np.zeros(D), NEV, TARGET, **_kw(pkg, 1))      # zero start vector
        good = pool.submit(op, _x0(rng, D, 1), NEV, TARGET, **_kw(pkg, 2))
        dropped = pool.submit(op, _x0(rng, D, 1), NEV, TARGET, **_kw(pkg, 3))
        pool.cancel(dropped)
        with pytest.raises(pkg._lib.PolfedArgumentError, match="nonzero"):
            pool.result(bad)
        vals, vecs = pool.result(good)
        _residuals_ok(H, vals, vecs)
        with pytest.raises(pkg._lib.PolfedArgumentError, match="unknown request"):
            pool.poll(dropped)
        st = pool.stats()
    assert st.failed == 1 and st.completed == 1 and st.submitted == 3


def test_cancelling_a_running_request_keeps_its_arrays(pkg, orc, cuda):
    """A request that has already started runs to the end after cancel and its
    worker still writes the host result arrays: the pool keeps them alive
    until it is closed, and goes on serving."""
    probs, rng = _problems(pkg, orc)
    op, H, s = probs[0]
    D = H.shape[0]
    big = pkg.xxz_hamiltonian(16, 8, 1.0, 1.0, 5.0, rng=np.random.default_rng(3))
    with pkg.SolverPool(workers=1) as pool:
        r = pool.submit(big, np.random.default_rng(4).random(big.dim), NEV, TARGET, **_kw(pkg, 5))
        for _ in range(2000):
            if pool.poll(r) != "queued":
                break
            time.sleep(0.005)
        pool.cancel(r)
        assert len(pool._cancelled) == 1
        vals, vecs = pool.result(pool.submit(op, _x0(rng, D, 1), NEV, TARGET, **_kw(pkg, 6)))
        _residuals_ok(H, vals, vecs)
    assert pool._cancelled == []


def _blocked_pool_order(pkg, policy, max_wait):
    """One worker: a blocker runs, then an earlier large and a later small
    request wait; returns the two waiting requests' start times (seconds)."""
    rng = np.random.default_rng(21)
    small = pkg.xxz_hamiltonian(12, 6, 1.0, 1.0, 5.0, rng=rng)       # D = 924
    large = pkg.xxz_hamiltonian(16, 8, 1.0, 1.0, 5.0, rng=rng)       # D = 12870
    kw = _kw(pkg, 4)
    with pkg.SolverPool(workers=1) as pool:
        pool.set_admission(policy, max_wait=max_wait)
        blocker = pool.submit(large, rng.random(large.dim), NEV, TARGET, **kw)
        big = pool.submit(large, rng.random(large.dim), NEV, TARGET, **kw)
        little = pool.submit(small, rng.random(small.dim), NEV, TARGET, **kw)
        assert pool.poll(big) == "queued" and pool.poll(little) == "queued"
        pool.result(blocker)
        tb, tl = None, None
        for rid in (big, little):
            pool.wait(rid)
        tb, tl = pool.times(big), pool.times(little)
        vb, _ = pool.result(big)
        vl, _ = pool.result(little)
    assert len(vb) >= 1 and len(vl) >= 1
    assert tb[0] < tl[0]                     # submitted in this order
    assert tb[1] >= 0 and tl[1] >= 0 and tb[2] >= tb[1] and tl[2] >= tl[1]
    return tb[1], tl[1]


def test_shortest_first_admission_lets_small_requests_pass(pkg, orc, cuda):
    """PF_ADMIT_SHORTEST: behind a running request, a later small request
    starts before an earlier large one."""
    t_big, t_little = _blocked_pool_order(pkg, "shortest", 600.0)
    assert t_little < t_big


def test_aged_requests_keep_arrival_order(pkg, orc, cuda):
    """PF_ADMIT_SHORTEST with max_wait = 0: every queued request has aged, so
    arrival order comes back (the large request starts first)."""
    t_big, t_little = _blocked_pool_order(pkg, "shortest", 0.0)
    assert t_big < t_little


def test_fifo_admission_keeps_arrival_order(pkg, orc, cuda):
    t_big, t_little = _blocked_pool_order(pkg, "fifo", 30.0)
    assert t_big < t_little


def test_infeasible_request_is_rejected(pkg, orc, cuda):
    """Requests the reference's planning cannot meet are rejected with its
    bisection error, counted apart from failures, and the pool goes on
    serving: more states than the whole space (the interval bisection), and
    a target near the spectrum's edge for which no order meets the cutoff
    (the order bisection; the oracle fails the same request the same way,
    with the same explicit KPM probes)."""
    probs, rng = _problems(pkg, orc)
    op, H, s = probs[0]
    D = H.shape[0]
    probes = orc.normalized_gaussian_probes(D, 24, np.random.default_rng(5))
    x_edge = np.random.default_rng(4).random(D)
    with pytest.raises(Exception, match="opposite signs"):
        orc.plan_only(orc.CSROperator(H), x_edge, 50, ("rescaled", 0.8), N=96, probes=probes)
    # the same kind of request with the pool's seeded probes: the first edge
    # target that the direct solve cannot plan
    dos = pkg.DoSConfig(N=96, R=24, seed=3)
    edge = None
    for eps in (0.8, 0.85, 0.9, 0.95):
        for nev in (50, 20):
            try:
                pkg.polfed(op, x_edge, nev, ("rescaled", eps), vecs=False, dos=dos)
            except pkg._lib.PolfedError as e:
                if "opposite signs" in str(e):
                    edge = (("rescaled", eps), nev)
                    break
        if edge:
            break
    assert edge is not None
    with pkg.SolverPool(workers=1) as pool:
        bad = pool.submit(op, _x0(rng, D, 1), D + 5, TARGET, **_kw(pkg, 1))
        bad2 = pool.submit(op, x_edge, edge[1], edge[0], vecs=False, dos=dos)
        good = pool.submit(op, _x0(rng, D, 1), NEV, TARGET, **_kw(pkg, 2))
        for r in (bad, bad2):
            assert pool.wait(r) == "rejected"
            with pytest.raises(pkg._lib.PolfedRejected, match="opposite signs"):
                pool.result(r)
        vals, vecs = pool.result(good)
        _residuals_ok(H, vals, vecs)
        st = pool.stats()
    assert st.rejected == 2 and st.failed == 0 and st.completed == 1


def test_destroy_wakes_waiting_threads(pkg, orc, cuda):
    """Closing a pool while another thread waits for a queued request fails
    that request ("pool destroyed") and returns the waiting thread."""
    import threading
    import time
    rng = np.random.default_rng(8)
    op = pkg.xxz_hamiltonian(16, 8, 1.0, 1.0, 5.0, rng=rng)       # D = 12870: the first solve takes a while
    D = op.dim
    pool = pkg.SolverPool(workers=1)
    pool.submit(op, rng.random(D), NEV, TARGET, **_kw(pkg, 1))
    queued = [pool.submit(op, rng.random(D), NEV, TARGET, **_kw(pkg, 2 + k)) for k in range(3)]
    outcome = {}

    def waiter():
        try:
            pool.result(queued[-1])
            outcome["r"] = "done"
        except pkg._lib.PolfedError as e:
            outcome["r"] = str(e)

    t = threading.Thread(target=waiter)
    t.start()
    time.sleep(0.5)                  # the waiter is now blocked in the native fetch
    pool.close()
    t.join(timeout=120)
    assert not t.is_alive()
    assert "pool destroyed" in outcome["r"] or "pool is closed" in outcome["r"], outcome


def test_batched_filter_matches_unbatched_uneven_dims(pkg, orc, cuda):
    """The filter engine runs the Clenshaw steps of every solve in flight as
    one launch per step.  Chain operators of different dimensions (XXZ L = 12,
    13, 14 and a J1-J2 L = 12 chain) and two Quantum Sun operators, all with
    s = 4, solved together with batching on, give the eigenpairs each gives
    alone on its own graph-captured filter, and the launches are shared."""
    rng = np.random.default_rng(31)
    probs = []
    for L in (12, 13, 14):
        f = 4 * (2 * rng.random(L) - 1)
        probs.append((pkg.xxz_hamiltonian(L, L // 2, 1.0, 1.0, 0.0, fields=f), orc.xxz_matrix(L, L // 2, 1.0, 1.0, f)))
    f = 3 * (2 * rng.random(12) - 1)
    probs.append((pkg.j1j2_hamiltonian(12, 6, 1.0, 0.5, 1.0, 0.8, 0.0, fields=f),
                  orc.j1j2_matrix(12, 6, 1.0, 0.5, 1.0, 0.8, f)))
    for Lloc in (7, 8):
        fq, nq, cq, gq = pkg.qsun_parameters(Lloc, 3, 0.75, rng=rng)
        probs.append((pkg.QSunOperator(Lloc, 3, 1.0, cq, nq, fq, gq), orc.qsun_matrix(Lloc, 3, 1.0, cq, nq, fq, gq)))
    x0s = [rng.random((H.shape[0], 4)) for _, H in probs]
    for op, _ in probs:
        pkg.autotune(op, 4, "fp64")
    alone = [pkg.polfed(op, x0, NEV, TARGET, **_kw(pkg, 40)) for (op, _), x0 in zip(probs, x0s)]
    with pkg.SolverPool(workers=len(probs)) as pool:
        pool.set_batching(True)
        res = pool.solve_batch([op for op, _ in probs], x0s, NEV, TARGET, **_kw(pkg, 40))
        st = pool.stats()
    for (op, H), (va, _), (vb, Vb) in zip(probs, alone, res):
        assert len(va) == len(vb) and len(vb) >= 1
        assert np.max(np.abs(va - vb) / np.maximum(1, np.abs(va))) < 1e-12
        _residuals_ok(H, vb, Vb)
    assert st.filter_launches > 0
    assert st.filter_instance_steps > 1.2 * st.filter_launches   # launches served several solves
    assert st.filter_bytes > 0 and st.filter_seconds > 0
