"""Serving loop scheduling (CPU): coalescing, orientation, admission, eviction, many clients.

The scheduler runs against DenseExecutor (each map a dense matrix), so these tests need no GPU; the
same scheduler drives the C ABI through GpuExecutor in tests/test_serving_gpu.py.
"""

import threading

import numpy as np
import pytest

from h2factory_b200.serving import AdmissionError, DenseExecutor, MatvecServer


def mats(rng, sizes, cplx=True):
    out = []
    for n in sizes:
        A = rng.standard_normal((n, n))
        if cplx:
            A = A + 1j * rng.standard_normal((n, n))
        out.append(A)
    return out


def test_results_all_orientations_and_coalescing():
    rng = np.random.default_rng(0)
    (A,) = mats(rng, [50])
    ex = DenseExecutor(delay=0.01)
    srv = MatvecServer(ex, budget_bytes=1e9, max_block=8, slots=1)
    srv.add_map("a", A)
    futs, xs = [], []
    for i in range(30):
        x = rng.standard_normal(50) + 1j * rng.standard_normal(50)
        mode = ("forward", "transpose", "adjoint")[i % 3]
        xs.append((x, mode))
        futs.append(srv.submit("a", x, mode))
    for (x, mode), f in zip(xs, futs):
        op = {"forward": A, "transpose": A.T, "adjoint": A.conj().T}[mode]
        assert np.allclose(f.result(timeout=10), op @ x, rtol=1e-13, atol=1e-12)
    st = srv.stats()
    srv.close()
    assert st["requests"] == 30
    assert st["mean_block"] > 1.0  # requests waiting behind a running block were coalesced
    assert max(srv.blocks) <= 8


def test_eviction_under_budget_and_reload():
    rng = np.random.default_rng(1)
    A, B = mats(rng, [40, 40])
    ex = DenseExecutor()
    one_map = ex.footprint(A, 4, 1)
    srv = MatvecServer(ex, budget_bytes=one_map * 1.5, max_block=4, slots=1)
    srv.add_map("a", A)
    srv.add_map("b", B)
    for i in range(6):
        key, M = (("a", A), ("b", B))[i % 2]
        x = rng.standard_normal(40)
        y = srv.submit(key, x).result(timeout=10)
        assert np.allclose(y, M @ x)
    assert ex.loads >= 6  # every switch evicted the idle map and reloaded the other
    assert srv.stats()["resident_maps"] == 1
    srv.close()


def test_admission_refused_when_map_exceeds_budget():
    rng = np.random.default_rng(2)
    (A,) = mats(rng, [64], cplx=False)
    srv = MatvecServer(DenseExecutor(), budget_bytes=100, max_block=4, slots=1)
    srv.add_map("big", A)
    fut = srv.submit("big", np.ones(64))
    with pytest.raises(AdmissionError):
        fut.result(timeout=10)
    srv.close()


def test_many_clients_each_result_as_if_alone():
    rng = np.random.default_rng(3)
    A, B = mats(rng, [30, 45])
    srv = MatvecServer(DenseExecutor(delay=0.002), budget_bytes=1e9, max_block=6, slots=2)
    srv.add_map("a", A)
    srv.add_map("b", B)
    errors = []

    def client(seed):
        r = np.random.default_rng(seed)
        for _ in range(20):
            key, M = (("a", A), ("b", B))[r.integers(2)]
            mode = ("forward", "transpose", "adjoint")[r.integers(3)]
            x = r.standard_normal(M.shape[0]) + 1j * r.standard_normal(M.shape[0])
            op = {"forward": M, "transpose": M.T, "adjoint": M.conj().T}[mode]
            y = srv.submit(key, x, mode).result(timeout=20)
            if not np.allclose(y, op @ x, rtol=1e-13, atol=1e-12):
                errors.append((key, mode))

    ts = [threading.Thread(target=client, args=(s,)) for s in range(8)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    st = srv.stats()
    srv.close()
    assert not errors
    assert st["requests"] == 160


def test_unknown_map_is_rejected():
    srv = MatvecServer(DenseExecutor(), budget_bytes=1e6)
    with pytest.raises(KeyError):
        srv.submit("missing", np.ones(3))
    srv.close()


def test_cancelled_requests_are_dropped_and_the_server_survives():
    """A client may cancel a request it no longer needs (an iterative solver that converged): a
    request cancelled before its block starts is dropped, the others are answered, and the
    scheduler keeps running."""
    rng = np.random.default_rng(5)
    (A,) = mats(rng, [30])
    srv = MatvecServer(DenseExecutor(delay=0.05), budget_bytes=1e9, max_block=4, slots=1)
    srv.add_map("a", A)
    xs = [rng.standard_normal(30) for _ in range(20)]
    futs = [srv.submit("a", x) for x in xs]
    cancelled = [f.cancel() for f in futs[8:16]]  # those still queued behind the first blocks
    assert any(cancelled)
    for x, f, c in zip(xs, futs, [False] * 8 + cancelled + [False] * 4):
        if c:
            assert f.cancelled()
        else:
            assert np.allclose(f.result(timeout=10), A @ x)
    assert np.allclose(srv.submit("a", xs[0]).result(timeout=10), A @ xs[0])  # still serving
    srv.close()


def test_a_client_that_dies_mid_stream_does_not_stop_the_others():
    """Clients are independent threads; one that dies after submitting (it never collects its
    result) leaves the server and the other clients' requests unaffected."""
    rng = np.random.default_rng(6)
    (A,) = mats(rng, [25])
    srv = MatvecServer(DenseExecutor(delay=0.002), budget_bytes=1e9, max_block=8, slots=2)
    srv.add_map("a", A)
    errors, done = [], []

    def client(i, die):
        r = np.random.default_rng(100 + i)
        for j in range(15):
            x = r.standard_normal(25)
            f = srv.submit("a", x, ("forward", "transpose", "adjoint")[j % 3])
            if die and j == 5:
                raise RuntimeError("client crashed")  # dies with a request in flight
            op = (A, A.T, A.conj().T)[j % 3]
            if not np.allclose(f.result(timeout=10), op @ x):
                errors.append((i, j))
        done.append(i)

    def run(i, die):
        try:
            client(i, die)
        except RuntimeError:
            pass

    ts = [threading.Thread(target=run, args=(i, i == 3)) for i in range(8)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=30)
    assert not errors and sorted(done) == [0, 1, 2, 4, 5, 6, 7]
    st = srv.stats()
    srv.close()
    assert st["requests"] >= 7 * 15 + 6  # the dead client's submitted requests were answered too


def test_replica_router_balances_maps_and_routes_requests():
    from h2factory_b200.serving import ReplicaRouter

    rng = np.random.default_rng(7)
    sizes = [40, 30, 40, 20, 30, 50]
    maps = mats(rng, sizes)
    exs = [DenseExecutor() for _ in range(3)]
    router = ReplicaRouter([MatvecServer(e, budget_bytes=1e9, max_block=4, slots=1) for e in exs])
    devs, load = [], [0, 0, 0]
    for i, M in enumerate(maps):
        need = exs[0].footprint(M, 4, 1)
        d = router.add_map(f"m{i}", M)
        assert load[d] == min(load)  # each map goes to the least-loaded device at its arrival
        load[d] += need
        devs.append(d)
    assert sorted(set(devs)) == [0, 1, 2] and router.assigned == load
    for i, M in enumerate(maps):
        x = rng.standard_normal(M.shape[0])
        assert np.allclose(router.submit(f"m{i}", x, "adjoint").result(timeout=10), M.conj().T @ x)
    st = router.stats()
    router.close()
    assert st["requests"] == len(maps)
    # each map was loaded by its own device only
    assert sum(e.loads for e in exs) == len(maps)
    for d, e in enumerate(exs):
        assert e.loads == devs.count(d)


def test_block_requests_mixed_with_vectors():
    """Requests of 1 and k right-hand sides share blocks; a block never exceeds max_block columns,
    every result has its request's shape, and a request wider than max_block is refused."""
    rng = np.random.default_rng(8)
    (A,) = mats(rng, [36])
    srv = MatvecServer(DenseExecutor(delay=0.005), budget_bytes=1e9, max_block=8, slots=1)
    srv.add_map("a", A)
    subs = []
    for i in range(40):
        k = (1, 3, 8, 1, 5)[i % 5]
        x = rng.standard_normal((36, k)) + 1j * rng.standard_normal((36, k))
        if k == 1 and i % 2:
            x = x[:, 0]
        mode = ("forward", "transpose", "adjoint")[i % 3]
        subs.append((x, mode, srv.submit("a", x, mode)))
    with pytest.raises(ValueError):
        srv.submit("a", np.zeros((36, 9)))
    for x, mode, f in subs:
        op = {"forward": A, "transpose": A.T, "adjoint": A.conj().T}[mode]
        y = f.result(timeout=10)
        assert y.shape == x.shape
        assert np.allclose(y, op @ x, rtol=1e-13, atol=1e-12)
    srv.close()
    assert max(srv.blocks) <= 8
    assert sum(srv.blocks) == sum(1 if x.ndim == 1 else x.shape[1] for x, _, _ in subs)


def test_inflight_cap_coalesces_and_serves_oldest_first():
    """With max_inflight blocks on the device at once, waiting requests coalesce into wider blocks
    and the queue whose oldest request waited longest launches next."""
    rng = np.random.default_rng(9)
    maps = mats(rng, [30, 30, 30], cplx=False)

    class Counting(DenseExecutor):
        def __init__(self):
            super().__init__(delay=0.01)
            self.live, self.peak, self.order = 0, 0, []

        def launch(self, slot, mode, xs):
            self.live += 1
            self.peak = max(self.peak, self.live)
            self.order.append(next(i for i, M in enumerate(maps) if slot.mat is M))
            return super().launch(slot, mode, xs)

        def results(self, slot, ticket, shapes):
            self.live -= 1
            return super().results(slot, ticket, shapes)

    ex = Counting()
    srv = MatvecServer(ex, budget_bytes=1e9, max_block=16, slots=2, max_inflight=1)
    for i, M in enumerate(maps):
        srv.add_map(i, M)
    subs = []
    for j in range(60):
        i = j % 3
        x = rng.standard_normal(30)
        subs.append((i, x, srv.submit(i, x)))
    for i, x, f in subs:
        assert np.allclose(f.result(timeout=20), maps[i] @ x)
    srv.close()
    assert ex.peak == 1
    assert np.mean(srv.blocks) > 3  # requests waited behind the single block and coalesced
    # round robin by age: no map waits for two launches of another while it has a request queued
    assert all(ex.order[k] != ex.order[k + 1] for k in range(min(6, len(ex.order) - 1)))


def test_open_loop_window_accounting(monkeypatch):
    """The serving benchmark's open-loop window (bench.py) against the CPU executor: arrivals follow
    the Poisson schedule, requests not started when the window closes are cancelled and dropped,
    every other request completes, and latency counts from the scheduled arrival."""
    import os
    import sys

    import torch

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    import bench

    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    rng = np.random.default_rng(12)
    maps = mats(rng, [24, 24], cplx=False)
    srv = MatvecServer(DenseExecutor(delay=0.004), budget_bytes=1e9, max_block=8, slots=1, max_inflight=1)
    for i, M in enumerate(maps):
        srv.add_map(i, M)
    xs = {(i, w): (rng.standard_normal(24) if w == 1 else rng.standard_normal((24, w))) for i in range(2) for w in (1, 4)}
    light = bench._open_loop(srv, xs, 2, 1, 200.0, 0.3, rng)      # well under capacity
    heavy = bench._open_loop(srv, xs, 2, 4, 20000.0, 0.3, rng)    # far over it
    srv.close()
    for r in (light, heavy):
        assert r["completed"] + r["cancelled"] == r["requests"]
        assert r["completed_in_window"] <= r["completed"]
        assert r["achieved_rhs_per_s"] == pytest.approx(r["achieved_req_per_s"] * r["rhs_per_request"])
    assert light["cancelled"] <= 2 and light["p99_ms"] < 100
    assert heavy["cancelled"] > 0 and heavy["mean_block_rhs"] > 4  # queued requests coalesced
    assert heavy["achieved_req_per_s"] < 20000.0
