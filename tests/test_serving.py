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
