"""Serving loop on the GPU: each result is the same alone and in the mix (GPU).

Several client threads issue forward / transpose / adjoint requests of one or three right-hand
sides on two resident maps; the server coalesces them into multi-RHS blocks on concurrent stream
slots. Every result must equal
the same product computed alone (one right-hand side, through h2b_matvec_host) to a relative
1e-12 -- the blocked kernels sum each column in the same order as the single-column ones up to
FP64 rounding.
"""

import threading

import numpy as np
import pytest
import torch

import h2factory_b200 as h2
from h2factory_b200 import methods
from h2factory_b200.serving import GpuExecutor, MatvecServer
from h2factory_b200.trees import build_tree

pytestmark = pytest.mark.gpu


def _maps():
    rng = np.random.default_rng(21)
    t = build_tree(rng.random((3000, 3)), depth=4, root_center=[0.5] * 3, root_halfsize=0.5)
    a = methods.interpolation_core(t, methods.laplace, 3, nodes="equispaced", couplings="toeplitz",
                                   precision="fp32")
    t2 = build_tree(rng.random((2000, 3)), maxvalues=40, root_center=[0.5] * 3, root_halfsize=0.5)
    b = methods.interpolation_core(t2, methods.helmholtz(3.0), 3)
    return {"laplace-toeplitz-fp32": a, "helmholtz-cheb": b}


@pytest.mark.parametrize("device_requests", [False, True])
def test_results_alone_and_in_the_mix(device_requests):
    maps = _maps()
    alone = {k: h2.H2Workspace(c, max_nrhs=1) for k, c in maps.items()}
    srv = MatvecServer(GpuExecutor(0), budget_bytes=40e9, max_block=8, slots=2)
    for k, c in maps.items():
        srv.add_map(k, c)
    jobs = []
    lock = threading.Lock()

    def client(seed):
        r = np.random.default_rng(seed)
        for _ in range(12):
            key = list(maps)[r.integers(2)]
            core = maps[key]
            mode = int(r.integers(3))
            n = core.trial.npoints
            shape = (n, 3) if r.integers(3) == 0 else (n,)  # some requests carry 3 right-hand sides
            x = r.standard_normal(shape)
            if core.field == "complex":
                x = x + 1j * r.standard_normal(shape)
            xs = torch.from_numpy(x).to("cuda:0") if device_requests else x
            if device_requests:
                torch.cuda.synchronize()
            fut = srv.submit(key, xs, mode)
            y = fut.result(timeout=120)
            y = y.cpu().numpy() if device_requests else y
            with lock:
                jobs.append((key, mode, x, y))

    ts = [threading.Thread(target=client, args=(s,)) for s in range(6)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    st = srv.stats()
    srv.close()
    assert len(jobs) == 72
    assert st["mean_block"] >= 1.0
    assert any(x.ndim == 2 for _, _, x, _ in jobs)
    for key, mode, x, y in jobs:
        assert y.shape == x.shape
        for xc, yc in zip(x.reshape(x.shape[0], -1).T, y.reshape(y.shape[0], -1).T):
            want = alone[key].matvec_host(np.ascontiguousarray(xc), mode)
            assert np.linalg.norm(yc - want) / np.linalg.norm(want) < 1e-12, (key, mode)
