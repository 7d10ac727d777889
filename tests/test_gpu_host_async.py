"""h2b_matvec_host_async (GPU): requests on host arrays enqueued on two workspaces and two
streams, with no wait between them, give the same results as the synchronous h2b_matvec_host and
the oracle (relative L2 1e-12, FP64 form), and the FP32 form within 1e-6 of its FP64 product."""

import copy

import numpy as np
import pytest
import torch

import h2factory_b200 as h2
from oracle import oracle
from test_gpu_parity import CASES, _x, rel

pytestmark = pytest.mark.gpu


def _pinned(a):
    """A Fortran-ordered copy of `a` in page-locked host memory (asynchronous copies)."""
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).pin_memory()
    return t.numpy().T


@pytest.mark.parametrize("name,nrhs", [("toeplitz-laplace", 4), ("cheb-helmholtz", 3)])
def test_host_async_two_workspaces(name, nrhs):
    core = CASES[name]()
    wss = [h2.H2Workspace(core, max_nrhs=nrhs) for _ in range(2)]
    streams = [torch.cuda.Stream() for _ in range(2)]
    n = core.test.npoints
    nreq = 6
    xs = [_x(core, nrhs, 40 + i, mode=i % 3) for i in range(nreq)]
    xp = [_pinned(x) for x in xs]
    yp = [_pinned(np.zeros((n, nrhs), dtype=core.dtype)) for _ in range(nreq)]
    for i in range(nreq):  # all enqueued before any result is read
        j = i % 2
        wss[j].matvec_host_async(xp[i], yp[i], i % 3, stream=streams[j].cuda_stream)
    torch.cuda.synchronize()
    desc = h2.flatten(core)
    for i in range(nreq):
        want = oracle.matvec(core, xs[i], i % 3, desc=desc)
        assert rel(yp[i], want) < 1e-12, (name, i)
        assert np.array_equal(yp[i], wss[i % 2].matvec_host(xs[i], i % 3)), (name, i)
    for w in wss:
        w.close()


def test_host_async_fp32_form_and_reuse():
    """One workspace, consecutive requests on one stream reuse its staging buffers: each result is
    that of its own input (the next request's copy in waits for the previous copy out)."""
    core = CASES["toeplitz-laplace"]()
    c32 = copy.copy(core)
    c32.precision = "fp32"
    ws64 = h2.H2Workspace(core, max_nrhs=8)
    ws32 = h2.H2Workspace(c32, max_nrhs=8)
    st = torch.cuda.Stream()
    n = core.test.npoints
    xs = [_x(core, 8, 60 + i) for i in range(4)]
    xp = [_pinned(x) for x in xs]
    yp = [_pinned(np.zeros((n, 8))) for _ in range(4)]
    for i in range(4):
        ws32.matvec_host_async(xp[i], yp[i], 0, stream=st.cuda_stream)
    st.synchronize()
    for i in range(4):
        assert rel(yp[i], ws64.matvec_host(xs[i], 0)) < 1e-6, i


def test_host_async_rejects_c_order():
    core = CASES["toeplitz-laplace"]()
    ws = h2.H2Workspace(core, max_nrhs=2)
    n = core.test.npoints
    with pytest.raises(ValueError):
        ws.matvec_host_async(np.zeros((n, 2)), np.zeros((n, 2)), 0)
