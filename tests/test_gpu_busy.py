"""A second call on a workspace that is inside a call gets H2B_BUSY (GPU).

H2Factory's workspaces carry an atomic ownership flag that every top-level operation takes with a
compare-and-swap and releases when it returns; a second operation on the same workspace -- or on
its transpose or adjoint view, which share the flag -- throws ConcurrentWorkspaceError
(src/maps/workspace.jl:284-329). The library keeps the same rule: h2b_matvec and friends return
H2B_BUSY (WorkspaceBusyError in Python) while another call holds the workspace.

The test holds a workspace inside h2b_profile_matvec, which waits for its stream before returning,
while a bounded delay kernel (torch.cuda._sleep) keeps that stream busy for a fraction of a second;
meanwhile a second thread calls the workspace and its transposed view and must be refused, a second
workspace on the same core must not be, and after the first call returns the workspace works again.
"""

import threading
import time

import numpy as np
import pytest
import torch

import h2factory_b200 as h2
from h2factory_b200 import methods
from h2factory_b200.trees import build_tree

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def test_second_call_on_a_busy_workspace_is_refused():
    rng = np.random.default_rng(2)
    t = build_tree(rng.random((2000, 3)), maxvalues=40, root_center=[0.5] * 3, root_halfsize=0.5)
    core = methods.interpolation_core(t, methods.laplace, 3)
    dcore = h2.DeviceCore(core)
    ws = h2.H2Workspace(dcore, max_nrhs=2)
    other = h2.similarworkspace(ws)
    n = core.trial.npoints
    x = torch.randn((2, n), dtype=torch.float64, device=DEV).t()
    y = torch.zeros((2, n), dtype=torch.float64, device=DEV).t()
    y2 = torch.zeros((2, n), dtype=torch.float64, device=DEV).t()
    h2.mul_(y, ws, x)
    torch.cuda.synchronize()
    want = y.clone()

    stream = torch.cuda.Stream(DEV)
    held = threading.Event()
    result = {}

    def holder():
        with torch.cuda.stream(stream):
            torch.cuda._sleep(int(1.5e9))  # about 0.75 s of device time at the B200's clock
        held.set()
        result["passes"] = h2.profilemul(ws, x, y=y2, stream=stream.cuda_stream)

    th = threading.Thread(target=holder)
    th.start()
    held.wait(timeout=30)
    time.sleep(0.2)  # the holder is now inside h2b_profile_matvec, waiting for its stream
    refused = []
    for view in (ws, h2.transpose(ws)):
        try:
            h2.mul_(torch.zeros_like(y), view, x)
        except h2.WorkspaceBusyError as e:
            refused.append(e.status)
    h2.mul_(torch.zeros((2, n), dtype=torch.float64, device=DEV).t(), other, x)  # another workspace: fine
    th.join(timeout=60)
    assert not th.is_alive()
    assert refused == [h2._abi.H2B_BUSY, h2._abi.H2B_BUSY]
    assert len(result["passes"]) > 2
    torch.cuda.synchronize()
    assert torch.allclose(y2, want, rtol=1e-12, atol=0)
    y3 = torch.zeros_like(y)
    h2.mul_(y3, ws, x)  # released: the workspace works again
    torch.cuda.synchronize()
    assert torch.allclose(y3, want, rtol=1e-12, atol=0)
