"""The timeout path of the tensor-core kernels' bounded waits (GPU).

Every mbarrier wait inside the tcgen05 kernels gives up after a bounded number of attempts; a wait
that gives up is counted (h2b_tensor_wait_timeouts), its CTA stops, waits for the products it has
already issued, frees its tensor memory and returns without writing its output tile, and
h2b_matvec_host reports the incomplete product as an error. The test makes waits give up by
lowering the bound to one attempt (h2b_set_tensor_wait_limit) -- nothing faults or hangs --, checks
the error and the counter, then restores the default bound and checks that the same workspace gives
a correct product again. This is the failure-detection form of H2Factory's
ConcurrentWorkspaceError tests (src/maps/workspace.jl:284-329) for a device-side wait.
"""

import copy

import numpy as np
import pytest

import h2factory_b200 as h2
from h2factory_b200 import _abi, methods
from h2factory_b200.trees import build_tree

pytestmark = pytest.mark.gpu


def _maps():
    rng = np.random.default_rng(5)
    t = build_tree(rng.random((4000, 3)), maxvalues=48, root_center=[0.5] * 3, root_halfsize=0.5)
    core = methods.interpolation_core(t, methods.helmholtz(4.0), 4)
    c32 = copy.copy(core)
    c32.precision = "fp32"
    return core, c32


def test_wait_timeout_reported_and_recovered():
    core, c32 = _maps()
    n = core.trial.npoints
    rng = np.random.default_rng(9)
    x = np.asfortranarray(rng.standard_normal((n, 8)) + 1j * rng.standard_normal((n, 8)))
    ws64 = h2.H2Workspace(core, max_nrhs=8)
    ws32 = h2.H2Workspace(c32, max_nrhs=8)
    want = ws64.matvec_host(x)
    before = _abi.tensor_wait_timeouts(0)
    try:
        _abi.set_tensor_wait_limit(1)
        with pytest.raises(_abi.H2BError) as err:
            ws32.matvec_host(x)
        assert err.value.status == _abi.H2B_ERR_CUDA
        assert "gave up" in str(err.value)
        assert _abi.tensor_wait_timeouts(0) > before
    finally:
        _abi.set_tensor_wait_limit(0)
    after = _abi.tensor_wait_timeouts(0)
    got = ws32.matvec_host(x)
    assert _abi.tensor_wait_timeouts(0) == after
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-6
