"""Parity at the benchmark configurations' sizes (GPU).

* The Toeplitz configuration at full size: Laplace, N = 262,144 points uniform in the unit cube,
  depth-5 octree (4,096 leaves), equispaced p = 4 with FFT'd M2L, 640,584 far pairs, 399 M near
  entries. The FP64 form must match the CPU oracle to 1e-12 relative L2, forward and transpose;
  the FP32 far-field form must stay within 1e-6 of the FP64 form.
* The sphere configuration's shape at 65,536 points (the full 1,048,576-point map is checked by
  the benchmark itself against the oracle and a 4,096-row direct sum): Helmholtz k = 8 pi x 0.45,
  Chebyshev p = 6, leaves <= 128 points, symmetry-reduced couplings, separable transfers. FP64 vs
  the oracle at 1e-12 (forward and adjoint, two right-hand sides: the oracle's cost grows with
  them), FP32 form vs FP64 within 1e-6 on 32 right-hand sides.
"""

import copy
import os
import sys

import numpy as np
import pytest
import torch

import h2factory_b200 as h2
from oracle import oracle

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
import bench  # noqa: E402  (the configurations' generators)

DEV = "cuda:0"
TOL64 = 1e-12
TOL32 = 1e-6


def _with_host_near(core):
    c = copy.copy(core)
    c.near_data, c.near_device = core.near_device.cpu().numpy(), None
    return c


def _cols(x):
    return torch.from_numpy(np.ascontiguousarray(x.T)).to(DEV).t()


def _mul(ws, mode, x):
    view = ws if mode == 0 else (h2.transpose(ws) if mode == 1 else h2.adjoint(ws))
    dt = torch.complex128 if ws.core.field == "complex" else torch.float64
    y = torch.zeros((x.shape[1], x.shape[0]), dtype=dt, device=DEV).t()
    h2.mul_(y, view, x)
    torch.cuda.synchronize()
    return y


def _rel_cols(a, b):
    return float(((a - b).norm(dim=0) / b.norm(dim=0)).max())


def test_toeplitz_configuration_full_size():
    _, core = bench.toeplitz_core(n=262144, depth=5, device=DEV)
    assert core.plans.far.shape[0] == 640584
    host = _with_host_near(core)
    d64 = h2.DeviceCore(core)
    d32 = h2.DeviceCore(bench.fp32_twin(core))
    core.near_device = None
    ws64, ws32 = h2.H2Workspace(d64, max_nrhs=16), h2.H2Workspace(d32, max_nrhs=16)
    rng = np.random.default_rng(5)
    n = core.trial.npoints
    desc = h2.flatten(host)
    for mode in (0, 1):
        xh = rng.standard_normal((n, 2))
        got = _mul(ws64, mode, _cols(xh)).cpu().numpy()
        want = oracle.matvec(host, xh, mode, desc=desc)
        assert np.linalg.norm(got - want) / np.linalg.norm(want) < TOL64, mode
        xb = _cols(rng.standard_normal((n, 16)))
        assert _rel_cols(_mul(ws32, mode, xb), _mul(ws64, mode, xb)) < TOL32, mode


def test_sphere_configuration_shape_65536():
    _, core = bench.sphere_core(65536, DEV)
    host = _with_host_near(core)
    d64 = h2.DeviceCore(core)
    d32 = h2.DeviceCore(bench.fp32_twin(core))
    core.near_device = None
    ws64, ws32 = h2.H2Workspace(d64, max_nrhs=32), h2.H2Workspace(d32, max_nrhs=32)
    rng = np.random.default_rng(6)
    n = core.trial.npoints
    desc = h2.flatten(host)
    for mode in (0, 2):
        xh = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
        got = _mul(ws64, mode, _cols(xh)).cpu().numpy()
        want = oracle.matvec(host, xh, mode, desc=desc)
        assert np.linalg.norm(got - want) / np.linalg.norm(want) < TOL64, mode
        xb = _cols(rng.standard_normal((n, 32)) + 1j * rng.standard_normal((n, 32)))
        assert _rel_cols(_mul(ws32, mode, xb), _mul(ws64, mode, xb)) < TOL32, mode
