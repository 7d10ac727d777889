"""The batched-uneven configuration's shape (GPU), scaled so the oracle checks it in seconds.

Maps drawn as that configuration draws them: point counts log-uniform (here in [2048, 5000]),
geometry uniform over {unit-cube volume, sphere surface, 4:1:1 ellipsoid surface}, kernel Laplace
or Helmholtz with k uniform in [1, 20], Chebyshev order p in {4, 5, 6}, leaves of at most 64
points, 1-16 right-hand sides, FP64 (plain) and FP32 (chosen) far fields, forward, transpose and
adjoint orientations mixed. The whole batch is captured once as a CUDA graph and replayed; each
map's replayed product must equal its eager product bit for bit, the FP64 maps the oracle
(relative L2 1e-12), and the FP32 maps their FP64 twins within 1e-6 (their far fields run on
the tcgen05 kernel when the right-hand sides make at least 4 FP32 columns)."""

import copy

import numpy as np
import pytest
import torch

from h2factory_b200 import batch, methods
from h2factory_b200.trees import build_tree
from oracle import oracle
from test_gpu_parity import rel

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _points(rng, n, geometry):
    if geometry == "cube":
        return rng.random((n, 3))
    i = np.arange(n) + 0.5
    phi, th = np.arccos(1 - 2 * i / n), np.pi * (1 + 5 ** 0.5) * i
    p = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], axis=1)
    p = p + 0.1 * np.sqrt(4 * np.pi / n) * rng.standard_normal(p.shape)
    scale = np.array([0.45, 0.45, 0.45]) if geometry == "sphere" else np.array([0.45, 0.1125, 0.1125])
    return 0.5 + p * scale


def _draw(seed, nmaps):
    rng = np.random.default_rng(seed)
    out = []
    for m in range(nmaps):
        n = int(np.exp(rng.uniform(np.log(2048), np.log(5000))))
        geometry = ("cube", "sphere", "ellipsoid")[rng.integers(3)]
        kernel = methods.laplace if rng.random() < 0.5 else methods.helmholtz(float(rng.uniform(1, 20)))
        p = int(rng.integers(4, 7))
        nrhs = int(rng.integers(1, 17))
        mode = int(rng.integers(3))
        tree = build_tree(_points(rng, n, geometry), maxvalues=64, root_center=[0.5] * 3, root_halfsize=0.5)
        core = methods.interpolation_core(tree, kernel, p, symmetry=True)
        out.append((core, nrhs, mode, geometry, p))
    return out


def test_batched_uneven_configuration_shape():
    maps = _draw(2026, 8)
    cores, nrhs, modes = [], [], []
    for core, r, mode, _, _ in maps:
        cores.append(core)
        nrhs.append(r)
        modes.append(mode)
        c32 = copy.copy(core)
        c32.precision = "fp32"
        cores.append(c32)
        nrhs.append(r)
        modes.append(mode)
    b = batch.BatchedMaps(cores, nrhs, device=0, modes=modes)
    rng = np.random.default_rng(7)
    xs_host = []
    for k, (c, r) in enumerate(zip(cores, nrhs)):
        n = c.trial.npoints if modes[k] == 0 else c.test.npoints
        x = rng.standard_normal((n, r))
        if c.field == "complex":
            x = x + 1j * rng.standard_normal((n, r))
        if k % 2 == 1:
            x = xs_host[k - 1]  # the FP32 twin multiplies the same block
        xs_host.append(x)
    b.set_inputs([torch.from_numpy(np.ascontiguousarray(x.T)).to(DEV).t() for x in xs_host])
    b.run_eager()
    torch.cuda.synchronize()
    eager = [y.clone() for y in b.outputs]
    b.capture()
    for y in b.outputs:
        y.zero_()
    b.replay()
    torch.cuda.synchronize()
    for k, (a, e) in enumerate(zip(b.outputs, eager)):
        assert torch.equal(a, e), k
    for i, (core, r, mode, geometry, p) in enumerate(maps):
        y64 = b.outputs[2 * i].cpu().numpy()
        y32 = b.outputs[2 * i + 1].cpu().numpy()
        want = oracle.matvec(core, xs_host[2 * i], mode)
        assert rel(y64, want) < 1e-12, (i, geometry, p, r, mode)
        assert rel(y32, y64) < 1e-6, (i, geometry, p, r, mode)
    b.close()
