"""Products captured in CUDA graphs (GPU): a matvec captured once and replayed gives the eager
result, and many maps of uneven size replay together from one graph (the batching pattern:
launch-bound small maps lose their per-kernel launch cost)."""

import numpy as np
import pytest
import torch

import h2factory_b200 as h2
from h2factory_b200 import batch, methods
from h2factory_b200.trees import build_tree

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _map(n, seed, kind):
    rng = np.random.default_rng(seed)
    if kind == "toeplitz":
        t = build_tree(rng.random((n, 3)), depth=3, root_center=[0.5] * 3, root_halfsize=0.5)
        return methods.interpolation_core(t, methods.laplace, 3, nodes="equispaced", couplings="toeplitz")
    t = build_tree(rng.random((n, 3)), maxvalues=40, root_center=[0.5] * 3, root_halfsize=0.5)
    return methods.interpolation_core(t, methods.helmholtz(2.0), 3)


def test_captured_matvec_equals_eager():
    core = _map(3000, 1, "toeplitz")
    ws = h2.H2Workspace(core, max_nrhs=4)
    x = torch.randn(4, 3000, dtype=torch.float64, device=DEV).t()
    want = torch.zeros(4, 3000, dtype=torch.float64, device=DEV).t()
    h2.mul_(want, h2.transpose(ws), x)
    y = torch.zeros_like(want)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        h2.mul_(y, h2.transpose(ws), x, stream=s.cuda_stream)
    for _ in range(3):
        y.zero_()
        g.replay()
    torch.cuda.synchronize()
    assert torch.equal(y, want)


def test_batched_uneven_maps_replay():
    cores = [_map(n, 10 + i, "toeplitz" if i % 2 else "dense") for i, n in enumerate((900, 2500, 1500, 4000))]
    nrhs = [1, 3, 2, 4]
    b = batch.BatchedMaps(cores, nrhs, device=0)
    xs = [torch.randn(r, c.trial.npoints, dtype=b.dtype(k), device=DEV).t() for k, (c, r) in enumerate(zip(cores, nrhs))]
    b.set_inputs(xs)
    b.run_eager()
    torch.cuda.synchronize()
    eager = [y.clone() for y in b.outputs]
    b.capture()
    for y in b.outputs:
        y.zero_()
    b.replay()
    torch.cuda.synchronize()
    for a, e in zip(b.outputs, eager):
        assert torch.equal(a, e)
