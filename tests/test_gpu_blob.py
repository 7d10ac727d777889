"""A core loaded from a map blob multiplies exactly like the core it was written from (GPU)."""

import numpy as np
import pytest
import torch

import h2factory_b200 as h2
from h2factory_b200 import methods
from h2factory_b200.trees import build_tree

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("sym", [False, True])
def test_blob_core_equals_direct_core(tmp_path, sym):
    rng = np.random.default_rng(8)
    t = build_tree(rng.random((3000, 3)), depth=4, root_center=[0.5] * 3, root_halfsize=0.5)
    core = methods.interpolation_core(t, methods.helmholtz(3.0), 3, nodes="equispaced", couplings="toeplitz",
                                      symmetry=sym)
    path = str(tmp_path / "m.h2b")
    h2.save_map(core, path)
    a = h2.H2Workspace(core, max_nrhs=2)
    b = h2.H2Workspace(h2.DeviceCore.from_blob(path), max_nrhs=2)
    assert b.shape == a.shape
    x = torch.randn(2, 3000, dtype=torch.complex128, device="cuda:0").t()
    for op in (lambda w: w, h2.transpose, h2.adjoint):
        ya = torch.zeros(2, 3000, dtype=torch.complex128, device="cuda:0").t()
        yb = torch.zeros_like(ya)
        h2.mul_(ya, op(a), x)
        h2.mul_(yb, op(b), x)
        torch.cuda.synchronize()
        assert torch.equal(ya, yb)
