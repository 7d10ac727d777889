"""The dense I2O for few right-hand sides, grouped by stored block (GPU).

Blocks of at most 4 field columns (1-4 real or 1-2 complex right-hand sides, times the moment
components) take the grouped kernel: pairs that read one stored (canonical) coupling block share
each staged piece of it, their symmetry permutations move to the moment gather and the output
rows, and a chunk's sums stay in shared memory. The maps here exercise what the grouping has to
get right: adaptive trees (receiving boxes on several levels, chunks cut at level changes),
symmetry-reduced couplings (every permutation on both operands), Petrov maps (different test and
trial trees), three moment components, and every orientation. FP64 against the oracle at 1e-12,
FP32 against FP64 at 1e-6, and the same product twice is bit-identical (no atomics).
"""

import copy

import numpy as np
import pytest
import torch

import h2factory_b200 as h2
from h2factory_b200 import methods
from h2factory_b200.trees import build_tree
from oracle import oracle

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
TOL64 = 1e-12
TOL32 = 1e-6


def clustered(n, seed, centers=5):
    rng = np.random.default_rng(seed)
    c = rng.random((centers, 3)) * 0.8 + 0.1
    w = rng.choice(centers, n)
    p = c[w] + rng.standard_normal((n, 3)) * rng.choice([0.02, 0.08, 0.2], centers)[w, None]
    return build_tree(np.clip(p, 0.0, 1.0), maxvalues=24, root_center=[0.5] * 3, root_halfsize=0.5)


def three_components(core):
    c = copy.copy(core)
    c.ncomp = 3
    scale = (1.0, -0.5, 2.0)
    c.collections_test = {n: np.concatenate([s * C for s in scale]) for n, C in core.collections_test.items()}
    c.collections_trial = c.collections_test
    return c


MAPS = {
    "laplace-sym": lambda: methods.interpolation_core(clustered(2500, 1), methods.laplace, 4, symmetry=True),
    "helmholtz-sym": lambda: methods.interpolation_core(clustered(2000, 2), methods.helmholtz(4.0), 3,
                                                        symmetry=True, transfers="separable"),
    "laplace-petrov": lambda: methods.interpolation_core(clustered(1500, 3), methods.laplace, 3,
                                                         trial=clustered(2200, 4, centers=3)),
    "laplace-3comp": lambda: three_components(
        methods.interpolation_core(clustered(1800, 5), methods.laplace, 3, symmetry=True)),
}


def _x(n, k, seed, cplx):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, k))
    return x + 1j * rng.standard_normal((n, k)) if cplx else x


def _mul(ws, mode, x, nout):
    view = ws if mode == 0 else (h2.transpose(ws) if mode == 1 else h2.adjoint(ws))
    dt = torch.complex128 if ws.core.field == "complex" else torch.float64
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).to(DEV).t()
    y = torch.zeros((x.shape[1], nout), dtype=dt, device=DEV).t()
    h2.mul_(y, view, xd)
    torch.cuda.synchronize()
    return y.cpu().numpy()


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("name", sorted(MAPS))
def test_grouped_i2o_matches_oracle(name):
    core = MAPS[name]()
    cplx = core.field == "complex"
    widths = [k for k in (1, 2, 3, 4) if (2 if cplx else 1) * core.ncomp * k <= 4]
    assert widths, "no block of this map takes the grouped kernel"
    levels = np.unique(core.test.level[np.unique(core.plans.far[:, 0])])
    assert levels.size > 1  # receiving boxes on several levels
    c32 = copy.copy(core)
    c32.precision = "fp32"
    for k in widths:
        ws64 = h2.H2Workspace(core, max_nrhs=k)
        ws32 = h2.H2Workspace(c32, max_nrhs=k)
        for mode in (0, 1, 2):
            nin = core.trial.npoints if mode == 0 else core.test.npoints
            nout = core.test.npoints if mode == 0 else core.trial.npoints
            x = _x(nin, k, 10 * k + mode, cplx)
            y64 = _mul(ws64, mode, x, nout)
            assert rel(y64, oracle.matvec(core, x, mode)) < TOL64, (name, k, mode)
            assert np.array_equal(y64, _mul(ws64, mode, x, nout)), (name, k, mode, "repeat")
            assert rel(_mul(ws32, mode, x, nout), y64) < TOL32, (name, k, mode, "fp32")
        ws64.close()
        ws32.close()
