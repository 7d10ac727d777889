"""Matrix-free near field on the device (GPU): entries K(x_i, y_j) computed from the points.

H2Factory accepts any matrix-like near operator with `mul!` (docs/src/near/storage.md:7-14); the
library's point-kernel near operator must give the product of the stored-block map to rounding.
Each case builds one map twice -- near blocks assembled on the host, and matrix-free -- and checks
the matrix-free device product against the CPU oracle run on the stored twin (relative L2 error
<= 1e-12, the bar of the other FP64 parity tests), in every orientation, with α/β, and near alone.
"""

import numpy as np
import pytest

import h2factory_b200 as h2
from h2factory_b200 import methods
from h2factory_b200.trees import build_tree
from oracle import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL64 = 1e-12


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def _cube(n, seed, **kw):
    rng = np.random.default_rng(seed)
    return build_tree(rng.random((n, 3)), root_center=[0.5] * 3, root_halfsize=0.5, **kw)


CASES = {
    "cheb-laplace": lambda near: methods.interpolation_core(_cube(3000, 21, maxvalues=40), methods.laplace, 3,
                                                            near=near),
    "toeplitz-laplace": lambda near: methods.interpolation_core(_cube(4000, 22, depth=4), methods.laplace, 4,
                                                                nodes="equispaced", couplings="toeplitz",
                                                                near=near),
    "cheb-helmholtz": lambda near: methods.interpolation_core(_cube(2500, 23, maxvalues=48),
                                                              methods.helmholtz(4.0), 3, near=near),
    "petrov-laplace": lambda near: methods.interpolation_core(_cube(2500, 24, maxvalues=20), methods.laplace, 3,
                                                              trial=_cube(900, 25, maxvalues=40), near=near),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def pair(request):
    return request.param, CASES[request.param]("host"), CASES[request.param]("free")


def dev(a):
    a = np.asarray(a)
    if a.ndim == 1:
        return __import__("torch").from_numpy(a.copy()).to(DEV)
    return __import__("torch").from_numpy(np.ascontiguousarray(a.T)).to(DEV).t()


def host(t):
    __import__("torch").cuda.synchronize()
    return t.cpu().numpy()


def _x(core, nrhs, seed, mode, out=False):
    rng = np.random.default_rng(seed)
    n = core.trial.npoints if (mode == 0) != out else core.test.npoints
    x = rng.standard_normal((n, nrhs))
    if core.field == "complex":
        x = x + 1j * rng.standard_normal((n, nrhs))
    return x[:, 0] if nrhs == 1 else x


ORIENT = [(0, lambda ws: ws), (1, h2.transpose), (2, h2.adjoint)]


def test_free_core_holds_no_near_blocks(pair):
    _, stored, free = pair
    info = h2.H2Workspace(free).dcore.info()
    assert info.near_entries == 0
    assert h2.H2Workspace(stored).dcore.info().near_entries > 0


@pytest.mark.parametrize("nrhs", [1, 2, 3, 16])
def test_matrix_free_matches_oracle(pair, nrhs):
    name, stored, free = pair
    ws = h2.H2Workspace(free, max_nrhs=nrhs)
    desc = h2.flatten(stored)
    for mode, op in ORIENT:
        x = _x(stored, nrhs, 31, mode)
        want = oracle.matvec(stored, x, mode, desc=desc)
        y = dev(np.zeros_like(_x(stored, nrhs, 0, mode, out=True)))
        h2.mul_(y, op(ws), dev(x))
        assert rel(host(y), want) < TOL64, (name, mode, nrhs)


def test_matrix_free_scaled_near_only(pair):
    name, stored, free = pair
    ws = h2.H2Workspace(free, max_nrhs=3)
    a, b = (0.75 - 0.5j, -1.25 + 0.3j) if stored.field == "complex" else (0.75, -1.25)
    desc = h2.flatten(stored)
    for mode, op in ORIENT:
        x = _x(stored, 3, 32, mode)
        y0 = _x(stored, 3, 33, mode, out=True)
        want = oracle.nearmul(stored, x, mode, alpha=a, beta=b, y=y0, desc=desc)
        y = dev(y0)
        h2.nearmul_(y, op(ws), dev(x), a, b)
        assert rel(host(y), want) < TOL64, (name, mode)
        want = oracle.matvec(stored, x, mode, alpha=a, beta=b, y=y0, desc=desc)
        y = dev(y0)
        h2.mul_(y, op(ws), dev(x), a, b)
        assert rel(host(y), want) < TOL64, (name, mode)
