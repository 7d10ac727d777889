"""Parity of the CUDA path with the CPU oracle and the closed-form golden fixtures (GPU).

Tolerances: the FP64 form must match the oracle to a relative L2 error of 1e-12 (the bar of
docs/src/implementing/example.md:205-222); the FP32 far-field form must match the FP64 oracle to
1e-6, the reduced-precision bar of the served form (its near field and final summation stay FP64).
"""

import os

import numpy as np
import pytest
import torch

import h2factory_b200 as h2
from h2factory_b200 import methods
from h2factory_b200.trees import build_tree
from oracle import oracle
from fakes import cluster_core, worked_example_core

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DEV = "cuda:0"
TOL64 = 1e-12
TOL32 = 1e-6


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def dev(a, dtype):
    """Column-major device copy of a host vector / matrix."""
    a = np.asarray(a, dtype=dtype)
    if a.ndim == 1:
        return torch.from_numpy(a.copy()).to(DEV)
    return torch.from_numpy(np.ascontiguousarray(a.T)).to(DEV).t()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def run(fn, A, x, y0=None, alpha=None, beta=None, nout=None):
    ws = A.ws if isinstance(A, h2.OrientedMap) else A
    dt = ws.core.dtype
    xd = dev(x, dt)
    n = nout if nout is not None else A.shape[0]
    if y0 is None:
        y0 = np.zeros((n,) + np.shape(x)[1:], dt)
    yd = dev(y0, dt)
    fn(yd, A, xd, alpha, beta)
    return host(yd)


ORIENT = [(0, lambda ws: ws), (1, h2.transpose), (2, h2.adjoint)]


# ---------------------------------------------------------------------------------------------
# closed-form golden cases
# ---------------------------------------------------------------------------------------------
def test_worked_example_gpu():
    g = np.load(os.path.join(GOLDEN, "worked_example.npz"))
    core, _ = worked_example_core()
    ws = h2.H2Workspace(core, max_nrhs=32)
    x = g["x"]
    for mode, op in ORIENT:
        y = run(h2.mul_, op(ws), x)
        assert rel(y, g[["y_fwd", "y_t", "y_h"][mode]]) < TOL64
        ys = run(h2.mul_, op(ws), x, y0=g["out0"], alpha=complex(g["alpha"]), beta=complex(g["beta"]))
        assert rel(ys, g[["ys_fwd", "ys_t", "ys_h"][mode]]) < TOL64
    # Matrix(A): all 32 columns at once
    M = run(h2.mul_, ws, np.eye(32, dtype=np.complex128))
    assert rel(M, g["F"]) < TOL64


def test_two_clusters_gpu():
    g = np.load(os.path.join(GOLDEN, "clusters_b4.npz"))
    pts = np.stack([g["points"], np.zeros(8), np.zeros(8)], axis=1)
    core, _, _ = cluster_core(pts, [0, 0, 0, 0, 1, 1, 1, 1], complex(g["c"]), minhalfsize=2.0)
    ws = h2.H2Workspace(core)
    for mode, op in ORIENT:
        y = run(h2.farmul_, op(ws), g["x"], y0=np.full(8, np.nan + 0j))
        assert rel(y, g[["y_fwd", "y_t", "y_h"][mode]]) < TOL64
    y = run(h2.farmul_, ws, g["x"], y0=g["y0"], alpha=complex(g["alpha"]), beta=complex(g["beta"]))
    assert rel(y, g["y_acc"]) < TOL64


@pytest.mark.parametrize("tag", ["c", "r"])
def test_many_clusters_gpu(tag):
    g = np.load(os.path.join(GOLDEN, "clusters_6x20.npz"))
    pts = np.stack([g["points"], np.zeros(120), np.zeros(120)], axis=1)
    field = "complex" if tag == "c" else "real"
    c = complex(g[f"{tag}_c"]) if tag == "c" else float(g[f"{tag}_c"])
    core, _, _ = cluster_core(pts, g["cid"], c, field=field, minhalfsize=1.0)
    ws = h2.H2Workspace(core)
    for mode, op in ORIENT:
        y = run(h2.farmul_, op(ws), g[f"{tag}_x"])
        assert rel(y, g[[f"{tag}_fwd", f"{tag}_t", f"{tag}_h"][mode]]) < TOL64


# ---------------------------------------------------------------------------------------------
# interpolation methods against the oracle
# ---------------------------------------------------------------------------------------------
def _cube(n, seed, **kw):
    rng = np.random.default_rng(seed)
    return build_tree(rng.random((n, 3)), root_center=[0.5] * 3, root_halfsize=0.5, **kw)


CASES = {
    "cheb-laplace-dense": lambda: methods.interpolation_core(_cube(3000, 1, maxvalues=40), methods.laplace, 4),
    "cheb-laplace-separable": lambda: methods.interpolation_core(_cube(3000, 1, maxvalues=40), methods.laplace, 4,
                                                                  transfers="separable"),
    "cheb-helmholtz": lambda: methods.interpolation_core(_cube(2500, 2, maxvalues=48), methods.helmholtz(4.0), 3),
    "toeplitz-laplace": lambda: methods.interpolation_core(_cube(4000, 3, depth=4), methods.laplace, 4,
                                                           nodes="equispaced", couplings="toeplitz"),
    "toeplitz-helmholtz": lambda: methods.interpolation_core(_cube(3000, 4, depth=4), methods.helmholtz(3.0), 3,
                                                             nodes="equispaced", couplings="toeplitz",
                                                             transfers="separable"),
    # one stored coupling per pair: too many per level for the grouped kernel's shared memory,
    # so the per-node Toeplitz kernel runs
    "toeplitz-laplace-unshared": lambda: _unshared(methods.interpolation_core(
        _cube(2000, 5, depth=3), methods.laplace, 4, nodes="equispaced", couplings="toeplitz")),
    # symmetry-reduced couplings: one canonical block / spectrum per orbit of the cube's signed
    # axis permutations, read through permutations
    "sym-cheb-laplace": lambda: methods.interpolation_core(_cube(3000, 1, maxvalues=40), methods.laplace, 4,
                                                           symmetry=True),
    "sym-cheb-helmholtz": lambda: methods.interpolation_core(_cube(2500, 2, maxvalues=48), methods.helmholtz(4.0),
                                                             3, symmetry=True),
    "sym-toeplitz-laplace": lambda: methods.interpolation_core(_cube(4000, 3, depth=4), methods.laplace, 4,
                                                               nodes="equispaced", couplings="toeplitz",
                                                               symmetry=True),
    "sym-toeplitz-helmholtz": lambda: methods.interpolation_core(_cube(3000, 4, depth=4), methods.helmholtz(3.0), 3,
                                                                 nodes="equispaced", couplings="toeplitz",
                                                                 transfers="separable", symmetry=True),
    # sphere, Chebyshev p = 6 (216 coefficients), Helmholtz, leaves <= 128 points, symmetry-reduced
    "sphere-cheb6-helmholtz-sym": lambda: methods.interpolation_core(
        _sphere(12000, 10, maxvalues=128), methods.helmholtz(8 * np.pi * 0.45), 6, symmetry=True),
    # Petrov (rectangular) maps: test and trial trees on different point sets and depths
    "petrov-cheb-laplace": lambda: methods.interpolation_core(
        _cube(3000, 6, maxvalues=40), methods.laplace, 4, trial=_cube(1100, 7, maxvalues=30)),
    "petrov-toeplitz-helmholtz": lambda: methods.interpolation_core(
        _cube(2500, 8, depth=4), methods.helmholtz(3.0), 3, nodes="equispaced", couplings="toeplitz",
        trial=_cube(4000, 9, depth=4)),
}


def _sphere(n, seed, **kw):
    """Fibonacci sphere (radius 0.45 in the unit cube) with jitter 0.1 x the point spacing: the
    geometry of the 1M-point Helmholtz configuration, at a size the oracle checks in seconds."""
    rng = np.random.default_rng(seed)
    i = np.arange(n) + 0.5
    phi, th = np.arccos(1 - 2 * i / n), np.pi * (1 + 5 ** 0.5) * i
    p = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], axis=1)
    p = p + 0.1 * np.sqrt(4 * np.pi / n) * rng.standard_normal(p.shape)
    return build_tree(0.5 + 0.45 * p, root_center=[0.5] * 3, root_halfsize=0.5, **kw)


def _unshared(core):
    core.couplings = [core.couplings[k] for k in core.pair_coupling]
    core.pair_coupling = np.arange(len(core.couplings), dtype=np.int64)
    return core


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    core = CASES[request.param]()
    return request.param, core


def _x(core, nrhs, seed, mode=0, out=False):
    """Right-hand sides of op(A) (out=False) or its outputs (out=True) for orientation `mode`."""
    rng = np.random.default_rng(seed)
    n = core.trial.npoints if (mode == 0) != out else core.test.npoints
    x = rng.standard_normal((n, nrhs))
    if core.field == "complex":
        x = x + 1j * rng.standard_normal((n, nrhs))
    return x[:, 0] if nrhs == 1 else x


@pytest.mark.parametrize("nrhs", [1, 5, 8, 13])
def test_methods_match_oracle(case, nrhs):
    name, core = case
    ws = h2.H2Workspace(core, max_nrhs=nrhs)
    desc = h2.flatten(core)
    for mode, op in ORIENT:
        x = _x(core, nrhs, 11, mode)
        want = oracle.matvec(core, x, mode, desc=desc)
        got = run(h2.mul_, op(ws), x)
        assert rel(got, want) < TOL64, (name, mode)


def test_methods_scaled_and_partial_products(case):
    name, core = case
    ws = h2.H2Workspace(core, max_nrhs=3)
    a, b = (0.75 - 0.5j, -1.25 + 0.3j) if core.field == "complex" else (0.75, -1.25)
    desc = h2.flatten(core)
    for mode, op in ORIENT:
        x = _x(core, 3, 12, mode)
        y0 = _x(core, 3, 13, mode, out=True)
        want = oracle.matvec(core, x, mode, alpha=a, beta=b, y=y0, desc=desc)
        assert rel(run(h2.mul_, op(ws), x, y0=y0, alpha=a, beta=b), want) < TOL64, (name, mode)
        want = oracle.farmul(core, x, mode, desc=desc)
        assert rel(run(h2.farmul_, op(ws), x, y0=np.full_like(y0, np.nan)), want) < TOL64
        want = oracle.farmul(core, x, mode, alpha=a, beta=b, y=y0, desc=desc)
        assert rel(run(h2.farmul_, op(ws), x, y0=y0, alpha=a, beta=b), want) < TOL64
        want = oracle.nearmul(core, x, mode, alpha=a, beta=b, y=y0, desc=desc)
        assert rel(run(h2.nearmul_, op(ws), x, y0=y0, alpha=a, beta=b), want) < TOL64


def test_fp32_far_field_form(case):
    name, core = case
    core32 = methods_copy_fp32(core)
    ws = h2.H2Workspace(core32, max_nrhs=5)
    for mode, op in ORIENT:
        x = _x(core, 5, 14, mode)
        want = oracle.matvec(core, x, mode)
        assert rel(run(h2.mul_, op(ws), x), want) < TOL32, (name, mode)


def methods_copy_fp32(core):
    import copy

    c = copy.copy(core)
    c.precision = "fp32"
    return c


def test_host_buffer_path(case):
    """h2b_matvec_host: host arrays in and out, the call a host-language binding makes."""
    name, core = case
    ws = h2.H2Workspace(core, max_nrhs=2)
    for mode in (0, 1, 2):
        x = _x(core, 2, 15, mode)
        got = ws.matvec_host(x, mode)
        assert rel(got, oracle.matvec(core, x, mode)) < TOL64, (name, mode)


def test_two_workspaces_share_one_core():
    core = CASES["toeplitz-laplace"]()
    a = h2.H2Workspace(core)
    b = h2.similarworkspace(a)
    assert b.dcore is a.dcore
    x = _x(core, 1, 16)
    ya = run(h2.mul_, a, x)
    yb = run(h2.mul_, b, x)
    assert rel(ya, yb) == 0.0


@pytest.mark.parametrize("ntest,ntrial", [(256, 16), (16, 256)])
def test_petrov_side_owned_transfers_gpu(ntest, ntrial):
    """test/farinteractions/test_rectangular.jl:103-154 on the device: all orientations equal the
    complete matrix of a rectangular map with distinct per-side transfers."""
    from fakes import petrov_core

    core, F, N = petrov_core(ntest, ntrial)
    ws = h2.H2Workspace(core, max_nrhs=2)
    rng = np.random.default_rng(20260720)
    x = rng.standard_normal((ntrial, 2)) + 1j * rng.standard_normal((ntrial, 2))
    y = rng.standard_normal((ntest, 2)) + 1j * rng.standard_normal((ntest, 2))
    assert rel(run(h2.farmul_, ws, x), F @ x) < TOL64
    assert rel(run(h2.farmul_, h2.transpose(ws), y), F.T @ y) < TOL64
    assert rel(run(h2.farmul_, h2.adjoint(ws), y), F.conj().T @ y) < TOL64
    assert rel(run(h2.mul_, ws, x), (F + N) @ x) < TOL64
    assert rel(run(h2.mul_, h2.adjoint(ws), y), (F + N).conj().T @ y) < TOL64


def test_single_leaf_map_has_no_far_field():
    """A tree that is one leaf: far = 0; 3-arg farmul! zero-fills, 5-arg leaves y alone."""
    rng = np.random.default_rng(5)
    t = build_tree(rng.random((50, 3)), maxvalues=100)
    core = methods.interpolation_core(t, methods.laplace, 2)
    assert core.plans.far.shape[0] == 0
    ws = h2.H2Workspace(core)
    x = rng.standard_normal(50)
    y0 = rng.standard_normal(50)
    assert np.all(run(h2.farmul_, ws, x, y0=y0) == 0)
    assert np.array_equal(run(h2.farmul_, ws, x, y0=y0, alpha=2.0, beta=3.0), y0)
    K = methods.kernel_matrix(methods.laplace, t.points, t.points)
    assert rel(run(h2.mul_, ws, x), K @ x) < TOL64


def test_c1_config_full_size():
    """Chebyshev p=4 Laplace, N=8192 uniform, leaves <= 64 points: oracle parity and method error."""
    rng = np.random.default_rng(0)
    pts = rng.random((8192, 3))
    t = build_tree(pts, maxvalues=64, root_center=[0.5] * 3, root_halfsize=0.5)
    core = methods.interpolation_core(t, methods.laplace, 4)
    assert core.plans.far.shape[0] == 56448
    ws = h2.H2Workspace(core)
    x = rng.standard_normal(8192)
    got = run(h2.mul_, ws, x)
    assert rel(got, oracle.matvec(core, x)) < TOL64
    K = methods.kernel_matrix(methods.laplace, pts, pts)
    assert rel(got, K @ x) < 5e-3


def test_sphere_helmholtz_32_rhs():
    """32 complex right-hand sides per product, forward and adjoint (the sphere configuration's
    block size), against the oracle."""
    core = CASES["sphere-cheb6-helmholtz-sym"]()
    ws = h2.H2Workspace(core, max_nrhs=32)
    desc = h2.flatten(core)
    for mode, op in (ORIENT[0], ORIENT[2]):
        x = _x(core, 32, 17, mode)
        want = oracle.matvec(core, x, mode, desc=desc)
        assert rel(run(h2.mul_, op(ws), x), want) < TOL64, mode
