"""Known-answer tests of the Toeplitz (FFT) M2L path, restated from the reference's own tests.

* test/farinteractions/test_toeplitz3d.jl:26-67 -- a genuinely three-dimensional coupling: the
  points are the 6 x 6 x 6 integer grid, the kernel exp(1.1 i |z|) / (|z| + 0.7), three
  equispaced nodes per axis, so every stored FFT'd tensor is (2n-1)^3 = 5 x 5 x 5 with no
  singleton axis and the dense coupling it encodes is neither diagonal nor symmetric. The FFT
  Toeplitz path must equal the dense coupling in all three orientations.
* test/moments/test_toeplitzmul.jl:47-182 -- the Hadamard product of an FFT'd translation and an
  FFT'd moment, with its alpha/beta contract. The library's couplings are scalar operators applied
  to every moment component (the "scalar tf" case of that test); the contract is checked through
  a closed form: a map whose D = 3 components carry the leaf bases scaled by s_c multiplies as
  (sum_c s_c^2) times the one-component map, in every orientation, with alpha/beta, for real and
  complex element types, and the input is never modified. The vector / matrix tf cases (moments
  mixing components through a D1 x D2 block of operators) have no counterpart in this library's
  descriptor, which holds one operator per translation.

The oracle parts run on the CPU; the device parts compare the CUDA path with the oracle.
"""

import copy

import numpy as np
import pytest

import h2factory_b200 as h2
from h2factory_b200 import methods
from h2factory_b200.trees import build_tree
from oracle import oracle

TOL64 = 1e-12
TOL32 = 1e-6
DEV = "cuda:0"


def kern3d(x, y):
    d = x[:, None, :] - y[None, :, :]
    r = np.sqrt(np.einsum("ijk,ijk->ij", d, d))
    return np.exp(1.1j * r) / (r + 0.7)


def grid_tree():
    g = np.arange(6.0)
    pts = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    return build_tree(pts, depth=3, root_center=[2.5] * 3, root_halfsize=4.0)


def grid_maps():
    tree = grid_tree()
    toep = methods.interpolation_core(tree, kern3d, 3, nodes="equispaced", couplings="toeplitz")
    dense = methods.interpolation_core(tree, kern3d, 3, nodes="equispaced", couplings="dense")
    return toep, dense


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def _x(n, nrhs, seed, cplx=True):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, nrhs))
    return x + 1j * rng.standard_normal((n, nrhs)) if cplx else x


# ---------------------------------------------------------------------------------------------
# the genuinely three-dimensional coupling
# ---------------------------------------------------------------------------------------------
def test_tensor_is_three_dimensional():
    toep, dense = grid_maps()
    assert toep.plans.far.shape[0] > 0
    spec = np.asarray(toep.couplings[int(toep.pair_coupling[0])])
    assert spec.shape == (5, 5, 5) and min(spec.shape) > 1
    S = np.asarray(dense.couplings[int(dense.pair_coupling[0])])
    assert S.shape == (27, 27)
    assert np.linalg.norm(S - np.diag(np.diag(S))) > 0          # not diagonal
    assert np.linalg.norm(S - S.T) / np.linalg.norm(S) > 1e-6   # off-axis displacement: not symmetric


def test_fft_path_equals_dense_coupling_oracle():
    toep, dense = grid_maps()
    for mode in (0, 1, 2):
        x = _x(toep.trial.npoints, 3, 40 + mode)
        assert rel(oracle.farmul(toep, x, mode), oracle.farmul(dense, x, mode)) < TOL64, mode
        assert rel(oracle.matvec(toep, x, mode), oracle.matvec(dense, x, mode)) < TOL64, mode


@pytest.mark.gpu
def test_fft_path_equals_dense_coupling_gpu():
    import torch

    toep, dense = grid_maps()
    for core in (toep, dense):
        for prec, tol in (("fp64", TOL64), ("fp32", TOL32)):
            c = copy.copy(core)
            c.precision = prec
            ws = h2.H2Workspace(c, max_nrhs=3)
            for mode in (0, 1, 2):
                x = _x(core.trial.npoints, 3, 40 + mode)
                want = oracle.matvec(dense, x, mode)
                xd = torch.from_numpy(np.ascontiguousarray(x.T)).to(DEV).t()
                y = torch.zeros((3, core.test.npoints), dtype=torch.complex128, device=DEV).t()
                view = ws if mode == 0 else (h2.transpose(ws) if mode == 1 else h2.adjoint(ws))
                h2.mul_(y, view, xd)
                torch.cuda.synchronize()
                assert rel(y.cpu().numpy(), want) < tol, (core.coupling_kind, prec, mode)


# ---------------------------------------------------------------------------------------------
# the Hadamard alpha/beta contract, scalar operator per component
# ---------------------------------------------------------------------------------------------
SCALES = (1.0, 0.5, -2.0)


def multicomponent(core):
    """The same map with three moment components whose leaf bases are s_c times the original's."""
    c = copy.copy(core)
    c.ncomp = 3
    c.collections_test = {n: np.concatenate([s * C for s in SCALES]) for n, C in core.collections_test.items()}
    c.collections_trial = (c.collections_test if core.collections_trial is core.collections_test else
                           {n: np.concatenate([s * C for s in SCALES]) for n, C in core.collections_trial.items()})
    return c


def contract_maps():
    rng = np.random.default_rng(11)
    t = build_tree(rng.random((1500, 3)), depth=3, root_center=[0.5] * 3, root_halfsize=0.5)
    real = methods.interpolation_core(t, methods.laplace, 3, nodes="equispaced", couplings="toeplitz")
    cplx = methods.interpolation_core(t, methods.helmholtz(3.0), 3, nodes="equispaced", couplings="toeplitz",
                                      transfers="separable")
    return {"real": real, "complex": cplx}


@pytest.mark.parametrize("field", ["real", "complex"])
def test_componentwise_operator_oracle(field):
    core = contract_maps()[field]
    multi = multicomponent(core)
    k = sum(s * s for s in SCALES)
    cp = field == "complex"
    for mode in (0, 1, 2):
        x = _x(core.trial.npoints, 2, 50 + mode, cp)
        one = oracle.farmul(core, x, mode)
        assert rel(oracle.farmul(multi, x, mode), k * one) < TOL64, mode
        a, b = (0.5 - 0.25j, 2.0 + 1.0j) if cp else (0.5, 2.0)
        y0 = _x(core.test.npoints, 2, 60 + mode, cp)
        for alpha, beta in ((1, 0), (0, 1), (1, 1), (a, b)):
            got = oracle.farmul(multi, x, mode, alpha=alpha, beta=beta, y=y0)
            want = oracle.farmul(core, x, mode, alpha=k * alpha, beta=beta, y=y0)
            assert rel(got, want) < TOL64, (mode, alpha, beta)


@pytest.mark.gpu
@pytest.mark.parametrize("field", ["real", "complex"])
def test_componentwise_operator_gpu(field):
    import torch

    core = contract_maps()[field]
    multi = multicomponent(core)
    k = sum(s * s for s in SCALES)
    cp = field == "complex"
    dt = torch.complex128 if cp else torch.float64
    for prec, tol in (("fp64", TOL64), ("fp32", 10 * TOL32)):
        m = copy.copy(multi)
        m.precision = prec
        ws = h2.H2Workspace(m, max_nrhs=2)
        for mode in (0, 1, 2):
            view = ws if mode == 0 else (h2.transpose(ws) if mode == 1 else h2.adjoint(ws))
            x = _x(core.trial.npoints, 2, 50 + mode, cp)
            xd = torch.from_numpy(np.ascontiguousarray(x.T)).to(DEV).t()
            x_before = xd.clone()
            a, b = (0.5 - 0.25j, 2.0 + 1.0j) if cp else (0.5, 2.0)
            y0 = _x(core.test.npoints, 2, 60 + mode, cp)
            for alpha, beta in ((1, 0), (0, 1), (1, 1), (a, b)):
                yd = torch.from_numpy(np.ascontiguousarray(y0.T)).to(DEV).t()
                h2.farmul_(yd, view, xd, alpha, beta)
                torch.cuda.synchronize()
                want = oracle.farmul(core, x, mode, alpha=k * alpha, beta=beta, y=y0)
                assert rel(yd.cpu().numpy(), want) < tol, (prec, mode, alpha, beta)
            assert torch.equal(xd, x_before), "the input was modified"
