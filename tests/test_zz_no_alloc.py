"""h2b_farmul_noalloc: the far product for callers that cannot allocate device memory (GPU).

Some hosts cannot call cudaMalloc when they multiply: their device memory is owned by another
allocator (a framework's caching pool), or their serving loop forbids allocation after start-up.
The entry point runs the far passes in a scratch array compiled into the library instead of a
workspace. This file checks, through the C ABI, that it gives the same result as the workspace
path (h2b_farmul) and as the CPU oracle on two calls in a row -- the second call finds the first
call's data in the shared scratch --, that the calls leave the device's free memory unchanged,
that blocks of 13 right-hand sides and a map that fills the scratch almost to its end work, and
that a map too large for the scratch is refused with a clear error.

The file name sorts last so that a run stopping at the first failure has run every other test.
"""

import ctypes as C

import numpy as np
import pytest
import torch

import h2factory_b200 as h2
from h2factory_b200 import _abi, methods
from h2factory_b200.trees import build_tree
from oracle import oracle

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
TOL64 = 1e-12   # same bar as the FP64 parity tests
TOL32 = 1e-6   # FP32 far field against the FP64 products


def _cols(a, dt):
    a = np.asarray(a, dtype=dt)
    return torch.from_numpy(np.ascontiguousarray(a.T)).to(DEV).t()


def _noalloc(dcore, mode, x, y, alpha=None, beta=None):
    lib = _abi.load_library()
    n_in, nrhs = x.shape
    ab = None
    if alpha is not None:
        a, b = complex(alpha), complex(beta)
        ab = ((C.c_double * 2)(a.real, a.imag), (C.c_double * 2)(b.real, b.imag))
    st = lib.h2b_farmul_noalloc(dcore.handle, mode, nrhs, C.c_void_p(x.data_ptr()), n_in,
                                C.c_void_p(y.data_ptr()), y.shape[0], ab[0] if ab else None,
                                ab[1] if ab else None,
                                C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, lib.h2b_last_error().decode()


def _maps():
    rng = np.random.default_rng(3)
    t = build_tree(rng.random((3000, 3)), depth=4, root_center=[0.5] * 3, root_halfsize=0.5)
    yield "toeplitz-laplace", methods.interpolation_core(
        t, methods.laplace, 3, nodes="equispaced", couplings="toeplitz"), TOL64
    t2 = build_tree(rng.random((2000, 3)), maxvalues=40, root_center=[0.5] * 3, root_halfsize=0.5)
    yield "chebyshev-helmholtz", methods.interpolation_core(t2, methods.helmholtz(3.0), 3), TOL64
    core32 = methods.interpolation_core(t2, methods.helmholtz(3.0), 3, precision="fp32")
    yield "chebyshev-helmholtz-fp32", core32, TOL32


def _rel(g, w):
    return np.linalg.norm(g - w) / np.linalg.norm(w)


def _check_twice(core, tol, nrhs, seed=7):
    """Two rounds of 3- and 5-argument calls in every orientation against h2b_farmul and the
    oracle. Every tensor is made before the calls, and the workspace products run first (they load
    every kernel the calls use), so the device's free memory must not move across the calls."""
    ws = h2.H2Workspace(core, max_nrhs=nrhs)
    dt = core.dtype
    rng = np.random.default_rng(seed)
    n = core.trial.npoints
    a, b = (0.5 - 0.25j, 2.0 + 1.0j) if core.field == "complex" else (0.5, 2.0)
    cases = []
    for call in range(2):  # two calls in a row share (and reuse) the scratch
        for mode, view in ((0, ws), (1, h2.transpose(ws)), (2, h2.adjoint(ws))):
            xh = rng.standard_normal((n, nrhs))
            y0 = rng.standard_normal((n, nrhs))
            if core.field == "complex":
                xh = xh + 1j * rng.standard_normal((n, nrhs))
                y0 = y0 + 1j * rng.standard_normal((n, nrhs))
            x = _cols(xh, dt)
            want3, want5 = _cols(np.zeros((n, nrhs)), dt), _cols(y0, dt)
            h2.farmul_(want3, view, x)
            h2.farmul_(want5, view, x, a, b)
            cases.append((call, mode, xh, y0, x, want3, want5,
                          _cols(np.full((n, nrhs), np.nan), dt), _cols(y0, dt)))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for call, mode, xh, y0, x, want3, want5, got3, got5 in cases:
        st, err = _noalloc(ws.dcore, mode, x, got3)
        assert st == 0, err
        st, err = _noalloc(ws.dcore, mode, x, got5, a, b)
        assert st == 0, err
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0, "a no-alloc call changed the device's free memory"
    for call, mode, xh, y0, x, want3, want5, got3, got5 in cases:
        g3, g5 = got3.cpu().numpy(), got5.cpu().numpy()
        assert _rel(g3, want3.cpu().numpy()) < tol, (call, mode)
        assert _rel(g5, want5.cpu().numpy()) < tol, (call, mode, "scaled")
        if call == 0:
            assert _rel(g3, oracle.farmul(core, xh, mode)) < tol, (mode, "oracle")
            assert _rel(g5, oracle.farmul(core, xh, mode, a, b, y=y0)) < tol, (mode, "oracle scaled")
    ws.close()
    return ws


@pytest.mark.parametrize("name", ["toeplitz-laplace", "chebyshev-helmholtz", "chebyshev-helmholtz-fp32"])
def test_noalloc_matches_workspace_farmul_twice(name):
    core, tol = next((c, t) for n, c, t in _maps() if n == name)
    _check_twice(core, tol, 3)


def test_noalloc_thirteen_rhs_toeplitz():
    """13 right-hand sides: the multi-RHS kernels (FP64 tensor-core sibling I2O, a partial 16-wide
    block) take their arenas from the scratch too (a depth-3 Toeplitz map, whose arenas for 13
    right-hand sides fit the scratch)."""
    rng = np.random.default_rng(4)
    t = build_tree(rng.random((1500, 3)), depth=3, root_center=[0.5] * 3, root_halfsize=0.5)
    core = methods.interpolation_core(t, methods.laplace, 3, nodes="equispaced", couplings="toeplitz")
    _check_twice(core, TOL64, 13, seed=11)


def test_noalloc_scratch_almost_full():
    """The largest block that fits: the four 256-byte aligned arenas end just inside the scratch."""
    core, tol = next((c, t) for n, c, t in _maps() if n == "toeplitz-laplace")
    info = h2.DeviceCore(core).info()
    al = lambda v: (v + 255) // 256 * 256  # noqa: E731

    def need(q):
        return 2 * al(info.moment_elems * q * 8) + 2 * al(info.spectrum_elems * q * 16)

    nrhs = 1
    while need(nrhs + 1) <= _abi.H2B_NOALLOC_SCRATCH_BYTES:
        nrhs += 1
    assert need(nrhs) > _abi.H2B_NOALLOC_SCRATCH_BYTES * 0.9
    _check_twice(core, tol, nrhs, seed=13)


def test_noalloc_refuses_maps_beyond_the_scratch():
    rng = np.random.default_rng(0)
    t = build_tree(rng.random((8192, 3)), maxvalues=64, root_center=[0.5] * 3, root_halfsize=0.5)
    core = methods.interpolation_core(t, methods.laplace, 4)
    dcore = h2.DeviceCore(core)
    per_rhs = 2 * dcore.info().moment_elems * 8
    nrhs = _abi.H2B_NOALLOC_SCRATCH_BYTES // per_rhs + 2
    x = torch.zeros((nrhs, 8192), dtype=torch.float64, device=DEV).t()
    y = torch.zeros((nrhs, 8192), dtype=torch.float64, device=DEV).t()
    st, err = _noalloc(dcore, 0, x, y)
    assert st == _abi.H2B_ERR_UNSUPPORTED
    assert "built-in scratch" in err
