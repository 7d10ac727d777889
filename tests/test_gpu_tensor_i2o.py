"""Dense I2O of the FP32 form on the tcgen05 tensor cores (three-term TF32 split), GPU.

The FP32 form takes the tensor-core kernel when its couplings are dense and the right-hand sides
make at least 4 FP32 columns (real maps: >= 4 right-hand sides, complex: >= 2; the MMA's N is
padded to 16). Each
case multiplies in every orientation and is compared with the FP64 form of the same map, which
test_gpu_parity.py pins to the oracle at 1e-12, and the sphere case directly with the oracle.
Tolerances: the whole product within 1e-6 relative L2 of the FP64 result (the served form's bar);
the far part alone within 1e-5, since the near field (FP64 in both forms) dilutes the far field's
error in the whole product. Shapes cover one and two 128-row tiles (64 and 216 coefficients), one
to three right-hand-side tiles (at most 64 FP32 columns each), rows and columns permuted by
symmetry-reduced couplings, and Petrov maps (source and receiver coefficient counts differ).
"""

import copy

import numpy as np
import pytest

import h2factory_b200 as h2
from h2factory_b200 import _abi, methods
from oracle import oracle
from test_gpu_parity import CASES, ORIENT, _x, rel, run

pytestmark = pytest.mark.gpu

TOL32 = 1e-5
BAR = 1e-6  # whole product vs the FP64 form: the reduced-precision bar of the served form


def _fp32(core):
    c = copy.copy(core)
    c.precision = "fp32"
    return c


@pytest.fixture(scope="module")
def cores():
    return {}


def _core(cores, name):
    if name not in cores:
        cores[name] = CASES[name]()
    return cores[name]


@pytest.mark.parametrize("name,nrhs", [
    ("cheb-laplace-dense", 4),
    ("cheb-laplace-dense", 7),
    ("cheb-laplace-dense", 16),
    ("cheb-laplace-dense", 130),
    ("cheb-helmholtz", 2),
    ("cheb-helmholtz", 3),
    ("cheb-helmholtz", 8),
    ("cheb-helmholtz", 32),
    ("cheb-helmholtz", 70),
    ("sym-cheb-laplace", 16),
    ("sym-cheb-helmholtz", 8),
    ("sym-cheb-helmholtz", 37),
    ("petrov-cheb-laplace", 24),
])
def test_tensor_i2o_matches_fp64(cores, name, nrhs):
    core = _core(cores, name)
    timeouts = _abi.tensor_wait_timeouts(0)
    ws64 = h2.H2Workspace(core, max_nrhs=nrhs)
    ws32 = h2.H2Workspace(_fp32(core), max_nrhs=nrhs)
    for mode, op in ORIENT:
        x = _x(core, nrhs, 21 + mode, mode)
        want = run(h2.mul_, op(ws64), x)
        got = run(h2.mul_, op(ws32), x)
        err = rel(got, want)
        assert err < BAR, (name, nrhs, mode, err)
        want_far = run(h2.farmul_, op(ws64), x)
        got_far = run(h2.farmul_, op(ws32), x)
        err_far = rel(got_far, want_far)
        assert err_far < TOL32, (name, nrhs, mode, err_far)
    assert _abi.tensor_wait_timeouts(0) == timeouts


def test_tensor_i2o_sphere_against_oracle(cores):
    """216 coefficients (two row tiles), 32 complex right-hand sides (one 64-column tile),
    symmetry-reduced couplings: forward and adjoint against the FP64 oracle."""
    core = _core(cores, "sphere-cheb6-helmholtz-sym")
    timeouts = _abi.tensor_wait_timeouts(0)
    ws32 = h2.H2Workspace(_fp32(core), max_nrhs=32)
    desc = h2.flatten(core)
    for mode, op in (ORIENT[0], ORIENT[2]):
        x = _x(core, 32, 27, mode)
        want = oracle.matvec(core, x, mode, desc=desc)
        assert rel(run(h2.mul_, op(ws32), x), want) < BAR, mode
        want_far = oracle.farmul(core, x, mode, desc=desc)
        assert rel(run(h2.farmul_, op(ws32), x), want_far) < TOL32, mode
    assert _abi.tensor_wait_timeouts(0) == timeouts


def test_tensor_i2o_repeatable(cores):
    """Two products of one block give bit-identical results (no atomics, fixed order)."""
    core = _core(cores, "cheb-helmholtz")
    ws32 = h2.H2Workspace(_fp32(core), max_nrhs=32)
    x = _x(core, 32, 31)
    a = run(h2.farmul_, ws32, x)
    b = run(h2.farmul_, ws32, x)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("name,nrhs", [
    ("cheb-laplace-dense", 1),
    ("cheb-laplace-dense", 3),
    ("cheb-helmholtz", 1),
    ("sym-cheb-laplace", 2),
    ("sym-cheb-helmholtz", 1),
    ("petrov-cheb-laplace", 3),
])
def test_small_blocks_fp32_dense(cores, name, nrhs):
    """Below the tensor-core kernel's range (fewer than 4 FP32 columns) the dense I2O of the FP32
    form runs the FMA / FP64 mma.sync tile products; it still matches its FP64 product within 1e-6."""
    core = _core(cores, name)
    ws64 = h2.H2Workspace(core, max_nrhs=nrhs)
    ws32 = h2.H2Workspace(_fp32(core), max_nrhs=nrhs)
    for mode, op in ORIENT:
        x = _x(core, nrhs, 51 + mode, mode)
        assert rel(run(h2.mul_, op(ws32), x), run(h2.mul_, op(ws64), x)) < BAR, (name, nrhs, mode)
