"""Pin the CPU oracle against the reference's closed-form known-answer tests (tests/golden).

The fixtures restate, as numbers, what the reference's tests check analytically; see
tests/golden/make_golden.py for the source lines of each.
"""

import os

import numpy as np
import pytest

from oracle import oracle
from fakes import b4points, cluster_core, worked_example_core

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def test_worked_example_all_orientations():
    """docs/src/implementing/example.md:205-222: forward/transpose/adjoint at rtol 1e-12."""
    g = load("worked_example.npz")
    core, F = worked_example_core()
    assert np.allclose(F, g["F"])
    x = g["x"]
    assert rel(oracle.matvec(core, x, 0), g["y_fwd"]) < 1e-12
    assert rel(oracle.matvec(core, x, 1), g["y_t"]) < 1e-12
    assert rel(oracle.matvec(core, x, 2), g["y_h"]) < 1e-12


def test_worked_example_scaled():
    """example.md:237-252: mul!(out, op(A), x, 2-i, 3+2i) on out = fill(2+i)."""
    g = load("worked_example.npz")
    core, _ = worked_example_core()
    for mode, key in ((0, "ys_fwd"), (1, "ys_t"), (2, "ys_h")):
        y = oracle.matvec(core, g["x"], mode, alpha=complex(g["alpha"]), beta=complex(g["beta"]),
                          y=g["out0"])
        assert rel(y, g[key]) < 1e-12


def test_worked_example_matrix_columns():
    """example.md:214: Matrix(A) == F column by column (multi-RHS identity input)."""
    g = load("worked_example.npz")
    core, _ = worked_example_core()
    n = g["F"].shape[0]
    M = oracle.matvec(core, np.eye(n, dtype=np.complex128), 0)
    assert rel(M, g["F"]) < 1e-12


def test_worked_example_has_far_and_near():
    """example.md:104-106: far pairs exist, some sources are not leaves, near is partial."""
    core, _ = worked_example_core()
    far = core.plans.far
    assert far.shape[0] > 0
    assert any(not core.trial.isleaf(int(b)) for b in far[:, 1])
    nnear = sum(core.test.values(int(a)).size * core.trial.values(int(b)).size
                for a, b in core.plans.near)
    assert 0 < nnear < 32 * 32


def test_two_cluster_farmul():
    """test/farinteractions/test_farmul.jl:17-97, closed form F[1:4,5:8] = F[5:8,1:4] = c."""
    g = load("clusters_b4.npz")
    pts = np.stack([g["points"], np.zeros(8), np.zeros(8)], axis=1)
    core, F, _ = cluster_core(pts, [0, 0, 0, 0, 1, 1, 1, 1], complex(g["c"]), minhalfsize=2.0)
    assert np.allclose(F, g["F"])
    x = g["x"]
    assert rel(oracle.farmul(core, x, 0), g["y_fwd"]) < 1e-12
    assert rel(oracle.farmul(core, x, 1), g["y_t"]) < 1e-12
    assert rel(oracle.farmul(core, x, 2), g["y_h"]) < 1e-12
    y = oracle.farmul(core, x, 0, alpha=complex(g["alpha"]), beta=complex(g["beta"]), y=g["y0"])
    assert rel(y, g["y_acc"]) < 1e-12
    # the only far pair sits two levels above the leaves (the hand-verifiable chain of the test)
    lv = core.test.level[core.plans.far[:, 0]]
    assert set(lv.tolist()) == {3}
    assert core.test.level[core.test.leaves()].min() == 5 or core.test.leaves().size == 2


def test_two_cluster_farmul_overwrites_stale_y():
    """3-argument farmul! zero-fills y first (farmul.jl:47-55)."""
    g = load("clusters_b4.npz")
    pts = np.stack([g["points"], np.zeros(8), np.zeros(8)], axis=1)
    core, _, _ = cluster_core(pts, [0, 0, 0, 0, 1, 1, 1, 1], complex(g["c"]), minhalfsize=2.0)
    y = oracle.farmul(core, g["x"], 0, y=np.full(8, np.nan + 0j))
    assert rel(y, g["y_fwd"]) < 1e-12


@pytest.mark.parametrize("tag", ["c", "r"])
def test_many_clusters_closed_form(tag):
    """test_component_harness.jl:88-118: F[i,j] = c iff clusters differ, all orientations."""
    g = load("clusters_6x20.npz")
    pts = np.stack([g["points"], np.zeros(120), np.zeros(120)], axis=1)
    field = "complex" if tag == "c" else "real"
    c = complex(g[f"{tag}_c"]) if tag == "c" else float(g[f"{tag}_c"])
    core, F, _ = cluster_core(pts, g["cid"], c, field=field, minhalfsize=1.0)
    x = g[f"{tag}_x"]
    assert rel(oracle.farmul(core, x, 0), g[f"{tag}_fwd"]) < 1e-12
    assert rel(oracle.farmul(core, x, 1), g[f"{tag}_t"]) < 1e-12
    assert rel(oracle.farmul(core, x, 2), g[f"{tag}_h"]) < 1e-12
    # every far pair joins different clusters
    cid = g["cid"]
    for a, b in core.plans.far:
        assert cid[core.test.values_below(a)[0] if hasattr(core.test, "values_below") else
                   _first_value(core.test, int(a))] != cid[_first_value(core.trial, int(b))]


def _first_value(tree, n):
    while not tree.isleaf(n):
        n = int(tree.children(n)[0])
    return int(tree.values(n)[0])


def test_toeplitz_operator_vs_dense():
    """test/H2Toeplitz/test_smoke.jl:38-78: FFT matvec == dense wrap-around multilevel Toeplitz."""
    g = load("toeplitz_smoke.npz")
    for q in range(6):
        kernel = g[f"kernel{q}"]
        khat = oracle.dft(kernel)
        assert np.allclose(khat, np.fft.fftn(kernel), rtol=1e-12, atol=1e-12)
        x = g[f"x{q}"]
        assert rel(oracle.toeplitz_apply(khat, x), g[f"Tx{q}"]) < 1e-9
        assert rel(oracle.toeplitz_apply(khat, x, adjoint=True), g[f"THx{q}"]) < 1e-9
        assert np.linalg.norm(g[f"Tx{q}"]) > 1e-8


def test_toeplitz_adjoint_duality():
    """test_smoke.jl:81-94: <y, A x> == <A' y, x>."""
    rng = np.random.default_rng(8)
    s = (3, 2, 2)
    kernel = rng.standard_normal(tuple(2 * v - 1 for v in s)) + 1j * rng.standard_normal(tuple(2 * v - 1 for v in s))
    khat = oracle.dft(kernel)
    n = int(np.prod(s))
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    lhs = np.vdot(y, oracle.toeplitz_apply(khat, x))
    rhs = np.vdot(oracle.toeplitz_apply(khat, y, adjoint=True), x)
    assert abs(lhs - rhs) <= 1e-9 * abs(lhs)


@pytest.mark.parametrize("ntest,ntrial", [(256, 16), (16, 256)])
def test_petrov_side_owned_transfers(ntest, ntrial):
    """test/farinteractions/test_rectangular.jl:103-154: rectangular map, different tree depths,
    distinct per-side transfers; forward/transpose/adjoint equal the complete matrix at 1e-12."""
    from fakes import petrov_core

    core, F, N = petrov_core(ntest, ntrial)
    assert F.shape == (ntest, ntrial)
    assert core.test.nlevels != core.trial.nlevels
    rng = np.random.default_rng(20260720)
    x = rng.standard_normal(ntrial) + 1j * rng.standard_normal(ntrial)
    y = rng.standard_normal(ntest) + 1j * rng.standard_normal(ntest)
    assert rel(oracle.farmul(core, x, 0), F @ x) < 1e-12
    yt = oracle.farmul(core, y, 1)
    ya = oracle.farmul(core, y, 2)
    assert rel(yt, F.T @ y) < 1e-12
    assert rel(ya, F.conj().T @ y) < 1e-12
    assert rel(ya, yt) > 0.1            # the conjugation path is exercised
    assert rel(oracle.matvec(core, x, 0), (F + N) @ x) < 1e-12


def test_petrov_side_swap_is_visible():
    """test_rectangular.jl:155-: with the two side constants swapped the product changes, so the
    tests above fail if the traversal resolves the wrong side."""
    from fakes import petrov_core

    core, F, _ = petrov_core()
    swapped, G, _ = petrov_core(c_trial=3.0, c_test=2.0)
    assert rel(G, F) > 0.1
    x = np.random.default_rng(1).standard_normal(16) + 0j
    assert rel(oracle.farmul(swapped, x, 0), F @ x) > 0.1
