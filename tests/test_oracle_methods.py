"""Oracle checks on real FMM methods (CPU): method error, storage equivalences, orientation.

* every (i, j) is covered exactly once by near + far (the plan invariant behind
  src/nearinteractions/nearmul.jl:54-111 and src/farinteractions/farmul.jl:91-133);
* Chebyshev/equispaced H2 products approximate the dense kernel to the interpolation error;
* separable and dense transfers give the same map (src/maps/leveltranslator.jl:84-265);
* Toeplitz and dense couplings give the same map for equispaced nodes
  (src/moments/toeplitz/toeplitzmul.jl vs i2otranslationcollection.jl:367-409);
* transpose/adjoint obey the factorisation identities of test/farinteractions/test_factorization.jl.
"""

import numpy as np
import pytest

from h2factory_b200 import methods
from h2factory_b200.trees import build_plans, build_tree
from oracle import oracle


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def cube_tree():
    rng = np.random.default_rng(1)
    pts = rng.random((1200, 3))
    return build_tree(pts, maxvalues=40, root_center=[0.5] * 3, root_halfsize=0.5)


def test_plan_partition_covers_each_pair_once(cube_tree):
    t = cube_tree
    plans = build_plans(t)
    n = t.npoints
    cover = np.zeros((n, n), np.int32)

    def dofs(node):
        stack, out = [int(node)], []
        while stack:
            m = stack.pop()
            if t.isleaf(m):
                out.extend(t.values(m).tolist())
            else:
                stack.extend(int(c) for c in t.children(m))
        return np.array(out, np.int64)

    for a, b in plans.far:
        cover[np.ix_(dofs(a), dofs(b))] += 1
    for a, b in plans.near:
        cover[np.ix_(t.values(int(a)), t.values(int(b)))] += 1
    assert cover.min() == 1 and cover.max() == 1
    # Galerkin plans are symmetric
    assert set(map(tuple, plans.far.tolist())) == set(map(tuple, plans.far[:, ::-1].tolist()))


def test_chebyshev_laplace_vs_dense(cube_tree):
    t = cube_tree
    core = methods.interpolation_core(t, methods.laplace, 4)
    K = methods.kernel_matrix(methods.laplace, t.points, t.points)
    x = np.random.default_rng(2).standard_normal(t.npoints)
    y = oracle.matvec(core, x)
    assert rel(y, K @ x) < 2e-3
    # near part alone is exact on its blocks
    yn = oracle.nearmul(core, x)
    far = core.plans.far
    assert far.shape[0] > 0 and np.isfinite(yn).all()


def test_separable_equals_dense_transfers(cube_tree):
    t = cube_tree
    x = np.random.default_rng(3).standard_normal(t.npoints)
    a = methods.interpolation_core(t, methods.laplace, 3, transfers="dense")
    b = methods.interpolation_core(t, methods.laplace, 3, transfers="separable")
    for mode in (0, 1, 2):
        assert rel(oracle.matvec(b, x, mode), oracle.matvec(a, x, mode)) < 1e-13


@pytest.fixture(scope="module")
def uniform_tree():
    rng = np.random.default_rng(4)
    pts = rng.random((3000, 3))
    return build_tree(pts, depth=4, root_center=[0.5] * 3, root_halfsize=0.5)


def test_toeplitz_equals_dense_couplings(uniform_tree):
    t = uniform_tree
    x = np.random.default_rng(5).standard_normal(t.npoints)
    dense = methods.interpolation_core(t, methods.laplace, 3, nodes="equispaced", couplings="dense")
    toep = methods.interpolation_core(t, methods.laplace, 3, nodes="equispaced", couplings="toeplitz")
    for mode in (0, 1, 2):
        assert rel(oracle.matvec(toep, x, mode), oracle.matvec(dense, x, mode)) < 1e-12
    K = methods.kernel_matrix(methods.laplace, t.points, t.points)
    assert rel(oracle.matvec(toep, x), K @ x) < 2e-2


def test_toeplitz_complex_kernel(uniform_tree):
    t = uniform_tree
    kern = methods.helmholtz(3.0)
    rng = np.random.default_rng(6)
    x = rng.standard_normal(t.npoints) + 1j * rng.standard_normal(t.npoints)
    dense = methods.interpolation_core(t, kern, 3, nodes="equispaced", couplings="dense")
    toep = methods.interpolation_core(t, kern, 3, nodes="equispaced", couplings="toeplitz")
    for mode in (0, 1, 2):
        assert rel(oracle.matvec(toep, x, mode), oracle.matvec(dense, x, mode)) < 1e-12


def test_orientation_identities_complex(cube_tree):
    """<y, A x> = <A^H y, x>; A^T x = conj(A^H conj(x)) (test_factorization.jl:132-177)."""
    t = cube_tree
    core = methods.interpolation_core(t, methods.helmholtz(2.0), 3)
    rng = np.random.default_rng(7)
    x = rng.standard_normal(t.npoints) + 1j * rng.standard_normal(t.npoints)
    y = rng.standard_normal(t.npoints) + 1j * rng.standard_normal(t.npoints)
    Ax = oracle.matvec(core, x, 0)
    AHy = oracle.matvec(core, y, 2)
    assert abs(np.vdot(y, Ax) - np.vdot(AHy, x)) < 1e-12 * abs(np.vdot(y, Ax))
    ATx = oracle.matvec(core, x, 1)
    assert rel(ATx, np.conj(oracle.matvec(core, np.conj(x), 2))) < 1e-13
    # complex-symmetric Galerkin kernel: the H2 approximation is symmetric too
    assert rel(ATx, Ax) < 1e-12


def test_scaled_mul_and_farmul_rules(cube_tree):
    """5-arg mul!: near (α, β) then far (α, 1); far 5-arg leaves non-receiving leaves alone."""
    t = cube_tree
    core = methods.interpolation_core(t, methods.helmholtz(1.0), 3)
    rng = np.random.default_rng(8)
    x = rng.standard_normal(t.npoints) + 1j * rng.standard_normal(t.npoints)
    y0 = rng.standard_normal(t.npoints) + 1j * rng.standard_normal(t.npoints)
    a, b = 0.3 - 1.1j, -0.7 + 0.25j
    for mode in (0, 1, 2):
        full = oracle.matvec(core, x, mode)
        y = oracle.matvec(core, x, mode, alpha=a, beta=b, y=y0)
        assert rel(y, a * full + b * y0) < 1e-13
        near = oracle.nearmul(core, x, mode)
        far = oracle.farmul(core, x, mode)
        assert rel(near + far, full) < 1e-13


def test_petrov_interpolation_vs_dense():
    """Rectangular map (test points != trial points, different depths) against the dense kernel
    in all orientations: the traversal pairs boxes of two trees on one root box."""
    rng = np.random.default_rng(6)
    test = build_tree(rng.random((3000, 3)), maxvalues=20, root_center=[0.5] * 3, root_halfsize=0.5)
    trial = build_tree(rng.random((300, 3)), maxvalues=40, root_center=[0.5] * 3, root_halfsize=0.5)
    core = methods.interpolation_core(test, methods.helmholtz(2.0), 4, trial=trial)
    assert core.test.nlevels != core.trial.nlevels
    K = methods.kernel_matrix(core.kernel, test.points, trial.points)
    for mode, op in ((0, K), (1, K.T), (2, K.conj().T)):
        x = rng.standard_normal(op.shape[1]) + 1j * rng.standard_normal(op.shape[1])
        y = oracle.matvec(core, x, mode)
        assert np.linalg.norm(y - op @ x) / np.linalg.norm(op @ x) < 5e-3


@pytest.mark.parametrize("kind", ["dense", "toeplitz"])
def test_symmetry_reduced_couplings_equal_unreduced(kind):
    """symmetryreduceddense.jl / symmetryreducedcollection.jl, test_toeplitz3d.jl:120-140: one
    stored coupling per orbit of the cube's signed axis permutations (about 20x fewer), read
    through permutations, gives the map of one coupling per translation, in every orientation."""
    rng = np.random.default_rng(7)
    if kind == "dense":
        tree = build_tree(rng.random((2000, 3)), maxvalues=40, root_center=[0.5] * 3, root_halfsize=0.5)
        mk = lambda sym: methods.interpolation_core(tree, methods.helmholtz(3.0), 3, symmetry=sym)
    else:
        tree = build_tree(rng.random((3000, 3)), depth=4, root_center=[0.5] * 3, root_halfsize=0.5)
        mk = lambda sym: methods.interpolation_core(tree, methods.laplace, 4, nodes="equispaced",
                                                    couplings="toeplitz", symmetry=sym)
    plain, reduced = mk(False), mk(True)
    assert len(plain.couplings) / len(reduced.couplings) > 5
    for mode in range(3):
        x = rng.standard_normal(tree.npoints) + 1j * rng.standard_normal(tree.npoints)
        if plain.field == "real":
            x = x.real
        a, b = oracle.matvec(plain, x, mode), oracle.matvec(reduced, x, mode)
        assert rel(b, a) < 1e-13
