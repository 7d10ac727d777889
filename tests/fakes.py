"""Closed-form test maps, restated from the reference's own known-answer tests.

H2Factory's tests build these through H2FactoryTestUtils (not part of the reference tree); here
they are rebuilt from the tests' descriptions:

* `worked_example_core`: docs/src/implementing/example.md:28-257 -- 32 points on [0, 1], kernel
  K(s, t) = 1 + 2s + 3t + (4+i)st, leaf bases [1; s], identity transfers, coupling
  C = [1 3; 2 4+i]; the H2 product is exact.
* `cluster_core`: test/farinteractions/test_farmul.jl:17-97 and
  test/farinteractions/test_component_harness.jl:88-118 -- charges summed up the tree
  (identity I2I), scaled by a complex constant c across well-separated clusters (scalar I2O),
  broadcast down (identity O2O): F[i, j] = c iff i and j sit in different clusters.
"""

import numpy as np

from h2factory_b200.core import H2Core
from h2factory_b200.trees import build_plans, build_tree


def worked_kernel(s, t):
    return 1 + 2 * s + 3 * t + (4 + 1j) * s * t


def worked_example_core(n: int = 32) -> tuple:
    coords = np.linspace(0.0, 1.0, n)
    tree = build_tree(coords[:, None], maxvalues=2)
    plans = build_plans(tree)
    shape = np.zeros((tree.nlevels + 1, 3), np.int32)
    shape[1:] = (2, 1, 1)
    colls = {}
    for leaf in tree.leaves():
        v = tree.values(int(leaf))
        c = np.zeros((1, 2, v.size), np.complex128)
        c[0, 0, :] = 1
        c[0, 1, :] = coords[v]
        colls[int(leaf)] = c
    eye = np.eye(2, dtype=np.complex128)
    transfers = {(l, s): eye for l in range(2, tree.nlevels + 1) for s in range(tree.nsectors)}
    Cmat = np.array([[1, 3], [2, 4 + 1j]], np.complex128)
    core = H2Core(field="complex", test=tree, trial=tree, plans=plans, ncomp=1, dim=1,
                  shape_test=shape, shape_trial=shape, collections_test=colls,
                  collections_trial=colls, transfers_test=transfers, transfers_trial=transfers,
                  transfer_kind="dense", coupling_kind="dense", couplings=[Cmat],
                  pair_coupling=np.zeros(plans.far.shape[0], np.int64), alpha=1.0,
                  conj_leaf_adjoint=True)
    blocks = []
    for a, b in plans.near:
        s = coords[tree.values(int(a))]
        t = coords[tree.values(int(b))]
        blocks.append(worked_kernel(s[:, None], t[None, :]).astype(np.complex128))
    core.set_near_blocks(blocks)
    F = worked_kernel(coords[:, None], coords[None, :])
    return core, F


def cluster_core(points, cluster_id, c, *, field="complex", maxvalues=None, minhalfsize=0.0,
                 near_kernel=None, alpha=1.0):
    """Scalar moments (ncoef = 1), identity transfers, coupling c on every far pair."""
    pts = np.asarray(points, np.float64)
    tree = build_tree(pts, maxvalues=maxvalues if maxvalues is not None else 0,
                      minhalfsize=minhalfsize)
    plans = build_plans(tree)
    dt = np.complex128 if field == "complex" else np.float64
    shape = np.zeros((tree.nlevels + 1, 3), np.int32)
    shape[1:] = (1, 1, 1)
    colls = {int(l): np.ones((1, 1, tree.values(int(l)).size), dt) for l in tree.leaves()}
    one = np.ones((1, 1), dt)
    transfers = {(l, s): one for l in range(2, tree.nlevels + 1) for s in range(tree.nsectors)}
    core = H2Core(field=field, test=tree, trial=tree, plans=plans, ncomp=1, dim=pts.shape[1],
                  shape_test=shape, shape_trial=shape, collections_test=colls,
                  collections_trial=colls, transfers_test=transfers, transfers_trial=transfers,
                  transfer_kind="dense", coupling_kind="dense",
                  couplings=[np.array([[c]], dt)],
                  pair_coupling=np.zeros(plans.far.shape[0], np.int64), alpha=alpha,
                  conj_leaf_adjoint=True)
    cid = np.asarray(cluster_id)
    F = np.where(cid[:, None] != cid[None, :], c, 0).astype(dt)
    N = np.zeros_like(F)
    if near_kernel is not None:
        blocks = []
        for a, b in plans.near:
            va, vb = tree.values(int(a)), tree.values(int(b))
            blk = near_kernel(pts[va, 0][:, None], pts[vb, 0][None, :]).astype(dt)
            N[np.ix_(va, vb)] = blk
            blocks.append(blk)
        core.set_near_blocks(blocks)
    else:
        core.set_near_blocks([np.zeros((tree.values(int(a)).size, tree.values(int(b)).size), dt)
                              for a, b in plans.near])
    return core, F, N


def b4points():
    """test/farinteractions/component_harness_fixtures.jl:4 -- two clusters of two pairs."""
    return np.array([0.0, 0.1, 5.0, 5.1, 40.0, 40.1, 45.0, 45.1])


def manyclusters(k, n, gap=100.0, spread=0.1):
    """component_harness_fixtures.jl:38-48: k clusters of n points on a line."""
    pts, cid = [], []
    for c in range(k):
        for j in range(n):
            pts.append((c * gap + spread * j / (n - 1), 0.0, 0.0))
            cid.append(c)
    return np.array(pts), np.array(cid)


def petrov_core(ntest=256, ntrial=16, c_trial=2.0, c_test=3.0, c_i2o=0.75 - 1.25j):
    """Rectangular Petrov map with side-owned scalar transfers.

    Restates test/farinteractions/test_rectangular.jl:44-76: uniform points on [0, 1] on each
    side (different counts, hence different tree depths), leaf bases of ones, every trial-side
    I2I/O2O equal to c_trial, every test-side one equal to c_test (real, so that the transposed
    and adjoint factors stay exact), and one complex coupling c_i2o. The complete matrix is
    F[i, j] = sum over far pairs (a, b) with i under a and j under b of
    c_test^(level(leaf(i)) - level(a)) * c_i2o * c_trial^(level(leaf(j)) - level(b)),
    assembled here from the trees alone. Near blocks hold 1 / (1 + |s - t|).
    """
    def side(n):
        pts = ((np.arange(n) + 0.5) / n)[:, None]
        return build_tree(pts, maxvalues=1, minhalfsize=0.004, root_center=[0.5], root_halfsize=0.5)

    test, trial = side(ntest), side(ntrial)
    plans = build_plans(test, trial)

    def shape(t):
        sh = np.zeros((t.nlevels + 1, 3), np.int32)
        sh[1:] = (1, 1, 1)
        return sh

    def colls(t):
        return {int(l): np.ones((1, 1, t.values(int(l)).size), np.complex128) for l in t.leaves()}

    def transfers(t, c):
        return {(l, s): np.full((1, 1), c, np.complex128) for l in range(2, t.nlevels + 1)
                for s in range(t.nsectors)}

    core = H2Core(field="complex", test=test, trial=trial, plans=plans, ncomp=1, dim=1,
                  shape_test=shape(test), shape_trial=shape(trial), collections_test=colls(test),
                  collections_trial=colls(trial), transfers_test=transfers(test, c_test),
                  transfers_trial=transfers(trial, c_trial), transfer_kind="dense",
                  coupling_kind="dense", couplings=[np.array([[c_i2o]], np.complex128)],
                  pair_coupling=np.zeros(plans.far.shape[0], np.int64), alpha=1.0,
                  conj_leaf_adjoint=True)

    def chains(t):
        """Per point: its leaf's level and its ancestor at every level (-1 below the leaf)."""
        anc = np.full((t.npoints, t.nlevels + 1), -1, np.int64)
        lvl = np.zeros(t.npoints, np.int64)
        for leaf in t.leaves():
            v = t.values(int(leaf))
            lvl[v] = t.level[leaf]
            n = int(leaf)
            while n >= 0:
                anc[v, t.level[n]] = n
                n = int(t.parent[n])
        return anc, lvl

    (ai, li), (aj, lj) = chains(test), chains(trial)
    F = np.zeros((ntest, ntrial), np.complex128)
    for a, b in plans.far:
        rows = np.nonzero(ai[:, test.level[a]] == a)[0]
        cols = np.nonzero(aj[:, trial.level[b]] == b)[0]
        F[np.ix_(rows, cols)] += (np.power(c_test, li[rows] - test.level[a])[:, None] * c_i2o
                                  * np.power(c_trial, lj[cols] - trial.level[b])[None, :])
    blocks, N = [], np.zeros_like(F)
    for a, b in plans.near:
        va, vb = test.values(int(a)), trial.values(int(b))
        blk = 1.0 / (1.0 + np.abs(test.points[va, 0][:, None] - trial.points[vb, 0][None, :]))
        blocks.append(blk.astype(np.complex128))
        N[np.ix_(va, vb)] = blk
    core.set_near_blocks(blocks)
    return core, F, N
