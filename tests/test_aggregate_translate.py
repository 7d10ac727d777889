"""Descriptors flattened from AggregateTranslateMode plans.

In H2Factory's AggregateTranslateMode the I2O translations of a level run right after the upward
pass has formed that level's moments (src/farinteractions/aggregation.jl:144-219): a receiving node
gets its translating partners level by level, finest level first
(`H2Trees.translatingnodes(plan, receivingnode, level)`, aggregation.jl:282-308), and only the
translating nodes' moments are kept past their level (`istranslatingnode` gates `modulate_in!`,
aggregation.jl:224-226 and 267-269; the even/odd transient level pools of
src/moments/allocatemoments.jl:273-293). A descriptor flattened from such a plan therefore holds
the AggregateMode descriptor's pairs, grouped per receiving node by the translating node's level
(bottom-up), with the store flags on the translating nodes only.

The library takes that descriptor as it is. The maps here are adaptive (clustered points, leaves
of at most a few points), so receiving nodes have partners on several levels and the regrouping
really reorders the lists; Petrov maps (different test and trial trees) are included. Products
agree with the AggregateMode descriptor's to rounding, on the oracle and on the GPU, in all three
orientations, FP64 and FP32.
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


def clustered(n, seed, centers=6):
    rng = np.random.default_rng(seed)
    c = rng.random((centers, 3)) * 0.8 + 0.1
    w = rng.choice(centers, n)
    p = c[w] + rng.standard_normal((n, 3)) * rng.choice([0.01, 0.05, 0.15], centers)[w, None]
    return build_tree(np.clip(p, 0.0, 1.0), maxvalues=12, root_center=[0.5] * 3, root_halfsize=0.5)


def maps():
    return {
        "galerkin-laplace": methods.interpolation_core(clustered(1800, 1), methods.laplace, 3),
        "galerkin-helmholtz-sym": methods.interpolation_core(clustered(1500, 2), methods.helmholtz(5.0), 3,
                                                             symmetry=True, transfers="separable"),
        "petrov-laplace": methods.interpolation_core(clustered(1200, 3), methods.laplace, 3,
                                                     trial=clustered(1600, 4, centers=4)),
    }


def _regroup(side, src_tree):
    """One side's receiving lists in AggregateTranslate order: per receiving node, the translating
    partners by level, finest first (node id within a level)."""
    s = copy.copy(side)
    recv = np.repeat(np.arange(side.i2o_ptr.size - 1), np.diff(side.i2o_ptr))
    order = np.lexsort((side.i2o_src, -src_tree.level[side.i2o_src], recv))
    s.i2o_src = side.i2o_src[order].astype(np.int32)
    s.i2o_pair = side.i2o_pair[order].astype(np.int64)
    return s, bool(np.any(order != np.arange(order.size)))


def aggregate_translate(core):
    """`core` with both sides' plans as an AggregateTranslatePlan lists them."""
    c = copy.copy(core)
    p = copy.copy(core.plans)
    # forward maps receive on the test side from trial nodes; transposed ones the other way round
    p.test, moved_test = _regroup(core.plans.test, core.trial)
    p.trial, moved_trial = _regroup(core.plans.trial, core.test)
    c.plans = p
    return c, moved_test or moved_trial


def _translating_flags_match(core):
    """Each side stores exactly the nodes that the other side's lists translate from."""
    for side, other in ((core.plans.test, core.plans.trial), (core.plans.trial, core.plans.test)):
        want = np.zeros_like(side.agg_store)
        want[np.unique(other.i2o_src)] = 1
        if not np.array_equal(side.agg_store, want):
            return False
    return True


def _x(n, nrhs, seed, cplx):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, nrhs))
    return x + 1j * rng.standard_normal((n, nrhs)) if cplx else x


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.mark.parametrize("name", ["galerkin-laplace", "galerkin-helmholtz-sym", "petrov-laplace"])
def test_aggregate_translate_descriptor_oracle(name):
    core = maps()[name]
    at, moved = aggregate_translate(core)
    assert moved, "the map has no receiving node with partners on two levels"
    assert _translating_flags_match(core) and _translating_flags_match(at)
    levels = {int(core.trial.level[s]) for s in core.plans.test.i2o_src}
    assert len(levels) > 1
    cplx = core.field == "complex"
    for mode in (0, 1, 2):
        n = core.trial.npoints if mode == 0 else core.test.npoints
        x = _x(n, 3, 70 + mode, cplx)
        want = oracle.matvec(core, x, mode)
        got = oracle.matvec(at, x, mode)
        assert rel(got, want) < TOL64, (name, mode)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["galerkin-laplace", "galerkin-helmholtz-sym", "petrov-laplace"])
def test_aggregate_translate_descriptor_gpu(name):
    import torch

    core = maps()[name]
    at, _ = aggregate_translate(core)
    cplx = core.field == "complex"
    dt = torch.complex128 if cplx else torch.float64
    for prec, tol in (("fp64", TOL64), ("fp32", TOL32)):
        c = copy.copy(at)
        c.precision = prec
        ws = h2.H2Workspace(c, max_nrhs=3)
        for mode in (0, 1, 2):
            nin = core.trial.npoints if mode == 0 else core.test.npoints
            nout = core.test.npoints if mode == 0 else core.trial.npoints
            x = _x(nin, 3, 70 + mode, cplx)
            want = oracle.matvec(core, x, mode)
            view = ws if mode == 0 else (h2.transpose(ws) if mode == 1 else h2.adjoint(ws))
            xd = torch.from_numpy(np.ascontiguousarray(x.T)).to(DEV).t()
            y = torch.zeros((3, nout), dtype=dt, device=DEV).t()
            h2.mul_(y, view, xd)
            torch.cuda.synchronize()
            assert rel(y.cpu().numpy(), want) < tol, (name, prec, mode)
        ws.close()
