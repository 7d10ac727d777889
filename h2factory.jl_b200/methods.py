"""Method data for the H2 maps: what an H2Factory *method* (iFMM, MLFMA, ...) supplies.

H2Factory owns no physics (its docs: docs/src/algorithm.md:34-46): the method provides leaf
moment collections, level transfers, I2O couplings and near blocks. This module builds them for
interpolation-based FMMs on a 2^D tree:

* Chebyshev interpolation (black-box FMM): dense or separable transfers, dense M2L blocks per
  unique translation;
* equispaced interpolation: identical, but the M2L block of two same-size boxes is multilevel
  Toeplitz, stored as the FFT of its wrap-around kernel (the H2Toeplitz storage of
  src/moments/toeplitz/toeplitzmoment.jl:28-30, ext/H2Toeplitz/H2Toeplitz.jl:19-47);

for the Laplace kernel 1/(4 pi |x-y|) and the Helmholtz kernel exp(ik|x-y|)/(4 pi |x-y|), with
the self term set to zero. Index conventions follow H2Factory's moments: one component array
of extents (p, p, p) per node, column-major.
"""

from __future__ import annotations

import numpy as np

from .core import H2Core
from .trees import Tree, build_plans

__all__ = ["laplace", "helmholtz", "chebyshev_nodes", "equispaced_nodes", "lagrange",
           "interpolation_core", "kernel_matrix"]


def laplace(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """1/(4 pi |x - y|) for rows of x against rows of y; zero where x == y."""
    d = x[:, None, :] - y[None, :, :]
    r = np.sqrt(np.einsum("ijk,ijk->ij", d, d))
    with np.errstate(divide="ignore"):
        k = np.where(r > 0, 1.0 / (4.0 * np.pi * np.where(r > 0, r, 1.0)), 0.0)
    return k


def helmholtz(wavenumber: float):
    """exp(i k |x - y|)/(4 pi |x - y|); zero where x == y."""

    def kern(x, y):
        d = x[:, None, :] - y[None, :, :]
        r = np.sqrt(np.einsum("ijk,ijk->ij", d, d))
        rs = np.where(r > 0, r, 1.0)
        return np.where(r > 0, np.exp(1j * wavenumber * rs) / (4.0 * np.pi * rs), 0.0)

    kern.wavenumber = wavenumber
    return kern


def kernel_matrix(kernel, x, y, chunk: int = 2048) -> np.ndarray:
    """Dense kernel matrix, in row chunks to bound temporaries."""
    out = None
    for s in range(0, x.shape[0], chunk):
        blk = kernel(x[s:s + chunk], y)
        if out is None:
            out = np.empty((x.shape[0], y.shape[0]), dtype=blk.dtype)
        out[s:s + chunk] = blk
    return out


def chebyshev_nodes(p: int) -> np.ndarray:
    """Chebyshev points of the first kind on [-1, 1]."""
    k = np.arange(p)
    return np.cos((2 * k + 1) * np.pi / (2 * p))


def equispaced_nodes(p: int) -> np.ndarray:
    """Cell-centred equispaced points on [-1, 1]: -1 + (2k+1)/p."""
    return -1.0 + (2.0 * np.arange(p) + 1.0) / p


def lagrange(nodes: np.ndarray, t: np.ndarray) -> np.ndarray:
    """L[k, j] = prod_{m != k} (t_j - xi_m) / (xi_k - xi_m)."""
    p = nodes.size
    t = np.asarray(t, dtype=np.float64)
    L = np.ones((p, t.size))
    for k in range(p):
        for m in range(p):
            if m != k:
                L[k] *= (t - nodes[m]) / (nodes[k] - nodes[m])
    return L


def _leaf_collection(tree: Tree, leaf: int, nodes: np.ndarray) -> np.ndarray:
    """(ncoef, nvalues) interpolation matrix of one leaf (column-major coefficient order)."""
    pts = tree.points[tree.values(leaf)]
    c, h = tree.center[leaf], tree.halfsize[leaf]
    p = nodes.size
    mats = [lagrange(nodes, (pts[:, d] - c[d]) / h) for d in range(tree.dim)]
    C = mats[0]
    for d in range(1, tree.dim):
        # a = a1 + p*a2 + p^2*a3: later axes vary slowest
        C = (mats[d][:, None, :] * C[None, :, :]).reshape(-1, pts.shape[0])
    return C


def _axis_factors(nodes: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Per-axis child->parent interpolation for the lower (-) and upper (+) child."""
    lo = lagrange(nodes, -0.5 + 0.5 * nodes)
    hi = lagrange(nodes, 0.5 + 0.5 * nodes)
    return lo, hi


def _grid_at(center, h, nodes, dim) -> np.ndarray:
    """Interpolation points of a box (centre, half size), ordered like the moment coefficients."""
    axes = [center[d] + h * nodes for d in range(dim)]
    grids = np.meshgrid(*axes, indexing="ij")
    return np.stack([g.ravel(order="F") for g in grids], axis=1).reshape(nodes.size ** dim, dim)


def _node_grid(tree: Tree, n: int, nodes: np.ndarray) -> np.ndarray:
    """Interpolation points of box n, ordered like the moment coefficients."""
    p = nodes.size
    c, h = tree.center[n], tree.halfsize[n]
    axes = [c[d] + h * nodes for d in range(tree.dim)]
    grids = np.meshgrid(*axes, indexing="ij")
    # column-major flattening: axis 0 fastest
    return np.stack([g.ravel(order="F") for g in grids], axis=1).reshape(p ** tree.dim, tree.dim)


def cube_symmetry(offs) -> tuple:
    """Canonical representative of an integer offset under the signed axis permutations, and
    the element (perm, signs) with offs = S c, (S v)_a = signs[a] * v[perm[a]].

    The canonical offset sorts the absolute components in descending order, so the up to 48
    offsets of one orbit (H2Trees' LatticeSymmetry group of the cube) share it.
    """
    offs = np.asarray(offs, np.int64)
    a = np.abs(offs)
    order = np.argsort(-a, kind="stable")
    canon = a[order]
    perm = np.empty_like(order)
    perm[order] = np.arange(order.size)      # canon[perm[a]] == |offs[a]|
    signs = np.where(offs < 0, -1, 1)
    return canon, perm, signs


def grid_permutation(p: int, dim: int, perm, signs) -> np.ndarray:
    """Node permutation of a p^dim interpolation grid under S: index of S xi_i for each i.

    Nodes symmetric about the box centre (xi_{p-1-k} = -xi_k, Chebyshev and equispaced) make
    a sign flip the index reversal k -> p - 1 - k (symmetryreducedcollection.jl:197-230).
    Coefficient order: axis 0 fastest.
    """
    idx = np.indices((p,) * dim).reshape(dim, -1)   # idx[a, lin] with axis 0 fastest below
    lin = np.ravel_multi_index(idx[::-1], (p,) * dim)  # C order over reversed axes = axis 0 fastest
    out = np.empty(p ** dim, np.int32)
    img = np.empty_like(idx)
    for a in range(dim):
        comp = idx[perm[a]]
        img[a] = comp if signs[a] > 0 else p - 1 - comp
    out[lin] = np.ravel_multi_index(img[::-1], (p,) * dim)
    return out


def toeplitz_permutation(ts: int, dim: int, perm, signs) -> np.ndarray:
    """Sample permutation of a padded (2p-1)^dim wrap-around tensor under S:
    t_{S d}[j] = t_d[perm[j]], the wrap position of S^-1 m_j (symmetryreducedcollection.jl:150-195).
    Valid for the FFT'd tensor too (S is orthogonal)."""
    idx = np.indices((ts,) * dim).reshape(dim, -1)
    signed = np.where(idx > ts // 2, idx - ts, idx)
    inv = np.empty(dim, np.int64)
    inv[np.asarray(perm)] = np.arange(dim)
    src = np.empty_like(signed)
    for b in range(dim):  # (S^-1 u)_b = signs[inv[b]] * u[inv[b]]
        src[b] = signs[inv[b]] * signed[inv[b]]
    src = np.mod(src, ts)
    lin = np.ravel_multi_index(idx[::-1], (ts,) * dim)
    out = np.empty(ts ** dim, np.int32)
    out[lin] = np.ravel_multi_index(src[::-1], (ts,) * dim)
    return out


def interpolation_core(tree: Tree, kernel, p: int, *, nodes: str = "chebyshev",
                       transfers: str = "dense", couplings: str = "dense",
                       field: str | None = None, precision: str = "fp64",
                       near: str = "host", alpha=1.0, trial: Tree | None = None,
                       symmetry: bool = False) -> H2Core:
    """H2 core of an interpolation FMM of order `p` for `kernel`.

    `tree` holds the test (row) points; `trial` the trial (column) points of a Petrov map
    (test/farinteractions/test_rectangular.jl), or None for a Galerkin map on one tree. The two
    trees must share the root box so that their boxes pair level by level.
    couplings = "dense" stores one M2L block per unique translation; "toeplitz" stores the
    FFT'd wrap-around kernel per unique translation (equispaced nodes, same-size boxes only).
    near = "host" assembles near blocks on the host; "none" leaves them to the caller
    (e.g. assembled on the device, see h2factory_b200.assembly); "free" computes the near entries
    on the device from the points (matrix-free; `laplace` and `helmholtz` kernels only).
    symmetry = True stores one coupling per orbit of the cube's signed axis permutations and
    reads the others through permutations (symmetry-reduced M2L, symmetryreduceddense.jl and
    symmetryreducedcollection.jl); it needs a radial kernel and cube moments.
    """
    xi = chebyshev_nodes(p) if nodes == "chebyshev" else equispaced_nodes(p)
    if couplings == "toeplitz" and nodes != "equispaced":
        raise ValueError("Toeplitz couplings need equispaced interpolation nodes")
    test = tree
    trial = tree if trial is None else trial
    if trial is not test and (not np.allclose(test.center[0], trial.center[0])
                              or not np.isclose(test.halfsize[0], trial.halfsize[0])):
        raise ValueError("test and trial trees need the same root box")
    plans = build_plans(test, trial)
    dim = tree.dim
    cplx = np.iscomplexobj(kernel(np.zeros((1, dim)), np.ones((1, dim))))
    if field is None:
        field = "complex" if cplx else "real"
    dtype = np.complex128 if field == "complex" else np.float64
    def side_shape(t):
        sh = np.zeros((t.nlevels + 1, 3), np.int32)
        sh[1:, :] = 1
        sh[1:, :dim] = p
        return sh

    def side_colls(t):
        return {int(n): _leaf_collection(t, int(n), xi).astype(dtype)[None] for n in t.leaves()}

    colls = side_colls(test)
    colls_trial = colls if trial is test else side_colls(trial)

    lo, hi = _axis_factors(xi)
    tdict = {}
    for lvl in range(2, max(test.nlevels, trial.nlevels) + 1):
        for s in range(tree.nsectors):
            facs = [(hi if (s >> d) & 1 else lo).astype(dtype) for d in range(dim)]
            if transfers == "separable":
                tdict[(lvl, s)] = tuple(facs)
            else:
                T = facs[0]
                for d in range(1, dim):
                    T = np.kron(facs[d], T)
                tdict[(lvl, s)] = T

    far = plans.far
    ca, cb = test.center[far[:, 0]], trial.center[far[:, 1]]
    hmin = np.minimum(test.halfsize[far[:, 0]], trial.halfsize[far[:, 1]])
    offs = np.round((cb - ca) / hmin[:, None] * 2).astype(np.int64)
    keys = np.concatenate([test.level[far[:, 0]][:, None].astype(np.int64),
                           trial.level[far[:, 1]][:, None].astype(np.int64), offs], axis=1)
    ukeys, first, inv = np.unique(keys, axis=0, return_index=True, return_inverse=True)
    blocks = []
    canon_of = rowperms = colperms = None
    if symmetry:
        canon_of, rowperms, colperms, cache = [], [], [], {}
        for u in range(ukeys.shape[0]):
            lr, lt = int(ukeys[u, 0]), int(ukeys[u, 1])
            c, prm, sg = cube_symmetry(ukeys[u, 2:])
            ck = (lr, lt, *c.tolist())
            if ck not in cache:
                cache[ck] = len(blocks)
                r, t = int(far[first[u], 0]), int(far[first[u], 1])
                hr, ht = test.halfsize[r], trial.halfsize[t]
                hmn = min(hr, ht)
                # canonical geometry: receiver at the origin, source at offset c (units hmin / 2)
                dc = -(hmn / 2.0) * c.astype(np.float64)
                if couplings == "toeplitz":
                    ts = 2 * p - 1
                    m = np.arange(ts)
                    m = np.where(m < p, m, m - ts)
                    grids = np.meshgrid(*([m] * dim), indexing="ij")
                    z = np.stack([dc[d] + (2.0 * hr / p) * grids[d] for d in range(dim)], axis=-1)
                    kv = kernel(z.reshape(-1, dim), np.zeros((1, dim)))[:, 0].reshape((ts,) * dim)
                    blocks.append(np.fft.fftn(kv.astype(np.complex128)))
                else:
                    xr = _grid_at(np.zeros(dim), hr, xi, dim)
                    yt = _grid_at(-dc, ht, xi, dim)
                    blocks.append(kernel(xr, yt).astype(dtype))
            canon_of.append(cache[ck])
            if couplings == "toeplitz":
                rowperms.append(toeplitz_permutation(2 * p - 1, dim, prm, sg))
                colperms.append(None)
            else:
                gp = grid_permutation(p, dim, prm, sg)
                rowperms.append(gp)
                colperms.append(gp)
    for u in range(ukeys.shape[0] if not symmetry else 0):
        r, t = int(far[first[u], 0]), int(far[first[u], 1])
        if couplings == "toeplitz":
            if test.level[r] != trial.level[t]:
                raise ValueError("Toeplitz couplings need same-level pairs (uniform trees)")
            h = test.halfsize[r]
            dc = test.center[r] - trial.center[t]
            ts = 2 * p - 1
            m = np.arange(ts)
            m = np.where(m < p, m, m - ts)          # wrap-around: index mod(i - j, ts)
            grids = np.meshgrid(*([m] * dim), indexing="ij")
            z = np.stack([dc[d] + (2.0 * h / p) * grids[d] for d in range(dim)], axis=-1)
            kv = kernel(z.reshape(-1, dim), np.zeros((1, dim)))[:, 0].reshape((ts,) * dim)
            blocks.append(np.fft.fftn(kv.astype(np.complex128)))
        else:
            B = kernel(_node_grid(test, r, xi), _node_grid(trial, t, xi)).astype(dtype)
            blocks.append(B)

    core = H2Core(field=field, test=test, trial=trial, plans=plans, ncomp=1, dim=dim,
                  shape_test=side_shape(test), shape_trial=side_shape(trial), collections_test=colls,
                  collections_trial=colls_trial, transfers_test=tdict, transfers_trial=tdict,
                  transfer_kind=transfers, coupling_kind=couplings, couplings=blocks,
                  pair_coupling=inv.reshape(-1).astype(np.int64), precision=precision,
                  alpha=alpha, conj_leaf_adjoint=(field == "complex"))
    if symmetry:
        core.coupling_canon = np.asarray(canon_of, np.int64)
        core.coupling_rowperm = rowperms
        core.coupling_colperm = colperms
    core.kernel = kernel
    if near == "free":
        if kernel is laplace:
            core.set_near_kernel("laplace")
        elif getattr(kernel, "wavenumber", None) is not None:
            core.set_near_kernel("helmholtz", kernel.wavenumber)
        else:
            raise ValueError("matrix-free near field: laplace or helmholtz kernels only")
    elif near == "host":
        core.set_near_blocks(near_blocks_from_kernel(trial, plans, kernel, dtype, test=test))
    return core


def near_blocks_from_kernel(tree: Tree, plans, kernel, dtype, test: Tree | None = None):
    """Dense near blocks K(values(a), values(b)) for every near leaf pair, in plan order."""
    test = tree if test is None else test
    out = []
    for a, b in plans.near:
        xa = test.points[test.values(int(a))]
        yb = tree.points[tree.values(int(b))]
        out.append(kernel(xa, yb).astype(dtype))
    return out
