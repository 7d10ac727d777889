"""2^D trees and the traversal plans H2Factory consumes.

H2Factory takes its trees and plans from H2Trees (not part of the reference tree); the matvec
only reads them through a handful of queries (`H2Trees.level/parent/children/sector/values/
isleaf`, `aggregationnodes/storenode`, `isdisaggregationnode/translatingnodes`,
`nearinteractions`), listed at their call sites:

* aggregation plan:    src/farinteractions/aggregation.jl:58-92, src/moments/allocatemoments.jl:242-250
* disaggregation plan: src/farinteractions/disaggregation.jl:235-271,
                       src/farinteractions/traversalhelpers.jl:103-112
* sectors:             src/maps/leveltranslator.jl:40-43
* near groups:         src/nearinteractions/nearmul.jl:54-111

This module restates those semantics for a 2^D box tree (binary, quad or octree) and a
dual-tree traversal with the standard adjacency admissibility: two boxes are near when their
closed boxes touch; a far pair is recorded when two boxes are not near but their parents were,
which yields the classic interaction lists (children of the parent's neighbours that are not
adjacent) on uniform trees. Everything is stored as flat integer arrays, the form the C ABI takes.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

__all__ = ["Tree", "build_tree", "Plans", "build_plans", "morton_order"]


@dataclass
class Tree:
    """A 2^D box tree. Node 0 is the root; nodes are numbered level by level (BFS)."""

    dim: int
    points: np.ndarray          # (npoints, dim)
    level: np.ndarray           # int32 [nnodes], root = 1
    parent: np.ndarray          # int32 [nnodes], -1 at the root
    sector: np.ndarray          # int32 [nnodes], child slot in the parent (bit d = upper half in axis d)
    child_ptr: np.ndarray       # int32 [nnodes+1]
    child: np.ndarray           # int32
    value_ptr: np.ndarray       # int32 [nnodes+1], dofs of leaves (empty for inner nodes)
    value: np.ndarray           # int32
    center: np.ndarray          # (nnodes, dim)
    halfsize: np.ndarray        # [nnodes]
    root_center: np.ndarray = field(default=None)
    root_halfsize: float = 0.0

    @property
    def nnodes(self) -> int:
        return int(self.level.shape[0])

    @property
    def nlevels(self) -> int:
        return int(self.level.max())

    @property
    def npoints(self) -> int:
        return int(self.points.shape[0])

    @property
    def nsectors(self) -> int:
        return 1 << self.dim

    def isleaf(self, n: int) -> bool:
        return self.child_ptr[n + 1] == self.child_ptr[n]

    def children(self, n: int) -> np.ndarray:
        return self.child[self.child_ptr[n]:self.child_ptr[n + 1]]

    def values(self, n: int) -> np.ndarray:
        return self.value[self.value_ptr[n]:self.value_ptr[n + 1]]

    def leaves(self) -> np.ndarray:
        return np.nonzero(np.diff(self.child_ptr) == 0)[0].astype(np.int32)

    def nodes_at(self, lvl: int) -> np.ndarray:
        return np.nonzero(self.level == lvl)[0].astype(np.int32)


def build_tree(points, *, maxvalues: int | None = None, depth: int | None = None,
               minhalfsize: float = 0.0, root_center=None, root_halfsize=None) -> Tree:
    """Build a 2^D tree over `points` (npoints x D).

    A node is split while it holds more than `maxvalues` points (every non-empty node is split
    until `depth` when `depth` is given instead), and its children would not be smaller than
    `minhalfsize`. Empty children are dropped. The root is the bounding cube unless given.
    """
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64))
    if pts.ndim == 1:
        pts = pts[:, None]
    npts, dim = pts.shape
    if dim < 1 or dim > 3:
        raise ValueError("points must have 1, 2 or 3 coordinates")
    if maxvalues is None and depth is None:
        raise ValueError("give maxvalues or depth")
    if root_center is None:
        lo, hi = pts.min(axis=0), pts.max(axis=0)
        root_center = 0.5 * (lo + hi)
        root_halfsize = 0.5 * float(np.max(hi - lo)) * (1.0 + 1e-12) + 1e-300
    root_center = np.asarray(root_center, dtype=np.float64).reshape(dim)
    root_halfsize = float(root_halfsize)

    levels = [np.array([1], np.int32)]
    parents = [np.array([-1], np.int32)]
    sectors = [np.array([0], np.int32)]
    centers = [root_center[None, :]]
    halves = [np.array([root_halfsize])]
    # point ownership at the current level, as a permutation grouped by node
    order = np.arange(npts, dtype=np.int64)
    seg = np.array([0, npts], np.int64)          # segment bounds of current-level nodes in `order`
    leaf_segments = {}                            # leaf node id -> its point indices
    lvl = 1
    cur_ids = np.array([0], np.int64)
    next_id = 1
    child_lists = {}
    while cur_ids.size:
        cnt = np.diff(seg)
        h = halves[-1]
        if depth is not None:
            split = (cnt > 0) & (lvl < depth)
        else:
            split = cnt > maxvalues
        split &= (0.5 * h >= minhalfsize)
        # leaves at this level keep their point lists
        for k in np.nonzero(~split)[0]:
            leaf_segments[int(cur_ids[k])] = order[seg[k]:seg[k + 1]].copy()
        if not split.any():
            break
        # assign points of split nodes to children
        sel_nodes = np.nonzero(split)[0]
        new_ids, new_par, new_sec, new_cen, new_half = [], [], [], [], []
        new_order, new_seg = [], [0]
        for k in sel_nodes:
            idx = order[seg[k]:seg[k + 1]]
            c = centers[-1][k]
            code = np.zeros(idx.size, np.int64)
            for d in range(dim):
                code |= (pts[idx, d] > c[d]).astype(np.int64) << d
            srt = np.argsort(code, kind="stable")
            idx = idx[srt]
            code = code[srt]
            present, starts = np.unique(code, return_index=True)
            stops = np.append(starts[1:], idx.size)
            kids = []
            for s_, a, b in zip(present, starts, stops):
                off = np.array([(1 if (s_ >> d) & 1 else -1) for d in range(dim)], np.float64)
                new_ids.append(next_id)
                kids.append(next_id)
                new_par.append(int(cur_ids[k]))
                new_sec.append(int(s_))
                new_cen.append(c + 0.5 * h[k] * off)
                new_half.append(0.5 * h[k])
                new_order.append(idx[a:b])
                new_seg.append(new_seg[-1] + (b - a))
                next_id += 1
            child_lists[int(cur_ids[k])] = kids
        lvl += 1
        cur_ids = np.array(new_ids, np.int64)
        levels.append(np.full(len(new_ids), lvl, np.int32))
        parents.append(np.array(new_par, np.int32))
        sectors.append(np.array(new_sec, np.int32))
        centers.append(np.array(new_cen).reshape(-1, dim))
        halves.append(np.array(new_half))
        order = np.concatenate(new_order) if new_order else np.zeros(0, np.int64)
        seg = np.array(new_seg, np.int64)

    level = np.concatenate(levels)
    nn = level.shape[0]
    parent = np.concatenate(parents)
    sector = np.concatenate(sectors)
    center = np.concatenate(centers, axis=0)
    halfsize = np.concatenate(halves)
    child_ptr = np.zeros(nn + 1, np.int32)
    for p, kids in child_lists.items():
        child_ptr[p + 1] = len(kids)
    child_ptr = np.cumsum(child_ptr).astype(np.int32)
    child = np.zeros(child_ptr[-1], np.int32)
    for p, kids in child_lists.items():
        child[child_ptr[p]:child_ptr[p + 1]] = kids
    value_ptr = np.zeros(nn + 1, np.int64)
    for n, idx in leaf_segments.items():
        value_ptr[n + 1] = idx.size
    value_ptr = np.cumsum(value_ptr)
    value = np.zeros(value_ptr[-1], np.int32)
    for n, idx in leaf_segments.items():
        value[value_ptr[n]:value_ptr[n + 1]] = np.sort(idx)
    if value_ptr[-1] != npts:
        raise AssertionError("every point must land in exactly one leaf")
    return Tree(dim=dim, points=pts, level=level, parent=parent, sector=sector,
                child_ptr=child_ptr, child=child, value_ptr=value_ptr.astype(np.int32),
                value=value, center=center, halfsize=halfsize,
                root_center=root_center, root_halfsize=root_halfsize)


def morton_order(points, bits: int = 10) -> np.ndarray:
    """Permutation that sorts points along a Morton curve of their bounding cube.

    Point sets generated in this order make every leaf's dofs a contiguous range, which keeps
    the x gathers and y scatters of the leaf kernels coalesced.
    """
    pts = np.asarray(points, dtype=np.float64)
    if pts.ndim == 1:
        pts = pts[:, None]
    lo, hi = pts.min(axis=0), pts.max(axis=0)
    span = max(float(np.max(hi - lo)), 1e-300)
    q = np.minimum(((pts - lo) / span * (1 << bits)).astype(np.int64), (1 << bits) - 1)
    code = np.zeros(pts.shape[0], np.int64)
    for b in range(bits - 1, -1, -1):
        for d in range(pts.shape[1] - 1, -1, -1):
            code = (code << 1) | ((q[:, d] >> b) & 1)
    return np.argsort(code, kind="stable")


# ---------------------------------------------------------------------------------------------
# Plans
# ---------------------------------------------------------------------------------------------

@dataclass
class SidePlans:
    """The two plans of one tree side, as flat arrays (see h2b_side_desc in include/h2b200.h)."""

    agg_level: np.ndarray
    agg_ptr: np.ndarray
    agg_node: np.ndarray
    agg_store: np.ndarray       # uint8 [nnodes]
    dis_level: np.ndarray
    dis_ptr: np.ndarray
    dis_node: np.ndarray
    dis_isnode: np.ndarray      # uint8 [nnodes]
    i2o_ptr: np.ndarray         # int32 [nnodes+1]
    i2o_src: np.ndarray         # int32, node ids on the other side
    i2o_pair: np.ndarray        # int64, index into Plans.far (the (test, trial) pair list)


@dataclass
class Plans:
    """Far pairs (test node receives from trial node), near leaf pairs and both sides' plans."""

    far: np.ndarray             # int32 (npairs, 2): (test node, trial node)
    near: np.ndarray            # int32 (nnear, 2): (test leaf, trial leaf)
    test: SidePlans
    trial: SidePlans


def _isnear(ca, ha, cb, hb):
    tol = 1e-9 * np.maximum(ha, hb)
    return np.all(np.abs(ca - cb) <= (ha + hb)[:, None] + tol[:, None], axis=1)


def _expand(tree: Tree, nodes: np.ndarray, split: np.ndarray):
    """For each entry: its children if split, else itself. Returns (counts, flat list)."""
    nch = (tree.child_ptr[nodes + 1] - tree.child_ptr[nodes]).astype(np.int64)
    cnt = np.where(split, nch, 1)
    flat = np.empty(int(cnt.sum()), np.int64)
    pos = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
    selfmask = ~split
    flat[pos[:-1][selfmask]] = nodes[selfmask]
    sidx = np.nonzero(split)[0]
    if sidx.size:
        lens = nch[sidx]
        dst = _ranges(pos[sidx], lens)
        src = _ranges(tree.child_ptr[nodes[sidx]].astype(np.int64), lens)
        flat[dst] = tree.child[src]
    return cnt, flat


def _ranges(starts, lens):
    """Concatenation of arange(starts[i], starts[i] + lens[i]); every lens[i] > 0."""
    total = int(lens.sum())
    out = np.ones(total, np.int64)
    out[0] = starts[0]
    cs = np.cumsum(lens)[:-1]
    out[cs] = starts[1:] - (starts[:-1] + lens[:-1]) + 1
    return np.cumsum(out)


def dual_traversal(test: Tree, trial: Tree):
    """Partition test x trial into far node pairs and near leaf pairs (level-synchronous)."""
    a = np.array([0], np.int64)
    b = np.array([0], np.int64)
    far_a, far_b, near_a, near_b = [], [], [], []
    while a.size:
        nearm = _isnear(test.center[a], test.halfsize[a], trial.center[b], trial.halfsize[b])
        far_a.append(a[~nearm])
        far_b.append(b[~nearm])
        a, b = a[nearm], b[nearm]
        la = np.diff(test.child_ptr)[a] == 0
        lb = np.diff(trial.child_ptr)[b] == 0
        both = la & lb
        near_a.append(a[both])
        near_b.append(b[both])
        a, b, la, lb = a[~both], b[~both], la[~both], lb[~both]
        ha, hb = test.halfsize[a], trial.halfsize[b]
        rel = 1e-9 * np.maximum(ha, hb)
        split_a = ~la & (lb | (ha >= hb - rel))
        split_b = ~lb & (la | (hb >= ha - rel))
        ca, fa = _expand(test, a, split_a)
        cb, fb = _expand(trial, b, split_b)
        # cartesian product per entry
        tot = ca * cb
        pa = np.concatenate([[0], np.cumsum(ca)])
        pb = np.concatenate([[0], np.cumsum(cb)])
        ent = np.repeat(np.arange(a.size), tot)
        start = np.concatenate([[0], np.cumsum(tot)])[:-1]
        k = np.arange(int(tot.sum())) - np.repeat(start, tot)
        cbr = cb[ent]
        a = fa[pa[ent] + k // cbr]
        b = fb[pb[ent] + k % cbr]
    far = np.stack([np.concatenate(far_a), np.concatenate(far_b)], axis=1).astype(np.int32)
    near = np.stack([np.concatenate(near_a), np.concatenate(near_b)], axis=1).astype(np.int32)
    far = far[np.lexsort((far[:, 1], far[:, 0]))]
    near = near[np.lexsort((near[:, 1], near[:, 0]))]
    return far, near


def _descendant_closure(tree: Tree, seeds: np.ndarray) -> np.ndarray:
    """uint8 mask of `seeds` and all their descendants (nodes are BFS numbered)."""
    mask = np.zeros(tree.nnodes, np.uint8)
    mask[seeds] = 1
    for n in range(1, tree.nnodes):  # parents precede children in BFS order
        if mask[tree.parent[n]]:
            mask[n] = 1
    return mask


def _stages(tree: Tree, mask: np.ndarray, bottom_up: bool):
    nodes = np.nonzero(mask)[0].astype(np.int32)
    if nodes.size == 0:
        return np.zeros(0, np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32)
    lv = tree.level[nodes]
    levels = np.unique(lv)
    if bottom_up:
        levels = levels[::-1]
    ptr = [0]
    out = []
    for L in levels:
        sel = nodes[lv == L]
        out.append(sel)
        ptr.append(ptr[-1] + sel.size)
    return levels.astype(np.int32), np.array(ptr, np.int32), np.concatenate(out).astype(np.int32)


def _side_plans(tree: Tree, translating: np.ndarray, recv: np.ndarray, src: np.ndarray,
                pair_index: np.ndarray) -> SidePlans:
    """Plans of a side that aggregates from `translating` and receives along (recv <- src)."""
    store = np.zeros(tree.nnodes, np.uint8)
    store[translating] = 1
    agg_mask = _descendant_closure(tree, translating)
    agg_level, agg_ptr, agg_node = _stages(tree, agg_mask, bottom_up=True)
    dis_mask = _descendant_closure(tree, np.unique(recv))
    dis_level, dis_ptr, dis_node = _stages(tree, dis_mask, bottom_up=False)
    order = np.lexsort((src, recv))
    recv, src, pair_index = recv[order], src[order], pair_index[order]
    counts = np.bincount(recv, minlength=tree.nnodes)
    i2o_ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return SidePlans(agg_level=agg_level, agg_ptr=agg_ptr, agg_node=agg_node, agg_store=store,
                     dis_level=dis_level, dis_ptr=dis_ptr, dis_node=dis_node, dis_isnode=dis_mask,
                     i2o_ptr=i2o_ptr, i2o_src=src.astype(np.int32),
                     i2o_pair=pair_index.astype(np.int64))


def build_plans(test: Tree, trial: Tree | None = None) -> Plans:
    """Far/near partition and the four side plans (test/trial x aggregation/disaggregation).

    Forward maps aggregate on the trial side and receive on the test side; transpose and
    adjoint maps use the other two plans, with each pair's roles swapped
    (src/maps/accessors.jl:232-242). For a Galerkin map pass one tree.
    """
    trial = test if trial is None else trial
    far, near = dual_traversal(test, trial)
    idx = np.arange(far.shape[0], dtype=np.int64)
    fa = far[:, 0].astype(np.int64)
    fb = far[:, 1].astype(np.int64)
    test_plans = _side_plans(test, np.unique(fa), fa, fb, idx)
    trial_plans = _side_plans(trial, np.unique(fb), fb, fa, idx)
    return Plans(far=far, near=near, test=test_plans, trial=trial_plans)
