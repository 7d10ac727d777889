"""Host side of the map: H2Factory's core/workspace split, flattened for the C ABI.

* `H2Core` holds the read-only method data (trees, plans, leaf collections, transfers,
  couplings, near blocks and the far prefactor), the fields an `AbstractH2Core` carries
  (src/maps/core.jl:17-33, docs/src/implementing/required.md:16-60).
* `DeviceCore` is that core copied into HBM by the CUDA library (h2b_core_create).
* `H2Workspace` is one request slot on a device core (H2Workspace / similarworkspace,
  src/maps/workspace.jl:81-113); `transpose(A)` and `adjoint(A)` give the oriented maps, and
  `mul_`, `farmul_`, `nearmul_` are `mul!`, `farmul!`, `nearmul!`
  (src/maps/abstracth2map.jl:42-86, src/farinteractions/farmul.jl:8-70,
  src/nearinteractions/nearmul.jl:8-14).
"""

from __future__ import annotations

import ctypes as C
import os
import threading
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .trees import Plans, Tree

__all__ = ["H2Core", "DeviceCore", "H2Workspace", "OrientedMap", "transpose", "adjoint",
           "mul_", "farmul_", "nearmul_", "similarworkspace", "flatten", "profilemul"]

_MODES = {"forward": _abi.H2B_FORWARD, "transpose": _abi.H2B_TRANSPOSE,
          "adjoint": _abi.H2B_ADJOINT}


@dataclass
class H2Core:
    """Read-only data of one H2 map (Galerkin when test is trial)."""

    field: str                      # "real" | "complex"
    test: Tree
    trial: Tree
    plans: Plans
    ncomp: int
    dim: int
    shape_test: np.ndarray          # int32 [(nlevels+1), 3]
    shape_trial: np.ndarray
    collections_test: dict          # leaf -> (ncomp, ncoef, nvalues)
    collections_trial: dict
    transfers_test: dict            # (child level, sector) -> matrix | tuple of per-axis matrices
    transfers_trial: dict
    transfer_kind: str              # "dense" | "separable"
    coupling_kind: str              # "dense" | "diagonal" | "toeplitz"
    couplings: list                 # unique blocks
    pair_coupling: np.ndarray       # int64 [npairs]: block of far pair (test node, trial node)
    precision: str = "fp64"         # far-field arithmetic: "fp64" | "fp32"
    alpha: object = 1.0             # scalar (-> α, α, conj α) or (forward, transpose, adjoint)
    conj_leaf_adjoint: bool = True  # leafmul(A, isAdjoint) = ConjugatedCollectionMul
    near_data: np.ndarray | None = None
    near_offset: np.ndarray | None = None
    near_device: object = None      # torch tensor holding near blocks on the device
    kernel: object = field(default=None, repr=False)
    near_kind: str = "stored"       # "stored" blocks, or a point kernel: "laplace" | "helmholtz"
    near_wavenumber: float = 0.0    # k of the Helmholtz point kernel
    # symmetry-reduced couplings: `couplings` holds one canonical block per orbit; key k (the
    # values of pair_coupling) reads couplings[coupling_canon[k]] through its permutations
    coupling_canon: np.ndarray | None = None
    coupling_rowperm: list | None = None  # per key: int32 array or None (identity)
    coupling_colperm: list | None = None  # per key (dense only)

    @property
    def dtype(self):
        return np.complex128 if self.field == "complex" else np.float64

    @property
    def size(self):
        return (self.test.npoints, self.trial.npoints)

    def alphas(self):
        a = self.alpha
        if np.ndim(a) == 0:
            a = complex(a)
            return (a, a, a.conjugate())
        return tuple(complex(v) for v in a)

    def set_near_blocks(self, blocks):
        """Near blocks in plan order (one dense (nvalues(a), nvalues(b)) array per near pair)."""
        sizes = np.array([b.size for b in blocks], np.int64)
        self.near_offset = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        data = np.empty(int(sizes.sum()), dtype=self.dtype)
        for off, blk in zip(self.near_offset, blocks):
            data[off:off + blk.size] = np.asarray(blk, dtype=self.dtype).ravel(order="F")
        self.near_data = data
        self.near_device = None

    def set_near_device(self, tensor, offsets):
        """Near blocks already on the device (flat, column-major blocks at `offsets`)."""
        self.near_device = tensor
        self.near_offset = np.asarray(offsets, np.int64)
        self.near_data = None

    def set_near_kernel(self, kind: str, wavenumber: float = 0.0):
        """Matrix-free near field: entries K(x_i, y_j) computed on the device from the points.

        A custom near storage in the sense of docs/src/near/storage.md:7-14 (any matrix-like
        operator with `mul!`): "laplace" is 1/(4 pi r), "helmholtz" exp(i k r)/(4 pi r), both 0 at
        r = 0 -- the kernels of h2factory_b200.methods -- over the same near leaf pairs.
        """
        if kind not in ("laplace", "helmholtz"):
            raise ValueError(kind)
        self.near_kind = kind
        self.near_wavenumber = float(wavenumber)
        self.near_data = self.near_offset = self.near_device = None

    def near_block(self, k: int) -> np.ndarray:
        a, b = self.plans.near[k]
        nr = self.test.value_ptr[a + 1] - self.test.value_ptr[a]
        nc = self.trial.value_ptr[b + 1] - self.trial.value_ptr[b]
        off = self.near_offset[k]
        return self.near_data[off:off + nr * nc].reshape((nr, nc), order="F")


def _as_f64(arr) -> np.ndarray:
    a = np.ascontiguousarray(arr)
    if np.iscomplexobj(a):
        return a.view(np.float64)
    return a.astype(np.float64, copy=False)


def _ptr(arr, ctype):
    return arr.ctypes.data_as(C.POINTER(ctype))


class _Keep(list):
    """Arrays whose memory the descriptor points into."""

    def add(self, arr, ctype):
        self.append(arr)
        return _ptr(arr, ctype)


def _side(core: H2Core, tree: Tree, shape: np.ndarray, colls: dict, transfers: dict,
          plans, keep: _Keep, other_is_trial: bool) -> _abi.SideDesc:
    s = _abi.SideDesc()
    s.nnodes, s.nlevels, s.root, s.ndofs = tree.nnodes, tree.nlevels, 0, tree.npoints
    i32 = C.c_int32
    s.level = keep.add(np.ascontiguousarray(tree.level, np.int32), i32)
    s.parent = keep.add(np.ascontiguousarray(tree.parent, np.int32), i32)
    s.sector = keep.add(np.ascontiguousarray(tree.sector, np.int32), i32)
    s.child_ptr = keep.add(np.ascontiguousarray(tree.child_ptr, np.int32), i32)
    s.child = keep.add(np.ascontiguousarray(tree.child, np.int32), i32)
    s.value_ptr = keep.add(np.ascontiguousarray(tree.value_ptr, np.int32), i32)
    s.value = keep.add(np.ascontiguousarray(tree.value, np.int32), i32)
    s.shape = keep.add(np.ascontiguousarray(shape, np.int32).ravel(), i32)
    s.agg_nstages = plans.agg_level.size
    s.agg_level = keep.add(np.ascontiguousarray(plans.agg_level, np.int32), i32)
    s.agg_ptr = keep.add(np.ascontiguousarray(plans.agg_ptr, np.int32), i32)
    s.agg_node = keep.add(np.ascontiguousarray(plans.agg_node, np.int32), i32)
    s.agg_store = keep.add(np.ascontiguousarray(plans.agg_store, np.uint8), C.c_uint8)
    s.dis_nstages = plans.dis_level.size
    s.dis_level = keep.add(np.ascontiguousarray(plans.dis_level, np.int32), i32)
    s.dis_ptr = keep.add(np.ascontiguousarray(plans.dis_ptr, np.int32), i32)
    s.dis_node = keep.add(np.ascontiguousarray(plans.dis_node, np.int32), i32)
    s.dis_isnode = keep.add(np.ascontiguousarray(plans.dis_isnode, np.uint8), C.c_uint8)
    s.i2o_ptr = keep.add(np.ascontiguousarray(plans.i2o_ptr, np.int32), i32)
    s.i2o_src = keep.add(np.ascontiguousarray(plans.i2o_src, np.int32), i32)
    # couplingkey: both sides look up the block stored for the (test, trial) pair
    coup = np.ascontiguousarray(core.pair_coupling[plans.i2o_pair], np.int64)
    s.i2o_coupling = keep.add(coup, C.c_int64)

    coff = np.full(tree.nnodes, -1, np.int64)
    parts, pos = [], 0
    for n in sorted(colls):
        Cn = np.asarray(colls[n], dtype=core.dtype)
        flat = np.ascontiguousarray(Cn.transpose(0, 2, 1)).ravel()  # (comp, j, a): a fastest
        coff[n] = pos
        parts.append(flat)
        pos += flat.size
    data = np.concatenate(parts) if parts else np.zeros(1, core.dtype)
    s.coll_offset = keep.add(coff, C.c_int64)
    s.coll = keep.add(_as_f64(data), C.c_double)
    s.coll_len = pos

    ns = core.test.nsectors
    toff = np.full((tree.nlevels + 1) * ns, -1, np.int64)
    parts, pos = [], 0
    for (lvl, sec), T in sorted(transfers.items()):
        if lvl > tree.nlevels:
            continue
        mats = T if isinstance(T, tuple) else (T,)
        flat = np.concatenate([np.asarray(m, dtype=core.dtype).ravel(order="F") for m in mats])
        toff[lvl * ns + sec] = pos
        parts.append(flat)
        pos += flat.size
    data = np.concatenate(parts) if parts else np.zeros(1, core.dtype)
    s.transfer_offset = keep.add(toff, C.c_int64)
    s.transfer = keep.add(_as_f64(data), C.c_double)
    s.transfer_len = pos
    return s


def flatten(core: H2Core):
    """The h2b_map_desc of `core` and the arrays it points into (keep both alive)."""
    keep = _Keep()
    d = _abi.MapDesc()
    d.field = _abi.H2B_COMPLEX if core.field == "complex" else _abi.H2B_REAL
    d.precision = _abi.H2B_FP32 if core.precision == "fp32" else _abi.H2B_FP64
    d.ncomp, d.dim, d.nsectors = core.ncomp, core.dim, core.test.nsectors
    d.transfer_kind = (_abi.H2B_TRANSFER_SEPARABLE if core.transfer_kind == "separable"
                       else _abi.H2B_TRANSFER_DENSE)
    d.coupling_kind = {"dense": _abi.H2B_COUPLING_DENSE, "diagonal": _abi.H2B_COUPLING_DIAGONAL,
                       "toeplitz": _abi.H2B_COUPLING_TOEPLITZ}[core.coupling_kind]
    d.conj_leaf_adjoint = int(bool(core.conj_leaf_adjoint))
    for m, a in enumerate(core.alphas()):
        d.alpha[m][0], d.alpha[m][1] = a.real, a.imag
    d.test = _side(core, core.test, core.shape_test, core.collections_test,
                   core.transfers_test, core.plans.test, keep, other_is_trial=True)
    d.trial = _side(core, core.trial, core.shape_trial, core.collections_trial,
                    core.transfers_trial, core.plans.trial, keep, other_is_trial=False)

    coffs, parts, pos = [], [], 0
    for blk in core.couplings:
        b = np.asarray(blk)
        if core.coupling_kind == "toeplitz":
            flat = _as_f64(np.asarray(b, np.complex128).ravel(order="F"))
        else:
            flat = _as_f64(np.asarray(b, dtype=core.dtype).ravel(order="F"))
        coffs.append(pos)
        parts.append(flat)
        pos += flat.size
    d.coupling = keep.add(np.concatenate(parts) if parts else np.zeros(1), C.c_double)
    d.coupling_len = pos
    if core.coupling_canon is None:
        d.ncouplings = len(coffs)
        d.coupling_offset = keep.add(np.array(coffs if coffs else [0], np.int64), C.c_int64)
    else:
        # one key per translation, sharing its orbit's canonical data, plus its permutations
        canon = np.asarray(core.coupling_canon, np.int64)
        d.ncouplings = canon.size
        d.coupling_offset = keep.add(np.array(coffs, np.int64)[canon] if canon.size else np.zeros(1, np.int64),
                                     C.c_int64)
        store, chunks, at = {}, [], 0

        def perm_offset(pm):
            nonlocal at
            if pm is None:
                return -1
            pm = np.ascontiguousarray(pm, np.int32)
            key = pm.tobytes()
            if key not in store:
                store[key] = at
                chunks.append(pm)
                at += pm.size
            return store[key]

        rows = np.array([perm_offset(pm) for pm in core.coupling_rowperm], np.int64)
        cols = np.array([perm_offset(pm) for pm in (core.coupling_colperm or [None] * canon.size)], np.int64)
        d.coupling_rowperm = keep.add(rows if rows.size else np.full(1, -1, np.int64), C.c_int64)
        d.coupling_colperm = keep.add(cols if cols.size else np.full(1, -1, np.int64), C.c_int64)
        d.coupling_perm = keep.add(np.concatenate(chunks) if chunks else np.zeros(1, np.int32), C.c_int32)
        d.coupling_perm_len = at

    near = core.plans.near
    rows, starts = np.unique(near[:, 0], return_index=True) if near.size else (np.zeros(0, np.int32), np.zeros(0, np.int64))
    ptr = np.append(starts, near.shape[0]).astype(np.int32)
    d.near_nrows = rows.size
    d.near_row = keep.add(np.ascontiguousarray(rows, np.int32), C.c_int32)
    d.near_ptr = keep.add(ptr, C.c_int32)
    d.near_col = keep.add(np.ascontiguousarray(near[:, 1], np.int32), C.c_int32)
    offs = core.near_offset if core.near_offset is not None else np.zeros(max(near.shape[0], 1), np.int64)
    d.near_offset = keep.add(np.ascontiguousarray(offs, np.int64), C.c_int64)
    if core.near_device is not None:
        t = core.near_device
        d.near = C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))
        d.near_len = t.numel()
        d.near_on_device = 1
        keep.append(t)
    else:
        data = core.near_data if core.near_data is not None else np.zeros(1, core.dtype)
        d.near = keep.add(_as_f64(data), C.c_double)
        d.near_len = data.size if core.near_data is not None else 0
        d.near_on_device = 0
    d.near_kind = {"stored": _abi.H2B_NEAR_STORED, "laplace": _abi.H2B_NEAR_LAPLACE,
                   "helmholtz": _abi.H2B_NEAR_HELMHOLTZ}[core.near_kind]
    d.near_wavenumber = core.near_wavenumber
    if core.near_kind != "stored":
        for name, tree in (("test_points", core.test), ("trial_points", core.trial)):
            pts = np.zeros((tree.npoints, 3))
            pts[:, :tree.dim] = tree.points
            setattr(d, name, keep.add(pts, C.c_double))
    return d, keep


# ---------------------------------------------------------------------------------------------
# Device objects
# ---------------------------------------------------------------------------------------------

@dataclass
class MapShape:
    """What a workspace needs of a core that was loaded from a map blob (no host-side H2Core)."""

    field: str
    size: tuple
    precision: str

    @property
    def dtype(self):
        return np.complex128 if self.field == "complex" else np.float64


def _aligned(nbytes: int) -> np.ndarray:
    """An 8-byte aligned uint8 buffer (the blob format's alignment)."""
    return np.zeros((nbytes + 7) // 8, np.uint64).view(np.uint8)[:nbytes]


def map_blob(core: H2Core) -> np.ndarray:
    """The core as one self-contained byte image (h2b_map_blob_write); near blocks held on the
    device are copied to the host first."""
    import copy

    if core.near_device is not None:
        c = copy.copy(core)
        c.near_data, c.near_device = core.near_device.cpu().numpy(), None
        core = c
    lib = _abi.load_library()
    desc, keep = flatten(core)
    size = C.c_size_t()
    _abi.check(lib.h2b_map_blob_write(C.byref(desc), None, 0, C.byref(size)))
    buf = _aligned(size.value)
    _abi.check(lib.h2b_map_blob_write(C.byref(desc), buf.ctypes.data_as(C.c_void_p), size.value, C.byref(size)))
    del keep
    return buf


def save_map(core: H2Core, path: str) -> int:
    """Write the map blob of `core` to `path`; returns its size in bytes."""
    buf = map_blob(core)
    with open(path, "wb") as f:
        f.write(buf.tobytes())
    return buf.size


def read_blob(blob) -> tuple:
    """(aligned buffer, h2b_map_desc pointing into it) of a blob given as bytes, array or path."""
    if isinstance(blob, (str, os.PathLike)):
        with open(blob, "rb") as f:
            data = f.read()
    else:
        data = bytes(np.asarray(blob, np.uint8).tobytes()) if not isinstance(blob, bytes) else blob
    buf = _aligned(len(data))
    buf[:] = np.frombuffer(data, np.uint8)
    desc = _abi.MapDesc()
    _abi.check(_abi.load_library().h2b_map_blob_read(buf.ctypes.data_as(C.c_void_p), buf.size, C.byref(desc)))
    return buf, desc


class DeviceCore:
    """The read-only core in HBM (h2b_core)."""

    def __init__(self, core: H2Core, device: int = 0):
        self.lib = _abi.load_library()
        self.core = core
        self.device = device
        desc, keep = flatten(core)
        h = C.c_void_p()
        _abi.check(self.lib.h2b_core_create(C.byref(desc), device, C.byref(h)))
        self.handle = h
        del keep

    @classmethod
    def from_blob(cls, blob, device: int = 0) -> "DeviceCore":
        """A core built straight from a map blob (bytes, uint8 array or file path)."""
        buf, desc = read_blob(blob)
        self = cls.__new__(cls)
        self.lib = _abi.load_library()
        self.device = device
        self.core = MapShape("complex" if desc.field == _abi.H2B_COMPLEX else "real",
                             (desc.test.ndofs, desc.trial.ndofs),
                             "fp32" if desc.precision == _abi.H2B_FP32 else "fp64")
        h = C.c_void_p()
        _abi.check(self.lib.h2b_core_create_from_blob(buf.ctypes.data_as(C.c_void_p), buf.size, device,
                                                       C.byref(h)))
        self.handle = h
        return self

    def info(self) -> _abi.CoreInfo:
        out = _abi.CoreInfo()
        _abi.check(self.lib.h2b_core_get_info(self.handle, C.byref(out)))
        return out

    def close(self):
        if getattr(self, "handle", None):
            self.lib.h2b_core_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _alphabeta(alpha, beta):
    if alpha is None and beta is None:
        return None, None
    a = complex(1.0 if alpha is None else alpha)
    b = complex(0.0 if beta is None else beta)
    return (C.c_double * 2)(a.real, a.imag), (C.c_double * 2)(b.real, b.imag)


def _colmajor(t, n: int):
    """(pointer, nrhs, ld) of a 1-D or column-major 2-D torch tensor with n rows."""
    if t.dim() == 1:
        if t.shape[0] != n or t.stride(0) != 1:
            raise ValueError(f"vector of length {n} with unit stride expected")
        return t.data_ptr(), 1, n
    if t.shape[0] != n or t.stride(0) != 1:
        raise ValueError(f"column-major ({n}, nrhs) tensor expected")
    return t.data_ptr(), t.shape[1], max(t.stride(1), n)


class H2Workspace:
    """One request slot on a device core; the map itself in forward orientation."""

    def __init__(self, dcore: DeviceCore | H2Core, max_nrhs: int = 1, device: int = 0):
        if isinstance(dcore, H2Core):
            dcore = DeviceCore(dcore, device)
        self.dcore = dcore
        self.lib = dcore.lib
        self.max_nrhs = max_nrhs
        h = C.c_void_p()
        _abi.check(self.lib.h2b_workspace_create(dcore.handle, max_nrhs, C.byref(h)))
        self.handle = h
        self.mode = _abi.H2B_FORWARD
        self._lock = threading.Lock()

    @property
    def core(self) -> H2Core:
        return self.dcore.core

    @property
    def shape(self):
        return self.core.size

    def close(self):
        if getattr(self, "handle", None):
            self.lib.h2b_workspace_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the C calls ------------------------------------------------------------------------
    def _call(self, fn, mode, y, x, alpha, beta, stream):
        import torch

        nrow, ncol = self.shape
        nout, nin = (nrow, ncol) if mode == _abi.H2B_FORWARD else (ncol, nrow)
        want = torch.complex128 if self.core.field == "complex" else torch.float64
        if x.dtype != want or y.dtype != want:
            raise TypeError(f"x and y must be {want}")
        xp, nrhs, ldx = _colmajor(x, nin)
        yp, nrhs_y, ldy = _colmajor(y, nout)
        if nrhs != nrhs_y:
            raise ValueError("x and y have different numbers of columns")
        a, b = _alphabeta(alpha, beta)
        if stream is None:
            stream = torch.cuda.current_stream(x.device).cuda_stream
        _abi.check(getattr(self.lib, fn)(self.handle, mode, nrhs, C.c_void_p(xp), ldx,
                                         C.c_void_p(yp), ldy, a, b, C.c_void_p(stream)))
        return y

    def matvec_host(self, x: np.ndarray, mode: int = _abi.H2B_FORWARD, alpha=None, beta=None,
                    y: np.ndarray | None = None) -> np.ndarray:
        """mul! on host arrays through h2b_matvec_host (copies in, multiplies, copies out)."""
        nrow, ncol = self.shape
        nout, nin = (nrow, ncol) if mode == _abi.H2B_FORWARD else (ncol, nrow)
        x = np.asfortranarray(x, dtype=self.core.dtype)
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        if y is None:
            y = np.zeros((nout,) if x.ndim == 1 else (nout, nrhs), dtype=self.core.dtype, order="F")
        a, b = _alphabeta(alpha, beta)
        _abi.check(self.lib.h2b_matvec_host(self.handle, mode, nrhs, x.ctypes.data_as(C.c_void_p),
                                            nin, y.ctypes.data_as(C.c_void_p), nout, a, b, None))
        return y

    def matvec_host_async(self, x: np.ndarray, y: np.ndarray, mode: int = _abi.H2B_FORWARD, stream=None,
                          alpha=None, beta=None) -> None:
        """Enqueue mul! on host arrays on `stream` (h2b_matvec_host_async) and return at once.

        x and y are Fortran-ordered arrays (page-locked memory for asynchronous copies) that must
        stay alive and untouched until the stream has passed this work."""
        nrow, ncol = self.shape
        nout, nin = (nrow, ncol) if mode == _abi.H2B_FORWARD else (ncol, nrow)
        if not (x.flags.f_contiguous and y.flags.f_contiguous) or x.dtype != self.core.dtype or y.dtype != x.dtype:
            raise ValueError("x and y must be Fortran-ordered arrays of the map's dtype")
        nrhs = 1 if x.ndim == 1 else x.shape[1]
        if x.shape[0] != nin or y.shape[0] != nout or (1 if y.ndim == 1 else y.shape[1]) != nrhs:
            raise ValueError("x / y shapes do not match the map")
        a, b = _alphabeta(alpha, beta)
        _abi.check(self.lib.h2b_matvec_host_async(self.handle, mode, nrhs, x.ctypes.data_as(C.c_void_p),
                                                  nin, y.ctypes.data_as(C.c_void_p), nout, a, b,
                                                  C.c_void_p(stream)))


def profilemul(A, x, y=None, alpha=None, beta=None, stream=None) -> list:
    """mul! with every pass timed on the device (h2b_profile_matvec), like H2Factory's
    Diagnostics.profilemul (src/diagnostics/timing.jl:150-160). Returns one record per launch,
    {"pass", "level", "ms"}, in launch order; `y` receives the product."""
    import torch

    ws, mode = _split(A)
    nrow, ncol = ws.shape
    nout, nin = (nrow, ncol) if mode == _abi.H2B_FORWARD else (ncol, nrow)
    xp, nrhs, ldx = _colmajor(x, nin)
    if y is None:
        y = torch.zeros((nrhs, nout), dtype=x.dtype, device=x.device).t() if x.dim() == 2 else \
            torch.zeros(nout, dtype=x.dtype, device=x.device)
    yp, nrhs_y, ldy = _colmajor(y, nout)
    if nrhs != nrhs_y:
        raise ValueError("x and y have different numbers of columns")
    a, b = _alphabeta(alpha, beta)
    if stream is None:
        stream = torch.cuda.current_stream(x.device).cuda_stream
    cap = 256
    recs = (_abi.PassTime * cap)()
    count = C.c_int32(0)
    _abi.check(ws.lib.h2b_profile_matvec(ws.handle, mode, nrhs, C.c_void_p(xp), ldx, C.c_void_p(yp), ldy, a, b,
                                         C.c_void_p(stream), recs, cap, C.byref(count)))
    return [{"pass": _abi.PASS_NAMES.get(r.pass_, str(r.pass_)), "level": int(r.level), "ms": float(r.milliseconds)}
            for r in recs[:min(cap, count.value)]]


class OrientedMap:
    """transpose(A) or adjoint(A) of a workspace (LinearMaps' TransposeMap / AdjointMap)."""

    def __init__(self, ws: H2Workspace, mode: int):
        self.ws = ws
        self.mode = mode

    @property
    def shape(self):
        r, c = self.ws.shape
        return (c, r) if self.mode != _abi.H2B_FORWARD else (r, c)


def transpose(A):
    if isinstance(A, OrientedMap):
        if A.mode == _abi.H2B_TRANSPOSE:
            return A.ws
        raise NotImplementedError("transpose of an adjoint map")
    return OrientedMap(A, _abi.H2B_TRANSPOSE)


def adjoint(A):
    if isinstance(A, OrientedMap):
        if A.mode == _abi.H2B_ADJOINT:
            return A.ws
        raise NotImplementedError("adjoint of a transposed map")
    return OrientedMap(A, _abi.H2B_ADJOINT)


def _split(A):
    if isinstance(A, OrientedMap):
        return A.ws, A.mode
    return A, _abi.H2B_FORWARD


def mul_(y, A, x, alpha=None, beta=None, stream=None):
    """mul!(y, A, x[, α, β]) on device tensors (src/maps/abstracth2map.jl:42-86)."""
    ws, mode = _split(A)
    return ws._call("h2b_matvec", mode, y, x, alpha, beta, stream)


def farmul_(y, A, x, alpha=None, beta=None, stream=None):
    """farmul!(y, A, x[, α, β]) (src/farinteractions/farmul.jl:8-70)."""
    ws, mode = _split(A)
    return ws._call("h2b_farmul", mode, y, x, alpha, beta, stream)


def nearmul_(y, A, x, alpha=None, beta=None, stream=None):
    """nearmul!(y, A, x[, α, β]) (src/nearinteractions/nearmul.jl:8-14)."""
    ws, mode = _split(A)
    return ws._call("h2b_nearmul", mode, y, x, alpha, beta, stream)


def similarworkspace(ws: H2Workspace, max_nrhs: int | None = None) -> H2Workspace:
    """A second workspace over the same device core (src/maps/workspace.jl:109-113)."""
    return H2Workspace(ws.dcore, max_nrhs or ws.max_nrhs)
