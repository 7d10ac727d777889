"""ctypes mirror of include/h2b200.h and the loader of the CUDA library.

The library is built in-tree (`build.py`) as libh2b200.so next to this file. Loading fails loudly
when it is missing: there is no CPU fallback for the product path.
"""

from __future__ import annotations

import ctypes as C
import os

H2B_OK = 0
H2B_ERR_INVALID = 1
H2B_ERR_CUDA = 2
H2B_ERR_NOMEM = 3
H2B_BUSY = 4
H2B_ERR_UNSUPPORTED = 5

H2B_REAL, H2B_COMPLEX = 0, 1
H2B_FP64, H2B_FP32 = 0, 1
H2B_FORWARD, H2B_TRANSPOSE, H2B_ADJOINT = 0, 1, 2
H2B_TRANSFER_DENSE, H2B_TRANSFER_SEPARABLE = 0, 1
H2B_COUPLING_DENSE, H2B_COUPLING_DIAGONAL, H2B_COUPLING_TOEPLITZ = 0, 1, 2

_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_u8p = C.POINTER(C.c_uint8)
_f64p = C.POINTER(C.c_double)


class SideDesc(C.Structure):
    _fields_ = [
        ("nnodes", C.c_int32), ("nlevels", C.c_int32), ("root", C.c_int32), ("ndofs", C.c_int32),
        ("level", _i32p), ("parent", _i32p), ("sector", _i32p), ("child_ptr", _i32p),
        ("child", _i32p), ("value_ptr", _i32p), ("value", _i32p), ("shape", _i32p),
        ("agg_nstages", C.c_int32), ("agg_level", _i32p), ("agg_ptr", _i32p), ("agg_node", _i32p),
        ("agg_store", _u8p),
        ("dis_nstages", C.c_int32), ("dis_level", _i32p), ("dis_ptr", _i32p), ("dis_node", _i32p),
        ("dis_isnode", _u8p), ("i2o_ptr", _i32p), ("i2o_src", _i32p), ("i2o_coupling", _i64p),
        ("coll_offset", _i64p), ("coll", _f64p), ("coll_len", C.c_int64),
        ("transfer_offset", _i64p), ("transfer", _f64p), ("transfer_len", C.c_int64),
    ]


class MapDesc(C.Structure):
    _fields_ = [
        ("field", C.c_int32), ("precision", C.c_int32), ("ncomp", C.c_int32), ("dim", C.c_int32),
        ("nsectors", C.c_int32), ("transfer_kind", C.c_int32), ("coupling_kind", C.c_int32),
        ("conj_leaf_adjoint", C.c_int32), ("alpha", (C.c_double * 2) * 3),
        ("test", SideDesc), ("trial", SideDesc),
        ("ncouplings", C.c_int64), ("coupling_offset", _i64p), ("coupling", _f64p),
        ("coupling_len", C.c_int64),
        ("near_nrows", C.c_int32), ("near_row", _i32p), ("near_ptr", _i32p), ("near_col", _i32p),
        ("near_offset", _i64p), ("near", _f64p), ("near_len", C.c_int64),
        ("near_on_device", C.c_int32),
        ("near_kind", C.c_int32), ("near_wavenumber", C.c_double), ("test_points", _f64p),
        ("trial_points", _f64p),
        ("coupling_rowperm", _i64p), ("coupling_colperm", _i64p), ("coupling_perm", _i32p),
        ("coupling_perm_len", C.c_int64),
    ]


class CoreInfo(C.Structure):
    _fields_ = [
        ("device_bytes", C.c_int64), ("near_entries", C.c_int64), ("npairs", C.c_int64 * 2),
        ("moment_elems", C.c_int64), ("spectrum_elems", C.c_int64), ("nrows", C.c_int32),
        ("ncols", C.c_int32),
    ]


class PassTime(C.Structure):
    _fields_ = [("pass_", C.c_int32), ("level", C.c_int32), ("milliseconds", C.c_double)]


# h2b_pass_time.pass values (H2B_PASS_*)
PASS_NAMES = {0: "near", 1: "leaf_aggregate", 2: "aggregate", 3: "modulate_in", 4: "i2o",
              5: "modulate_out", 6: "disaggregate", 7: "leaf_disaggregate"}

LIB_NAME = "libh2b200.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

# every symbol include/h2b200.h declares
EXPORTS = [
    "h2b_version", "h2b_last_error", "h2b_core_create", "h2b_core_destroy", "h2b_core_get_info",
    "h2b_workspace_create", "h2b_workspace_destroy", "h2b_matvec", "h2b_matvec_host",
    "h2b_farmul", "h2b_nearmul", "h2b_farmul_noalloc", "h2b_map_blob_write", "h2b_map_blob_read",
    "h2b_core_create_from_blob", "h2b_tensor_wait_timeouts", "h2b_matvec_host_async",
    "h2b_profile_matvec", "h2b_set_tensor_wait_limit",
]

H2B_NOALLOC_SCRATCH_BYTES = 16 << 20

H2B_NEAR_STORED, H2B_NEAR_LAPLACE, H2B_NEAR_HELMHOLTZ = 0, 1, 2


class H2BError(RuntimeError):
    """A failed h2b_* call; `status` is the h2b_status code."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"h2b status {status}: {msg}")
        self.status = status


class WorkspaceBusyError(H2BError):
    """Concurrent use of one workspace (H2Factory's ConcurrentWorkspaceError)."""


_lib = None


def load_library(path: str | None = None) -> C.CDLL:
    """Load libh2b200.so (once) and declare its signatures."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(f"{p} is missing: build it with h2factory_b200.build.build_library() "
                          "(the CUDA library is the only implementation; there is no fallback)")
    lib = C.CDLL(p)
    vp = C.c_void_p
    lib.h2b_version.restype = C.c_int32
    lib.h2b_last_error.restype = C.c_char_p
    lib.h2b_core_create.argtypes = [C.POINTER(MapDesc), C.c_int32, C.POINTER(vp)]
    lib.h2b_core_destroy.argtypes = [vp]
    lib.h2b_core_get_info.argtypes = [vp, C.POINTER(CoreInfo)]
    lib.h2b_map_blob_write.argtypes = [C.POINTER(MapDesc), vp, C.c_size_t, C.POINTER(C.c_size_t)]
    lib.h2b_map_blob_read.argtypes = [vp, C.c_size_t, C.POINTER(MapDesc)]
    lib.h2b_core_create_from_blob.argtypes = [vp, C.c_size_t, C.c_int32, C.POINTER(vp)]
    lib.h2b_workspace_create.argtypes = [vp, C.c_int32, C.POINTER(vp)]
    lib.h2b_workspace_destroy.argtypes = [vp]
    lib.h2b_tensor_wait_timeouts.argtypes = [C.c_int32, C.POINTER(C.c_uint32)]
    lib.h2b_set_tensor_wait_limit.argtypes = [C.c_int32, C.c_uint32]
    mv = [vp, C.c_int32, C.c_int32, vp, C.c_int64, vp, C.c_int64, _f64p, _f64p, vp]
    for name in ("h2b_matvec", "h2b_matvec_host", "h2b_matvec_host_async", "h2b_farmul", "h2b_nearmul"):
        getattr(lib, name).argtypes = mv
    # far part in the library's built-in scratch: takes the core instead of a workspace
    lib.h2b_farmul_noalloc.argtypes = mv
    lib.h2b_profile_matvec.argtypes = mv + [C.POINTER(PassTime), C.c_int32, C.POINTER(C.c_int32)]
    for name in EXPORTS:
        if name not in ("h2b_version", "h2b_last_error"):
            getattr(lib, name).restype = C.c_int
    if path is None:
        _lib = lib
    return lib


def check(status: int) -> None:
    """Raise H2BError for a non-zero h2b_status."""
    if status != H2B_OK:
        msg = load_library().h2b_last_error().decode(errors="replace")
        if status == H2B_BUSY:
            raise WorkspaceBusyError(status, msg)
        raise H2BError(status, msg)


def set_tensor_wait_limit(limit: int, device: int = 0) -> None:
    """Bound of the tensor-core kernels' mbarrier waits on `device` (0 restores the default)."""
    check(load_library().h2b_set_tensor_wait_limit(device, limit))


def tensor_wait_timeouts(device: int = 0) -> int:
    """Bounded mbarrier waits of the tensor-core kernels that gave up on `device` (0 when healthy)."""
    n = C.c_uint32(0)
    check(load_library().h2b_tensor_wait_timeouts(device, C.byref(n)))
    return int(n.value)
