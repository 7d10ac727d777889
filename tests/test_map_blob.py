"""Map blob (CPU): the descriptor as one byte image, written and read back through the C ABI.

A core stored this way loads in another process without its builder. Read back, every field must
equal the original descriptor's; truncated or altered images are refused with an error, never
read out of bounds.
"""

import ctypes as C

import numpy as np
import pytest

import h2factory_b200 as h2
from h2factory_b200 import _abi, methods
from h2factory_b200.trees import build_tree


def _core(kind):
    rng = np.random.default_rng(4)
    if kind == "toeplitz-sym":
        t = build_tree(rng.random((1500, 3)), depth=3, root_center=[0.5] * 3, root_halfsize=0.5)
        return methods.interpolation_core(t, methods.helmholtz(2.0), 3, nodes="equispaced",
                                          couplings="toeplitz", symmetry=True)
    t = build_tree(rng.random((1200, 3)), maxvalues=30, root_center=[0.5] * 3, root_halfsize=0.5)
    if kind == "free":
        return methods.interpolation_core(t, methods.laplace, 3, near="free")
    return methods.interpolation_core(t, methods.laplace, 3, transfers="separable")


def _arr(ptr, n, dt):
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt) if n else np.zeros(0, dt)


@pytest.mark.parametrize("kind", ["dense", "free", "toeplitz-sym"])
def test_blob_round_trip(kind):
    core = _core(kind)
    desc, keep = h2.flatten(core)
    buf, back = h2.read_blob(h2.map_blob(core))
    for name, _ in _abi.MapDesc._fields_:
        a, b = getattr(desc, name), getattr(back, name)
        if isinstance(a, (int, float)):
            assert a == b, name
    assert np.array_equal(np.ctypeslib.as_array(desc.alpha), np.ctypeslib.as_array(back.alpha))
    for side in ("test", "trial"):
        s, r = getattr(desc, side), getattr(back, side)
        nn = s.nnodes
        for name in ("level", "parent", "sector"):
            assert np.array_equal(_arr(getattr(s, name), nn, np.int32), _arr(getattr(r, name), nn, np.int32))
        nv = s.value_ptr[nn]
        assert np.array_equal(_arr(s.value, nv, np.int32), _arr(r.value, nv, np.int32))
        npair = s.i2o_ptr[nn]
        assert np.array_equal(_arr(s.i2o_coupling, npair, np.int64), _arr(r.i2o_coupling, npair, np.int64))
        fw = 2 if core.field == "complex" else 1
        assert np.array_equal(_arr(s.coll, fw * s.coll_len, np.float64), _arr(r.coll, fw * r.coll_len, np.float64))
        assert np.array_equal(_arr(s.transfer, fw * s.transfer_len, np.float64),
                              _arr(r.transfer, fw * r.transfer_len, np.float64))
    assert np.array_equal(_arr(desc.coupling, desc.coupling_len, np.float64),
                          _arr(back.coupling, back.coupling_len, np.float64))
    if core.near_kind == "stored":
        n = desc.near_len * (2 if core.field == "complex" else 1)
        assert np.array_equal(_arr(desc.near, n, np.float64), _arr(back.near, n, np.float64))
    else:
        assert np.array_equal(_arr(desc.test_points, 3 * desc.test.ndofs, np.float64),
                              _arr(back.test_points, 3 * back.test.ndofs, np.float64))
    if core.coupling_canon is not None:
        assert np.array_equal(_arr(desc.coupling_perm, desc.coupling_perm_len, np.int32),
                              _arr(back.coupling_perm, back.coupling_perm_len, np.int32))
    # the oracle on the read-back descriptor gives the original product
    from oracle import oracle

    x = np.random.default_rng(0).standard_normal(core.trial.npoints)
    if core.field == "complex":
        x = x + 0j
    if core.near_kind == "stored":
        for mode in (0, 2):
            a = oracle.matvec(core, x, mode)
            assert np.array_equal(a, oracle.matvec(core, x, mode, desc=(back, buf)))
    del keep, buf


def test_bad_blobs_are_refused():
    lib = _abi.load_library()
    good = h2.map_blob(_core("dense"))
    out = _abi.MapDesc()

    def read(b):
        buf = np.zeros((b.size + 7) // 8 + 1, np.uint64).view(np.uint8)[:b.size]
        buf[:] = b
        return lib.h2b_map_blob_read(buf.ctypes.data_as(C.c_void_p), buf.size, C.byref(out)), \
            lib.h2b_last_error().decode()

    assert read(good)[0] == _abi.H2B_OK
    st, msg = read(good[: good.size // 2])
    assert st == _abi.H2B_ERR_INVALID and ("truncated" in msg or "bounds" in msg or "entries" in msg)
    bad = good.copy()
    bad[:8] = np.frombuffer(b"NOTABLOB", np.uint8)
    assert read(bad) == (_abi.H2B_ERR_INVALID, "h2b_map_blob_read: not a map blob")
    bad = good.copy()
    bad[8:16] = np.frombuffer(np.uint64(3).tobytes(), np.uint8)  # record count
    assert read(bad)[0] == _abi.H2B_ERR_INVALID
    bad = good.copy()
    # the first array record's count (after the 16-byte head and the scalars record)
    sc = int(np.frombuffer(good[20:24].tobytes(), np.uint32)[0])
    at = 16 + 16 + ((sc + 7) & ~7) + 8
    bad[at:at + 8] = np.frombuffer(np.int64(1 << 40).tobytes(), np.uint8)
    assert read(bad)[0] == _abi.H2B_ERR_INVALID


def test_blob_file(tmp_path):
    core = _core("dense")
    path = tmp_path / "map.h2b"
    n = h2.save_map(core, str(path))
    assert path.stat().st_size == n
    buf, desc = h2.read_blob(str(path))
    assert desc.test.ndofs == core.test.npoints
