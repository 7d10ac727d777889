"""The C ABI library loads, exports every declared symbol, and rejects malformed maps (CPU).

Descriptor validation runs on the host before any CUDA call, so these tests need no GPU: they are
the host-side fault tests of the boundary (malformed plans must fail loudly, never reach a kernel).
"""

import ctypes as C
import os
import re

import numpy as np
import pytest

from h2factory_b200 import _abi, methods
from h2factory_b200.core import flatten
from h2factory_b200.trees import build_tree

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "h2b200.h")).read()
    return sorted(set(re.findall(r"^(?:h2b_status|int32_t|const char \*)\s*(h2b_\w+)\(", txt, re.M)))


@pytest.fixture(scope="module")
def lib():
    from h2factory_b200 import build

    build.build_library()
    return _abi.load_library()


def test_exports_every_declared_symbol(lib):
    names = header_functions()
    assert len(names) >= 11
    assert sorted(names) == sorted(_abi.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n


def test_version(lib):
    assert lib.h2b_version() >> 16 == 1


def test_struct_layout_matches_header():
    # field order/count of the ctypes mirror against the header
    txt = open(os.path.join(ROOT, "include", "h2b200.h")).read()
    side = txt[txt.index("typedef struct h2b_side_desc"):txt.index("} h2b_side_desc;")]
    names = re.findall(r"\*?(\w+);", side)
    fields = [f for f, _ in _abi.SideDesc._fields_]
    assert [n for n in names if n in fields] == fields
    mapd = txt[txt.index("typedef struct h2b_map_desc"):txt.index("} h2b_map_desc;")]
    mapd = re.sub(r"/\*.*?\*/", "", mapd, flags=re.S)
    names = re.findall(r"\b(\w+)(?:\[[^\]]*\])*;", mapd)
    fields = [f for f, _ in _abi.MapDesc._fields_]
    assert [n for n in names if n in fields] == fields


@pytest.fixture
def small_core():
    # rebuilt per test: the descriptor points into the core's own arrays, which tests mutate
    rng = np.random.default_rng(0)
    t = build_tree(rng.random((1500, 3)), maxvalues=16, root_center=[0.5] * 3, root_halfsize=0.5)
    assert t.nlevels >= 4
    return methods.interpolation_core(t, methods.laplace, 2)


def create(lib, desc):
    h = C.c_void_p()
    st = lib.h2b_core_create(C.byref(desc), 0, C.byref(h))
    if st == 0:
        lib.h2b_core_destroy(h)
    return st, lib.h2b_last_error().decode()


@pytest.mark.parametrize("mutate, msg", [
    (lambda d, k: setattr(d, "field", 7), "field"),
    (lambda d, k: setattr(d, "ncomp", 0), "ncomp"),
    (lambda d, k: setattr(d, "coupling_kind", 9), "coupling kind"),
    (lambda d, k: k.bad_value(d), "dof id"),
    (lambda d, k: k.dup_value(d), "in two leaves"),
    (lambda d, k: k.bad_coupling(d), "coupling index"),
    (lambda d, k: k.bad_near(d), "near block"),
    (lambda d, k: k.bad_stage_order(d), "aggregation"),
    (lambda d, k: k.bad_parent(d), "parent"),
    (lambda d, k: setattr(d, "near_kind", 7), "near kind"),
    (lambda d, k: setattr(d, "near_kind", _abi.H2B_NEAR_LAPLACE), "without points"),
    (lambda d, k: k.helmholtz_on_real(d), "Helmholtz near kernel on a real map"),
])
def test_malformed_maps_are_rejected(lib, small_core, mutate, msg):
    desc, keep = flatten(small_core)

    class K:
        @staticmethod
        def bad_value(d):
            n = d.test.value_ptr[d.test.nnodes]
            arr = np.ctypeslib.as_array(d.test.value, shape=(n,))
            arr[3] = d.test.ndofs + 5

        @staticmethod
        def dup_value(d):
            n = d.test.value_ptr[d.test.nnodes]
            arr = np.ctypeslib.as_array(d.test.value, shape=(n,))
            arr[3] = arr[n - 1]

        @staticmethod
        def bad_coupling(d):
            n = d.test.i2o_ptr[d.test.nnodes]
            arr = np.ctypeslib.as_array(d.test.i2o_coupling, shape=(n,))
            arr[0] = d.ncouplings

        @staticmethod
        def bad_near(d):
            arr = np.ctypeslib.as_array(d.near_offset, shape=(d.near_ptr[d.near_nrows],))
            arr[-1] = d.near_len

        @staticmethod
        def bad_stage_order(d):
            arr = np.ctypeslib.as_array(d.trial.agg_level, shape=(d.trial.agg_nstages,))
            arr[:] = arr[::-1].copy()

        @staticmethod
        def bad_parent(d):
            arr = np.ctypeslib.as_array(d.test.parent, shape=(d.test.nnodes,))
            arr[5] = d.test.nnodes + 3

        @staticmethod
        def helmholtz_on_real(d):
            pts = np.zeros(3 * max(d.test.ndofs, d.trial.ndofs))
            keep.append(pts)
            d.test_points = d.trial_points = pts.ctypes.data_as(C.POINTER(C.c_double))
            d.near_kind = _abi.H2B_NEAR_HELMHOLTZ

    mutate(desc, K)
    st, err = create(lib, desc)
    assert st == _abi.H2B_ERR_INVALID
    assert msg in err
    del keep


def test_bad_permutations_are_rejected(lib):
    rng = np.random.default_rng(2)
    t = build_tree(rng.random((800, 3)), maxvalues=16, root_center=[0.5] * 3, root_halfsize=0.5)
    core = methods.interpolation_core(t, methods.laplace, 2, symmetry=True)
    for how, msg in (("dup", "not a permutation"), ("range", "not a permutation"), ("off", "out of range")):
        desc, keep = flatten(core)
        arr = np.ctypeslib.as_array(desc.coupling_perm, shape=(desc.coupling_perm_len,))
        offs = np.ctypeslib.as_array(desc.coupling_rowperm, shape=(desc.ncouplings,))
        if how == "dup":
            arr[1] = arr[0]
        elif how == "range":
            arr[0] = 99
        else:
            offs[offs >= 0] = desc.coupling_perm_len
        st, err = create(lib, desc)
        assert st == _abi.H2B_ERR_INVALID and msg in err, (how, err)
        del keep


def test_bad_call_arguments_without_device(lib):
    st = lib.h2b_matvec(None, 0, 1, None, 1, None, 1, None, None, None)
    assert st == _abi.H2B_ERR_INVALID
    st = lib.h2b_workspace_create(None, 1, C.byref(C.c_void_p()))
    assert st == _abi.H2B_ERR_INVALID
