"""The Julia descriptor mirrors written out for a binding match the C ABI (CPU only).

A Julia package binds the library through isbits mirrors of h2b_side_desc / h2b_map_desc. Julia is
not installed here, so the mirrors cannot be compiled; this test parses the two `struct` blocks out
of the binding's integration notes and checks them field by field against the ctypes mirror the
Python host uses (which `test_abi.py` checks against the header's layout): the same names in the same
order, and for each field the same size, alignment and pointee type, so that the C layout rules
Julia applies to isbits structs place every field at the ctypes offset.
"""

import ctypes as C
import os
import re

from h2factory_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCALARS = {"Int32": C.c_int32, "Int64": C.c_int64, "UInt8": C.c_uint8, "Float64": C.c_double}


def julia_structs():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    out = {}
    for name, body in re.findall(r"^struct (\w+)\n(.*?)^end$", text, flags=re.S | re.M):
        out[name] = [tuple(p.strip() for p in line.split("::")) for line in body.strip().splitlines()]
    return out


def layout(fields, structs):
    """(name, size, align, offset) of each field under the C rules, from the Julia types."""
    out, off, maxal = [], 0, 1
    for name, jt in fields:
        if jt.startswith("Ptr{"):
            size = align = 8
        elif jt in SCALARS:
            size = align = C.sizeof(SCALARS[jt])
        elif (m := re.fullmatch(r"NTuple\{(\d+),(\w+)\}", jt)):
            size, align = int(m.group(1)) * C.sizeof(SCALARS[m.group(2)]), C.sizeof(SCALARS[m.group(2)])
        else:
            sub = layout(structs[jt], structs)
            size, align = sub[-1][0], sub[-1][1]
        off = (off + align - 1) // align * align
        out.append((name, size, align, off))
        off += size
        maxal = max(maxal, align)
    total = (off + maxal - 1) // maxal * maxal
    return out + [(total, maxal)]


def _pointee(ct):
    return getattr(ct, "_type_", None)


def check(jname, ctype, structs):
    fields = structs[jname]
    assert [f for f, _ in fields] == [f for f, _ in ctype._fields_]
    lay = layout(fields, structs)
    (total, _), lay = lay[-1], lay[:-1]
    assert total == C.sizeof(ctype)
    for (name, jt), (_, size, _, off), (_, ct) in zip(fields, lay, ctype._fields_):
        assert getattr(ctype, name).offset == off, name
        assert C.sizeof(ct) == size, name
        if jt.startswith("Ptr{"):
            assert _pointee(ct) is SCALARS[jt[4:-1]], name


def test_side_desc_mirror():
    check("H2BSideDesc", _abi.SideDesc, julia_structs())


def test_map_desc_mirror():
    structs = julia_structs()
    assert set(structs) >= {"H2BSideDesc", "H2BMapDesc"}
    check("H2BMapDesc", _abi.MapDesc, structs)
