"""The ctypes mirrors of the C ABI's structs (idi_b200/_native.py) against
include/idiwf.h: same members in the same order, and the same offsets under
the C layout rules that ctypes follows (natural alignment)."""

import ctypes
import os
import re

import pytest

from idi_b200 import _native as nat

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "idiwf.h")
C_SIZES = {"int32_t": 4, "uint32_t": 4, "int64_t": 8, "uint64_t": 8, "double": 8, "float": 4}


def _c_struct(name):
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, flags=re.S)
    assert m, name
    members = []
    for decl in m.group(1).split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        mt = re.match(r"(?:const )?([A-Za-z_0-9]+)\s+(.*)$", decl)
        assert mt, decl
        ctype, rest = mt.groups()
        for d in rest.split(","):
            md = re.match(r"\s*(\*?)\s*(?:const\s+)?(\*?)\s*([A-Za-z_0-9]+)(?:\[(\d+)\])?\s*$", d)
            assert md, d
            ptr = md.group(1) or md.group(2)
            field, count = md.group(3), md.group(4)
            size = 8 if ptr else C_SIZES[ctype] * (int(count) if count else 1)
            align = 8 if ptr else C_SIZES[ctype]
            members.append((field, size, align))
    offsets, off = [], 0
    for field, size, align in members:
        off = (off + align - 1) // align * align
        offsets.append((field, off))
        off += size
    return offsets


@pytest.mark.parametrize("cname,pyname", [("idiwf_geom", "Geom"), ("idiwf_config", "Config"),
                                          ("idiwf_batch", "Batch"), ("idiwf_rng", "Rng"),
                                          ("idiwf_emitters_desc", "EmittersDesc")])
def test_ctypes_mirror_matches_header(cname, pyname):
    cls = getattr(nat, pyname)
    c_fields = _c_struct(cname)
    py_fields = [(f[0], getattr(cls, f[0]).offset) for f in cls._fields_]
    assert py_fields == c_fields
