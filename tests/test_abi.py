"""The C-ABI library: it loads, exports every symbol include/idiwf.h
declares, and rejects bad arguments on the host (no GPU needed)."""

import ctypes
import os
import re

import numpy as np
import pytest

from idi_b200 import _native as nat
from idi_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(nat.LIB_PATH):
        build.build()
    return nat.load()


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "idiwf.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(idiwf_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(lib):
    syms = header_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(nat.EXPORTED)


def test_version(lib):
    assert lib.idiwf_version() >> 16 == 1


def _geom(nx=8, ny=8, k=1e4, flags=0):
    g = nat.Geom()
    g.nx, g.ny, g.flags = nx, ny, flags
    g.pixelsize, g.detz, g.k = 75.0, 1e5, k
    for i in range(9):
        g.rot[i] = 1.0 if i % 4 == 0 else 0.0
    return g


def _batch(offsets):
    off = np.asarray(offsets, np.int64)
    b = nat.Batch()
    b.n_images = off.size - 1
    b.offsets = off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    b.atoms = ctypes.c_void_p(4096)  # never dereferenced on the host
    b.amplitudes = None
    return b, off


def test_workspace_size_validates(lib):
    b, _keep = _batch([0, 10, 30])
    assert lib.idiwf_forward_workspace_size(ctypes.byref(_geom()), ctypes.byref(b), nat.SPLIT, None) > 0
    assert lib.idiwf_forward_workspace_size(ctypes.byref(_geom(nx=0)), ctypes.byref(b), nat.SPLIT, None) == 0
    assert lib.idiwf_forward_workspace_size(ctypes.byref(_geom(k=-1)), ctypes.byref(b), nat.SPLIT, None) == 0
    assert lib.idiwf_forward_workspace_size(ctypes.byref(_geom()), ctypes.byref(b), 7, None) == 0
    bad, _keep2 = _batch([0, 10, 5])
    assert lib.idiwf_forward_workspace_size(ctypes.byref(_geom()), ctypes.byref(bad), nat.SPLIT, None) == 0
    # workspace grows with padded emitters
    b2, _keep3 = _batch([0, 100000])
    assert lib.idiwf_forward_workspace_size(ctypes.byref(_geom()), ctypes.byref(b2), nat.SPLIT, None) > 100000 * 52


def _fwd(lib, g, b, precision=nat.SPLIT, out_kind=nat.OUT_C128, out=4096, ws=4096, ws_bytes=1 << 20, cfg=None):
    return lib.idiwf_forward(ctypes.byref(g), ctypes.byref(b), precision, out_kind, ctypes.c_void_p(out),
                             ctypes.c_void_p(ws), ws_bytes, ctypes.byref(cfg) if cfg else None, None)


def test_forward_rejects_bad_arguments(lib):
    b, _keep = _batch([0, 10])
    assert _fwd(lib, _geom(nx=-1), b) == nat.ERR_INVALID_ARGUMENT
    assert b"positive" in lib.idiwf_last_error_string()
    assert _fwd(lib, _geom(), b, precision=9) == nat.ERR_INVALID_ARGUMENT
    assert _fwd(lib, _geom(), b, out_kind=9) == nat.ERR_INVALID_ARGUMENT
    assert _fwd(lib, _geom(), b, out=0) == nat.ERR_INVALID_ARGUMENT
    assert _fwd(lib, _geom(flags=64), b) == nat.ERR_INVALID_ARGUMENT
    # workspace too small / misaligned
    assert _fwd(lib, _geom(), b, ws_bytes=16) == nat.ERR_WORKSPACE
    assert _fwd(lib, _geom(), b, ws=4096 + 8) == nat.ERR_WORKSPACE
    # misaligned atoms
    b.atoms = ctypes.c_void_p(4096 + 8)
    assert _fwd(lib, _geom(), b) == nat.ERR_INVALID_ARGUMENT
    # bad kernel shapes
    b.atoms = ctypes.c_void_p(4096)
    cfg = nat.Config(threads=100)
    assert _fwd(lib, _geom(), b, cfg=cfg) == nat.ERR_INVALID_ARGUMENT
    cfg = nat.Config(emitters_per_tile=100)
    assert _fwd(lib, _geom(), b, cfg=cfg) == nat.ERR_INVALID_ARGUMENT
    cfg = nat.Config(pixels_per_thread=3)
    assert _fwd(lib, _geom(), b, cfg=cfg) == nat.ERR_INVALID_ARGUMENT


def test_empty_batch_rejected(lib):
    b, _keep = _batch([0])
    assert _fwd(lib, _geom(), b) == nat.ERR_INVALID_ARGUMENT


def test_time_path_validation(lib):
    g = _geom()
    ws = ctypes.c_void_p(4096)
    at = ctypes.c_void_p(4096)
    n_max = lib.idiwf_time_max_emitters()
    assert n_max >= 20000
    # above the on-chip table the global-memory kernel needs a workspace that grows with n
    assert lib.idiwf_time_workspace_size(ctypes.byref(g), n_max + 1) > 1 << 20
    assert lib.idiwf_time_forward(ctypes.byref(g), at, at, n_max + 1, 0.3, 2.0, ws, ws, 1 << 20, None) == nat.ERR_WORKSPACE
    assert lib.idiwf_time_forward(ctypes.byref(g), at, at, (1 << 28) + 1, 0.3, 2.0, ws, ws, 1 << 20, None) == nat.ERR_UNSUPPORTED
    assert lib.idiwf_time_forward(ctypes.byref(g), at, at, 0, 0.3, 2.0, ws, ws, 1 << 20, None) == nat.ERR_INVALID_ARGUMENT
    assert lib.idiwf_time_forward(ctypes.byref(g), at, at, 10, -1.0, 2.0, ws, ws, 1 << 20, None) == nat.ERR_INVALID_ARGUMENT
    g.offset[0] = 1.0
    assert lib.idiwf_time_forward(ctypes.byref(g), at, at, 10, 0.3, 2.0, ws, ws, 1 << 20, None) == nat.ERR_INVALID_ARGUMENT
    g.offset[0] = 0.0
    g.flags = nat.SECONDORDER
    assert lib.idiwf_time_forward(ctypes.byref(g), at, at, 10, 0.3, 2.0, ws, ws, 1 << 20, None) == nat.ERR_UNSUPPORTED


def test_backward_validation(lib):
    b, _keep = _batch([0, 10])
    g = _geom()
    z = ctypes.c_void_p(4096)
    assert lib.idiwf_backward(ctypes.byref(g), ctypes.byref(b), None, z, z, None, z, 1 << 30, None, None) == nat.ERR_INVALID_ARGUMENT
    assert lib.idiwf_backward(ctypes.byref(g), ctypes.byref(b), z, z, z, None, z, 16, None, None) == nat.ERR_WORKSPACE
    assert lib.idiwf_backward_workspace_size(ctypes.byref(g), ctypes.byref(b), None) > 0


def test_microbench_validation(lib):
    r = ctypes.c_double()
    assert lib.idiwf_microbench(9, ctypes.c_void_p(4096), None, ctypes.byref(r)) == nat.ERR_INVALID_ARGUMENT


def test_product_has_no_cpu_fallback(monkeypatch):
    """Compute calls fail loudly when the library is missing."""
    import importlib

    monkeypatch.setattr(nat, "LIB_PATH", "/nonexistent/libidiwf.so")
    monkeypatch.setattr(nat, "_lib", None)
    with pytest.raises(nat.NativeLibraryMissing):
        nat.load()
    importlib.reload(nat)
