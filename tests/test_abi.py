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


def test_fft_autocorr_validation(lib):
    """``idiwf_fft_autocorr``: its workspace size and the argument checks
    that come before any device work."""
    vp = ctypes.c_void_p
    al = lambda b: (b + 255) // 256 * 256  # noqa: E731
    # twiddles (N = max(2 n0, 2 n1) double pairs), then T (n1 + 1) x n0 and
    # C (n1 + 1) x (n0 + 1) complex values per image of a group
    need = lib.idiwf_fft_autocorr_workspace_size(1, 8, 16, nat.F64)
    assert need == al(32 * 16) + al(17 * 8 * 16) + al(17 * 9 * 16)
    assert lib.idiwf_fft_autocorr_workspace_size(3, 8, 16, nat.F32) == al(32 * 16) + al(3 * 17 * 8 * 8) + al(
        3 * 17 * 9 * 8)
    # 1024^2 FP64: 33.6 MB of T and C per image, groups of at most 7 images
    # (256 MB), balanced: 8 images run as two groups of 4
    assert lib.idiwf_fft_autocorr_workspace_size(8, 1024, 1024, nat.F64) == al(2048 * 16) + al(
        4 * 1025 * 1024 * 16) + al(4 * 1025 * 1025 * 16)
    # other lengths: padded to fastlen(2 n); tables of G1, G0 and L1 values,
    # T m x n0 and C m x (n0 + 1), m = G1 / 2 + 1.  6 x 8: G0 = 12, G1 = L1 = 16
    assert lib.idiwf_fft_autocorr_workspace_size(1, 6, 8, nat.F64) == 3 * 256 + al(9 * 6 * 16) + al(9 * 7 * 16)
    # padded lengths above 4096 (fastlen(4098) = 4116, fastlen(6000) = 6000)
    for n0, n1 in ((8, 2049), (8, 8192), (0, 8), (3000, 8), (8, 0)):
        assert lib.idiwf_fft_autocorr_workspace_size(1, n0, n1, nat.F64) == 0, (n0, n1)
    # 5 x 13: G1 = 27 is odd, the inverse has L1 = 26 values (Hp = 13 by
    # Bluestein through FFTs of M = fastlen(2 Hp - 1) = 25): tables of 27, 10,
    # 26 and chirp 13, filter and twiddles 25
    assert lib.idiwf_fft_autocorr_workspace_size(1, 5, 13, nat.F64) == (
        al(27 * 16) + al(10 * 16) + al(26 * 16) + al(13 * 16) + 2 * al(25 * 16) + al(14 * 5 * 16) + al(14 * 6 * 16))
    assert lib.idiwf_fft_autocorr_workspace_size(1, 8, 8, 7) == 0
    assert lib.idiwf_fft_autocorr_workspace_size(0, 8, 8, nat.F64) == 0

    def call(x=4096, dtype=nat.F64, batch=1, n0=8, n1=16, norm=None, mode=-1, ws=4096, ws_bytes=need, out=8192):
        return lib.idiwf_fft_autocorr(vp(x), dtype, batch, n0, n1, vp(norm) if norm else None, mode, 0.5, vp(out),
                                      vp(ws), ws_bytes, None)

    assert call(x=0) == nat.ERR_INVALID_ARGUMENT
    assert call(out=0) == nat.ERR_INVALID_ARGUMENT
    assert call(batch=0) == nat.ERR_INVALID_ARGUMENT
    assert call(n1=3000) == nat.ERR_UNSUPPORTED
    assert b"not supported" in lib.idiwf_last_error_string()
    # the closed-form pair count does not hold for an odd padded width
    ws_odd = lib.idiwf_fft_autocorr_workspace_size(1, 5, 13, nat.F64)
    assert call(n0=5, n1=13, mode=2, ws_bytes=ws_odd) == nat.ERR_UNSUPPORTED
    assert call(mode=3) == nat.ERR_INVALID_ARGUMENT
    assert call(mode=0) == nat.ERR_INVALID_ARGUMENT  # no norm
    assert call(ws_bytes=need - 1) == nat.ERR_WORKSPACE
    assert call(batch=2) == nat.ERR_WORKSPACE  # sized for one image
    assert call(ws=4096 + 128) == nat.ERR_WORKSPACE
    assert call(x=4096 + 8) == nat.ERR_INVALID_ARGUMENT
    assert call(out=8192 + 8) == nat.ERR_INVALID_ARGUMENT
    assert call(dtype=9) == nat.ERR_INVALID_ARGUMENT


def test_fft_autocorr_shape_predicate():
    import torch

    from idi_b200.reconstruction import cusimple

    assert cusimple._hand_ok((1024, 1024), torch.float64)
    assert cusimple._hand_ok((4, 4096), torch.float32)
    assert cusimple._hand_ok((2, 8), torch.float64)
    assert cusimple._hand_ok((15, 33), torch.float64)
    assert cusimple._hand_ok((30,), torch.float64)
    assert cusimple._hand_ok((13,), torch.float64)
    assert cusimple._hand_ok((8, 13), torch.float64)
    assert not cusimple._hand_ok((8, 3000), torch.float64)
    assert not cusimple._hand_ok((8, 8192), torch.float64)
    assert not cusimple._hand_ok((8, 8, 8), torch.float64)
    assert not cusimple._hand_ok((8, 8), torch.float16)


def test_fft_autocorr_1d_validation(lib):
    """``idiwf_fft_autocorr_1d``: lines run as images of up to 1024 rows;
    the workspace holds two twiddle tables and T of one group of images."""
    vp = ctypes.c_void_p
    al = lambda b: (b + 255) // 256 * 256  # noqa: E731
    # 3000 lines of 1000: images of 1024 rows (2 + a remainder of 952), G = 2000, m = 1001
    assert lib.idiwf_fft_autocorr_1d_workspace_size(3000, 1000, nat.F64) == 2 * al(2000 * 16) + al(
        2 * 1001 * 1024 * 16)
    assert lib.idiwf_fft_autocorr_1d_workspace_size(10, 30, nat.F32) == 2 * al(60 * 16) + al(31 * 10 * 8)
    assert lib.idiwf_fft_autocorr_1d_workspace_size(1, 13, nat.F64) > 0  # fastlen(26) = 27: Bluestein
    assert lib.idiwf_fft_autocorr_1d_workspace_size(1, 3000, nat.F64) == 0
    assert lib.idiwf_fft_autocorr_1d_workspace_size(0, 30, nat.F64) == 0
    assert lib.idiwf_fft_autocorr_1d_workspace_size(1, 30, 7) == 0
    need = lib.idiwf_fft_autocorr_1d_workspace_size(4, 30, nat.F64)

    def call(x=4096, dtype=nat.F64, lines=4, n=30, mode=-1, ws=4096, ws_bytes=need, out=8192):
        return lib.idiwf_fft_autocorr_1d(vp(x), dtype, lines, n, None, mode, 0.5, vp(out), vp(ws), ws_bytes, None)

    assert call(x=0) == nat.ERR_INVALID_ARGUMENT
    assert call(lines=0) == nat.ERR_INVALID_ARGUMENT
    assert call(dtype=9) == nat.ERR_INVALID_ARGUMENT
    assert call(n=3000) == nat.ERR_UNSUPPORTED
    assert call(mode=5) == nat.ERR_INVALID_ARGUMENT
    assert call(mode=1) == nat.ERR_INVALID_ARGUMENT  # no norm
    assert call(ws_bytes=need - 1) == nat.ERR_WORKSPACE
    assert call(ws=4096 + 64) == nat.ERR_WORKSPACE
