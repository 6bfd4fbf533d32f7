"""Host-side core: geometry, settings, workspaces and the tensor-level calls
into the CUDA library.  Everything here takes and returns torch tensors on a
CUDA device; the reference-compatible entry points in :mod:`.cuda`,
:mod:`.cutime` and :mod:`.autograd` are built on these functions.
"""

from __future__ import annotations

import ctypes
import math
import threading
from typing import Optional, Sequence

import numpy as np
import torch

from .. import _native as nat

__all__ = [
    "rotation",
    "parse_settings",
    "make_geom",
    "forward",
    "backward",
    "time_forward",
    "time_order",
    "tune",
    "microbench",
    "workspace_error",
    "ErrorWord",
    "photons",
    "chargesharing",
    "emitters",
    "qcorr_radial",
    "qcorr_3d",
]


def rotation(alpha, beta, gamma):
    """Yaw-pitch-roll rotation matrix, as ``idi/util/__init__.py:348-372``
    (same expression order, so the detector positions agree bit for bit)."""
    cosa, cosb, cosg = math.cos(alpha), math.cos(beta), math.cos(gamma)
    sina, sinb, sing = math.sin(alpha), math.sin(beta), math.sin(gamma)
    return np.array(
        [
            [cosb * cosg, sina * sinb * cosg - cosa * sing, cosa * sinb * cosg + sina * sing],
            [cosb * sing, sina * sinb * sing + cosa * cosg, cosa * sinb * sing - sina * cosg],
            [-sinb, sina * cosb, cosa * cosb],
        ]
    )


def parse_settings(settings: str, default_precision: str = "double"):
    """Map the reference's ``settings`` substrings (``idi/simulation/cuda.py:51-65``)
    to (geometry flags, precision, complex64 output).

    ``single`` -> split-precision kernel with complex64 output; ``split`` ->
    split-precision kernel with complex128 output; ``double`` (or neither) ->
    all-FP64 kernel; ``accurate`` -> all-FP64 kernel with the cancellation-free
    near-field path difference.  ``nf``, ``scale``, ``secondorder`` select the geometry.
    ``nofast`` and unknown substrings are ignored, as in the reference.
    """
    s = settings or ""
    flags = 0
    if "nf" in s:
        flags |= nat.NF
    if "scale" in s:
        flags |= nat.SCALE
    if "secondorder" in s:
        flags |= nat.SECONDORDER
    if "accurate" in s:
        # FP64 near field without the reference's |d-r| - d_z cancellation
        return flags | nat.ACCURATE, nat.DOUBLE, False
    if "split" in s:
        return flags, nat.SPLIT, False
    if "single" in s:
        return flags, nat.SPLIT, True
    if "double" in s:
        return flags, nat.DOUBLE, False
    return flags, (nat.SPLIT if default_precision == "split" else nat.DOUBLE), False


def ndet_pair(Ndet):
    if np.size(Ndet) == 1:
        n = int(np.ravel([Ndet])[0])
        return [n, n]
    return [int(Ndet[0]), int(Ndet[1])]


def make_geom(Ndet, pixelsize, detz, k, detangles=(0, 0), detoffset=(0, 0), flags=0) -> nat.Geom:
    nx, ny = ndet_pair(Ndet)
    g = nat.Geom()
    g.nx, g.ny = nx, ny
    g.flags = int(flags)
    g.pixelsize, g.detz, g.k = float(pixelsize), float(detz), float(k)
    g.offset[0], g.offset[1] = float(detoffset[0]), float(detoffset[1])
    if np.any(detangles):
        M = rotation(float(detangles[0]), float(detangles[1]), 0.0)
        g.has_rot = 1
        for i, v in enumerate(M.ravel()):
            g.rot[i] = float(v)
    else:
        g.has_rot = 0
        for i in range(9):
            g.rot[i] = 1.0 if i % 4 == 0 else 0.0
    return g


# ---------------------------------------------------------------------------
# workspaces
# ---------------------------------------------------------------------------
class _Workspaces:
    """One growing uint8 buffer per (device, role); released with :func:`release`."""

    def __init__(self):
        self._bufs = {}
        self._lock = threading.Lock()

    def get(self, nbytes: int, device: torch.device, role: str = "main") -> torch.Tensor:
        key = (device.index if device.index is not None else torch.cuda.current_device(), role)
        with self._lock:
            buf = self._bufs.get(key)
            if buf is None or buf.numel() < nbytes:
                self._bufs.pop(key, None)
                buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
                self._bufs[key] = buf
            return buf

    def drop(self, device: torch.device, role: str):
        key = (device.index if device.index is not None else torch.cuda.current_device(), role)
        with self._lock:
            self._bufs.pop(key, None)

    def release(self):
        with self._lock:
            self._bufs.clear()


WORKSPACES = _Workspaces()


def release():
    """Free the cached workspaces (the reference's ``idiwf_release``)."""
    WORKSPACES.release()


def _stream(device: torch.device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _require_cuda(t: torch.Tensor, name: str, dtype=None):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def _offsets_array(offsets, n_atoms: int) -> np.ndarray:
    off = np.ascontiguousarray(np.asarray(offsets, dtype=np.int64))
    if off.ndim != 1 or off.size < 2 or off[0] != 0 or off[-1] != n_atoms or np.any(np.diff(off) < 0):
        raise ValueError("offsets must be non-decreasing, start at 0 and end at the emitter count")
    return off


def _batch(atoms: torch.Tensor, off: np.ndarray, amplitudes: Optional[torch.Tensor]) -> nat.Batch:
    b = nat.Batch()
    b.n_images = int(off.size - 1)
    b.offsets = off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    b.atoms = ctypes.c_void_p(atoms.data_ptr() if atoms.numel() else 0)
    if amplitudes is None:
        b.amplitudes = None
        b.amp_dtype = nat.F64
    else:
        b.amplitudes = ctypes.c_void_p(amplitudes.data_ptr())
        b.amp_dtype = nat.F32 if amplitudes.dtype == torch.float32 else nat.F64
    return b


_OUT_DTYPES = {
    nat.OUT_C128: torch.complex128,
    nat.OUT_C64: torch.complex64,
    nat.OUT_I64: torch.float64,
    nat.OUT_I32: torch.float32,
}


def _config(config) -> Optional[nat.Config]:
    if config is None:
        return None
    if isinstance(config, nat.Config):
        return config
    c = nat.Config()
    c.threads = int(config.get("threads", 0))
    c.pixels_per_thread = int(config.get("pixels_per_thread", 0))
    c.emitters_per_tile = int(config.get("emitters_per_tile", 0))
    c.ctas_per_sm = int(config.get("ctas_per_sm", 0))
    c.pixel_groups = int(config.get("pixel_groups", 0))
    return c


def _check_amplitudes(amplitudes, atoms):
    if amplitudes is None:
        return None
    _require_cuda(amplitudes, "amplitudes")
    if amplitudes.dtype not in (torch.float32, torch.float64):
        raise ValueError("amplitudes must be float32 or float64")
    if amplitudes.numel() != atoms.shape[0]:
        raise ValueError("amplitudes must have one entry per emitter")
    return amplitudes


class ErrorWord:
    """Device-side accumulator of the kernels' error words, checked later.

    The library records device-side errors (emitters out of the split range, a
    near-field image outside the split kernels' range, a bounded wait that ran
    out) in the workspace header, and every call clears them.  Calls given an
    ``ErrorWord`` OR their word into this 256-byte device buffer (laid out like
    a workspace header) on their stream, without synchronising; :meth:`check`
    reads it once (synchronises) and raises with the library's message."""

    def __init__(self, device):
        self.device = torch.device(device)
        self.buf = torch.zeros(256, dtype=torch.uint8, device=self.device)
        self._word = self.buf[4:8].view(torch.int32)

    def collect(self, workspace: torch.Tensor):
        self._word.bitwise_or_(workspace[4:8].view(torch.int32))

    def check(self):
        lib = nat.load()
        st = lib.idiwf_workspace_error(ctypes.c_void_p(self.buf.data_ptr()), _stream(self.device))
        self._word.zero_()
        nat.check(st)


def forward(
    atoms: torch.Tensor,
    offsets: Sequence[int],
    geom: nat.Geom,
    precision: int = nat.SPLIT,
    out_kind: int = nat.OUT_C128,
    amplitudes: Optional[torch.Tensor] = None,
    out: Optional[torch.Tensor] = None,
    config=None,
    role: str = "main",
    errors: Optional[ErrorWord] = None,
) -> torch.Tensor:
    """Direct sum of a batch of images: ``atoms`` (N,4) float64 on the GPU,
    image b = rows ``offsets[b]:offsets[b+1]``.  Returns (B, nx, ny).
    With ``errors``, the call's device error word is added to it."""
    lib = nat.load()
    _require_cuda(atoms, "atoms", torch.float64)
    if atoms.ndim != 2 or atoms.shape[1] != 4:
        raise ValueError("atoms must have shape (N, 4): x, y, z, phase")
    amplitudes = _check_amplitudes(amplitudes, atoms)
    off = _offsets_array(offsets, atoms.shape[0])
    B = off.size - 1
    dev = atoms.device
    if out is None:
        out = torch.empty((B, geom.nx, geom.ny), dtype=_OUT_DTYPES[out_kind], device=dev)
    else:
        _require_cuda(out, "out", _OUT_DTYPES[out_kind])
        if tuple(out.shape) != (B, geom.nx, geom.ny):
            raise ValueError("out has the wrong shape")
    batch = _batch(atoms, off, amplitudes)
    cfg = _config(config)
    cfg_p = ctypes.byref(cfg) if cfg is not None else None
    nbytes = lib.idiwf_forward_workspace_size(ctypes.byref(geom), ctypes.byref(batch), precision, cfg_p)
    if nbytes == 0:
        nat.check(nat.ERR_INVALID_ARGUMENT)
    ws = WORKSPACES.get(nbytes, dev, role)
    nat.check(lib.idiwf_forward(ctypes.byref(geom), ctypes.byref(batch), precision, out_kind,
                                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
                                cfg_p, _stream(dev)))
    if errors is not None:
        errors.collect(ws)
    return out


def tune(atoms, offsets, geom, precision=nat.SPLIT, out_kind=nat.OUT_I32, amplitudes=None, role="main") -> dict:
    """Autotune the forward kernel shape on this batch (synchronises)."""
    lib = nat.load()
    _require_cuda(atoms, "atoms", torch.float64)
    amplitudes = _check_amplitudes(amplitudes, atoms)
    off = _offsets_array(offsets, atoms.shape[0])
    out = torch.empty((off.size - 1, geom.nx, geom.ny), dtype=_OUT_DTYPES[out_kind], device=atoms.device)
    batch = _batch(atoms, off, amplitudes)
    nbytes = lib.idiwf_forward_workspace_size(ctypes.byref(geom), ctypes.byref(batch), precision, None)
    ws = WORKSPACES.get(nbytes, atoms.device, role)
    best = nat.Config()
    nat.check(lib.idiwf_tune(ctypes.byref(geom), ctypes.byref(batch), precision, out_kind,
                             ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
                             _stream(atoms.device), ctypes.byref(best)))
    return {"threads": best.threads, "pixels_per_thread": best.pixels_per_thread,
            "emitters_per_tile": best.emitters_per_tile, "ctas_per_sm": best.ctas_per_sm,
            "pixel_groups": best.pixel_groups}


def cta_times(device=None, role="main") -> np.ndarray:
    """Per-CTA busy time (ns) of the last forward launch on ``device``."""
    lib = nat.load()
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    ws = WORKSPACES.get(256, dev, role)
    buf = (ctypes.c_uint64 * 4096)()
    n = ctypes.c_int32(0)
    nat.check(lib.idiwf_forward_cta_times(ctypes.c_void_p(ws.data_ptr()), buf, 4096, ctypes.byref(n), _stream(dev)))
    return np.frombuffer(buf, dtype=np.uint64, count=n.value).copy()


def backward_workspace_error(device=None):
    """Raise if the last adjoint call recorded a device-side error (synchronises)."""
    workspace_error(device, "backward")


def workspace_error(device=None, role="main"):
    """Raise if a kernel recorded a device-side error in the workspace (synchronises)."""
    lib = nat.load()
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    ws = WORKSPACES.get(256, dev, role)
    nat.check(lib.idiwf_workspace_error(ctypes.c_void_p(ws.data_ptr()), _stream(dev)))


def backward(
    atoms: torch.Tensor,
    offsets: Sequence[int],
    geom: nat.Geom,
    field: torch.Tensor,
    grad_intensity: torch.Tensor,
    amplitudes: Optional[torch.Tensor] = None,
    want_amp: bool = True,
    config=None,
    errors: Optional[ErrorWord] = None,
):
    """Adjoint of I = |E|^2: returns (grad_atoms (N,4) [dx,dy,dz,dphase], grad_amp (N) or None).
    ``config``: ``pixels_per_thread`` = emitters per thread (4 or 8), ``pixel_groups`` = -1 for an
    FP64 phase per pair instead of per run of 4 pixels.  With ``errors``, the call's device
    error word is added to it."""
    lib = nat.load()
    _require_cuda(atoms, "atoms", torch.float64)
    _require_cuda(field, "field", torch.complex128)
    _require_cuda(grad_intensity, "grad_intensity", torch.float64)
    amplitudes = _check_amplitudes(amplitudes, atoms)
    off = _offsets_array(offsets, atoms.shape[0])
    B = off.size - 1
    if tuple(field.shape) != (B, geom.nx, geom.ny) or tuple(grad_intensity.shape) != (B, geom.nx, geom.ny):
        raise ValueError("field and grad_intensity must be (B, nx, ny)")
    batch = _batch(atoms, off, amplitudes)
    dev = atoms.device
    grad_atoms = torch.empty((atoms.shape[0], 4), dtype=torch.float64, device=dev)
    grad_amp = torch.empty((atoms.shape[0],), dtype=torch.float64, device=dev) if want_amp else None
    cfg = _config(config)
    cfg_p = ctypes.byref(cfg) if cfg is not None else None
    nbytes = lib.idiwf_backward_workspace_size(ctypes.byref(geom), ctypes.byref(batch), cfg_p)
    if nbytes == 0:
        nat.check(nat.ERR_INVALID_ARGUMENT)
    ws = WORKSPACES.get(nbytes, dev, "backward")
    nat.check(lib.idiwf_backward(ctypes.byref(geom), ctypes.byref(batch), ctypes.c_void_p(field.data_ptr()),
                                 ctypes.c_void_p(grad_intensity.data_ptr()), ctypes.c_void_p(grad_atoms.data_ptr()),
                                 ctypes.c_void_p(grad_amp.data_ptr()) if grad_amp is not None else None,
                                 ctypes.c_void_p(ws.data_ptr()), ws.numel(), cfg_p, _stream(dev)))
    if errors is not None:
        errors.collect(ws)
    return grad_atoms, grad_amp


def time_max_emitters() -> int:
    return int(nat.load().idiwf_time_max_emitters())


def time_forward(atoms: torch.Tensor, times: torch.Tensor, geom: nat.Geom, c: float, tau: float,
                 out: Optional[torch.Tensor] = None, digest: bool = False, stats: Optional[dict] = None):
    """Time-dependent intensity (nx, ny) float64 of one image.  With ``digest``,
    returns (intensity, per-pixel order digests as (nx, ny) int64 holding the
    uint64 bits).  A ``stats`` dict receives (synchronising) how many pixels
    took the full sort and how many warm-started sorts were given up (on-chip
    kernel, up to 20480 emitters; both 0 for larger counts)."""
    lib = nat.load()
    _require_cuda(atoms, "atoms", torch.float64)
    _require_cuda(times, "times", torch.float64)
    if times.numel() != atoms.shape[0]:
        raise ValueError("one emission time per emitter")
    dev = atoms.device
    if out is None:
        out = torch.empty((geom.nx, geom.ny), dtype=torch.float64, device=dev)
    nbytes = lib.idiwf_time_workspace_size(ctypes.byref(geom), atoms.shape[0])
    ws = WORKSPACES.get(nbytes, dev, "time")
    if digest:
        dig = torch.empty((geom.nx, geom.ny), dtype=torch.int64, device=dev)
        nat.check(lib.idiwf_time_forward_digest(ctypes.byref(geom), ctypes.c_void_p(atoms.data_ptr()),
                                                ctypes.c_void_p(times.data_ptr()), atoms.shape[0], float(c),
                                                float(tau), ctypes.c_void_p(out.data_ptr()),
                                                ctypes.c_void_p(dig.data_ptr()), ctypes.c_void_p(ws.data_ptr()),
                                                ws.numel(), _stream(dev)))
    else:
        nat.check(lib.idiwf_time_forward(ctypes.byref(geom), ctypes.c_void_p(atoms.data_ptr()),
                                         ctypes.c_void_p(times.data_ptr()), atoms.shape[0], float(c), float(tau),
                                         ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()),
                                         ws.numel(), _stream(dev)))
    if stats is not None:
        # workspace header words 3 and 4 (uint32)
        w = ws[12:20].cpu().numpy().view(np.uint32)
        stats["full_sorts"], stats["warm_given_up"] = int(w[0]), int(w[1])
    return (out, dig) if digest else out


def time_order(atoms: torch.Tensor, times: torch.Tensor, geom: nat.Geom, c: float, ix: int, iy: int):
    """Sorted emitter order and arrival times of pixel (ix, iy), as the time path sorts them."""
    lib = nat.load()
    _require_cuda(atoms, "atoms", torch.float64)
    _require_cuda(times, "times", torch.float64)
    dev = atoms.device
    n = atoms.shape[0]
    order = torch.empty(n, dtype=torch.int32, device=dev)
    keys = torch.empty(n, dtype=torch.float64, device=dev)
    nbytes = lib.idiwf_time_workspace_size(ctypes.byref(geom), n)
    ws = WORKSPACES.get(nbytes, dev, "time")
    nat.check(lib.idiwf_time_order(ctypes.byref(geom), ctypes.c_void_p(atoms.data_ptr()),
                                   ctypes.c_void_p(times.data_ptr()), n, float(c), int(ix), int(iy),
                                   ctypes.c_void_p(order.data_ptr()), ctypes.c_void_p(keys.data_ptr()),
                                   ctypes.c_void_p(ws.data_ptr()), ws.numel(), _stream(dev)))
    return order, keys


MICROBENCH_KINDS = {"mufu_sincos": 0, "fp64_fma": 1, "fp32_fma": 2, "fp32x2_fma": 3}


def microbench(kind: str, device=None) -> float:
    """Measured pipe throughput: MUFU ops/s, or flop/s for the FMA pipes."""
    lib = nat.load()
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    scratch = torch.empty(4 << 20, dtype=torch.uint8, device=dev)
    rate = ctypes.c_double(0)
    nat.check(lib.idiwf_microbench(MICROBENCH_KINDS[kind], ctypes.c_void_p(scratch.data_ptr()), _stream(dev),
                                   ctypes.byref(rate)))
    return rate.value


# ---------------------------------------------------------------------------
# detector stage
# ---------------------------------------------------------------------------
_ELEM_CODE = {torch.float64: nat.F64, torch.float32: nat.F32, torch.int32: nat.I32, torch.int64: nat.I64}
if hasattr(torch, "uint32"):
    _ELEM_CODE[torch.uint32] = nat.U32


def make_rng(key, stream: int = 0, first_image: int = 0) -> nat.Rng:
    r = nat.Rng()
    r.key[0] = int(key[0]) & (2**64 - 1)
    r.key[1] = int(key[1]) & (2**64 - 1)
    r.stream = int(stream) & (2**64 - 1)
    r.first_image = int(first_image) & (2**64 - 1)
    return r


def photons(probs: torch.Tensor, n_photons: float, key, stream: int = 0, dtype=torch.float64,
            out: Optional[torch.Tensor] = None, first_image: int = 0, check: bool = False) -> torch.Tensor:
    """Poisson photon counts of ``probs`` (..., nx, ny) on its CUDA device: rate
    ``probs * (n_photons / sum over the last two axes)`` (``idi/simulation/common.py:17``).
    ``check`` synchronises and raises ValueError on a negative/NaN probability or an all-zero image."""
    lib = nat.load()
    _require_cuda(probs, "probs")
    if probs.dtype not in (torch.float64, torch.float32):
        raise ValueError("probs must be float64 or float32")
    if probs.dim() < 2:
        raise ValueError("probs needs at least two (detector) axes")
    if dtype not in _ELEM_CODE:
        raise ValueError(f"unsupported count dtype {dtype}")
    npix = probs.shape[-1] * probs.shape[-2]
    B = probs.numel() // npix if npix else 0
    if out is None:
        out = torch.empty(probs.shape, dtype=dtype, device=probs.device)
    elif out.shape != probs.shape or out.dtype != dtype or not out.is_contiguous():
        raise ValueError("out must be a contiguous tensor of probs' shape and the count dtype")
    if B == 0 or npix == 0:
        return out
    dev = probs.device
    ws = WORKSPACES.get(lib.idiwf_photons_workspace_size(B, npix), dev, "photons")
    rng = make_rng(key, stream, first_image)
    nat.check(lib.idiwf_photons(ctypes.c_void_p(probs.data_ptr()), _ELEM_CODE[probs.dtype], B, npix,
                                float(n_photons), ctypes.byref(rng), ctypes.c_void_p(out.data_ptr()),
                                _ELEM_CODE[dtype], ctypes.c_void_p(ws.data_ptr()), ws.numel(), _stream(dev)))
    if check:
        _value_check(dev, "photons")
    return out


def _value_check(dev, role):
    try:
        workspace_error(dev, role)
    except nat.IdiwfError as e:
        if e.status == nat.ERR_INVALID_ARGUMENT:
            raise ValueError(str(e)) from None
        raise


def chargesharing(counts: torch.Tensor, s: float, ns: float = 0.0, key=(0, 0), stream: int = 0,
                  positions: Optional[torch.Tensor] = None, scales: Optional[torch.Tensor] = None,
                  out: Optional[torch.Tensor] = None, first_image: int = 0, check: bool = False) -> torch.Tensor:
    """Charge sharing (``idi/simulation/common.py:26-67``) of photon counts
    (..., nx, ny) on their CUDA device; float64 result.  ``positions`` (P, 2)
    and ``scales`` inject the per-photon draws in the reference's photon order."""
    lib = nat.load()
    _require_cuda(counts, "counts")
    if counts.dtype not in _ELEM_CODE:
        raise ValueError(f"unsupported counts dtype {counts.dtype}")
    if counts.dim() < 2:
        raise ValueError("counts needs at least two (detector) axes")
    nx, ny = counts.shape[-2], counts.shape[-1]
    B = counts.numel() // (nx * ny) if nx * ny else 0
    if out is None:
        out = torch.empty(counts.shape, dtype=torch.float64, device=counts.device)
    if B == 0:
        return out
    dev = counts.device
    npos = 0
    if positions is not None:
        _require_cuda(positions, "positions", torch.float64)
        if positions.dim() != 2 or positions.shape[1] != 2:
            raise ValueError("positions must be (photons, 2)")
        npos = positions.shape[0]
    if scales is not None:
        _require_cuda(scales, "scales", torch.float64)
        need = npos if (s > 0) else counts.numel()
        if scales.numel() != need:
            raise ValueError(f"scales must hold {need} values")
    injected = int(positions is not None and s > 0)
    pos_ptr = None
    if positions is not None:
        # any non-NULL pointer selects injected draws, also for zero photons
        pos_ptr = ctypes.c_void_p(positions.data_ptr() or out.data_ptr())
    ws = WORKSPACES.get(lib.idiwf_chargesharing_workspace_size(B, nx, ny, injected), dev, "charge")
    rng = make_rng(key, stream, first_image)
    nat.check(lib.idiwf_chargesharing(
        ctypes.c_void_p(counts.data_ptr()), _ELEM_CODE[counts.dtype], B, nx, ny, float(s), float(ns),
        ctypes.byref(rng), pos_ptr,
        ctypes.c_void_p(scales.data_ptr()) if scales is not None else None, npos,
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(), _stream(dev)))
    if check:
        _value_check(dev, "charge")
    return out


# ---------------------------------------------------------------------------
# emitter sources
# ---------------------------------------------------------------------------
def _vec3(x, pad):
    """A scalar repeated on three axes, or up to three per-axis values padded with ``pad``."""
    a = np.atleast_1d(np.asarray(x, np.float64)).ravel()
    if a.size == 1:
        return np.repeat(a, 3)
    return np.concatenate([a[:3], np.full(max(0, 3 - a.size), pad)])


def emitters_desc(kind, random_phase=True, r=0.0, fwhm=(0.0, 0.0, 0.0), rho=(2.0, 2.0, 2.0), depth=0.0,
                  attenuation=float("inf"), rot=None, orientation=0, axis=(0.0, 0.0, 1.0), weighted=False,
                  sites: Optional[torch.Tensor] = None) -> nat.EmittersDesc:
    d = nat.EmittersDesc()
    d.kind = int(kind)
    d.random_phase = int(bool(random_phase))
    d.orientation = int(orientation)
    d.weighted = int(bool(weighted))
    d.r = float(r)
    f = _vec3(fwhm, 1.0)
    g = _vec3(rho, 2.0)
    for a in range(3):
        d.fwhm[a] = float(f[a])
        d.rho[a] = float(g[a])
        d.axis[a] = float(axis[a])
    d.depth = float(depth)
    d.attenuation = float(attenuation)
    M = np.eye(3) if rot is None else np.asarray(rot, np.float64).reshape(3, 3)
    for i, v in enumerate(M.ravel()):
        d.rot[i] = float(v)
    if sites is not None:
        _require_cuda(sites, "sites", torch.float64)
        d.sites = ctypes.c_void_p(sites.data_ptr())
        d.n_sites = int(sites.shape[0])
    return d


def emitters(desc: nat.EmittersDesc, n_images: int, n: int, key, stream: int = 0, first_image: int = 0,
             device=None, out: Optional[torch.Tensor] = None, check: bool = False,
             keep: Optional[torch.Tensor] = None) -> torch.Tensor:
    """(n_images * n, 4) float64 emitter rows [x, y, z, phase] drawn on the
    device.  ``keep`` holds a tensor that ``desc`` points into alive for the call."""
    lib = nat.load()
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    if out is None:
        out = torch.empty((n_images * n, 4), dtype=torch.float64, device=dev)
    elif out.shape != (n_images * n, 4) or out.dtype != torch.float64 or not out.is_contiguous():
        raise ValueError("out must be a contiguous (n_images * n, 4) float64 tensor")
    ws = WORKSPACES.get(lib.idiwf_emitters_workspace_size(ctypes.byref(desc), n_images, n), dev, "emitters")
    rng = make_rng(key, stream, first_image)
    nat.check(lib.idiwf_emitters(ctypes.byref(desc), int(n_images), int(n), ctypes.byref(rng),
                                 ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
                                 _stream(dev)))
    if check:
        _value_check(dev, "emitters")
    return out


# ---------------------------------------------------------------------------
# direct q-space correlators
# ---------------------------------------------------------------------------
def qcorr_radial(q: torch.Tensor, images: torch.Tensor, qmax: int) -> torch.Tensor:
    """(B, qmax) float64 radial correlation of float32 images (B, nr, nc);
    q: (nr * nc, 4) float32 [qx, qy, qz, 0] on the same device."""
    lib = nat.load()
    _require_cuda(q, "q", torch.float32)
    _require_cuda(images, "images", torch.float32)
    B, nr, nc = images.shape
    dev = images.device
    out = torch.empty((B, int(qmax)), dtype=torch.float64, device=dev)
    ws = WORKSPACES.get(lib.idiwf_qcorr_workspace_size(nr, nc), dev, "qcorr")
    nat.check(lib.idiwf_qcorr_radial(ctypes.c_void_p(q.data_ptr()), ctypes.c_void_p(images.data_ptr()), B, nr, nc,
                                     int(qmax), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()),
                                     ws.numel(), _stream(dev)))
    return out


def qcorr_3d(zd: torch.Tensor, images: torch.Tensor, qmax: int, maxdqz: int, xcenter: float, ycenter: float,
             z: float) -> torch.Tensor:
    """(B, 2 maxdqz, 2 qmax, 2 qmax) float64 3d correlation of float32 images
    (B, nr, nc); zd: (nr, nc) float32 z / d on the same device."""
    lib = nat.load()
    _require_cuda(zd, "zd", torch.float32)
    _require_cuda(images, "images", torch.float32)
    B, nr, nc = images.shape
    dev = images.device
    out = torch.empty((B, 2 * int(maxdqz), 2 * int(qmax), 2 * int(qmax)), dtype=torch.float64, device=dev)
    ws = WORKSPACES.get(lib.idiwf_qcorr_workspace_size(nr, nc), dev, "qcorr")
    nat.check(lib.idiwf_qcorr_3d(ctypes.c_void_p(zd.data_ptr()), ctypes.c_void_p(images.data_ptr()), B, nr, nc,
                                 int(qmax), int(maxdqz), float(xcenter), float(ycenter), float(z),
                                 ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
                                 _stream(dev)))
    return out
