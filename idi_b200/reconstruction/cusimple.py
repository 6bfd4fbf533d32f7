"""Drop-in for ``idi.reconstruction.cusimple``: FFT autocorrelation on the GPU
(``idi/reconstruction/cusimple.py:6-121``).

One or two correlated axes go through this library's own FFTs end to end
(``idiwf_fft_autocorr``: the padded transform, the power spectrum, the
inverse, the fftshift, the crop and the normalisation) whenever the library
takes the shape: powers of two from 4 to 4096, or padded lengths
``fastlen(2 n)`` up to 4096 (an odd last one by Bluestein's algorithm, for
the reference's inverse of one value fewer).
Other shapes (and three axes) use cuFFT's transforms (through ``torch.fft``)
with this library's power-spectrum and crop kernels around them
(``idiwf_power_spectrum``, ``idiwf_corr_crop``).  The correlator's running mean / variance is
``idiwf_welford_update``.  Inputs may be numpy arrays or CUDA tensors;
results are numpy unless ``returngpu``.
"""

from __future__ import annotations

import ctypes
import functools

import numpy as np
import torch

from .. import _native as nat
from ..simulation import _core

__all__ = ["corr", "correlator2d", "fastlen"]


@functools.lru_cache(maxsize=None)
def fastlen(x, factors=(2, 3, 5, 7, 11)):
    """Smallest N >= x whose prime factors are all in ``factors`` (FFT-friendly length)."""
    n = max(1, int(np.ceil(x)))
    while True:
        m = n
        for f in factors:
            while m % f == 0:
                m //= f
        if m == 1:
            return n
        n += 1


def _device():
    return torch.device("cuda", torch.cuda.current_device())


def _code(t):
    if t.dtype == torch.float64 or t.dtype == torch.complex128:
        return nat.F64
    if t.dtype == torch.float32 or t.dtype == torch.complex64:
        return nat.F32
    raise ValueError(f"unsupported dtype {t.dtype}")


def _stream(dev):
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _power_(spec):
    nat.check(nat.load().idiwf_power_spectrum(ctypes.c_void_p(spec.data_ptr()), spec.numel(), _code(spec),
                                              _stream(spec.device)))
    return spec


def _crop(full, nax, halves, norm=None, mode=0, threshold=0.0):
    """Centre crop of the last ``nax`` axes of ``full`` (batch leading)."""
    full = full.contiguous()
    g = (ctypes.c_int32 * nax)(*full.shape[-nax:])
    n = (ctypes.c_int32 * nax)(*halves)
    lead = full.shape[:-nax]
    batch = int(np.prod(lead)) if lead else 1
    out = torch.empty(tuple(lead) + tuple(2 * h for h in halves), dtype=full.dtype, device=full.device)
    if norm is not None:
        norm = norm.to(full.dtype).contiguous()
    nat.check(nat.load().idiwf_corr_crop(
        ctypes.c_void_p(full.data_ptr()), _code(full), batch, nax, g, n,
        ctypes.c_void_p(norm.data_ptr()) if norm is not None else None, int(mode), float(threshold),
        ctypes.c_void_p(out.data_ptr()), _stream(full.device)))
    return out


def _autocorr(x, nax, fftshape):
    """Autocorrelation along the last ``nax`` axes, uncropped: irfftn(|rfftn(x, s)|^2)
    with the inverse's default sizes, as the reference's calls."""
    dims = tuple(range(-nax, 0))
    spec = torch.fft.rfftn(x, s=fftshape, dim=dims)
    _power_(spec)
    return torch.fft.irfftn(spec, dim=dims)


def _hand_ok(shape, dtype):
    """Whether ``idiwf_fft_autocorr`` (two correlated axes) or
    ``idiwf_fft_autocorr_1d`` (one) takes this shape."""
    if len(shape) not in (1, 2) or dtype not in (torch.float32, torch.float64):
        return False
    code = nat.F64 if dtype == torch.float64 else nat.F32
    lib = nat.load()
    if len(shape) == 1:
        return lib.idiwf_fft_autocorr_1d_workspace_size(1, int(shape[0]), code) > 0
    return lib.idiwf_fft_autocorr_workspace_size(1, int(shape[0]), int(shape[1]), code) > 0


def _hand_autocorr_1d(x, mode=-1, norm=None, threshold=0.0):
    """Autocorrelation of every line of the last axis (length n) by
    ``idiwf_fft_autocorr_1d``; ``mode`` as ``idiwf_fft_autocorr`` (norm: 2n
    values)."""
    n = int(x.shape[-1])
    x = x.contiguous()
    if norm is not None:
        norm = norm.to(x.dtype).contiguous()
    lines = x.numel() // n
    out = torch.empty(tuple(x.shape[:-1]) + (2 * n,), dtype=x.dtype, device=x.device)
    lib = nat.load()
    code = _code(x)
    nbytes = lib.idiwf_fft_autocorr_1d_workspace_size(lines, n, code)
    ws = _core.WORKSPACES.get(nbytes, x.device, "fftcorr")
    nat.check(lib.idiwf_fft_autocorr_1d(
        ctypes.c_void_p(x.data_ptr()), code, lines, n,
        ctypes.c_void_p(norm.data_ptr()) if norm is not None else None, int(mode), float(threshold),
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(), _stream(x.device)))
    return out


def _hand_autocorr(x, mode=-1, norm=None, threshold=0.0):
    """Shifted autocorrelation ((2 n0) x (2 n1), no crop needed) of the last two axes of
    ``x`` (power-of-two lengths) by ``idiwf_fft_autocorr``; ``mode`` as there
    (-1 none, 0 / 1 divide by ``norm``, 2 divide by the pair count)."""
    x = x.contiguous()
    if x.data_ptr() % (2 * x.element_size()):
        x = x.clone()  # rows are read as pairs of values
    n0, n1 = int(x.shape[-2]), int(x.shape[-1])
    lead = tuple(x.shape[:-2])
    batch = int(np.prod(lead)) if lead else 1
    out = torch.empty(lead + (2 * n0, 2 * n1), dtype=x.dtype, device=x.device)
    if norm is not None:
        norm = norm.to(x.dtype).contiguous()
    lib = nat.load()
    code = _code(x)
    nbytes = lib.idiwf_fft_autocorr_workspace_size(batch, n0, n1, code)
    ws = _core.WORKSPACES.get(nbytes, x.device, "fftcorr")
    nat.check(lib.idiwf_fft_autocorr(
        ctypes.c_void_p(x.data_ptr()), code, batch, n0, n1,
        ctypes.c_void_p(norm.data_ptr()) if norm is not None else None, int(mode), float(threshold),
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(), _stream(x.device)))
    return out


def corr(input, axes=(-1, -2), norm=False, returngpu=False, **kwargs):
    """Autocorrelation of ``input`` along ``axes`` (default the last two),
    output 2n per correlated axis with zero shift at index n.  ``norm``
    divides by the mean over the other axes (over everything when there are
    none) and by the pair count, with NaN where fewer than 0.9 pairs overlap."""
    x = input if isinstance(input, torch.Tensor) else torch.from_numpy(np.asarray(input))
    x = x.to(_device())
    if not x.is_floating_point():
        x = x.to(torch.float64)
    axes = sorted([x.ndim + a if a < 0 else a for a in axes])
    others = [i for i in range(x.ndim) if i not in axes]
    sizes = [x.shape[a] for a in axes]
    fftshape = [fastlen(2 * s) for s in sizes]
    if norm:
        x = x * (1 / x.mean(dim=others if others else None, keepdim=bool(others)))
    moved = torch.movedim(x, axes, list(range(x.ndim - len(axes), x.ndim))).contiguous()
    if _hand_ok(sizes, x.dtype):
        f = _hand_autocorr if len(sizes) == 2 else _hand_autocorr_1d
        if not norm:
            ret = f(moved, mode=-1)
        elif fastlen(2 * sizes[-1]) % 2 == 0:
            # the pair count in closed form: the transform of ones in the
            # reference rounds to the same integers, and the same < 0.9 positions
            ret = f(moved, mode=2, threshold=0.9)
        else:
            # an odd last padded length: the reference's inverse has one
            # value fewer, and its pair count is the same transform of ones
            pairs = f(torch.ones(sizes, dtype=x.dtype, device=x.device), mode=-1)
            ret = f(moved, mode=0, norm=pairs, threshold=0.9)
    else:
        full = _autocorr(moved, len(axes), fftshape)
        pairs = None
        if norm:
            ones = torch.ones(sizes, dtype=x.dtype, device=x.device)
            pairs = _crop(_autocorr(ones, len(axes), fftshape), len(axes), sizes)
        ret = _crop(full, len(axes), sizes, norm=pairs, mode=0, threshold=0.9)
    ret = torch.movedim(ret, list(range(x.ndim - len(axes), x.ndim)), axes)
    if returngpu:
        return ret
    return ret.cpu().numpy()


class correlator2d:
    """Running 2D autocorrelation divided by the mask autocorrelation
    (``idi/reconstruction/cusimple.py:40-121``), FP32 like the reference:
    ``add(image, mask=None)`` accumulates, ``mean`` / ``std`` / ``n`` report."""

    def __init__(self, mask=None, norm=True) -> None:
        self._fftshape = None
        self._dev = _device()
        if mask is not None:
            m = torch.as_tensor(np.asarray(mask) if not isinstance(mask, torch.Tensor) else mask)
            self._mask = m.to(self._dev, torch.float32)
            self._maskcorr = self._corr(self._mask)
        else:
            self._mask = None
            self._maskcorr = None
        self._mean = None
        self._nvar = None
        self._n = 0
        self._norm = norm

    def _corr(self, x):
        if self._fftshape is None:
            self._fftshape = [fastlen(2 * s) for s in x.shape[-2:]]
        if _hand_ok(x.shape[-2:], x.dtype):
            return _hand_autocorr(x)
        return _crop(_autocorr(x, 2, self._fftshape), 2, list(x.shape[-2:]))

    def add(self, input, mask=None) -> None:
        if np.ndim(input) != 2:
            raise ValueError("input must be 2D.")
        x = input if isinstance(input, torch.Tensor) else torch.from_numpy(np.asarray(input))
        x = x.to(self._dev, torch.float32).clone()
        if self._norm:
            x /= x.mean()
        if mask is not None:
            m = torch.as_tensor(np.asarray(mask) if not isinstance(mask, torch.Tensor) else mask)
            m = m.to(self._dev, torch.float32)
            x *= m
            maskcorr = self._corr(m)
        elif self._mask is not None:
            x *= self._mask
            maskcorr = self._maskcorr
        elif self._maskcorr is not None:
            maskcorr = self._maskcorr
        else:
            maskcorr = self._corr(torch.ones_like(x))
            self._maskcorr = maskcorr
        if _hand_ok(x.shape, x.dtype):
            c = _hand_autocorr(x, mode=1, norm=maskcorr, threshold=0.5)
        else:
            c = _crop(_autocorr(x, 2, self._fftshape or [fastlen(2 * s) for s in x.shape]), 2, list(x.shape),
                      norm=maskcorr, mode=1, threshold=0.5)
        if self._mean is None:
            self._mean = torch.empty_like(c)
            self._nvar = torch.empty_like(c)
        self._n += 1
        nat.check(nat.load().idiwf_welford_update(ctypes.c_void_p(c.data_ptr()), ctypes.c_void_p(self._mean.data_ptr()),
                                                  ctypes.c_void_p(self._nvar.data_ptr()), c.numel(), self._n,
                                                  _stream(self._dev)))

    @property
    def mean(self) -> np.ndarray:
        return self._mean.cpu().numpy()

    @property
    def n(self) -> int:
        return self._n

    @property
    def std(self) -> np.ndarray:
        return torch.sqrt(self._nvar / self._n).cpu().numpy()
