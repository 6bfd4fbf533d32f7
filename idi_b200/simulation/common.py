"""Drop-in for ``idi.simulation.common``: ``randomphotons`` and ``chargesharing``
on the GPU (``idi/simulation/common.py:11-67``).

Both accept numpy arrays (the reference's host path; the result comes back as
numpy) or CUDA tensors (the reference's cupy path; the result stays on the
device).  The draws come from the library's counter-based Philox4x64-10
streams instead of numpy's / numba's generators, so the numbers differ from
the reference's while the distributions are the same; the rates, the
reduction and the charge-sharing arithmetic follow the reference.  Charge
sharing also takes the reference's own draws (``positions``, ``scales``) and
then reproduces its output.

``rng``: None (a fresh seed from ``np.random.randint``, as the reference),
an int seed, a ``numpy.random.Generator`` (one 63-bit key is drawn from it,
as the reference's cupy branch does), or a :class:`DeviceRNG` (advances one
stream per call, reproducible across calls).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _core

__all__ = ["randomphotons", "chargesharing", "DeviceRNG"]


class DeviceRNG:
    """Key and stream counter for the device samplers.  Each call that draws
    takes the next stream, so a sequence of calls is reproducible from the seed."""

    def __init__(self, seed=None):
        if seed is None:
            seed = np.random.randint(2**63)
        self.key = tuple(int(x) for x in np.random.SeedSequence(int(seed)).generate_state(2, np.uint64))
        self.stream = 0

    def take(self):
        s = self.stream
        self.stream += 1
        return self.key, s


def _key_stream(rng):
    if isinstance(rng, DeviceRNG):
        return rng.take()
    if rng is None:
        return (int(np.random.randint(2**63)), 0), 0
    if isinstance(rng, np.random.Generator):
        # the reference's integers(high=2**63), [0, 2**63), in the form numpy 2 accepts
        return (int(rng.integers(2**63)), 0), 0
    if isinstance(rng, (int, np.integer)):
        return (int(rng), 0), 0
    raise TypeError("rng must be None, an int seed, a numpy Generator or a DeviceRNG")


_TORCH_COUNT = {
    np.dtype(np.float64): torch.float64,
    np.dtype(np.float32): torch.float32,
    np.dtype(np.int32): torch.int32,
    np.dtype(np.int64): torch.int64,
}
if hasattr(torch, "uint32"):
    _TORCH_COUNT[np.dtype(np.uint32)] = torch.uint32


def _count_dtype(dtype):
    """(device dtype, final numpy dtype or None) for the reference's ``dtype``."""
    if isinstance(dtype, torch.dtype):
        return dtype, None
    nd = np.dtype(dtype)
    return _TORCH_COUNT.get(nd, torch.float64), nd


def _device():
    return torch.device("cuda", torch.cuda.current_device())


def randomphotons(probs, Nphotons, rng=None, dtype=float):
    """Poisson photon counts with ``Nphotons`` expected photons per image
    (sum over the last two axes), ``idi/simulation/common.py:11-23``.

    Infinite ``Nphotons`` returns ``probs`` unchanged.  A negative or NaN
    probability, or an image that sums to zero, raises ValueError (numpy's
    ``poisson`` does the same).  Inputs other than numpy arrays and torch
    tensors return None, as in the reference.
    """
    if not np.isfinite(Nphotons):
        return probs
    if isinstance(probs, torch.Tensor):
        tdt, _ = _count_dtype(dtype)
        key, stream = _key_stream(rng)
        p = probs if probs.is_cuda else probs.to(_device())
        if p.dtype not in (torch.float64, torch.float32):
            p = p.to(torch.float64)
        out = _core.photons(p.contiguous(), Nphotons, key, stream, dtype=tdt, check=True)
        return out if probs.is_cuda else out.cpu()
    if isinstance(probs, np.ndarray):
        tdt, nd = _count_dtype(dtype)
        key, stream = _key_stream(rng)
        a = probs if probs.dtype in (np.float64, np.float32) else probs.astype(np.float64)
        d = torch.from_numpy(np.ascontiguousarray(a)).to(_device())
        out = _core.photons(d, Nphotons, key, stream, dtype=tdt, check=True).cpu().numpy()
        return out if nd is None or out.dtype == nd else out.astype(nd)
    return None


def chargesharing(img, s, ns=0, rng=None, positions=None, scales=None):
    """Charge sharing between neighbouring pixels, ``idi/simulation/common.py:26-67``.

    Every count in ``img`` (..., nx, ny) becomes a photon at a uniform position
    inside its pixel whose charge spreads as a Gaussian of width ``s`` pixels
    over the pixels within ``ceil(2 s)``; charge leaving the detector is lost;
    ``ns > 0`` scales each photon's charge by ``1 + ns N(0,1)``.  For
    ``s <= 0`` the result is ``img`` (``ns == 0``) or ``img * (1 + ns N(0,1))``.
    ``positions`` ((photons, 2) offsets in [-0.5, 0.5)) and ``scales`` inject
    the draws, in the reference's photon order; the result is float64.
    """
    if not s > 0 and ns == 0:
        return img
    is_torch = isinstance(img, torch.Tensor)
    if is_torch:
        d = img if img.is_cuda else img.to(_device())
    else:
        a = np.asarray(img)
        if a.dtype not in (np.float64, np.float32, np.int32, np.int64, np.uint32):
            a = a.astype(np.int64) if np.issubdtype(a.dtype, np.integer) else a.astype(np.float64)
        d = torch.from_numpy(np.ascontiguousarray(a)).to(_device())
    if d.dtype not in _core._ELEM_CODE:
        d = d.to(torch.float64)
    dev = d.device

    def _dev64(x):
        if x is None:
            return None
        t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64))
        return t.to(dev, torch.float64).contiguous()

    pos = _dev64(positions)
    sc = _dev64(scales)
    if pos is not None:
        pos = pos.reshape(-1, 2)
    if sc is not None:
        sc = sc.reshape(-1)
    key, stream = ((0, 0), 0) if (pos is not None or (not s > 0 and sc is not None)) else _key_stream(rng)
    out = _core.chargesharing(d.contiguous(), float(s), float(ns), key, stream, positions=pos, scales=sc, check=True)
    if is_torch:
        return out if img.is_cuda else out.cpu()
    return out.cpu().numpy()
