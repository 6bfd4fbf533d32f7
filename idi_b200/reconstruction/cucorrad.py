"""Drop-in for ``idi.reconstruction.cucorrad``: radial autocorrelation with q
correction on the GPU (``idi/reconstruction/cucorrad.py:10-152``), through
``idiwf_qcorr_radial``."""

from __future__ import annotations

import contextlib
import warnings

import numpy as np
import torch

from ..simulation import _core
from . import _geometry

__all__ = ["corrfunction"]


@contextlib.contextmanager
def corrfunction(shape, z, maxq, xcenter=None, ycenter=None, return_gpu=False):
    """Radial autocorrelation with q correction.

    ``shape`` (Nr, Nc) of the images in pixels, ``z`` detector distance in
    pixels, ``maxq`` the number of radial bins (clamped to [15, 511]),
    ``xcenter`` / ``ycenter`` the beam position (default the middle).  Yields
    ``corr(image)``: float64 (maxq,) with the sum of v(p) v(p') over pixel
    pairs binned by round(|q(p) - q(p')|) (a CUDA tensor with
    ``return_gpu``); an image stack (B, Nr, Nc) gives (B, maxq).
    """
    if not 15 <= maxq <= 511:
        warnings.warn("maxq will be clamped between 15 and 511")
    qmax = int(max(15, min(511, maxq)))
    shape = (int(shape[0]), int(shape[1]))
    dev = torch.device("cuda", torch.cuda.current_device())
    state = {"q": torch.from_numpy(_geometry.q_rows(shape, z, xcenter, ycenter)).to(dev)}

    def corr(input):
        q = state["q"]
        if q is None:
            raise ValueError("already closed, use within with statement")
        img = input if isinstance(input, torch.Tensor) else torch.from_numpy(np.asarray(input))
        img = img.to(dev, torch.float32).contiguous()
        if tuple(img.shape[-2:]) != shape:
            raise ValueError("input has not the shape specified in init!")
        out = _core.qcorr_radial(q, img.reshape(-1, *shape), qmax)
        out = out.reshape(img.shape[:-2] + (qmax,))
        return out if return_gpu else out.cpu().numpy()

    try:
        yield corr
    finally:
        state["q"] = None
