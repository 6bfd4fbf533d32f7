"""Drop-in for ``idi.reconstruction.cucor``: 3d autocorrelation with q
correction on the GPU (``idi/reconstruction/cucor.py:10-128``), through
``idiwf_qcorr_3d``."""

from __future__ import annotations

import contextlib
import warnings

import numpy as np
import torch

from ..simulation import _core
from . import _geometry

__all__ = ["corrfunction"]


@contextlib.contextmanager
def corrfunction(shape, z, maxq, xcenter=None, ycenter=None):
    """3d autocorrelation with q correction.

    ``shape`` (Nr, Nc), ``z`` detector distance in pixels, ``maxq`` the half
    width in q (clamped to [32, 1024], and to the image), optional beam
    position.  Yields ``corr(image)``: float64 (2 maxdqz, 2 qmax, 2 qmax) with
    val(dqz, dqy, dqx) = sum over pixel pairs of v(p) v(p'), symmetric about
    the centre; an image stack (B, Nr, Nc) gives one such array per image.
    """
    nr, nc = int(shape[0]), int(shape[1])
    if not 32 <= maxq <= 1024:
        warnings.warn("maxq will be clamped between 32 and 1024")
    qmax = int(max(32, min(1024, maxq, nr, nc)))
    zd, maxdqz, xc, yc = _geometry.zd_grid((nr, nc), z, xcenter, ycenter)
    dev = torch.device("cuda", torch.cuda.current_device())
    state = {"zd": torch.from_numpy(zd).to(dev)}
    cz = float(np.float32(z))

    def corr(input):
        d_zd = state["zd"]
        if d_zd is None:
            raise ValueError("already closed, use within with statement")
        img = input if isinstance(input, torch.Tensor) else torch.from_numpy(np.asarray(input))
        img = img.to(dev, torch.float32).contiguous()
        if tuple(img.shape[-2:]) != (nr, nc):
            raise ValueError("input has not the shape specified in init!")
        out = _core.qcorr_3d(d_zd, img.reshape(-1, nr, nc), qmax, maxdqz, float(xc), float(yc), cz)
        out = out.reshape(img.shape[:-2] + out.shape[1:]).cpu().numpy()
        return out

    try:
        yield corr
    finally:
        state["zd"] = None
