"""Detector geometry of the q-space correlators, with the reference's
conventions (``idi/reconstruction/cucorrad.py:30-38``, ``cucor.py:36-47``):
pixel (r, c) at (r - xcenter, c - ycenter, z) in pixel units, the centre
rounded to float32 (defaults Nr/2, Nc/2, also for a centre of 0), FP64
distances, float32 results.  Kept arithmetic for arithmetic so the bins of
every pair are the reference's."""

from __future__ import annotations

import math

import numpy as np


def centre(shape, xcenter, ycenter):
    return np.float32(xcenter or shape[0] / 2), np.float32(ycenter or shape[1] / 2)


def _offsets(shape, xc, yc, z):
    x = np.arange(shape[0], dtype=np.float64)[:, None] - xc
    y = np.arange(shape[1], dtype=np.float64)[None, :] - yc
    d = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    return x, y, d


def q_rows(shape, z, xcenter=None, ycenter=None) -> np.ndarray:
    """(nr * nc, 4) float32 rows [qx, qy, qz, 0] with q = k z / d."""
    xc, yc = centre(shape, xcenter, ycenter)
    x, y, d = _offsets(shape, xc, yc, z)
    out = np.zeros((shape[0] * shape[1], 4), np.float32)
    for i, k in enumerate((x, y, z)):
        out[:, i] = np.broadcast_to((k * z / d).astype(np.float32), d.shape).ravel()
    return out


def zd_grid(shape, z, xcenter=None, ycenter=None):
    """(zd (nr, nc) float32 = z / d, maxdqz, xcenter, ycenter) of the 3d correlator."""
    xc, yc = centre(shape, xcenter, ycenter)
    _, _, d = _offsets(shape, xc, yc, z)
    zd = np.array(z / d, np.float32)
    maxdqz = int(math.ceil(z * (np.max(zd) - np.min(zd)))) | 1
    return zd, maxdqz, xc, yc
