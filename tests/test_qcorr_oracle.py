"""Direct q-space correlators on the CPU: the oracle's restatement of the
reference's kernels (``idi/reconstruction/cucorrad.py``, ``cucor.py``) against
outputs of those kernels (committed fixtures, made by running them under
numba's CUDA simulator) and against the reference's own known-answer tests
(``tests/test_recon.py:85-104``), with the host geometry of
``idi_b200.reconstruction``."""

import math
import os

import numpy as np
import pytest

import oracle
from idi_b200.reconstruction import _geometry
from tests.conftest import GOLDEN


@pytest.fixture(scope="module")
def golden():
    path = os.path.join(GOLDEN, "qcorr_ref.npz")
    return np.load(path)


def _centre(meta):
    return (None if math.isnan(meta[2]) else meta[2]), (None if math.isnan(meta[3]) else meta[3])


@pytest.mark.parametrize("name", ["rad_12x10", "rad_14x16_centre"])
def test_radial_matches_reference_kernel(golden, name):
    img = golden[f"{name}__image"]
    z, maxq = golden[f"{name}__meta"][:2]
    xc, yc = _centre(golden[f"{name}__meta"])
    qmax = int(max(15, min(511, maxq)))
    q = _geometry.q_rows(img.shape, z, xc, yc)
    out = oracle.qcorr_radial(q, img, qmax)[0]
    np.testing.assert_allclose(out, golden[f"{name}__out"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name", ["cube_16x16", "cube_10x14_centre"])
def test_3d_matches_reference_kernel(golden, name):
    img = golden[f"{name}__image"]
    z, maxq = golden[f"{name}__meta"][:2]
    xc, yc = _centre(golden[f"{name}__meta"])
    qmax = int(max(32, min(1024, maxq, *img.shape)))
    zd, maxdqz, xcf, ycf = _geometry.zd_grid(img.shape, z, xc, yc)
    out = oracle.qcorr_3d(zd, img, qmax, maxdqz, xcf, ycf, np.float32(z))[0]
    ref = golden[f"{name}__out"]
    assert out.shape == ref.shape
    np.testing.assert_allclose(out, ref, rtol=1e-6, atol=1e-6)


def test_radial_known_answer():
    """ones(32, 32), z = 100, 16 bins: 16 values, the smallest is the
    zero-offset bin, t.sum() (the reference's test_cucorrrad)."""
    t = np.ones((32, 32))
    out = oracle.qcorr_radial(_geometry.q_rows(t.shape, 100.0), t, 16)[0]
    assert len(out) == 16
    assert out.min() == t.sum()


def test_3d_known_answer():
    """ones(32, 32), z = 1000, maxq 32: (.., 64, 64), maximum t.sum() at the
    centre (the reference's test_cucor)."""
    t = np.ones((32, 32))
    zd, maxdqz, xc, yc = _geometry.zd_grid(t.shape, 1000.0)
    out = oracle.qcorr_3d(zd, t, 32, maxdqz, xc, yc, np.float32(1000.0))[0]
    assert out.shape[1:] == (64, 64) and len(out) > 1
    assert out.max() == t.sum()
    assert np.unravel_index(np.argmax(out), out.shape) == tuple(i // 2 for i in out.shape)
