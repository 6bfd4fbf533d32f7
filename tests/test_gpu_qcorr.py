"""Direct q-space correlators on the device (idiwf_qcorr_radial /
idiwf_qcorr_3d) against the oracle's restatement of the reference's kernels,
the reference's own outputs (fixtures) and its known-answer tests."""

import math
import os

import numpy as np
import pytest
import torch

import oracle
from idi_b200.reconstruction import _geometry, cucor, cucorrad
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "qcorr_ref.npz"))


def _centre(meta):
    return (None if math.isnan(meta[2]) else meta[2]), (None if math.isnan(meta[3]) else meta[3])


@pytest.mark.parametrize("name", ["rad_12x10", "rad_14x16_centre"])
def test_radial_reference_outputs(golden, name):
    img = golden[f"{name}__image"]
    z, maxq = golden[f"{name}__meta"][:2]
    xc, yc = _centre(golden[f"{name}__meta"])
    with cucorrad.corrfunction(img.shape, z, int(maxq), xc, yc) as f:
        out = f(img)
    np.testing.assert_allclose(out, golden[f"{name}__out"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name", ["cube_16x16", "cube_10x14_centre"])
def test_3d_reference_outputs(golden, name):
    img = golden[f"{name}__image"]
    z, maxq = golden[f"{name}__meta"][:2]
    xc, yc = _centre(golden[f"{name}__meta"])
    with cucor.corrfunction(img.shape, z, int(maxq), xc, yc) as f:
        out = f(img)
    np.testing.assert_allclose(out, golden[f"{name}__out"], rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("shape,z,maxq,centre", [((64, 48), 120.0, 40, (None, None)),
                                                 ((96, 128), 300.0, 64, (40.5, 70.0)),
                                                 ((33, 200), 80.0, 511, (None, None))])
def test_radial_vs_oracle(shape, z, maxq, centre):
    g = np.random.default_rng(sum(shape))
    imgs = g.exponential(1.0, (2,) + shape).astype(np.float32)
    with cucorrad.corrfunction(shape, z, maxq, *centre) as f:
        out = f(imgs)
    qmax = int(max(15, min(511, maxq)))
    ref = oracle.qcorr_radial(_geometry.q_rows(shape, z, *centre), imgs, qmax)
    assert out.shape == (2, qmax)
    np.testing.assert_allclose(out, ref, rtol=1e-11, atol=1e-9)


@pytest.mark.parametrize("shape,z,maxq,centre", [((48, 40), 60.0, 32, (None, None)),
                                                 ((40, 72), 150.0, 50, (15.0, 30.5))])
def test_3d_vs_oracle(shape, z, maxq, centre):
    g = np.random.default_rng(sum(shape) + 1)
    imgs = g.exponential(1.0, (2,) + shape).astype(np.float32)
    with cucor.corrfunction(shape, z, maxq, *centre) as f:
        out = f(imgs)
    qmax = int(max(32, min(1024, maxq, *shape)))
    zd, maxdqz, xc, yc = _geometry.zd_grid(shape, z, *centre)
    ref = oracle.qcorr_3d(zd, imgs, qmax, maxdqz, xc, yc, np.float32(z))
    assert out.shape == ref.shape
    np.testing.assert_allclose(out, ref, rtol=1e-11, atol=1e-9)


def test_known_answers():
    t = np.ones((32, 32))
    with cucorrad.corrfunction(t.shape, 100, 16) as f:
        c = f(t)
        assert len(c) == 16 and c.min() == t.sum()
    with cucor.corrfunction(t.shape, 1000, 32) as f:
        c = f(t)
        assert c.shape[1:] == (64, 64) and len(c) > 1
        assert c.max() == t.sum()
        assert np.unravel_index(np.argmax(c), c.shape) == tuple(i // 2 for i in c.shape)


def test_closed_and_device_output():
    t = np.ones((20, 20))
    with cucorrad.corrfunction(t.shape, 50, 16, return_gpu=True) as f:
        c = f(torch.ones((20, 20), device="cuda"))
        assert c.is_cuda and c.shape == (16,)
    with pytest.raises(ValueError):
        f(t)
    with cucor.corrfunction(t.shape, 50, 32) as g:
        with pytest.raises(ValueError):
            g(np.ones((20, 21)))
