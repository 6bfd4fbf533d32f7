"""FFT autocorrelation on the device (cuFFT transforms, this library's power
spectrum / crop / running-statistics kernels) against the reference's numpy
twin ``idi/reconstruction/cpusimple.py`` (fixtures) and the reference's own
checks against scipy (``tests/test_recon.py:106-121``)."""

import os

import numpy as np
import pytest
import torch

from idi_b200.reconstruction import cusimple
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "fftcorr_ref.npz"))


def test_corr_known_answers():
    import scipy.signal as ss

    t = np.arange(32 * 16).reshape(32, 16).astype(float)
    c = cusimple.corr(t)
    np.testing.assert_allclose(c[1:, 1:], ss.correlate(t, t, "full", "fft"), atol=1e-7)
    t = np.arange(15 * 33).reshape(15, 33).astype(float)
    c = cusimple.corr(t, norm=True)
    gc = ss.correlate(t / t.mean(), t / t.mean(), "full", "fft")
    gn = ss.correlate(np.ones_like(t), np.ones_like(t), "full", "fft")
    g = gc / gn
    g[gn < 0.9] = np.nan
    np.testing.assert_allclose(c[1:, 1:], g, atol=1e-7)


@pytest.mark.parametrize("name,kw", [("corr_arange", {}), ("corr_arange_norm", {"norm": True})])
def test_corr_reference(golden, name, kw):
    out = cusimple.corr(golden[f"{name}__in"], **kw)
    ref = golden[f"{name}__out"]
    np.testing.assert_allclose(out, ref, rtol=1e-10, atol=1e-9 * np.nanmax(np.abs(ref)))


def test_corr_stack_and_line(golden):
    st = golden["corr_stack__in"]
    for key, kw in (("corr_stack__out", {}), ("corr_stack_norm__out", {"norm": True})):
        ref = golden[key]
        np.testing.assert_allclose(cusimple.corr(st, **kw), ref, rtol=1e-10, atol=1e-10 * np.nanmax(np.abs(ref)))
    ref = golden["corr_line__out"]
    np.testing.assert_allclose(cusimple.corr(golden["corr_line__in"], axes=(-1,)), ref, rtol=1e-10,
                               atol=1e-10 * np.abs(ref).max())
    g = cusimple.corr(torch.from_numpy(st).cuda(), returngpu=True)
    assert g.is_cuda and g.shape == (3, 40, 48)


@pytest.mark.parametrize("name", ["plain", "mask", "addmask"])
def test_correlator2d_reference(golden, name):
    imgs, mask = golden["c2d__images"], golden["c2d__mask"]
    c = cusimple.correlator2d(mask=mask) if name == "mask" else cusimple.correlator2d()
    for im in imgs:
        if name == "addmask":
            c.add(im, mask=mask)
        else:
            c.add(im)
    assert c.n == len(imgs)
    for attr in ("mean", "std"):
        ref = golden[f"c2d_{name}__{attr}"]
        np.testing.assert_allclose(getattr(c, attr), ref, rtol=2e-4, atol=2e-4 * np.abs(ref).max())


def test_corr_pow2_reference(golden):
    """Power-of-two shapes: this library's own FFTs (idiwf_fft_autocorr)."""
    st = golden["corr_pow2__in"]
    for key, kw in (("corr_pow2__out", {}), ("corr_pow2_norm__out", {"norm": True})):
        ref = golden[key]
        out = cusimple.corr(st, **kw)
        assert out.shape == ref.shape
        np.testing.assert_array_equal(np.isnan(out), np.isnan(ref))
        np.testing.assert_allclose(out, ref, rtol=1e-10, atol=1e-10 * np.nanmax(np.abs(ref)))


@pytest.mark.parametrize("name", ["plain", "mask", "addmask"])
def test_correlator2d_pow2_reference(golden, name):
    imgs, mask = golden["c2dp__images"], golden["c2dp__mask"]
    c = cusimple.correlator2d(mask=mask) if name == "mask" else cusimple.correlator2d()
    for im in imgs:
        if name == "addmask":
            c.add(im, mask=mask)
        else:
            c.add(im)
    for attr in ("mean", "std"):
        ref = golden[f"c2dp_{name}__{attr}"]
        np.testing.assert_allclose(getattr(c, attr), ref, rtol=2e-4, atol=2e-4 * np.abs(ref).max())


def _pair_count(n0, n1, dtype):
    i = torch.arange(2 * n0, dtype=torch.float64)
    j = torch.arange(2 * n1, dtype=torch.float64)
    c = (n0 - (i - n0).abs())[:, None] * (n1 - (j - n1).abs())[None, :]
    return c.to(dtype).cuda()


@pytest.mark.parametrize("shape,dtype", [((4, 4), torch.float64), ((8, 64), torch.float64),
                                         ((256, 128), torch.float64), ((1024, 1024), torch.float64),
                                         ((2048, 16), torch.float64), ((64, 32), torch.float32),
                                         ((512, 512), torch.float32)])
def test_hand_fft_vs_cufft(shape, dtype):
    """The hand-written FFT autocorrelation against cuFFT's transforms with the
    same crop, on a batch of 3, plain and divided by the pair count."""
    g = torch.Generator(device="cuda").manual_seed(sum(shape))
    x = torch.empty((3,) + shape, dtype=dtype, device="cuda").exponential_(1.0, generator=g)
    tol = 1e-12 if dtype == torch.float64 else 2e-5
    ref = cusimple._crop(cusimple._autocorr(x, 2, [2 * s for s in shape]), 2, list(shape))
    hand = cusimple._hand_autocorr(x)
    assert hand.shape == ref.shape
    assert (hand - ref).abs().max().item() <= tol * ref.abs().max().item()
    count = _pair_count(*shape, dtype)
    hn = cusimple._hand_autocorr(x, mode=2, threshold=0.9)
    rn = torch.where(count < 0.9, torch.full_like(ref, float("nan")), ref / count)
    assert torch.equal(torch.isnan(hn), torch.isnan(rn))
    ok = ~torch.isnan(rn)
    assert ((hn - rn).abs() * count)[ok].max().item() <= 2 * tol * ref.abs().max().item()


def test_other_shapes_take_cufft():
    # fastlen(6000) = 6000 is above the hand-written FFTs' 4096; cuFFT takes it
    assert not cusimple._hand_ok((12, 3000), torch.float64)
    x = torch.ones((12, 3000), dtype=torch.float64, device="cuda")
    c = cusimple.corr(x, returngpu=True)
    assert c.shape == (24, 6000)


@pytest.mark.parametrize("shape,dtype", [((15, 33), torch.float64), ((13, 10), torch.float64),
                                         ((1, 30), torch.float64), ((3, 5), torch.float64),
                                         ((2, 9), torch.float64), ((7, 50), torch.float64),
                                         ((40, 12), torch.float64), ((100, 75), torch.float64),
                                         ((300, 500), torch.float64), ((1000, 1050), torch.float64),
                                         ((1500, 7), torch.float64), ((6, 2000), torch.float64),
                                         ((100, 75), torch.float32), ((300, 500), torch.float32),
                                         ((4, 1), torch.float64), ((1, 1), torch.float64), ((2, 2), torch.float64),
                                         ((5, 1), torch.float32), ((1, 3), torch.float64)])
def test_hand_fft_general_vs_cufft(shape, dtype):
    """Other lengths: mixed-radix passes (2, 3, 4, 5, 7, 8, 11) on the padded
    lengths fastlen(2 n), cropped, against cuFFT's transforms with the same
    crop; plain and divided by the pair count."""
    fs = [cusimple.fastlen(2 * s) for s in shape]
    assert cusimple._hand_ok(shape, dtype) and fs[1] % 2 == 0
    g = torch.Generator(device="cuda").manual_seed(sum(shape) + 7)
    x = torch.empty((3,) + shape, dtype=dtype, device="cuda").exponential_(1.0, generator=g)
    tol = 1e-12 if dtype == torch.float64 else 2e-5
    ref = cusimple._crop(cusimple._autocorr(x, 2, fs), 2, list(shape))
    hand = cusimple._hand_autocorr(x)
    assert hand.shape == ref.shape
    assert (hand - ref).abs().max().item() <= tol * ref.abs().max().item()
    count = _pair_count(*shape, dtype)
    hn = cusimple._hand_autocorr(x, mode=2, threshold=0.9)
    rn = torch.where(count < 0.9, torch.full_like(ref, float("nan")), ref / count)
    assert torch.equal(torch.isnan(hn), torch.isnan(rn))
    ok = ~torch.isnan(rn)
    assert ((hn - rn).abs() * count)[ok].max().item() <= 2 * tol * ref.abs().max().item()


@pytest.mark.parametrize("lead,n", [((5, 2), 4), ((5, 2), 30), ((5, 2), 1000), ((5, 2), 1024), ((5, 2), 1500),
                                    ((2500,), 100), ((1030,), 7), ((3,), 1), ((3,), 2), ((4,), 3)])
def test_hand_fft_1d_vs_cufft(lead, n):
    """One correlated axis (idiwf_fft_autocorr_1d; more than 1024 lines run as
    several images plus a remainder) against cuFFT's 1D transforms."""
    g = torch.Generator(device="cuda").manual_seed(n)
    x = torch.empty(lead + (n,), dtype=torch.float64, device="cuda").exponential_(1.0, generator=g)
    ref = cusimple._crop(cusimple._autocorr(x, 1, [cusimple.fastlen(2 * n)]), 1, [n])
    hand = cusimple._hand_autocorr_1d(x)
    assert hand.shape == ref.shape == lead + (2 * n,)
    assert (hand - ref).abs().max().item() <= 1e-12 * ref.abs().max().item()
    j = torch.arange(2 * n, dtype=torch.float64, device="cuda")
    count = n - (j - n).abs()
    hn = cusimple._hand_autocorr_1d(x, mode=2, threshold=0.9)
    rn = torch.where(count < 0.9, torch.full_like(ref, float("nan")), ref / count)
    assert torch.equal(torch.isnan(hn), torch.isnan(rn))
    ok = ~torch.isnan(rn)
    assert ((hn - rn).abs() * count)[ok].max().item() <= 2e-12 * ref.abs().max().item()


@pytest.mark.parametrize("shape,dtype", [((5, 13), torch.float64), ((9, 17), torch.float64),
                                         ((12, 31), torch.float64), ((4, 38), torch.float64),
                                         ((7, 61), torch.float64), ((300, 301), torch.float64),
                                         ((1000, 344), torch.float64), ((64, 337), torch.float32)])
def test_hand_fft_odd_width_vs_cufft(shape, dtype):
    """An odd last padded length fastlen(2 n1): the reference's inverse has
    one value fewer, which is never a product of 2, 3, 5, 7, 11 -- the
    inverse by Bluestein's algorithm -- and norm=True divides by the same
    transform of ones.  Against cuFFT's transforms with the same lengths."""
    fs = [cusimple.fastlen(2 * s) for s in shape]
    assert fs[1] % 2 == 1 and cusimple._hand_ok(shape, dtype)
    g = torch.Generator(device="cuda").manual_seed(sum(shape) + 11)
    x = torch.empty((3,) + shape, dtype=dtype, device="cuda").exponential_(1.0, generator=g)
    tol = 1e-12 if dtype == torch.float64 else 2e-5
    ref = cusimple._crop(cusimple._autocorr(x, 2, fs), 2, list(shape))
    hand = cusimple._hand_autocorr(x)
    assert hand.shape == ref.shape
    assert (hand - ref).abs().max().item() <= tol * ref.abs().max().item()
    ones = torch.ones(shape, dtype=dtype, device="cuda")
    pairs = cusimple._crop(cusimple._autocorr(ones, 2, fs), 2, list(shape))
    rn = cusimple._crop(cusimple._autocorr(x, 2, fs), 2, list(shape), norm=pairs, mode=0, threshold=0.9)
    hn = cusimple.corr(x, axes=(1, 2), returngpu=True, norm=False)
    assert torch.equal(hn, cusimple._hand_autocorr(x))
    # corr(norm=True) divides by the mean first; compare on the same input
    xm = x * (1 / x.mean(dim=0, keepdim=True))
    hn = cusimple.corr(x, axes=(1, 2), norm=True, returngpu=True)
    rn = cusimple._crop(cusimple._autocorr(xm, 2, fs), 2, list(shape), norm=pairs, mode=0, threshold=0.9)
    assert torch.equal(torch.isnan(hn), torch.isnan(rn))
    ok = ~torch.isnan(rn)
    assert ((hn - rn).abs() * pairs)[ok].max().item() <= 4 * tol * (rn.abs() * pairs)[ok].max().item()


@pytest.mark.parametrize("n", [13, 38, 301])
def test_hand_fft_1d_odd_vs_cufft(n):
    """One axis with an odd padded length, plain and divided by the
    transform of ones."""
    G = cusimple.fastlen(2 * n)
    assert G % 2 == 1
    g = torch.Generator(device="cuda").manual_seed(n)
    x = torch.empty((7, n), dtype=torch.float64, device="cuda").exponential_(1.0, generator=g)
    ref = cusimple._crop(cusimple._autocorr(x, 1, [G]), 1, [n])
    hand = cusimple._hand_autocorr_1d(x)
    assert (hand - ref).abs().max().item() <= 1e-12 * ref.abs().max().item()
    ones = torch.ones((n,), dtype=torch.float64, device="cuda")
    pairs = cusimple._crop(cusimple._autocorr(ones, 1, [G]), 1, [n])
    hn = cusimple._hand_autocorr_1d(x, mode=0, norm=pairs, threshold=0.9)
    rn = torch.where(pairs < 0.9, torch.full_like(ref, float("nan")), ref / pairs)
    assert torch.equal(torch.isnan(hn), torch.isnan(rn))
    ok = ~torch.isnan(rn)
    assert ((hn - rn).abs() * pairs)[ok].max().item() <= 2e-12 * ref.abs().max().item()
