"""Device photon sampling and charge sharing (idi/simulation/common.py:11-67)
through the C ABI, against the oracle (bit-exact draws from the same streams)
and against the reference's own outputs (committed fixtures)."""

import os

import numpy as np
import pytest
import torch

import oracle
from idi_b200.simulation import _core, common
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "detector_ref.npz"))


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


@pytest.mark.parametrize("name", ["photons_low", "photons_high"])
def test_photons_bit_exact_vs_oracle_on_reference_rates(golden, name):
    probs = golden[f"{name}__probs"]
    n = float(golden[f"{name}__n_photons"])
    key = (0x1234567890ABCDEF, 42)
    gpu = _core.photons(_dev(probs), n, key, 7, check=True).cpu().numpy()
    orc, rates = oracle.photons(probs, n, key, 7, return_rates=True)
    np.testing.assert_array_equal(gpu, orc)
    assert np.abs(rates - golden[f"{name}__rates"]).max() <= 4 * np.spacing(rates.max())


def test_photons_large_batch_bit_exact_and_chunk_invariant():
    g = np.random.default_rng(11)
    probs = g.gamma(0.4, 1.0, (5, 300, 257)) * g.uniform(0.2, 3.0, (5, 1, 1))
    key = (99, 2**63 + 1)
    whole = _core.photons(_dev(probs), 3.0e6, key, 3).cpu().numpy()
    np.testing.assert_array_equal(whole, oracle.photons(probs, 3.0e6, key, 3))
    parts = [_core.photons(_dev(probs[i:i + 2]), 3.0e6, key, 3, first_image=i).cpu().numpy() for i in (0, 2, 4)]
    np.testing.assert_array_equal(whole, np.concatenate(parts))
    again = _core.photons(_dev(probs), 3.0e6, key, 3).cpu().numpy()
    np.testing.assert_array_equal(whole, again)


def test_photons_quad_and_pixel_threads_vs_oracle():
    """A mean rate below 1 takes the kernel with one thread per pixel quad,
    above 1 the one with one thread per pixel; both against the oracle on
    images mixing inversion and PTRS pixels, with pixel counts that are not
    multiples of 4."""
    g = np.random.default_rng(12)
    probs = g.exponential(1.0, (3, 101, 67))
    probs[:, ::13, ::7] *= 400.0  # hot pixels: rates above 10 at either mean
    key = (5, 6)
    for n in (0.4 * probs[0].size, 30.0 * probs[0].size):
        gpu = _core.photons(_dev(probs), n, key, 2).cpu().numpy()
        orc, rates = oracle.photons(probs, n, key, 2, return_rates=True)
        assert (rates < 10).any() and (rates >= 10).any()
        np.testing.assert_array_equal(gpu, orc)


@pytest.mark.parametrize("dtype", [torch.float32, torch.int32, torch.int64] +
                         ([torch.uint32] if hasattr(torch, "uint32") else []))
def test_photons_out_dtypes(dtype):
    g = np.random.default_rng(2)
    probs = g.uniform(0, 1, (2, 64, 48))
    ref = _core.photons(_dev(probs), 5e4, (5, 6), 0).cpu().numpy()
    out = _core.photons(_dev(probs), 5e4, (5, 6), 0, dtype=dtype)
    assert out.dtype == dtype
    np.testing.assert_array_equal(out.to(torch.float64).cpu().numpy() if dtype != getattr(torch, "uint32", None)
                                  else out.cpu().numpy().astype(np.float64), ref)


def test_photons_float32_probs():
    g = np.random.default_rng(4)
    p32 = g.uniform(0, 1, (3, 40, 40)).astype(np.float32)
    gpu = _core.photons(_dev(p32), 1e4, (8, 8), 1).cpu().numpy()
    np.testing.assert_array_equal(gpu, oracle.photons(p32.astype(np.float64), 1e4, (8, 8), 1))


def test_photons_statistics():
    """Per-pixel means over 400 images against the rates, and the image totals
    against Poisson(N)."""
    g = np.random.default_rng(5)
    base = g.uniform(0.05, 1.0, (1, 32, 32))
    probs = np.repeat(base, 400, 0)
    n = 2000.0
    c = _core.photons(_dev(probs), n, (2024, 1), 0).cpu().numpy()
    lam = base[0] * (n / base.sum())
    z = (c.mean(0) - lam) / np.sqrt(lam / c.shape[0])
    assert abs(z.mean()) < 0.2 and 0.8 < z.std() < 1.2
    tot = c.sum((1, 2))
    assert abs(tot.mean() - n) < 5 * np.sqrt(n / tot.size)
    assert 0.8 < tot.var() / n < 1.25


def test_randomphotons_mirror_numpy_and_torch():
    g = np.random.default_rng(6)
    probs = g.uniform(0, 1, (2, 30, 20))
    out = common.randomphotons(probs, 1000, rng=17)
    assert isinstance(out, np.ndarray) and out.dtype == np.float64 and out.shape == probs.shape
    np.testing.assert_array_equal(out, oracle.photons(probs, 1000, (17, 0), 0))
    u = common.randomphotons(probs, 1000, rng=17, dtype=np.uint32)
    assert u.dtype == np.uint32
    np.testing.assert_array_equal(u.astype(np.float64), out)
    t = common.randomphotons(_dev(probs), 1000, rng=17)
    assert t.is_cuda
    np.testing.assert_array_equal(t.cpu().numpy(), out)
    r = common.DeviceRNG(3)
    a = common.randomphotons(probs, 1000, rng=r)
    b = common.randomphotons(probs, 1000, rng=r)
    assert not np.array_equal(a, b)


def test_randomphotons_invalid_inputs_raise():
    p = np.ones((8, 8))
    p[2, 3] = -1.0
    with pytest.raises(ValueError):
        common.randomphotons(p, 100, rng=1)
    with pytest.raises(ValueError):
        common.randomphotons(np.zeros((2, 8, 8)), 100, rng=1)
    q = np.ones((8, 8))
    q[0, 0] = np.nan
    with pytest.raises(ValueError):
        common.randomphotons(q, 100, rng=1)
    # the context is still usable afterwards
    ok = common.randomphotons(np.ones((8, 8)), 100, rng=1)
    assert ok.sum() > 0


@pytest.mark.parametrize("name", ["cs_w2", "cs_w1_noise", "cs_w3_edges"])
def test_chargesharing_injected_matches_reference(golden, name):
    s, ns = golden[f"{name}__meta"]
    counts = golden[f"{name}__counts"]
    out = common.chargesharing(counts, s, ns, positions=golden[f"{name}__positions"],
                               scales=golden[f"{name}__scales"])
    np.testing.assert_allclose(out, golden[f"{name}__out"], rtol=1e-13, atol=1e-15)


def test_chargesharing_noshare_matches_reference(golden):
    name = "cs_noshare_noise"
    s, ns = golden[f"{name}__meta"]
    out = common.chargesharing(golden[f"{name}__counts"], s, ns, scales=golden[f"{name}__scales"])
    np.testing.assert_array_equal(out, golden[f"{name}__out"])


@pytest.mark.parametrize("s,ns", [(0.45, 0.0), (0.9, 0.15), (1.6, 0.0)])
def test_chargesharing_generated_vs_oracle(s, ns):
    g = np.random.default_rng(int(s * 100))
    counts = g.poisson(0.6, (3, 41, 37)).astype(np.int32)
    counts[1, 0, :] += 1  # edge photons
    key = (77, 88)
    gpu = _core.chargesharing(_dev(counts), s, ns, key, 5, check=True).cpu().numpy()
    orc = oracle.chargesharing(counts, s, ns, key=key, stream=5)
    np.testing.assert_allclose(gpu, orc, rtol=1e-12, atol=1e-14)
    parts = np.concatenate([_core.chargesharing(_dev(counts[i:i + 1]), s, ns, key, 5, first_image=i).cpu().numpy()
                            for i in range(3)])
    np.testing.assert_array_equal(parts, gpu)


def test_chargesharing_count_types_and_empty():
    g = np.random.default_rng(9)
    c = g.poisson(0.8, (17, 19))
    pos = g.uniform(-0.5, 0.5, (int(c.sum()), 2))
    ref = oracle.chargesharing(c, 0.7, 0.0, positions=pos)
    for dt in (np.int64, np.int32, np.float64, np.float32):
        out = common.chargesharing(c.astype(dt), 0.7, 0, positions=pos)
        np.testing.assert_allclose(out, ref, rtol=1e-13, atol=1e-15)
    fr = c.astype(np.float64) + 0.7  # astype(int) truncation of fractional counts
    np.testing.assert_allclose(common.chargesharing(fr, 0.7, 0, positions=pos), ref, rtol=1e-13, atol=1e-15)
    z = common.chargesharing(np.zeros((6, 5), np.int64), 0.7, 0, rng=1)
    assert not z.any()


def test_chargesharing_position_count_mismatch_raises():
    c = np.ones((4, 4), np.int64)
    with pytest.raises(ValueError):
        common.chargesharing(c, 0.5, 0, positions=np.zeros((15, 2)))
    with pytest.raises(ValueError):
        common.chargesharing(-c, 0.5, 0, rng=3)
    ok = common.chargesharing(c, 0.5, 0, positions=np.zeros((16, 2)))
    assert ok.sum() > 0


def test_simulate_photons_pipeline_matches_two_step():
    """simulate_photons == randomphotons(|simulate|^2) on the same streams, for
    host output (chunked, pipelined) and device output."""
    from idi_b200.simulation import cuda as sim
    from tests.helpers import rng, sphere
    from idi_b200.simulation.simobj import fixed

    g = rng(31)
    n, nimg = 300, 9
    pos = sphere(g, n, 0.01)
    phases = g.uniform(0, 2 * np.pi, (nimg, n))
    mk = lambda: fixed(6400.0, pos, phases)  # noqa: E731
    E = sim.simulate(nimg, mk(), 48, 75.0, 1e5, settings="double", verbose=False)
    I = np.abs(E) ** 2
    want = oracle.photons(I, 5e3, (123, 0), 0)
    got = sim.simulate_photons(nimg, mk(), 48, 75.0, 1e5, 5e3, settings="double", verbose=False, rng=123)
    assert got.dtype == np.uint32 and got.shape == (nimg, 48, 48)
    # |E|^2 of the device (re^2 + im^2) and numpy's |E|**2 may differ in the
    # last ulp, which can move a draw across a boundary: allow a few pixels
    assert (got.astype(np.float64) != want).mean() < 1e-3
    gpu = sim.simulate_photons(nimg, mk(), 48, 75.0, 1e5, 5e3, settings="double", returngpu=True, rng=123,
                               dtype=np.float64)
    np.testing.assert_array_equal(gpu.cpu().numpy(), got.astype(np.float64))
    cs = sim.simulate_photons(nimg, mk(), 48, 75.0, 1e5, 5e3, settings="double", verbose=False, rng=123,
                              chargesharing=(0.5, 0.0))
    ref_cs = oracle.chargesharing(got.astype(np.int64), 0.5, 0.0, key=(123, 0), stream=0)
    np.testing.assert_allclose(cs, ref_cs, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("s,mean,ns", [(2.6, 0.4, 0.0), (0.5, 40.0, 0.0), (0.5, 40.0, 0.1)])
def test_chargesharing_wide_and_crowded_vs_oracle(s, mean, ns):
    """w = ceil(2 s) above the tiled kernel's 4, and images so crowded that a
    tile's region holds more photons than its shared memory: both take the
    per-pixel gather, which must agree with the tiled one's order and sums."""
    g = np.random.default_rng(int(s * 10 + mean))
    counts = g.poisson(mean, (2, 37, 45)).astype(np.int64)
    key = (12, 34)
    gpu = _core.chargesharing(_dev(counts), s, ns, key, 3, check=True).cpu().numpy()
    orc = oracle.chargesharing(counts, s, ns, key=key, stream=3)
    np.testing.assert_allclose(gpu, orc, rtol=1e-12, atol=1e-12)
