"""Detector stage (photon sampling, charge sharing) on the CPU: the oracle's
random streams against numpy's Philox, the oracle against the reference's own
``idi/simulation/common.py`` (committed fixtures, and live where the reference
tree is present), the sampler's distribution, and the host-side behaviour of
the ``idi_b200.simulation.common`` mirror that needs no GPU."""

import os

import numpy as np
import pytest
from scipy import stats

import oracle
from tests.conftest import GOLDEN


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "detector_ref.npz"))


@pytest.mark.parametrize("counter,key", [([0, 5, 7, 9], [123, 456]), ([41, 2**40, 3, 2**63 + 5], [2**64 - 1, 7])])
def test_philox_matches_numpy(counter, key):
    raw = np.random.Philox(counter=np.array(counter, np.uint64), key=np.array(key, np.uint64)).random_raw(12)
    for j in range(3):
        c = list(counter)
        c[0] += j + 1
        np.testing.assert_array_equal(oracle.philox4x64(c, key), raw[4 * j:4 * j + 4])


def test_uniform_stream_matches_numpy_generator():
    key = (2**62 + 3, 99)
    for c1, c2, c3 in [(0, 0, 0), (12345, 7, 2), (2**40, 2**63 | 3, 11)]:
        u = oracle.uniforms(c1, c2, c3, key, 21)
        bg = np.random.Philox(counter=np.array([0, c1, c2, c3], np.uint64), key=np.array(key, np.uint64))
        g = np.random.Generator(bg).random(21)
        np.testing.assert_array_equal(u, g)


@pytest.mark.parametrize("name", ["photons_low", "photons_high"])
def test_rates_match_reference(golden, name):
    """rate = p * (N / sum p), against the rates the reference's randomphotons
    passed to its generator (within 4 ulps: the sums are reduced in different
    orders)."""
    probs = golden[f"{name}__probs"]
    ref = golden[f"{name}__rates"]
    _, rates = oracle.photons(probs, float(golden[f"{name}__n_photons"]), (1, 2), 0, return_rates=True)
    ulps = np.abs(rates - ref) / np.spacing(np.abs(ref))
    assert ulps.max() <= 4


def test_image_sum_close_to_numpy():
    g = np.random.default_rng(3)
    for n in (1, 7, 2048, 2049, 300000):
        x = g.gamma(0.3, 1.0, n)
        assert abs(oracle.image_sum(x) - x.sum()) <= 1e-14 * x.sum()


@pytest.mark.parametrize("lam", [0.03, 0.7, 4.0, 9.99, 10.0, 37.0, 1500.0])
def test_poisson_sampler_distribution(lam):
    """Chi-square of 40k draws at one rate against the Poisson pmf."""
    p = np.ones((1, 200, 200))
    c = oracle.photons(p, lam * p.size, (int(lam * 1000) + 17, 5), 3).ravel()
    ks = np.arange(int(max(0, lam - 7 * np.sqrt(lam) - 2)), int(lam + 7 * np.sqrt(lam) + 4))
    expect = stats.poisson.pmf(ks, lam) * c.size
    obs = np.array([(c == k).sum() for k in ks])
    keep = expect >= 10
    e = np.concatenate([expect[keep], [c.size - expect[keep].sum()]])
    o = np.concatenate([obs[keep], [c.size - obs[keep].sum()]])
    chi = ((o - e) ** 2 / np.maximum(e, 1e-12)).sum()
    assert stats.chi2.sf(chi, len(e) - 1) > 1e-4
    assert abs(c.mean() - lam) < 5 * np.sqrt(lam / c.size)


def test_quad_block_uniforms_match_numpy_philox():
    """Below rate 10 pixel p inverts word p % 4 of the Philox4x64-10 block with
    counter (2^63, p / 4, image, stream): numpy's generator, started one block
    earlier, gives that block as its first raw output."""
    key, stream = (0xDEADBEEF12345678, 77), 5
    npix, lam = 32, 3.0
    probs = np.ones((2, 4, 8))                  # two images of 32 pixels; rate exactly n / npix
    got = oracle.photons(probs, lam * npix, key, stream).reshape(2, npix)
    assert len(np.unique(got)) >= 4
    for b in range(2):
        for p in range(npix):
            ctr = np.array([2**63 - 1, p // 4, b, stream], np.uint64)
            w = np.random.Philox(counter=ctr, key=np.array(key, np.uint64)).random_raw(4)[p % 4]
            u = float(int(w) >> 11) * 2.0**-53
            k, term = 0, np.exp(-lam)
            F = term
            while u > F:
                k += 1
                term = term * lam / k
                F += term
            assert got[b, p] == k, (b, p)


def test_photons_first_image_offsets_the_stream():
    g = np.random.default_rng(1)
    p = g.uniform(0.1, 1.0, (4, 9, 7))
    whole = oracle.photons(p, 500.0, (9, 9), 4)
    parts = np.concatenate([oracle.photons(p[:1], 500.0, (9, 9), 4),
                            oracle.photons(p[1:], 500.0, (9, 9), 4, first_image=1)])
    np.testing.assert_array_equal(whole, parts)


@pytest.mark.parametrize("name", ["cs_w2", "cs_w1_noise", "cs_w3_edges"])
def test_chargesharing_matches_reference(golden, name):
    s, ns = golden[f"{name}__meta"]
    out = oracle.chargesharing(golden[f"{name}__counts"], s, ns, positions=golden[f"{name}__positions"],
                               scales=golden[f"{name}__scales"])
    ref = golden[f"{name}__out"]
    np.testing.assert_allclose(out, ref, rtol=1e-13, atol=1e-15)


def test_chargesharing_noshare_fixture(golden):
    name = "cs_noshare_noise"
    np.testing.assert_array_equal(golden[f"{name}__counts"] * golden[f"{name}__scales"], golden[f"{name}__out"])


def test_chargesharing_conserves_charge_inside():
    """Far from the edges a photon deposits its charge up to the Gaussian tail
    beyond w = ceil(2 s) pixels, which the reference's kernel leaves out."""
    c = np.zeros((1, 15, 15), np.int64)
    c[0, 7, 7] = 5
    out = oracle.chargesharing(c, 0.4, 0.0, key=(3, 4), stream=1)
    assert 0.99 * 5 < out.sum() <= 5
    assert out[0, 7, 7] == out.max()
    one = np.zeros((1, 15, 15), np.int64)
    one[0, 7, 7] = 1
    centred = oracle.chargesharing(one, 0.1, 0.0, positions=np.zeros((1, 2)))
    assert abs(centred.sum() - 1) < 1e-12


def test_chargesharing_live_reference(reference):
    """The oracle against the reference's chargesharing run here, with its
    numba draws read back after seeding (as the fixture generator does)."""
    import numba

    @numba.njit
    def nb_seed(seed):
        np.random.seed(seed)

    @numba.njit
    def nb_draws(n):
        return np.random.rand(n, 2) - 0.5

    img = np.random.default_rng(8).poisson(1.1, (11, 13))
    nb_seed(77)
    ref = reference.common.chargesharing(img, 0.8, 0)
    nb_seed(77)
    mu = nb_draws(int(img.sum()))
    np.testing.assert_allclose(oracle.chargesharing(img, 0.8, 0.0, positions=mu), ref, rtol=1e-13, atol=1e-15)


# ---------------------------------------------------------------------------
# host behaviour of the mirror (no device work)
# ---------------------------------------------------------------------------
def test_mirror_passthrough_cases():
    from idi_b200.simulation import common

    p = np.ones((4, 4))
    assert common.randomphotons(p, np.inf) is p
    assert common.randomphotons([1, 2], 10) is None
    img = np.ones((3, 3))
    assert common.chargesharing(img, 0, 0) is img
    assert common.chargesharing(img, -1.0, 0) is img


def test_device_rng_streams_advance():
    from idi_b200.simulation import common

    r = common.DeviceRNG(5)
    k1, s1 = r.take()
    k2, s2 = r.take()
    assert k1 == k2 and (s1, s2) == (0, 1)
    assert common.DeviceRNG(5).key == k1 and common.DeviceRNG(6).key != k1
    g = np.random.Generator(np.random.PCG64(1))
    key, stream = common._key_stream(g)
    assert key[0] == np.random.Generator(np.random.PCG64(1)).integers(2**63) and stream == 0
    with pytest.raises(TypeError):
        common._key_stream("seed")
