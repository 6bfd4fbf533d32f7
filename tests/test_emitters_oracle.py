"""Emitter sources on the CPU: the host-built lattices and emitter counts
against the reference's own simobj (bit for bit), the oracle's restatement of
the device draws against samples of the reference's generators
(distribution tests) and against the reference's fwhm weights and weighted
choice without replacement."""

import os
import warnings

import numpy as np
import pytest
from scipy import stats

import oracle
from idi_b200.simulation import _core, simobj
from tests.conftest import GOLDEN


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "emitters_ref.npz"))


LATTICES = {
    "sc": lambda: simobj.sc(8000.0, 500, 3.6e-4, repeats=[5, 6, 7]),
    "fcc": lambda: simobj.fcc(8000.0, 3000, 3.6e-4, repeats=[6, 5, 4]),
    "hcp": lambda: simobj.hcp(8000.0, 800, 3.2e-4, repeats=[5, 5, 6]),
    "cuso4": lambda: simobj.cuso4(700, 8000.0, repeats=[4, 3, 5]),
    "fcc_rot_fwhm": lambda: simobj.fcc(8000.0, 3000, 3.6e-4, rotangles=(0.1, 0.2, 0.3), fwhm=0.002),
}


@pytest.mark.parametrize("name", sorted(LATTICES))
def test_lattice_sites_bit_exact(golden, name):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        obj = LATTICES[name]()
    ref = golden[f"lattice_{name}__sites"]
    assert obj._allpos.dtype == ref.dtype
    np.testing.assert_array_equal(obj._allpos, ref)


def test_foil_emitter_counts(golden):
    cases = [
        dict(E=8000.0, excitation=1e6, thickness=0.01, fwhm=0.1),
        dict(E=8000.0, excitation=3e5, thickness=0.02, fwhm=(0.1, 0.2), attenuationlength=0.01, rho=(2, 4),
             rotangles=(0.3, 0, 0)),
        dict(E=6400.0, excitation=2e5, thickness=0.005, fwhm=0.3, attenuationlength=0.002, rho=3),
    ]
    np.testing.assert_array_equal([simobj.foil(**kw).N for kw in cases], golden["foil__N"])


def test_crystal_weights_match_reference(golden):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        obj = simobj.fcc(8000.0, 3000, 3.6e-4, rotangles=(0.1, 0.2, 0.3), fwhm=0.002)
    w = oracle.site_weights(obj._allpos.astype(np.float64), 0.002)
    np.testing.assert_allclose(w / w.sum(), golden["crystal_weights__p"], rtol=1e-12)


def _ks(a, b):
    return stats.ks_2samp(a, b).pvalue


def test_sphere_distribution(golden):
    ref = golden["sample_sphere"]
    ours = oracle.emit("sphere", 1, ref.shape[0], (11, 12), r=0.01)[:, :3]
    for a in range(3):
        assert _ks(ours[:, a], ref[:, a]) > 1e-3
    assert _ks(np.linalg.norm(ours, axis=1), np.linalg.norm(ref, axis=1)) > 1e-3
    assert np.linalg.norm(ours, axis=1).max() <= 0.01 * (1 + 1e-12)


@pytest.mark.parametrize("name,kw", [("sample_gnorm2", dict(fwhm=(0.01, 0.02, 0.03), rho=2)),
                                     ("sample_gennorm4", dict(fwhm=0.01, rho=4))])
def test_gnorm_distribution(golden, name, kw):
    ref = golden[name]
    ours = oracle.emit("gnorm", 1, ref.shape[0], (13, 14), **kw)[:, :3]
    for a in range(3):
        assert _ks(ours[:, a], ref[:, a]) > 1e-3


def test_foil_distribution(golden):
    ref = golden["sample_foil"]
    R = _core.rotation(0.2, 0, 0)
    ours = oracle.emit("foil", 1, ref.shape[0], (15, 16), fwhm=(0.1, 0.2), depth=0.01 / R[2, 2],
                       attenuation=0.005, rot=R)[:, :3]
    for a in range(3):
        assert _ks(ours[:, a], ref[:, a]) > 1e-3


def test_weighted_choice_inclusion_frequencies(golden):
    """Per-site inclusion counts of 3000 draws of 40 of 216 sites, the
    oracle's exponential keys against the reference's numpy choice."""
    sites = golden["choice_sc__sites"].astype(np.float64)
    ref = golden["choice_sc__counts"]
    _, sel = oracle.emit_sites(sites, 3000, 40, (17, 18), weighted=True, fwhm=0.003)
    ours = np.bincount(sel, minlength=sites.shape[0])
    assert ours.sum() == ref.sum() == 3000 * 40
    both = ours + ref
    keep = both > 0
    chi = (((ours - ref)[keep]) ** 2 / both[keep]).sum()
    assert stats.chi2.sf(chi, keep.sum() - 1) > 1e-4


def test_site_selection_properties():
    g = np.random.default_rng(3)
    sites = g.normal(size=(500, 3))
    rows, sel = oracle.emit_sites(sites, 4, 120, (1, 2), orientation=1)
    for b in range(4):
        s = sel[b * 120:(b + 1) * 120]
        assert np.all(np.diff(s) > 0)  # distinct, in site order
        M = oracle.site_rotation(1, (1, 2), 0, b)
        np.testing.assert_allclose(rows[b * 120:(b + 1) * 120, :3], sites[s] @ M.T, rtol=0, atol=1e-14)
    rows, sel = oracle.emit_sites(sites, 1, 1234, (1, 2))
    for r0 in range(0, 1000, 500):
        assert len(np.unique(sel[r0:r0 + 500])) == 500  # every round without replacement
    assert len(np.unique(sel[1000:])) == 234


def test_random_rotations_are_uniform():
    zs = np.array([oracle.site_rotation(1, (5, 6), 0, b) for b in range(3000)])
    for M in zs[:20]:
        np.testing.assert_allclose(M @ M.T, np.eye(3), atol=1e-13)
        assert abs(np.linalg.det(M) - 1) < 1e-13
    assert _ks(zs[:, 2, 2], np.random.default_rng(0).uniform(-1, 1, 20000)) > 1e-3
    ax = np.array([oracle.site_rotation(2, (5, 6), 0, b, axis=(0, 0, 2.0)) for b in range(50)])
    np.testing.assert_allclose(ax[:, 2, 2], 1.0, atol=1e-14)  # rotations about z keep z


def test_device_sources_host_side():
    """Constructors and descriptors need no GPU."""
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        c = simobj.fcc(8000.0, 50000, 3.6e-4, seed=3)
    assert c.ondevice and c.N == 50000 and c._allpos.shape[1] == 3
    f = simobj.foil(8000.0, 1e6, 0.01, 0.1, seed=1)
    assert f.ondevice and f.N > 0
    g = simobj.gauss(8000.0, 100, 0.01, seed=2)
    assert g.ondevice and np.all(g.rho == 2)
    s = simobj.sphere(8000.0, 100, 0.01, rng=np.random.default_rng(1))
    assert not s.ondevice and s.get2()[0].shape == (100, 3)
