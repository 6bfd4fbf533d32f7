"""Emitter sources drawn on the device (idiwf_emitters) against the oracle's
restatement on the same streams, and the simulate loops fed by them."""

import warnings

import numpy as np
import pytest
import torch

import oracle
from idi_b200 import _native as nat
from idi_b200.simulation import _core, cuda, simobj

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)
KEY = (0xABCDEF0123456789, 77)


def _emit(kind, n_images, n, first=0, **kw):
    desc = _core.emitters_desc(kind, **kw)
    return _core.emitters(desc, n_images, n, KEY, 3, first, DEV, check=True).cpu().numpy()


def _close(a, b):
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-15 * max(1.0, float(np.abs(b).max())))


@pytest.mark.parametrize("kw", [dict(r=0.01), dict(r=2.5, random_phase=False)])
def test_sphere_vs_oracle(kw):
    gpu = _emit(nat.EMIT_SPHERE, 3, 5000, **kw)
    _close(gpu, oracle.emit("sphere", 3, 5000, KEY, 3, **kw))


@pytest.mark.parametrize("kw", [dict(fwhm=(0.01, 0.02, 0.03)), dict(fwhm=0.01, rho=4.0),
                                dict(fwhm=(0.01, 0.02, 0.015), rho=(2.0, 3.0, 6.0), rot=_core.rotation(0.1, 0.2, 0.3))])
def test_gnorm_vs_oracle(kw):
    gpu = _emit(nat.EMIT_GNORM, 2, 4000, **kw)
    _close(gpu, oracle.emit("gnorm", 2, 4000, KEY, 3, **kw))


@pytest.mark.parametrize("kw", [dict(fwhm=(0.1, 0.2), depth=0.01),
                                dict(fwhm=(0.1, 0.2), depth=0.01, attenuation=0.004, rot=_core.rotation(0.3, 0, 0)),
                                dict(fwhm=0.2, rho=3.0, depth=0.02, attenuation=0.01)])
def test_foil_vs_oracle(kw):
    gpu = _emit(nat.EMIT_FOIL, 2, 4000, **kw)
    _close(gpu, oracle.emit("foil", 2, 4000, KEY, 3, **kw))


@pytest.mark.parametrize("kw", [dict(), dict(weighted=True, fwhm=1.5), dict(orientation=nat.ORIENT_RANDOM),
                                dict(weighted=True, fwhm=(1.0, 2.0, 1.5), rho=(2.0, 4.0, 2.0),
                                     orientation=nat.ORIENT_AXIS, axis=(0.2, 0.5, 1.0), rot=_core.rotation(0.1, 0, 0.2))])
def test_sites_vs_oracle(kw):
    g = np.random.default_rng(5)
    sites = g.normal(size=(3000, 3))
    d_sites = torch.from_numpy(sites).to(DEV)
    for n in (700, 3000, 7100):  # one round, all sites, three rounds
        desc = _core.emitters_desc(nat.EMIT_SITES, sites=d_sites, **kw)
        gpu = _core.emitters(desc, 3, n, KEY, 3, 0, DEV, check=True).cpu().numpy()
        rows, sel = oracle.emit_sites(sites, 3, n, KEY, 3, **kw)
        _close(gpu, rows)


def test_sites_large_lattice_and_chunks():
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        c = simobj.fcc(8000.0, 50000, 3.6e-4, seed=9)
    sites = torch.from_numpy(c._allpos.astype(np.float64)).to(DEV)
    desc = _core.emitters_desc(nat.EMIT_SITES, sites=sites, orientation=nat.ORIENT_RANDOM)
    whole = _core.emitters(desc, 4, 50000, KEY, 0, 0, DEV).cpu().numpy()
    parts = np.concatenate([_core.emitters(desc, 2, 50000, KEY, 0, f, DEV).cpu().numpy() for f in (0, 2)])
    np.testing.assert_array_equal(whole, parts)
    rows, _ = oracle.emit_sites(c._allpos.astype(np.float64), 1, 50000, KEY, 0, first_image=3,
                                orientation=nat.ORIENT_RANDOM)
    _close(whole[3 * 50000:], rows)


def test_sites_too_few_weights_raises():
    sites = torch.from_numpy(np.array([[0.0, 0, 0], [100.0, 0, 0], [200.0, 0, 0]])).to(DEV)
    desc = _core.emitters_desc(nat.EMIT_SITES, sites=sites, weighted=True, fwhm=0.01)
    with pytest.raises(ValueError):
        _core.emitters(desc, 1, 2, KEY, 0, 0, DEV, check=True)
    ok = _core.emitters(_core.emitters_desc(nat.EMIT_SPHERE, r=1.0), 1, 10, KEY, 0, 0, DEV, check=True)
    assert torch.isfinite(ok).all()


def test_source_objects():
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        c = simobj.fcc(8000.0, 2000, 3.6e-4, fwhm=0.003, seed=4)
    rows = c.device_batch(3).cpu().numpy()
    assert rows.shape == (6000, 4)
    lattice = {tuple(p) for p in np.round(c._allpos.astype(np.float64), 12)}
    assert all(tuple(p) in lattice for p in np.round(rows[:, :3], 12))
    pos, ph = c.get2()  # the 4th image
    assert pos.shape == (2000, 3) and ph.shape == (2000, 1)
    c.rndPos = False
    a = c.device_batch(2).cpu().numpy()
    b = c.device_batch(1).cpu().numpy()
    np.testing.assert_array_equal(a[:2000, :3], a[2000:, :3])
    np.testing.assert_array_equal(a[:2000, :3], b[:, :3])
    assert not np.array_equal(a[:2000, 3], a[2000:, 3])
    c.rndPhase = False
    assert not c.device_batch(1)[:, 3].any()
    f = simobj.foil(8000.0, 1e6, 0.01, 0.1, seed=1)
    assert f.device_batch(2).shape == (2 * f.N, 4)
    s = simobj.sphere(8000.0, 500, 0.01, seed=3)
    s.ondevice = True
    assert np.linalg.norm(s.get2()[0], axis=1).max() <= 0.01


def test_simulate_with_device_source():
    """simulate() on a device source equals the forward of the same rows."""
    mk = lambda: simobj.fcc(6400.0, 2900, 3.6e-4, seed=12)  # noqa: E731  (9^3 cells, 2916 sites)
    E = cuda.simulate(5, mk(), 64, 75.0, 1e5, settings="nf double", verbose=False)
    rows = mk().device_batch(5)
    geom = _core.make_geom(64, 75.0, 1e5, mk().k, flags=nat.NF)
    ref = _core.forward(rows, np.arange(6) * 2900, geom, nat.DOUBLE, nat.OUT_C128).cpu().numpy()
    np.testing.assert_array_equal(E, ref)
    Eg = cuda.simulate(5, mk(), 64, 75.0, 1e5, settings="nf double", returngpu=True, verbose=False)
    np.testing.assert_array_equal(Eg.cpu().numpy(), ref)
    gen = cuda.simulate_gen(mk(), 64, 75.0, 1e5, settings="nf double", maximg=5, batch=2)
    np.testing.assert_array_equal(np.stack(list(gen)), ref)
