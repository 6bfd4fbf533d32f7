"""Host-side logic of the reference-compatible API (no GPU)."""

import numpy as np
import pytest

import oracle
from idi_b200 import _native as nat
from idi_b200.simulation import _core, simobj


def test_parse_settings():
    assert _core.parse_settings("double") == (0, nat.DOUBLE, False)
    assert _core.parse_settings("") == (0, nat.DOUBLE, False)
    assert _core.parse_settings("single") == (0, nat.SPLIT, True)
    assert _core.parse_settings("nf split scale") == (nat.NF | nat.SCALE, nat.SPLIT, False)
    assert _core.parse_settings("secondorder nofast whatever") == (nat.SECONDORDER, nat.DOUBLE, False)
    assert _core.parse_settings("", "split") == (0, nat.SPLIT, False)


def test_geometry_and_rotation():
    g = _core.make_geom(16, 75.0, 1e5, 3e4, (0.1, 0.2), (3.0, -4.0), nat.NF)
    assert (g.nx, g.ny, g.flags, g.has_rot) == (16, 16, nat.NF, 1)
    M = np.array(list(g.rot)).reshape(3, 3)
    assert np.array_equal(M, oracle.rotation(0.1, 0.2, 0))
    assert np.allclose(M @ M.T, np.eye(3))
    g2 = _core.make_geom([4, 6], 1.0, 2.0, 3.0)
    assert (g2.nx, g2.ny, g2.has_rot) == (4, 6, 0)
    assert list(g2.rot) == [1, 0, 0, 0, 1, 0, 0, 0, 1]


def test_rotation_matches_reference(reference):
    for a in [(0.1, 0.2, 0.0), (2.0, -1.0, 0.5)]:
        assert np.array_equal(_core.rotation(*a), reference.util.rotation(*a))


def test_offsets_validation():
    assert list(_core._offsets_array([0, 3, 3, 7], 7)) == [0, 3, 3, 7]
    for bad in ([1, 3], [0, 5, 3], [0, 3]):
        with pytest.raises(ValueError):
            _core._offsets_array(bad, 5)


def test_simobj_contract():
    """Mirrors the reference's tests/test_sim.py:16-53 for the sources provided."""
    o = simobj.sphere(E=1, N=1e3, r=10, rng=np.random.default_rng(1))
    assert abs(o.k - 2 * np.pi / 1.24) < 1e-12
    assert o.N == 1000
    o.rndPos = False
    o.rndPhase = False
    t = o.get()
    assert t.shape == (1000, 4)
    assert np.all(np.linalg.norm(t[:, :3], axis=1) < 10)
    assert np.allclose(t[:, 3], 0)
    o.rndPhase = True
    pos2, ph2 = o.get2()
    assert np.allclose(pos2, t[:, :3])
    assert abs(ph2.mean() - np.pi) < 0.2
    o.rndPos = True
    pos3, _ = o.get2()
    assert not np.allclose(pos3, pos2)
    f = simobj.fixed(6400, np.zeros((5, 3)), phases=np.arange(10.0).reshape(2, 5))
    assert np.array_equal(f.get()[:, 3], np.arange(5.0))
    assert np.array_equal(f.get()[:, 3], np.arange(5.0, 10.0))
