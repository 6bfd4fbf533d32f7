"""Split precision in the near field outside the paraxial regime.

The split kernels expand the path difference |d - r| - |d| to second order
where the dropped remainder is below 1e-7 rad, take an exact per-pair
remainder where it is not, and refuse images whose remainder would exceed
2 rad (or whose emitters reach a quarter of the detector distance).  These
tests run geometries where the second-order expansion alone is off by up to
0.1 rad -- the reference's own unit-test geometry among them, sphere(100,
100, 10) on 4x4 pixels of 10 um at 1000 um (tests/test_sim.py:124-135) --
and compare the forward and the adjoint with the FP64 oracle, which
computes the distance exactly as idi/simulation/cpu.py:42-55 does.
"""

import numpy as np
import pytest
import torch

import oracle
from idi_b200 import _native as nat
from idi_b200.simulation import _core, cuda, simobj
from idi_b200.simulation.autograd import intensity
from tests.helpers import atoms, rel_field_err, rng, sphere

pytestmark = pytest.mark.gpu

SPLIT_REL_MASKED = 1e-4  # relative intensity over pixels with I >= 1e-3 <I>
SPLIT_FIELD = 2e-5       # max |dE| / rms |E|
ADJ_REL = 1e-4           # relative norm error of each gradient


def k_of(E_ev):
    return 2 * np.pi / (1.24 / E_ev)


# name: (photon energy eV, sphere radius um, emitters, Ndet, pixel um, detz um,
#        k * max remainder of the second-order expansion, rad)
GEOMS = {
    # the reference's unit-test object and detector (tests/test_sim.py:124-135)
    "reference_test": (100.0, 10.0, 100, 4, 10.0, 1000.0),
    # a 1 um object at 1 cm, 8 keV: remainder ~8e-5 rad
    "micron_at_1cm": (8000.0, 1.0, 2000, 48, 50.0, 1e4),
}


def _gpu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _case(name, seed, n_img=2, amplitudes=False):
    E_ev, r, n, ndet, ps, dz = GEOMS[name]
    g0 = rng(seed)
    pos = sphere(g0, n, r)
    ph = g0.uniform(0, 2 * np.pi, (n_img, n))
    amp = g0.uniform(0.5, 1.5, n) if amplitudes else None
    return E_ev, pos, ph, amp, ndet, ps, dz


def _check_field(E, ref, what):
    assert rel_field_err(E, ref) < SPLIT_FIELD, (what, rel_field_err(E, ref))
    m = oracle.intensity_metrics(np.abs(E) ** 2, np.abs(ref) ** 2)
    assert m["max_rel_masked"] < SPLIT_REL_MASKED, (what, m)


def test_expansion_alone_would_fail_here():
    """The geometries are outside the second-order regime: the remainder the
    expansion drops is far above the split tolerance (numpy, FP64)."""
    for name, (E_ev, r, n, ndet, ps, dz) in GEOMS.items():
        k = k_of(E_ev)
        pos = sphere(rng(1), n, r)
        ix, iy = np.meshgrid(np.arange(ndet), np.arange(ndet), indexing="ij")
        d = np.stack([(ix - ndet / 2) * ps, (iy - ndet / 2) * ps, np.full(ix.shape, dz)], -1).reshape(-1, 3)
        D = np.linalg.norm(d, axis=1)[:, None]
        s = pos @ (d / D).T
        rp = (pos ** 2).sum(1)[:, None] - s ** 2
        L = np.linalg.norm(d[None] - pos[:, None], axis=2)
        remainder = k * np.abs(rp / (D.T + L - s) - rp / (2 * D.T))
        assert remainder.max() > 1e-5, (name, remainder.max())


@pytest.mark.parametrize("name", sorted(GEOMS))
@pytest.mark.parametrize("settings", ["nf split", "nf single", "nf scale split"])
def test_forward_exact_near_field_vs_oracle(name, settings):
    E_ev, pos, ph, amp, ndet, ps, dz = _case(name, 7, amplitudes=True)
    k = k_of(E_ev)
    flags, prec, c64 = _core.parse_settings(settings)
    geom = _core.make_geom(ndet, ps, dz, k, flags=flags)
    at = np.concatenate([atoms(pos, p) for p in ph])
    n = pos.shape[0]
    off = np.arange(ph.shape[0] + 1) * n
    amps = np.tile(amp, ph.shape[0])
    E = _core.forward(_gpu(at), off, geom, prec, nat.OUT_C64 if c64 else nat.OUT_C128, amplitudes=_gpu(amps))
    _core.workspace_error()
    E = E.cpu().numpy()
    og = oracle.geometry(ndet, ps, dz, k)
    of = oracle.flags_from_settings(settings)
    for b in range(ph.shape[0]):
        _check_field(E[b], oracle.wavefield(og, of, atoms(pos, ph[b]), amp), (name, settings, b))


def test_reference_test_geometry_through_simulate():
    """cuda.simulate(2, sphere(100, 100, 10), 4, 10, 1000, k, settings="nf single"),
    the reference's unit-test call with the split kernel, against the oracle."""
    E_ev, pos, ph, _, ndet, ps, dz = _case("reference_test", 11)
    obj = simobj.fixed(E_ev, pos, phases=ph)
    for settings in ("nf single", "nf split", "nf scale single"):
        res = cuda.simulate(2, obj, ndet, ps, dz, obj.k, settings=settings, verbose=False)
        assert res.shape == (2, 4, 4)
        of = oracle.flags_from_settings(settings)
        for b in range(2):
            ref = oracle.wavefield(oracle.geometry(ndet, ps, dz, obj.k), of, atoms(pos, ph[b]))
            _check_field(res[b], ref, (settings, b))


def test_mixed_batch_paraxial_exact_and_empty():
    """One launch holding a paraxial image, an exact-path image and an empty
    image: each kernel takes its own images, all match the oracle."""
    k = k_of(8000.0)
    g0 = rng(21)
    small = sphere(g0, 1500, 0.01)   # 10 nm: second order suffices
    large = sphere(g0, 900, 1.0)     # 1 um at 1 cm: exact remainder
    ph = [g0.uniform(0, 2 * np.pi, 1500), g0.uniform(0, 2 * np.pi, 900)]
    at = np.concatenate([atoms(small, ph[0]), atoms(large, ph[1])])
    off = [0, 1500, 1500, 2400]
    og = oracle.geometry([40, 32], 50.0, 1e4, k)
    for settings in ("nf split", "nf scale split"):
        flags, prec, _ = _core.parse_settings(settings)
        geom = _core.make_geom([40, 32], 50.0, 1e4, k, flags=flags)
        E = _core.forward(_gpu(at), off, geom, prec, nat.OUT_C128)
        _core.workspace_error()
        E = E.cpu().numpy()
        of = oracle.flags_from_settings(settings)
        _check_field(E[0], oracle.wavefield(og, of, atoms(small, ph[0])), (settings, "paraxial"))
        assert np.all(E[1] == 0), settings
        _check_field(E[2], oracle.wavefield(og, of, atoms(large, ph[1])), (settings, "exact"))


def test_outside_split_range_is_reported_not_wrong():
    """A 100 um sphere at 1000 um (remainder ~100 rad): the split kernels
    refuse the image (IDIWF_ERR_UNSUPPORTED through the workspace and
    through simulate), the FP64 kernel computes it."""
    g0 = rng(31)
    pos = sphere(g0, 200, 100.0)
    ph = g0.uniform(0, 2 * np.pi, (1, 200))
    obj = simobj.fixed(100.0, pos, phases=ph)
    with pytest.raises(nat.IdiwfError) as ei:
        cuda.simulate(1, obj, 4, 10.0, 1000.0, obj.k, settings="nf split", verbose=False)
    assert ei.value.status == nat.ERR_UNSUPPORTED
    with pytest.raises(nat.IdiwfError):
        list(cuda.simulate_gen(obj, 4, 10.0, 1000.0, obj.k, settings="nf single", maximg=1))
    # a batch with one such image among valid ones reports it too
    geom = _core.make_geom(4, 10.0, 1000.0, obj.k, flags=nat.NF)
    ok = sphere(g0, 50, 1.0)
    at = np.concatenate([atoms(ok, ph[0, :50]), atoms(pos, ph[0])])
    _core.forward(_gpu(at), [0, 50, 250], geom, nat.SPLIT)
    with pytest.raises(nat.IdiwfError) as ei:
        _core.workspace_error()
    assert ei.value.status == nat.ERR_UNSUPPORTED
    # the FP64 kernel has no such limit
    res = cuda.simulate(1, obj, 4, 10.0, 1000.0, obj.k, settings="nf double", verbose=False)
    ref = oracle.wavefield(oracle.geometry(4, 10.0, 1000.0, obj.k), oracle.NF, atoms(pos, ph[0]))
    assert rel_field_err(res[0], ref) < 1e-10


def _adjoint_case(name, settings, seed):
    E_ev, pos, ph, amp, ndet, ps, dz = _case(name, seed, n_img=1, amplitudes=True)
    k = k_of(E_ev)
    g0 = rng(seed + 1)
    flags, _, _ = _core.parse_settings(settings)
    geom = _core.make_geom(ndet, ps, dz, k, flags=flags)
    og = oracle.geometry(ndet, ps, dz, k)
    of = oracle.flags_from_settings(settings)
    r = GEOMS[name][1]
    target = np.abs(oracle.wavefield(og, of, atoms(pos + g0.normal(0, 1e-3 * r, pos.shape), ph[0]), amp)) ** 2
    return pos, ph[0], amp, geom, og, of, target


@pytest.mark.parametrize("name", sorted(GEOMS))
@pytest.mark.parametrize("settings", ["nf", "nf scale"])
def test_adjoint_exact_near_field_vs_oracle(name, settings):
    """The exact adjoint (full projector, exact 1/|d - r| gradient) against the
    oracle's FP64 adjoint, every gradient within 1e-4 relative norm."""
    pos, ph, amp, geom, og, of, target = _adjoint_case(name, settings, 41)
    n = pos.shape[0]
    at = atoms(pos, ph)
    E = _core.forward(_gpu(at), [0, n], geom, nat.SPLIT, nat.OUT_C128, amplitudes=_gpu(amp))
    I = E.real ** 2 + E.imag ** 2
    gI = (2 * (I - _gpu(target)[None])).contiguous()
    ga, gamp = _core.backward(_gpu(at), [0, n], geom, E, gI, amplitudes=_gpu(amp))
    _core.backward_workspace_error()
    ga, gamp = ga.cpu().numpy(), gamp.cpu().numpy()
    E_o = oracle.wavefield(og, of, at, amp)
    _, gpos_o, gpsi_o, gamp_o = oracle.adjoint(og, of, at, amp, E_o, target)

    def err(g, g_ref):
        return float(np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref))

    assert err(ga[:, :3], gpos_o) < ADJ_REL, err(ga[:, :3], gpos_o)
    assert err(ga[:, 3], gpsi_o) < ADJ_REL, err(ga[:, 3], gpsi_o)
    assert err(gamp, gamp_o) < ADJ_REL, err(gamp, gamp_o)


def test_autograd_reports_geometry_outside_split_range():
    g0 = rng(51)
    pos = torch.from_numpy(sphere(g0, 100, 100.0)).cuda().requires_grad_(True)
    ph = torch.from_numpy(g0.uniform(0, 2 * np.pi, 100)).cuda().requires_grad_(True)
    I = intensity(pos, ph, Ndet=4, pixelsize=10.0, detz=1000.0, k=k_of(100.0), settings="nf")
    with pytest.raises(nat.IdiwfError):
        I.sum().backward()
