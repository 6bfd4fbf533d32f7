"""Adjoint direct sum on the GPU: against the FP64 oracle adjoint, against
autograd through a small pure-torch FP64 reference, and against FP64 central
differences on the differentiation geometry."""

import numpy as np
import pytest
import torch

import oracle
from idi_b200 import _native as nat
from idi_b200.simulation import _core
from idi_b200.simulation.autograd import intensity
from tests.helpers import K64, atoms, rng, sphere

pytestmark = pytest.mark.gpu


def _gpu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _norm_err(g, g_ref):
    return float(np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref))


@pytest.mark.parametrize("settings", ["nf", "", "secondorder", "nf scale", "scale"])
def test_adjoint_matches_oracle(settings):
    g0 = rng(41)
    n = 700
    pos = sphere(g0, n, 0.012)
    ph = g0.uniform(0, 2 * np.pi, n)
    amp = g0.uniform(0.5, 1.5, n)
    ndet, ps, dz, ang, off = [48, 40], 200.0, 1e5, (0.03, 0.01), (500.0, -300.0)
    flags, _, _ = _core.parse_settings(settings)
    geom = _core.make_geom(ndet, ps, dz, K64, ang, off, flags)
    og = oracle.geometry(ndet, ps, dz, K64, ang, off)
    of = oracle.flags_from_settings(settings)
    target = np.abs(oracle.wavefield(og, of, atoms(pos + g0.normal(0, 5e-5, pos.shape), ph), amp)) ** 2
    at = atoms(pos, ph)
    E = _core.forward(_gpu(at), [0, n], geom, nat.SPLIT, nat.OUT_C128, amplitudes=_gpu(amp))
    I = (E.real ** 2 + E.imag ** 2)
    gI = 2 * (I - _gpu(target)[None])
    ga, gamp = _core.backward(_gpu(at), [0, n], geom, E, gI.contiguous(), amplitudes=_gpu(amp))
    torch.cuda.synchronize()
    ga = ga.cpu().numpy()
    gamp = gamp.cpu().numpy()
    E_o = oracle.wavefield(og, of, at, amp)
    _, gpos_o, gpsi_o, gamp_o = oracle.adjoint(og, of, at, amp, E_o, target)
    assert _norm_err(ga[:, :3], gpos_o) < 1e-4
    assert _norm_err(ga[:, 3], gpsi_o) < 1e-4
    assert _norm_err(gamp, gamp_o) < 1e-4


@pytest.mark.parametrize("settings", ["nf", "", "secondorder", "nf scale"])
def test_adjoint_pixel_runs_vs_per_pair_and_oracle(settings):
    """The adjoint with one FP64 base phase per emitter and run of 4 pixels
    (the default where the image's bound holds: here 0.78 rad) and with an
    FP64 phase per pair, both against the oracle adjoint."""
    g0 = rng(43)
    n = 700
    pos = sphere(g0, n, 0.008)
    ph = g0.uniform(0, 2 * np.pi, n)
    amp = g0.uniform(0.5, 1.5, n)
    ndet, ps, dz, ang, off = [48, 40], 200.0, 1e5, (0.03, 0.01), (500.0, -300.0)
    flags, _, _ = _core.parse_settings(settings)
    geom = _core.make_geom(ndet, ps, dz, K64, ang, off, flags)
    og = oracle.geometry(ndet, ps, dz, K64, ang, off)
    of = oracle.flags_from_settings(settings)
    target = np.abs(oracle.wavefield(og, of, atoms(pos + g0.normal(0, 5e-5, pos.shape), ph), amp)) ** 2
    at = atoms(pos, ph)
    E = _core.forward(_gpu(at), [0, n], geom, nat.SPLIT, nat.OUT_C128, amplitudes=_gpu(amp))
    I = (E.real ** 2 + E.imag ** 2)
    gI = (2 * (I - _gpu(target)[None])).contiguous()
    E_o = oracle.wavefield(og, of, at, amp)
    _, gpos_o, gpsi_o, gamp_o = oracle.adjoint(og, of, at, amp, E_o, target)
    res = []
    for cfg in ({"pixel_groups": 1}, {"pixel_groups": -1}):
        ga, gamp = _core.backward(_gpu(at), [0, n], geom, E, gI, amplitudes=_gpu(amp), config=cfg)
        torch.cuda.synchronize()
        ga, gamp = ga.cpu().numpy(), gamp.cpu().numpy()
        assert _norm_err(ga[:, :3], gpos_o) < 1e-4, cfg
        assert _norm_err(ga[:, 3], gpsi_o) < 1e-4, cfg
        assert _norm_err(gamp, gamp_o) < 1e-4, cfg
        res.append(ga)
    assert not np.array_equal(res[0], res[1])  # the run path was taken


def _torch_intensity_nf(pos, phase, det, k):
    """Plain torch FP64 near-field intensity (the expression of cpu.py:44-55)."""
    d = det[:, None, :] - pos[None, :, :]
    dist = torch.sqrt((d ** 2).sum(-1))
    ph = (dist - det[:, None, 2] + pos[None, :, 2]) * k + phase[None, :]
    return torch.cos(ph).sum(1) ** 2 + torch.sin(ph).sum(1) ** 2


def test_adjoint_matches_torch_fp64_autograd():
    """500 emitters uniform in a 15 nm sphere, 64x64 pixels of a 512x512,
    0.1 m, 6.4 keV detector: split adjoint vs torch FP64 autograd."""
    g0 = rng(51)
    n = 500
    pos = sphere(g0, n, 0.015)
    ph = g0.uniform(0, 2 * np.pi, n)
    target = np.abs(oracle.wavefield(oracle.geometry([64, 64], 75.0, 1e5, K64, (0, 0), (128 * 75.0, 64 * 75.0)),
                                     oracle.NF, atoms(pos + g0.normal(0, 5e-5, pos.shape), ph))) ** 2
    ix, iy = np.meshgrid(np.arange(64), np.arange(64), indexing="ij")
    det = np.stack([(ix - 32) * 75.0 + 128 * 75.0, (iy - 32) * 75.0 + 64 * 75.0, np.full(ix.shape, 1e5)], -1)
    p_t = torch.tensor(pos, dtype=torch.float64, requires_grad=True)
    q_t = torch.tensor(ph, dtype=torch.float64, requires_grad=True)
    I_t = _torch_intensity_nf(p_t, q_t, torch.tensor(det.reshape(-1, 3)), K64)
    L_t = ((I_t - torch.tensor(target.reshape(-1))) ** 2).sum()
    L_t.backward()

    p_g = _gpu(pos).requires_grad_(True)
    q_g = _gpu(ph).requires_grad_(True)
    I_g = intensity(p_g, q_g, Ndet=[64, 64], pixelsize=75.0, detz=1e5, k=K64, settings="nf",
                    detoffset=(128 * 75.0, 64 * 75.0))
    L_g = ((I_g[0] - _gpu(target)) ** 2).sum()
    L_g.backward()
    assert abs(L_g.item() - L_t.item()) <= 1e-4 * L_t.item()
    assert _norm_err(p_g.grad.cpu().numpy(), p_t.grad.numpy()) < 2e-4
    assert _norm_err(q_g.grad.cpu().numpy(), q_t.grad.numpy()) < 2e-4


@pytest.mark.parametrize("settings", ["nf", ""])
def test_adjoint_finite_differences_full_geometry(settings):
    """10,000 emitters in a 15 nm sphere, 512x512 detector at 0.1 m, 6.4 keV,
    target = intensity after a 0.05 nm Gaussian displacement, L = sum (I - T)^2.
    64 random coordinates: FP64 central differences (step 1e-4 nm, all-FP64
    forward) against the split-precision adjoint."""
    g0 = rng(61)
    n = 10000
    pos = sphere(g0, n, 0.015)
    ph = g0.uniform(0, 2 * np.pi, n)
    flags, _, _ = _core.parse_settings(settings)
    geom = _core.make_geom(512, 75.0, 1e5, K64, flags=flags)
    at = _gpu(atoms(pos, ph))
    tgt_at = _gpu(atoms(pos + g0.normal(0, 5e-5, pos.shape), ph))
    T = _core.forward(tgt_at, [0, n], geom, nat.DOUBLE, nat.OUT_I64)

    def loss(a):
        I = _core.forward(a, [0, n], geom, nat.DOUBLE, nat.OUT_I64)
        return float(((I - T) ** 2).sum().item())

    E = _core.forward(at, [0, n], geom, nat.SPLIT, nat.OUT_C128)
    I = E.real ** 2 + E.imag ** 2
    ga, _ = _core.backward(at, [0, n], geom, E, (2 * (I - T)).contiguous(), want_amp=False)
    ga = ga.cpu().numpy()
    h = 1e-7
    idx = g0.choice(n, 64, replace=False)
    dims = g0.integers(0, 3, 64)
    fd = np.empty(64)
    for m, (j, d) in enumerate(zip(idx, dims)):
        a1 = at.clone(); a1[j, d] += h
        a2 = at.clone(); a2[j, d] -= h
        fd[m] = (loss(a1) - loss(a2)) / (2 * h)
    ad = ga[idx, dims]
    # near field: the FP64 forward follows the reference's |d - r| - d_z
    # rounding, whose k*ulp(|d|) ~ 5e-7 rad noise limits the difference quotient
    tol = 3e-3 if settings == "nf" else 5e-4
    assert np.max(np.abs(ad - fd)) <= tol * np.max(np.abs(fd)), np.max(np.abs(ad - fd)) / np.max(np.abs(fd))


def test_autograd_interface_amplitudes_and_batches():
    g0 = rng(71)
    counts = [300, 0, 120]
    pos = _gpu(sphere(g0, sum(counts), 0.01)).requires_grad_(True)
    ph = _gpu(g0.uniform(0, 2 * np.pi, sum(counts))).requires_grad_(True)
    amp = _gpu(g0.uniform(0.5, 1.5, sum(counts)).astype(np.float32)).requires_grad_(True)
    off = np.concatenate([[0], np.cumsum(counts)])
    I = intensity(pos, ph, amp, Ndet=[16, 12], pixelsize=75.0, detz=1e5, k=K64, settings="nf", offsets=off)
    assert tuple(I.shape) == (3, 16, 12) and I.dtype == torch.float64
    assert torch.all(I[1] == 0)
    (I ** 2).sum().backward()
    assert pos.grad.shape == pos.shape and ph.grad.shape == ph.shape
    assert amp.grad.dtype == torch.float32
    # d(sum I^2)/d a_j = sum 2 I dI/da_j; check the amplitude gradient against the oracle
    a64 = amp.detach().double().cpu().numpy()
    at = atoms(pos.detach().cpu().numpy(), ph.detach().cpu().numpy())
    og = oracle.geometry([16, 12], 75.0, 1e5, K64)
    E = oracle.wavefield(og, oracle.NF, at[:300], a64[:300])
    # L = sum I^2 = sum (I - 0)^2 -> the oracle's adjoint with a zero target
    _, gp, gq, ga = oracle.adjoint(og, oracle.NF, at[:300], a64[:300], E, np.zeros((16, 12)))
    assert _norm_err(amp.grad.double().cpu().numpy()[:300], ga) < 1e-4
    assert _norm_err(pos.grad.cpu().numpy()[:300], gp) < 1e-4
