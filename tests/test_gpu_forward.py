"""Forward direct sum on the GPU against the reference (golden fixtures made
by the reference's own cpu.simulate) and against the oracle."""

import numpy as np
import pytest
import torch

import oracle
from idi_b200 import _native as nat
from idi_b200.simulation import _core, cuda, simobj
from tests.helpers import E_EV, K64, atoms, rel_field_err, rng, sphere

pytestmark = pytest.mark.gpu

# split precision: <= 1e-4 relative intensity over pixels with I >= 1e-3 <I>,
# and the field error relative to the rms field
SPLIT_REL_MASKED = 1e-4
SPLIT_FIELD = 2e-5
# FP64 mode: <= 1e-5 relative intensity per pixel (it reproduces the
# reference's rounding; sin/cos differ by at most an ulp)
DOUBLE_REL = 1e-5


def _gpu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _run(at, offsets, geom, precision, out_kind=nat.OUT_C128, amps=None, config=None):
    E = _core.forward(_gpu(at), offsets, geom, precision, out_kind,
                      amplitudes=None if amps is None else _gpu(amps), config=config)
    torch.cuda.synchronize()
    _core.workspace_error()
    return E.cpu().numpy()


def _golden_cases(golden_forward):
    names = sorted({k.split("__")[0] for k in golden_forward.files})
    for name in names:
        nx, ny, ps, dz, a0, a1, o0, o1, k = golden_forward[f"{name}__meta"]
        settings = str(golden_forward[f"{name}__settings"])
        flags, _, _ = _core.parse_settings(settings)
        geom = _core.make_geom([int(nx), int(ny)], ps, dz, k, (a0, a1), (o0, o1), flags)
        pos = golden_forward[f"{name}__pos"]
        ph = golden_forward[f"{name}__phases"]
        at = np.concatenate([atoms(pos, p) for p in ph])
        offsets = np.arange(ph.shape[0] + 1) * pos.shape[0]
        yield name, geom, at, offsets, golden_forward[f"{name}__field"]


def test_double_matches_reference_golden(golden_forward):
    for name, geom, at, off, ref in _golden_cases(golden_forward):
        E = _run(at, off, geom, nat.DOUBLE)
        assert rel_field_err(E, ref) < 1e-12, name
        m = oracle.intensity_metrics(np.abs(E) ** 2, np.abs(ref) ** 2, floor=0.0)
        assert m["max_rel_masked"] < DOUBLE_REL, (name, m)


def test_split_matches_reference_golden(golden_forward):
    for name, geom, at, off, ref in _golden_cases(golden_forward):
        E = _run(at, off, geom, nat.SPLIT)
        assert rel_field_err(E, ref) < SPLIT_FIELD, name
        m = oracle.intensity_metrics(np.abs(E) ** 2, np.abs(ref) ** 2)
        assert m["max_rel_masked"] < SPLIT_REL_MASKED, (name, m)


@pytest.mark.parametrize("settings", ["", "nf", "scale", "nf scale", "secondorder", "secondorder scale"])
@pytest.mark.parametrize("precision", [nat.DOUBLE, nat.SPLIT])
def test_modes_amplitudes_vs_oracle(settings, precision):
    g0 = rng(11)
    n = 1500
    pos = sphere(g0, n, 0.015)
    ph = g0.uniform(0, 2 * np.pi, n)
    amp = g0.uniform(0.5, 1.5, n).astype(np.float32)
    flags, _, _ = _core.parse_settings(settings)
    geom = _core.make_geom([33, 20], 75.0, 1e5, K64, (0.02, -0.03), (40.0, 10.0), flags)
    ref = oracle.wavefield(oracle.geometry([33, 20], 75.0, 1e5, K64, (0.02, -0.03), (40.0, 10.0)),
                           oracle.flags_from_settings(settings), atoms(pos, ph), amp.astype(np.float64))
    E = _run(atoms(pos, ph), [0, n], geom, precision, amps=amp)[0]
    if precision == nat.DOUBLE:
        assert rel_field_err(E, ref) < 1e-12
    else:
        assert rel_field_err(E, ref) < SPLIT_FIELD
        m = oracle.intensity_metrics(np.abs(E) ** 2, np.abs(ref) ** 2)
        assert m["max_rel_masked"] < SPLIT_REL_MASKED, m


@pytest.mark.parametrize("precision", [nat.DOUBLE, nat.SPLIT])
def test_batched_uneven_and_edge_sizes(precision):
    """Ragged batch incl. an empty image, a single emitter and non-tile sizes;
    odd detector sizes exercise the pixel tail."""
    g0 = rng(21)
    counts = [0, 1, 7, 64, 65, 300, 1000, 2500]
    imgs = [atoms(sphere(g0, c, 0.01), g0.uniform(0, 2 * np.pi, c)) for c in counts]
    at = np.concatenate(imgs)
    off = np.concatenate([[0], np.cumsum(counts)])
    for ndet in ([13, 7], [1, 1], [5, 129], [9, 12]):
        geom = _core.make_geom(ndet, 75.0, 1e5, K64, flags=nat.NF)
        og = oracle.geometry(ndet, 75.0, 1e5, K64)
        E = _run(at, off, geom, precision)
        assert E.shape == (len(counts), ndet[0], ndet[1])
        for b, a in enumerate(imgs):
            ref = oracle.wavefield(og, oracle.NF, a) if len(a) else np.zeros((ndet[0], ndet[1]), complex)
            if len(a) == 0:
                assert np.all(E[b] == 0)
                continue
            tol = 1e-12 if precision == nat.DOUBLE else 1e-5
            assert np.abs(E[b] - ref).max() <= tol * max(np.sqrt(len(a)), 1.0), (ndet, counts[b])


def test_output_kinds():
    g0 = rng(5)
    n = 700
    at = atoms(sphere(g0, n, 0.01), g0.uniform(0, 2 * np.pi, n))
    geom = _core.make_geom([40, 24], 75.0, 1e5, K64, flags=nat.NF)
    E = _run(at, [0, n], geom, nat.SPLIT, nat.OUT_C128)[0]
    E64 = _run(at, [0, n], geom, nat.SPLIT, nat.OUT_C64)[0]
    I64 = _run(at, [0, n], geom, nat.SPLIT, nat.OUT_I64)[0]
    I32 = _run(at, [0, n], geom, nat.SPLIT, nat.OUT_I32)[0]
    assert E64.dtype == np.complex64 and I32.dtype == np.float32
    assert np.allclose(E64, E, rtol=0, atol=1e-5 * np.abs(E).max())
    assert np.allclose(I64, np.abs(E) ** 2, rtol=1e-12)
    assert np.allclose(I32, np.abs(E) ** 2, rtol=1e-6)


def test_kernel_shapes_agree():
    """Every tile/thread shape gives identical sums (the summation order per
    pixel does not depend on the shape)."""
    g0 = rng(8)
    n = 2100
    at = atoms(sphere(g0, n, 0.012), g0.uniform(0, 2 * np.pi, n))
    geom = _core.make_geom([37, 29], 75.0, 1e5, K64, flags=nat.NF)
    base = _run(at, [0, n], geom, nat.SPLIT)
    for cfg in ({"threads": 128, "pixels_per_thread": 4, "emitters_per_tile": 128},
                {"threads": 256, "pixels_per_thread": 2, "emitters_per_tile": 512, "ctas_per_sm": 2},
                {"threads": 64, "pixels_per_thread": 8, "emitters_per_tile": 64}):
        assert np.array_equal(_run(at, [0, n], geom, nat.SPLIT, config=cfg), base), cfg
    dbase = _run(at, [0, n], geom, nat.DOUBLE)
    for cfg in ({"threads": 256, "pixels_per_thread": 1, "emitters_per_tile": 64},
                {"threads": 64, "pixels_per_thread": 4, "emitters_per_tile": 32}):
        assert np.array_equal(_run(at, [0, n], geom, nat.DOUBLE, config=cfg), dbase), cfg


@pytest.mark.parametrize("settings", ["", "nf", "nf scale", "scale", "secondorder"])
def test_pixel_runs_vs_per_pixel_and_oracle(settings):
    """Split forward with one FP64 base phase per run of 4 pixels plus FP32
    offsets (the default wherever the image's bound holds) and with an FP64
    phase per pixel: both against the oracle.  Rotated, offset detector whose
    rows are a multiple of 4 pixels long; amplitudes."""
    g0 = rng(17)
    n = 3000
    pos = sphere(g0, n, 0.02)  # k * 1.5 px * 75 um / 0.1 m * 0.02 um = 0.73 rad: runs in use
    ph = g0.uniform(0, 2 * np.pi, n)
    amp = g0.uniform(0.5, 1.5, n).astype(np.float32)
    flags, _, _ = _core.parse_settings(settings)
    geom = _core.make_geom([36, 44], 75.0, 1e5, K64, (0.02, -0.03), (40.0, 10.0), flags)
    ref = oracle.wavefield(oracle.geometry([36, 44], 75.0, 1e5, K64, (0.02, -0.03), (40.0, 10.0)),
                           oracle.flags_from_settings(settings), atoms(pos, ph), amp.astype(np.float64))
    E_run = _run(atoms(pos, ph), [0, n], geom, nat.SPLIT, amps=amp, config={"pixel_groups": 1})[0]
    E_pix = _run(atoms(pos, ph), [0, n], geom, nat.SPLIT, amps=amp, config={"pixel_groups": -1})[0]
    assert not np.array_equal(E_run, E_pix)  # the run path was taken
    for E in (E_run, E_pix):
        assert rel_field_err(E, ref) < SPLIT_FIELD
        m = oracle.intensity_metrics(np.abs(E) ** 2, np.abs(ref) ** 2)
        assert m["max_rel_masked"] < SPLIT_REL_MASKED, m


def test_pixel_runs_fall_back_beyond_their_bound():
    """An object too large for the runs' 1 rad offset bound (and rows that are
    not a multiple of 4 long) takes the per-pixel path: identical results."""
    g0 = rng(18)
    n = 1200
    at = atoms(sphere(g0, n, 0.05), g0.uniform(0, 2 * np.pi, n))  # bound 1.8 rad
    geom = _core.make_geom([24, 32], 75.0, 1e5, K64, flags=nat.NF)
    assert np.array_equal(_run(at, [0, n], geom, nat.SPLIT, config={"pixel_groups": 1}),
                          _run(at, [0, n], geom, nat.SPLIT, config={"pixel_groups": -1}))
    at = atoms(sphere(g0, n, 0.01), g0.uniform(0, 2 * np.pi, n))
    geom = _core.make_geom([24, 30], 75.0, 1e5, K64, flags=nat.NF)
    assert np.array_equal(_run(at, [0, n], geom, nat.SPLIT, config={"pixel_groups": 1}),
                          _run(at, [0, n], geom, nat.SPLIT, config={"pixel_groups": -1}))


@pytest.mark.parametrize("ndet", [[40, 64], [8, 12]])
def test_mixed_batch_runs_and_per_pixel_kernels(ndet):
    """One batch whose images take different kernels: small objects the
    pixel-run kernel, large ones (beyond the 1 rad bound) the per-pixel
    kernel, each from its own work counter.  Every image against the oracle
    and against the all-per-pixel result; the small detector also splits the
    work over emitter chunks."""
    g0 = rng(33)
    radii = [0.01, 0.06, 0.015, 0.08, 0.005]  # bound 0.37, 2.2, 0.55, 2.9, 0.18 rad
    counts = [1500, 1100, 2600, 700, 1234]
    imgs = [atoms(sphere(g0, c, r), g0.uniform(0, 2 * np.pi, c)) for c, r in zip(counts, radii)]
    at = np.concatenate(imgs)
    off = np.concatenate([[0], np.cumsum(counts)])
    geom = _core.make_geom(ndet, 75.0, 1e5, K64, flags=nat.NF)
    og = oracle.geometry(ndet, 75.0, 1e5, K64)
    E = _run(at, off, geom, nat.SPLIT)
    E_pix = _run(at, off, geom, nat.SPLIT, config={"pixel_groups": -1})
    for b, a in enumerate(imgs):
        ref = oracle.wavefield(og, oracle.NF, a)
        for X in (E[b], E_pix[b]):
            assert rel_field_err(X, ref) < SPLIT_FIELD, (ndet, b)
        if radii[b] > 0.03:  # beyond the bound: the per-pixel kernel, bit for bit
            assert np.array_equal(E[b], E_pix[b]), b
        else:
            assert not np.array_equal(E[b], E_pix[b]), b


def test_pixel_runs_shapes_agree():
    """With pixel runs the sums are still the same for every kernel shape: a
    run's base phase is fixed by the detector, not by the thread layout."""
    g0 = rng(9)
    n = 2100
    at = atoms(sphere(g0, n, 0.012), g0.uniform(0, 2 * np.pi, n))
    geom = _core.make_geom([37, 28], 75.0, 1e5, K64, flags=nat.NF)
    base = _run(at, [0, n], geom, nat.SPLIT)
    assert not np.array_equal(base, _run(at, [0, n], geom, nat.SPLIT, config={"pixel_groups": -1}))
    for cfg in ({"threads": 128, "pixels_per_thread": 4, "emitters_per_tile": 128},
                {"threads": 256, "pixels_per_thread": 2, "emitters_per_tile": 512, "ctas_per_sm": 2},
                {"threads": 64, "pixels_per_thread": 8, "emitters_per_tile": 64}):
        assert np.array_equal(_run(at, [0, n], geom, nat.SPLIT, config=cfg), base), cfg


def test_split_accuracy_against_accurate_fp64():
    """Split precision against the cancellation-free FP64 oracle (error floor
    ~1e-9 rad), on a window of the 8 keV, 0.2 m, 50 um precision geometry:
    50,000 fcc emitters, detector corner (largest angles)."""
    g0 = rng(99)
    a = 3.6e-4
    m = int(np.ceil(0.012 / a))
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    cells = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 1, 3)
    sites = ((cells + base[None]) * a).reshape(-1, 3) - 0.006
    pos = sites[g0.choice(len(sites), 50000, replace=False)] + g0.normal(0, 1e-5, (50000, 3))
    ph = g0.uniform(0, 2 * np.pi, 50000)
    k8 = 2 * np.pi / (1.24 / 8000.0)
    off = (448 * 50.0, 448 * 50.0)
    geom = _core.make_geom([64, 64], 50.0, 2e5, k8, (0, 0), off, nat.NF)
    truth = oracle.wavefield(oracle.geometry([64, 64], 50.0, 2e5, k8, (0, 0), off), oracle.NF | oracle.ACCURATE,
                             atoms(pos, ph))
    E = _run(atoms(pos, ph), [0, 50000], geom, nat.SPLIT)[0]
    m_split = oracle.intensity_metrics(np.abs(E) ** 2, np.abs(truth) ** 2)
    assert m_split["max_rel_masked"] < SPLIT_REL_MASKED, m_split
    assert m_split["max_rel_to_mean"] < 1e-5, m_split


def test_reference_api_shapes():
    """Mirrors the reference's tests/test_sim.py:124-135 (cuda.simulate shape)."""
    obj = simobj.sphere(100, 100, 10, rng=np.random.default_rng(0))
    res = cuda.simulate(2, obj, 4, 10, 1000, obj.k, verbose=False)
    assert res.shape == (2, 4, 4) and res.dtype == np.complex128
    gen = cuda.simulate_gen(obj, [4, 6], 10, 1000, obj.k, settings="single", maximg=3)
    imgs = list(gen)
    assert len(imgs) == 3 and imgs[0].shape == (4, 6) and imgs[0].dtype == np.complex64
    g = cuda.simulate(2, obj, 8, 10, 1000, settings="nf split", returngpu=True, verbose=False)
    assert isinstance(g, torch.Tensor) and g.is_cuda and tuple(g.shape) == (2, 8, 8)


def test_simulate_matches_reference_simulate(golden_forward):
    """The drop-in simulate() against the reference's own cpu.simulate: every
    fixture of forward_ref.npz was made by calling the reference's
    cpu.simulate(2, obj, Ndet, pixelsize, detz, k, settings, detangles,
    detoffset) on an object that hands out the stored positions and phases;
    here cuda.simulate gets the same call with the same object sequence."""
    names = sorted({k.split("__")[0] for k in golden_forward.files})
    assert len(names) >= 6
    for name in names:
        nx, ny, ps, dz, a0, a1, o0, o1, k = golden_forward[f"{name}__meta"]
        settings = str(golden_forward[f"{name}__settings"])
        pos = golden_forward[f"{name}__pos"]
        ph = golden_forward[f"{name}__phases"]
        ref = golden_forward[f"{name}__field"]
        for prec, tol in (("double", 1e-12), ("split", SPLIT_FIELD)):
            obj = simobj.fixed(E_EV, pos, phases=ph)
            ours = cuda.simulate(ph.shape[0], obj, [int(nx), int(ny)], ps, dz, k, settings=f"{settings} {prec}",
                                 verbose=False, detangles=(a0, a1), detoffset=(o0, o1))
            assert ours.shape == ref.shape and ours.dtype == np.complex128
            assert rel_field_err(ours, ref) < tol, (name, prec, rel_field_err(ours, ref))


def test_range_check_reports_error():
    """Emitters too far out for the split phase range are reported, not wrapped."""
    at = np.zeros((4, 4))
    at[0, 0] = 1e4
    geom = _core.make_geom([8, 8], 75.0, 1e5, K64)
    _core.forward(_gpu(at), [0, 4], geom, nat.SPLIT)
    with pytest.raises(nat.IdiwfError) as ei:
        _core.workspace_error()
    assert ei.value.status == nat.ERR_UNSUPPORTED
    # the next call clears the error word
    at[0, 0] = 0.0
    _core.forward(_gpu(at), [0, 4], geom, nat.SPLIT)
    _core.workspace_error()


def test_accurate_fp64_mode_vs_oracle():
    """settings='accurate': the FP64 kernel with the cancellation-free near-field
    path difference against the oracle's same form (field error ~1e-13)."""
    g0 = rng(123)
    n = 3000
    at = atoms(sphere(g0, n, 0.012), g0.uniform(0, 2 * np.pi, n))
    flags, prec, _ = _core.parse_settings("nf scale accurate")
    assert prec == nat.DOUBLE and flags & nat.ACCURATE
    geom = _core.make_geom([40, 30], 50.0, 2e5, K64, (0.01, 0.02), (2e4, -1e4), flags)
    og = oracle.geometry([40, 30], 50.0, 2e5, K64, (0.01, 0.02), (2e4, -1e4))
    E = _run(at, [0, n], geom, nat.DOUBLE)[0]
    truth = oracle.wavefield(og, oracle.NF | oracle.SCALE | oracle.ACCURATE, at)
    # with a 2e4 um detector offset the pixel constant k (|d| - d_z) is ~5e7 rad,
    # so two FP64 evaluations of it differ by ~1e-8 rad (a per-pixel phase)
    assert rel_field_err(E, truth) < 2e-7
    assert oracle.intensity_metrics(np.abs(E) ** 2, np.abs(truth) ** 2, floor=0.0)["max_rel_masked"] < 1e-9
    # the reference-sequence FP64 kernel differs from the truth by its own rounding noise
    E_ref = _run(at, [0, n], _core.make_geom([40, 30], 50.0, 2e5, K64, (0.01, 0.02), (2e4, -1e4),
                                             nat.NF | nat.SCALE), nat.DOUBLE)[0]
    assert 1e-12 < rel_field_err(E_ref, truth) < 1e-5


def test_simulate_pipelined_chunks_match_direct():
    """simulate() with host output splits large jobs into chunks whose copies
    overlap compute; results equal one direct batched launch."""
    g0 = rng(555)
    n, nimg = 300, 9
    pos = sphere(g0, n, 0.01)
    ph = g0.uniform(0, 2 * np.pi, (nimg, n))
    for settings in ("nf split", "nf single"):
        obj = simobj.fixed(E_EV, pos, phases=ph)
        res = cuda.simulate(nimg, obj, 1024, 75.0, 1e5, K64, settings=settings, verbose=False)
        assert res.shape == (nimg, 1024, 1024) and res.dtype == np.complex128
        at = np.concatenate([atoms(pos, p) for p in ph])
        flags, prec, c64 = _core.parse_settings(settings)
        geom = _core.make_geom(1024, 75.0, 1e5, K64, flags=flags)
        direct = _core.forward(torch.from_numpy(at).cuda(), np.arange(nimg + 1) * n, geom, prec,
                               nat.OUT_C64 if c64 else nat.OUT_C128).cpu().numpy()
        assert np.array_equal(res, direct.astype(np.complex128))


@pytest.mark.parametrize("flags", [0, nat.NF])
def test_small_config_full_image_fp64_and_split_vs_oracle(flags):
    """The CPU-runnable configuration at full size (2,000 emitters in a 10 nm
    sphere, 256x256 @ 75 um, 0.1 m, 6.4 keV): the FP64 kernel against the
    oracle per pixel (1e-9 of the intensity; in practice the last bits of
    sin/cos), and the split kernel within 1e-4 on the masked pixels."""
    g = rng(505)
    at = atoms(sphere(g, 2000, 0.01), g.uniform(0, 2 * np.pi, 2000))
    geom = _core.make_geom(256, 75.0, 1e5, K64, flags=flags)
    d_at = torch.from_numpy(at).cuda()
    Ed = _core.forward(d_at, [0, 2000], geom, nat.DOUBLE, nat.OUT_C128).cpu().numpy()[0]
    Is = _core.forward(d_at, [0, 2000], geom, nat.SPLIT, nat.OUT_I64).cpu().numpy()[0]
    ref = oracle.wavefield(oracle.geometry(256, 75.0, 1e5, K64), flags, at)
    Iref = np.abs(ref) ** 2
    m = oracle.intensity_metrics(np.abs(Ed) ** 2, Iref)
    assert m["max_rel_masked"] < 1e-9 and m["max_rel_to_mean"] < 1e-10
    assert oracle.intensity_metrics(Is, Iref)["max_rel_masked"] < 1e-4
