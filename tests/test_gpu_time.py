"""Time-dependent path on the GPU: arrival-time ordering bit-exact against
the reference's own sort (golden fixtures) and the oracle; intensities
against the reference and the oracle."""

import numpy as np
import pytest
import torch

import oracle
from idi_b200.simulation import _core, cutime, simobj
from tests.helpers import K64, atoms, rng, sphere

pytestmark = pytest.mark.gpu


def _gpu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _cases(golden_time):
    for name in sorted({k.split("__")[0] for k in golden_time.files}):
        nx, ny, ps, dz, a0, a1, c, tau, pw, k = golden_time[f"{name}__meta"]
        settings = str(golden_time[f"{name}__settings"])
        flags, _, _ = _core.parse_settings(settings)
        geom = _core.make_geom([int(nx), int(ny)], ps, dz, k, (a0, a1), (0, 0), flags)
        at = atoms(golden_time[f"{name}__pos"], golden_time[f"{name}__phases"][0])
        yield name, geom, at, golden_time[f"{name}__times"], c, tau, golden_time


def test_time_order_bit_exact_vs_reference(golden_time):
    for name, geom, at, times, c, tau, gt in _cases(golden_time):
        sk = gt[f"{name}__sorted_keys"]
        keys = gt[f"{name}__keys"]
        for p in range(geom.nx * geom.ny):
            order, sorted_keys = _core.time_order(_gpu(at), _gpu(times), geom, c, p // geom.ny, p % geom.ny)
            order = order.cpu().numpy()
            sorted_keys = sorted_keys.cpu().numpy()
            assert np.array_equal(sorted_keys, sk[p]), (name, p)      # the reference's sorted sequence, bitwise
            assert np.array_equal(keys[p][order], sk[p]), (name, p)   # and the permutation that produces it


def test_time_image_vs_reference(golden_time):
    for name, geom, at, times, c, tau, gt in _cases(golden_time):
        img = _core.time_forward(_gpu(at), _gpu(times), geom, c, tau).cpu().numpy()
        ref = gt[f"{name}__image"]
        assert np.max(np.abs(img - ref) / np.abs(ref)) < 1e-10, name


@pytest.mark.parametrize("settings", ["", "nf", "scale", "nf scale"])
def test_time_vs_oracle(settings):
    g0 = rng(81)
    n = 3000
    at = atoms(sphere(g0, n, 0.01), g0.uniform(0, 2 * np.pi, n))
    times = g0.normal(0, 5.0 / 2.35, n)
    flags, _, _ = _core.parse_settings(settings)
    geom = _core.make_geom([10, 7], 75.0, 1e5, K64, (0.02, 0.04), (0, 0), flags)
    og = oracle.geometry([10, 7], 75.0, 1e5, K64, (0.02, 0.04))
    of = oracle.flags_from_settings(settings)
    img, dig = _core.time_forward(_gpu(at), _gpu(times), geom, 0.3, 2.0, digest=True)
    img = img.cpu().numpy()
    ref, ref_dig, _ = oracle.time_image_digest(og, of, at, times, 0.3, 2.0)
    assert np.max(np.abs(img - ref) / np.abs(ref)) < 1e-10
    assert np.array_equal(dig.cpu().numpy().view(np.uint64), ref_dig)
    assert np.array_equal(_core.time_forward(_gpu(at), _gpu(times), geom, 0.3, 2.0).cpu().numpy(), img)
    for ix, iy in [(0, 0), (5, 3), (9, 6)]:
        order, _ = _core.time_order(_gpu(at), _gpu(times), geom, 0.3, ix, iy)
        assert np.array_equal(order.cpu().numpy(), oracle.time_order(og, of, at, times, 0.3, ix, iy))


def test_time_full_size_every_pixel():
    """The time-dependent configuration at full size -- 20,000 emitters in a
    10 nm sphere, 256x256 detector at 0.1 m, 6.4 keV, 5 fs FWHM emission
    times, tau = 2 fs -- on every pixel against the oracle's full image: the
    intensity within 1e-10 (the bar is 1e-5), and the sorted order through the
    per-pixel order digest.  The oracle finds no equal neighbouring keys, so
    the order is unique and any argsort of the reference's keys gives it."""
    g0 = rng(91)
    n = 20000
    at = atoms(sphere(g0, n, 0.01), g0.uniform(0, 2 * np.pi, n))
    times = g0.normal(0, 5.0 / 2.35, n)
    geom = _core.make_geom(256, 75.0, 1e5, K64)
    og = oracle.geometry(256, 75.0, 1e5, K64)
    img, dig = _core.time_forward(_gpu(at), _gpu(times), geom, 0.3, 2.0, digest=True)
    img, dig = img.cpu().numpy(), dig.cpu().numpy().view(np.uint64)
    ref, ref_dig, ties = oracle.time_image_digest(og, 0, at, times, 0.3, 2.0)
    assert ties.max() == 0
    assert np.array_equal(dig, ref_dig), int(np.sum(dig != ref_dig))
    assert np.max(np.abs(img - ref) / np.abs(ref)) < 1e-10
    # and the full order and sorted keys on a few pixels
    for ix, iy in [(0, 0), (128, 128), (17, 201), (255, 3)]:
        order, keys = _core.time_order(_gpu(at), _gpu(times), geom, 0.3, ix, iy)
        o_ref = oracle.time_order(og, 0, at, times, 0.3, ix, iy)
        assert np.array_equal(order.cpu().numpy(), o_ref)
        assert oracle.order_digest(o_ref) == int(ref_dig[ix, iy])
        t_ref, _ = oracle.time_keys(og, 0, at, times, 0.3, ix, iy)
        assert np.array_equal(keys.cpu().numpy(), t_ref[o_ref])


def test_np_inner_on_this_host_matches_the_fma_chain():
    """The reference's arrival keys t = -np.inner(q, r)/c + t0 (time.py:77-88)
    take their last bits from the BLAS kernel numpy calls on the host that
    runs it; the oracle and the device evaluate np.inner as
    fma(q2, z, fma(q1, y, q0 x)).  This runs the reference's expressions with
    numpy on this host (the GPU machine in the GPU pass) -- pixels in blocks of
    4 as the reference's default, the time-dependent configuration's 20,000
    emitters and 256x256 detector -- and requires the same keys bit for bit."""
    g0 = rng(91)
    n, nd, c = 20000, 256, 0.3
    at = atoms(sphere(g0, n, 0.01), g0.uniform(0, 2 * np.pi, n))
    times = g0.normal(0, 5.0 / 2.35, n)
    dets = np.array(np.meshgrid(75.0 * (np.arange(nd) - nd / 2), 75.0 * (np.arange(nd) - nd / 2), 1e5)).T.reshape(-1, 3)
    og = oracle.geometry(nd, 75.0, 1e5, K64)
    blocks = dets.reshape(-1, 4, 3)
    for j in np.linspace(0, blocks.shape[0] - 1, 48).astype(int):
        det = blocks[j]
        d = np.linalg.norm(det, axis=-1)[:, None]
        q = det / d
        q[..., -1] -= 1
        s = np.inner(q, at[:, :3])
        t = -s / c + times.T
        for b in range(4):
            p = 4 * j + b
            # row p of np.array(meshgrid(x, y, z)).T.reshape(-1, 3) is (x[p // ny], y[p % ny], z)
            ix, iy = p // nd, p % nd
            assert np.array_equal(t[b], oracle.time_keys(og, 0, at, times, c, ix, iy)[0]), (j, b)


def test_cutime_reference_api_shape():
    """Mirrors tests/test_sim.py:137-141 of the reference."""
    obj = simobj.sphere(100, 100, 10, rng=np.random.default_rng(0))
    res = cutime.simulate(obj, 4, 10, 1000, obj.k, 1.0, 1.0, 1.0)
    assert res.shape == (4, 4) and res.dtype == np.float64
    gen = cutime.simulate_gen(obj, 4, 10, 1000, obj.k, 1.0, 1.0, 1.0, maximg=2)
    assert len(list(gen)) == 2


def test_time_sort_fallback_and_degenerate_keys():
    """Keys that defeat the bucket sort (one far outlier puts every other key
    in one bucket -> radix fallback) and all-equal keys keep the exact order."""
    g0 = rng(101)
    n = 5000
    at = atoms(sphere(g0, n, 0.01), g0.uniform(0, 2 * np.pi, n))
    geom = _core.make_geom([3, 2], 75.0, 1e5, K64)
    og = oracle.geometry([3, 2], 75.0, 1e5, K64)
    times = np.zeros(n)
    times[1234] = 1e6
    for tt in (times, np.zeros(n)):
        for ix, iy in [(0, 0), (2, 1)]:
            order, keys = _core.time_order(_gpu(at), _gpu(tt), geom, 0.3, ix, iy)
            assert np.array_equal(order.cpu().numpy(), oracle.time_order(og, 0, at, tt, 0.3, ix, iy))
        img = _core.time_forward(_gpu(at), _gpu(tt), geom, 0.3, 2.0).cpu().numpy()
        ref = oracle.time_image(og, 0, at, tt, 0.3, 2.0)
        assert np.max(np.abs(img - ref) / np.abs(ref)) < 1e-10
    # a single emitter
    one = at[:1]
    img = _core.time_forward(_gpu(one), _gpu(np.zeros(1)), geom, 0.3, 2.0).cpu().numpy()
    assert np.allclose(img, oracle.time_image(og, 0, one, np.zeros(1), 0.3, 2.0), rtol=1e-12)


@pytest.mark.parametrize("n,settings,outlier", [(30000, "", False), (70000, "nf scale", False),
                                                (25000, "nf", True)])
def test_time_large_emitter_counts(n, settings, outlier):
    """Emitter counts above the on-chip table (the global-memory kernel):
    intensities against the oracle and the sorted order bit for bit; with
    one far outlying emission time every other key falls in one bucket and
    the radix fallback sorts them."""
    assert n > _core.time_max_emitters()
    g0 = rng(n)
    at = atoms(sphere(g0, n, 0.01), g0.uniform(0, 2 * np.pi, n))
    times = g0.normal(0, 5.0 / 2.35, n)
    if outlier:
        times[n // 3] = 1e6
    flags, _, _ = _core.parse_settings(settings)
    geom = _core.make_geom([4, 3], 75.0, 1e5, K64, (0.02, 0.0), (0, 0), flags)
    og = oracle.geometry([4, 3], 75.0, 1e5, K64, (0.02, 0.0))
    of = oracle.flags_from_settings(settings)
    img, dig = _core.time_forward(_gpu(at), _gpu(times), geom, 0.3, 2.0, digest=True)
    img = img.cpu().numpy()
    ref, ref_dig, _ = oracle.time_image_digest(og, of, at, times, 0.3, 2.0)
    assert np.max(np.abs(img - ref) / np.abs(ref)) < 1e-9
    assert np.array_equal(dig.cpu().numpy().view(np.uint64), ref_dig)  # every pixel's order
    for ix, iy in ((0, 0), (3, 2)):
        order, keys = _core.time_order(_gpu(at), _gpu(times), geom, 0.3, ix, iy)
        np.testing.assert_array_equal(order.cpu().numpy(), oracle.time_order(og, of, at, times, 0.3, ix, iy))
        assert np.all(np.diff(keys.cpu().numpy()) >= 0)


def test_time_large_emitter_counts_many_pixels():
    """More pixels than SMs: the workspace-resident kernel's grid is as large
    as the slices the workspace holds (one per resident CTA)."""
    n = 21000
    g0 = rng(909)
    at = atoms(sphere(g0, n, 0.01), g0.uniform(0, 2 * np.pi, n))
    times = g0.normal(0, 5.0 / 2.35, n)
    geom = _core.make_geom([20, 20], 75.0, 1e5, K64)
    img = _core.time_forward(_gpu(at), _gpu(times), geom, 0.3, 2.0).cpu().numpy()
    ref = oracle.time_image(oracle.geometry([20, 20], 75.0, 1e5, K64), 0, at, times, 0.3, 2.0)
    assert np.max(np.abs(img - ref) / np.abs(ref)) < 1e-9


def _all_pixels_vs_oracle(at, times, nd, c, tau, settings="", tol=1e-10):
    flags, _, _ = _core.parse_settings(settings)
    geom = _core.make_geom(nd, 75.0, 1e5, K64, (0, 0), (0, 0), flags)
    og = oracle.geometry(nd, 75.0, 1e5, K64)
    stats = {}
    img, dig = _core.time_forward(_gpu(at), _gpu(times), geom, c, tau, digest=True, stats=stats)
    ref, ref_dig, ties = oracle.time_image_digest(og, oracle.flags_from_settings(settings), at, times, c, tau)
    assert np.array_equal(dig.cpu().numpy().view(np.uint64), ref_dig), int(np.sum(dig.cpu().numpy().view(np.uint64) != ref_dig))
    assert np.max(np.abs(img.cpu().numpy() - ref) / np.abs(ref)) < tol
    return stats, ties


def test_time_warm_start_with_ties():
    """Each CTA starts a pixel's sort from its previous pixel's order and
    repairs it with window insertion sorts.  Every emitter twice (same
    position, phase and emission time) makes every key appear twice, so each
    pixel's order depends on the (key, emitter index) tie rule; 144x144 pixels
    give the kernel claims of 16 neighbouring pixels.  Every pixel's order
    digest and intensity against the oracle, and most pixels warm-started."""
    g0 = rng(303)
    n0 = 1500
    pos = sphere(g0, n0, 0.01)
    ph = g0.uniform(0, 2 * np.pi, n0)
    t0 = g0.normal(0, 5.0 / 2.35, n0)
    at = atoms(np.concatenate([pos, pos]), np.concatenate([ph, ph]))
    times = np.concatenate([t0, t0])
    stats, ties = _all_pixels_vs_oracle(at, times, 144, 0.3, 2.0)
    assert ties.min() >= n0  # every key appears (at least) twice
    assert stats["full_sorts"] < 144 * 144 // 4, stats


@pytest.mark.parametrize("settings", ["", "nf scale"])
def test_time_warm_start_given_up_for_geometric_keys(settings):
    """All emission times equal: the keys are the geometric path differences
    alone, whose order turns with the pixel direction (fastest near the beam
    axis), so the window passes cannot always repair the previous order and
    the kernel falls back to the full sort.  Every pixel against the oracle."""
    g0 = rng(404)
    n = 3000
    at = atoms(sphere(g0, n, 0.5), g0.uniform(0, 2 * np.pi, n))
    times = np.zeros(n)
    stats, _ = _all_pixels_vs_oracle(at, times, 48, 0.3, 0.5, settings, tol=1e-9)
    assert stats["full_sorts"] > 148, stats  # beyond each CTA's first pixel
