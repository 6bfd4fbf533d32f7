"""Generate the golden fixtures in this directory from the reference itself.

    python tests/golden/make_golden.py

Runs the reference's own CPU implementations -- ``idi/simulation/cpu.py``
``simulate``, ``idi/simulation/time.py`` ``simulate`` and
``idi/simulation/common.py`` ``randomphotons`` / ``chargesharing``, the
simulation objects of ``idi/simulation/simobj.py`` and
``idi/reconstruction/cpusimple.py`` -- unmodified, through
``oracle/refshim.py``, on seeded inputs (numpy Philox), and stores inputs and
outputs.  For the time path it also records, per pixel, the arrival-time keys
the reference computes and the order its ``_psort`` puts them in, by wrapping
the module's ``_integral`` (the reference calls it once per pixel block with
the keys; the wrapper copies them before and after the in-place sort and then
calls the original).

Needs the reference tree (``IDI_REFERENCE``, or ``oracle.refshim.REF_ROOT``).
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import refshim  # noqa: E402

E_EV = 6400.0
K = 2 * np.pi / (1.24 / E_EV)

FWD_CASES = [
    # name, settings, Ndet, pixelsize, detz, detangles, detoffset
    ("ff", "", (24, 16), 75.0, 1e5, (0, 0), (0, 0)),
    ("nf", "nf", (24, 16), 75.0, 1e5, (0, 0), (0, 0)),
    ("ff_scale", "scale", (24, 16), 75.0, 1e5, (0, 0), (0, 0)),
    ("nf_scale", "nf scale", (24, 16), 75.0, 1e5, (0, 0), (0, 0)),
    ("nf_rot_off", "nf", (17, 12), 60.5, 8e4, (0.1, 0.2), (30.0, -20.0)),
    ("ff_rot_off", "", (17, 12), 60.5, 8e4, (0.1, 0.2), (30.0, -20.0)),
]

TIME_CASES = [
    # name, settings, Ndet, pixelsize, detz, detangles, c, tau, pulsewidth
    ("time_ff", "", (4, 4), 75.0, 1e5, (0, 0), 0.3, 2.0, 5.0),
    ("time_ff_scale_rot", "scale", (4, 4), 75.0, 1e5, (0.05, 0.1), 0.3, 2.0, 5.0),
]


def sphere(rng, n, r):
    t = rng.uniform(-1, 1, n)
    p = rng.uniform(0, 2 * np.pi, n)
    u = r * rng.uniform(0, 1, n) ** (1 / 3)
    s = np.sqrt(1 - t ** 2)
    return np.stack([u * t, u * s * np.sin(p), u * s * np.cos(p)], -1)


def make_forward(ref):
    out = {}
    for i, (name, settings, ndet, ps, dz, ang, off) in enumerate(FWD_CASES):
        rng = np.random.Generator(np.random.Philox(1000 + i))
        n = 400
        pos = sphere(rng, n, 0.01)
        ph = rng.uniform(0, 2 * np.pi, (2, n))
        obj = refshim.InjectedObject(E_EV, pos, ph)
        res = ref.cpu.simulate(2, obj, list(ndet), ps, dz, K, settings=settings, detangles=ang, detoffset=off)
        out[f"{name}__pos"] = pos
        out[f"{name}__phases"] = ph
        out[f"{name}__field"] = res
        out[f"{name}__meta"] = np.array([ndet[0], ndet[1], ps, dz, ang[0], ang[1], off[0], off[1], K])
        out[f"{name}__settings"] = np.array(settings)
    return out


def make_time(ref):
    out = {}
    tmod = ref.time
    for i, (name, settings, ndet, ps, dz, ang, c, tau, pw) in enumerate(TIME_CASES):
        rng = np.random.Generator(np.random.Philox(2000 + i))
        n = 200
        pos = sphere(rng, n, 0.01)
        ph = rng.uniform(0, 2 * np.pi, (1, n))
        obj = refshim.InjectedObject(E_EV, pos, ph)
        keys, sorted_keys = [], []
        orig = tmod._integral

        def spy(amp, t0, tau_):
            t2 = np.atleast_2d(t0)
            keys.append(t2.copy())
            r = orig(amp, t0, tau_)
            sorted_keys.append(np.atleast_2d(t0).copy())
            return r

        tmod._integral = spy
        try:
            np.random.seed(3000 + i)  # the reference draws emission times from the global RNG
            img = tmod.simulate(obj, list(ndet), ps, dz, K, c, tau, pw, detangles=ang, settings=settings)
        finally:
            tmod._integral = orig
        np.random.seed(3000 + i)
        times = np.random.randn(n) * (pw / 2.35)
        out[f"{name}__pos"] = pos
        out[f"{name}__phases"] = ph
        out[f"{name}__times"] = times
        out[f"{name}__image"] = img
        out[f"{name}__keys"] = np.concatenate(keys, 0)          # (npix, n) unsorted, emitter order
        out[f"{name}__sorted_keys"] = np.concatenate(sorted_keys, 0)
        out[f"{name}__meta"] = np.array([ndet[0], ndet[1], ps, dz, ang[0], ang[1], c, tau, pw, K])
        out[f"{name}__settings"] = np.array(settings)
    return out


class _RateSpy:
    """Stands in for the Generator handed to the reference's ``randomphotons``:
    records the Poisson rates it is asked for and returns zeros."""

    def __init__(self):
        self.rates = []

    def poisson(self, lam):
        self.rates.append(np.array(lam, copy=True))
        return np.zeros(np.shape(lam))


PHOTON_CASES = [
    # name, image shape, n_photons (low rates: inversion; high rates: PTRS)
    ("photons_low", (2, 24, 20), 300.0),
    ("photons_high", (2, 24, 20), 2.0e5),
]

CHARGE_CASES = [
    # name, image shape, mean count, s, ns
    ("cs_w2", (16, 12), 0.7, 0.6, 0.0),
    ("cs_w1_noise", (16, 12), 1.5, 0.3, 0.1),
    ("cs_w3_edges", (9, 7), 2.0, 1.3, 0.0),
    ("cs_noshare_noise", (10, 8), 3.0, 0.0, 0.2),
]


def make_detector(ref):
    """Rates of ``common.randomphotons`` (recorded through a stand-in rng) and
    ``common.chargesharing`` outputs together with the random draws the
    reference made: its photon offsets come from numba's generator
    (``common.py:50``), seeded here through a jitted ``np.random.seed`` and read
    back by a jitted function drawing the same sequence; the s <= 0 branch
    draws from numpy's global generator (``common.py:39``)."""
    import numba

    @numba.njit
    def nb_seed(seed):
        np.random.seed(seed)

    @numba.njit(fastmath=True)
    def nb_draws(n, ns):
        mu = np.random.rand(n, 2) - 0.5
        scale = np.ones(n)
        if ns > 0:
            scale = 1 + np.random.randn(n) * ns
        return mu, scale

    out = {}
    for i, (name, shape, nph) in enumerate(PHOTON_CASES):
        rng = np.random.Generator(np.random.Philox(4000 + i))
        probs = rng.gamma(0.5, 1.0, shape) * rng.uniform(0.5, 1.5, shape[:1] + (1, 1))
        spy = _RateSpy()
        ref.common.randomphotons(probs, nph, rng=spy)
        out[f"{name}__probs"] = probs
        out[f"{name}__n_photons"] = np.array(nph)
        out[f"{name}__rates"] = spy.rates[0]
    for i, (name, shape, mean, s, ns) in enumerate(CHARGE_CASES):
        rng = np.random.Generator(np.random.Philox(5000 + i))
        img = rng.poisson(mean, shape)
        img[0, 0] += 2  # photons in the corner: charge leaves the detector
        seed = 6000 + i
        if s > 0:
            nb_seed(seed)
            res = ref.common.chargesharing(img, s, ns)
            nb_seed(seed)
            mu, scale = nb_draws(int(img.sum()), ns)
        else:
            np.random.seed(seed)
            res = ref.common.chargesharing(img, s, ns)
            np.random.seed(seed)
            mu = np.zeros((0, 2))
            scale = 1 + ns * np.random.randn(*img.shape)
        out[f"{name}__counts"] = img
        out[f"{name}__meta"] = np.array([s, ns])
        out[f"{name}__positions"] = mu
        out[f"{name}__scales"] = scale
        out[f"{name}__out"] = res
    return out


LATTICE_CASES = [
    # name, class, args, kwargs
    ("sc", "sc", (8000.0, 500, 3.6e-4), dict(repeats=[5, 6, 7])),
    ("fcc", "fcc", (8000.0, 3000, 3.6e-4), dict(repeats=[6, 5, 4])),
    ("hcp", "hcp", (8000.0, 800, 3.2e-4), dict(repeats=[5, 5, 6])),
    ("cuso4", "cuso4", (700, 8000.0), dict(repeats=[4, 3, 5])),
    ("fcc_rot_fwhm", "fcc", (8000.0, 3000, 3.6e-4), dict(rotangles=(0.1, 0.2, 0.3), fwhm=0.002)),
]

FOIL_CASES = [
    dict(E=8000.0, excitation=1e6, thickness=0.01, fwhm=0.1),
    dict(E=8000.0, excitation=3e5, thickness=0.02, fwhm=(0.1, 0.2), attenuationlength=0.01, rho=(2, 4),
         rotangles=(0.3, 0, 0)),
    dict(E=6400.0, excitation=2e5, thickness=0.005, fwhm=0.3, attenuationlength=0.002, rho=3),
]


def make_emitters(ref):
    """Lattices (bit-exact targets), foil emitter counts, the crystal's fwhm
    weights, and samples of the reference's own generators (sphere, gnorm,
    rndgennorm, foil; numpy draws) plus per-site inclusion counts of its
    weighted choice without replacement, for distribution tests."""
    sim = ref.simobj
    out = {}
    for name, cls, args, kw in LATTICE_CASES:
        obj = getattr(sim, cls)(*args, **kw)
        out[f"lattice_{name}__sites"] = obj._allpos
    obj = sim.fcc(8000.0, 3000, 3.6e-4, rotangles=(0.1, 0.2, 0.3), fwhm=0.002)
    obj.updatePos()
    out["crystal_weights__p"] = obj._p
    out["foil__N"] = np.array([sim.foil(**kw).N for kw in FOIL_CASES])
    n = 8000
    # sphere.updatePos and foil.updatePos call rndSphere / rndtruncexp
    # without a generator (fresh OS entropy each run); wrapped here to pass a
    # seeded one so the fixture is reproducible
    orig_sphere, orig_texp = sim._rndSphere, sim._rndtruncexp
    sim._rndSphere = lambda r, N: ref.util.rndSphere(r, N, rng=np.random.default_rng(7005))
    sim._rndtruncexp = lambda lam, b, N: ref.util.rndtruncexp(lam, b, N, rng=np.random.default_rng(7006))
    s = sim.sphere(6400.0, n, 0.01)
    s.rng = np.random.default_rng(7000)
    out["sample_sphere"] = s.get2()[0]
    g = sim.gnorm(6400.0, n, np.array([0.01, 0.02, 0.03]), 2)
    g.rng = np.random.default_rng(7001)
    out["sample_gnorm2"] = g.get2()[0]
    out["sample_gennorm4"] = ref.util.rndgennorm(0, 0.01, 4, (n, 3), np.random.default_rng(7002))
    f = sim.foil(8000.0, 1e6, 0.01, (0.1, 0.2), attenuationlength=0.005, rotangles=(0.2, 0, 0))
    f.rng = np.random.default_rng(7003)
    f._N = n
    out["sample_foil"] = f.get2()[0]
    sim._rndSphere, sim._rndtruncexp = orig_sphere, orig_texp
    # weighted choice without replacement: 3000 draws of 40 of 216 sc sites
    c = sim.sc(8000.0, 40, 1e-3, repeats=[6, 6, 6], fwhm=0.003)
    c.rng = np.random.default_rng(7004)
    counts = np.zeros(len(c._allpos), np.int64)
    for _ in range(3000):
        c.updatePos()
        idx = np.flatnonzero((c._allpos[:, None, :] == c._pos[None, :, :]).all(-1).any(1))
        counts[idx] += 1
    out["choice_sc__sites"] = c._allpos
    out["choice_sc__counts"] = counts
    return out


def make_fftcorr(ref):
    """``idi/reconstruction/cpusimple.py`` (the numpy twin of the cupy
    ``cusimple``, which needs cupy): ``corr`` on the reference test's inputs
    and on seeded stacks, and ``correlator2d`` with and without masks."""
    simple = refshim.load_module("reconstruction.cpusimple")
    out = {}
    t1 = np.arange(32 * 16).reshape(32, 16).astype(float)
    out["corr_arange__in"] = t1
    out["corr_arange__out"] = simple.corr(t1)
    t2 = np.arange(15 * 33).reshape(15, 33).astype(float)
    out["corr_arange_norm__in"] = t2
    out["corr_arange_norm__out"] = simple.corr(t2, norm=True)
    g = np.random.Generator(np.random.Philox(9000))
    st = g.exponential(1.0, (3, 20, 24))
    out["corr_stack__in"] = st
    out["corr_stack__out"] = simple.corr(st)
    # cusimple turns the axes positive before picking the mean's axes
    # (cusimple.py:13,17); cpusimple compares the negative defaults and would
    # average over everything, so pass them positive to get cusimple's result
    out["corr_stack_norm__out"] = simple.corr(st, axes=(1, 2), norm=True)
    line = g.exponential(1.0, (4, 30))
    out["corr_line__in"] = line
    out["corr_line__out"] = simple.corr(line, axes=(-1,))
    imgs = g.exponential(1.0, (3, 20, 24)).astype(np.float32)
    mask = (g.uniform(0, 1, (20, 24)) > 0.2).astype(np.float32)
    out["c2d__images"] = imgs
    out["c2d__mask"] = mask
    for name, kw, per_add in (("plain", {}, None), ("mask", {"mask": mask}, None), ("addmask", {}, mask)):
        c = simple.correlator2d(**kw)
        for im in imgs:
            c.add(im, mask=per_add) if per_add is not None else c.add(im)
        out[f"c2d_{name}__mean"] = c.mean
        out[f"c2d_{name}__std"] = c.std
    # power-of-two shapes (the GPU library's own FFTs take these)
    st2 = g.exponential(1.0, (2, 32, 64))
    out["corr_pow2__in"] = st2
    out["corr_pow2__out"] = simple.corr(st2)
    out["corr_pow2_norm__out"] = simple.corr(st2, axes=(1, 2), norm=True)
    imgs2 = g.exponential(1.0, (3, 16, 32)).astype(np.float32)
    mask2 = (g.uniform(0, 1, (16, 32)) > 0.2).astype(np.float32)
    out["c2dp__images"] = imgs2
    out["c2dp__mask"] = mask2
    for name, kw, per_add in (("plain", {}, None), ("mask", {"mask": mask2}, None), ("addmask", {}, mask2)):
        c = simple.correlator2d(**kw)
        for im in imgs2:
            c.add(im, mask=per_add) if per_add is not None else c.add(im)
        out[f"c2dp_{name}__mean"] = c.mean
        out[f"c2dp_{name}__std"] = c.std
    return out


def main():
    if not refshim.available():
        raise SystemExit("reference tree not available")
    ref = refshim.load()
    np.savez_compressed(os.path.join(HERE, "forward_ref.npz"), **make_forward(ref))
    np.savez_compressed(os.path.join(HERE, "time_ref.npz"), **make_time(ref))
    np.savez_compressed(os.path.join(HERE, "detector_ref.npz"), **make_detector(ref))
    np.savez_compressed(os.path.join(HERE, "emitters_ref.npz"), **make_emitters(ref))
    np.savez_compressed(os.path.join(HERE, "fftcorr_ref.npz"), **make_fftcorr(ref))
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
