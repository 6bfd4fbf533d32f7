"""The near-field bound behind the split kernels' path choice, on the CPU.

With s = d_hat . r, r_perp^2 = |r|^2 - s^2 and L = |d - r|, the path
difference is exactly |d - r| - |d| = -s + N with N = r_perp^2 / (|d| + L - s).
The split kernels use N ~ r_perp^2 / (2|d|) where the remainder
R = N - r_perp^2 / (2|d|) is small; the classifier bounds it per image by
kNfBoundC r^3 / D^2 for r = max |r| <= D / 4 and D = the detector plane's
distance from the origin (a lower bound on every |d|).  These tests check the
identity and the bound over random emitters and tilted, offset detectors,
with the constants read from the library's source.
"""

import os
import re

import numpy as np
import pytest

from tests.helpers import rng

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "idi_b200", "csrc",
                   "idiwf_internal.cuh")


def _const(name):
    m = re.search(rf"constexpr double {name} = ([0-9.eE+-]+);", open(HDR).read())
    assert m, name
    return float(m.group(1))


def _split(d, r):
    D = np.linalg.norm(d, axis=-1)
    s = (d * r).sum(-1) / D
    rp = (r * r).sum(-1) - s * s
    L = np.linalg.norm(d - r, axis=-1)
    return D, s, rp, L


def test_exact_identity():
    g = rng(3)
    d = g.normal(0, 1, (20000, 3)) * [50.0, 50.0, 10.0] + [0, 0, 1000.0]
    r = g.normal(0, 40.0, (20000, 3))
    D, s, rp, L = _split(d, r)
    N = rp / (D + L - s)
    assert np.allclose(L - D, -s + N, rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("seed", range(4))
def test_remainder_bound_holds(seed):
    """|R| <= kNfBoundC r^3 / D^2 for every emitter with |r| <= r <= D/4 and
    every pixel of a tilted, offset detector whose plane is D from the origin."""
    c = _const("kNfBoundC")
    g = rng(100 + seed)
    for _ in range(20):
        # random detector plane: normal n, distance D; pixels spread over it
        n = g.normal(0, 1, 3)
        n /= np.linalg.norm(n)
        Dp = g.uniform(100.0, 1e5)
        u = np.cross(n, [1.0, 0, 0] if abs(n[0]) < 0.9 else [0, 1.0, 0])
        u /= np.linalg.norm(u)
        v = np.cross(n, u)
        a, b = g.uniform(-3, 3, (2, 400)) * Dp
        d = Dp * n + a[:, None] * u + b[:, None] * v
        rho = g.uniform(1e-3, 0.25)
        rmax = rho * Dp
        # emitters inside the ball, many on its surface (where the bound is tight)
        r = g.normal(0, 1, (400, 3))
        r *= (rmax * np.where(g.uniform(size=400) < 0.5, 1.0, g.uniform(size=400) ** (1 / 3))
              / np.linalg.norm(r, axis=1))[:, None]
        dd, rr = np.broadcast_arrays(d[:, None, :], r[None, :, :])
        D, s, rp, L = _split(dd, rr)
        R = rp / (D + L - s) - rp / (2 * D)
        assert np.all(np.abs(R) <= c * rmax ** 3 / Dp ** 2), (rho, np.abs(R).max() / (rmax ** 3 / Dp ** 2))


def test_bound_is_close_to_tight_for_small_objects():
    """At r << D the largest remainder approaches r^3 / (3 sqrt(3) D^2) on the
    axis pixel: the classifier's constant is conservative by less than 2x."""
    c = _const("kNfBoundC")
    Dp, rmax = 1e4, 1.0
    d = np.array([0.0, 0.0, Dp])
    t = np.linspace(-1, 1, 20001)
    r = rmax * np.stack([np.sqrt(1 - t * t), np.zeros_like(t), t], -1)
    D, s, rp, L = _split(np.broadcast_to(d, r.shape), r)
    R = np.abs(rp / (D + L - s) - rp / (2 * D)).max()
    tight = rmax ** 3 / (3 * np.sqrt(3) * Dp ** 2)
    assert abs(R / tight - 1) < 1e-3
    assert 1.0 < c / (1 / (3 * np.sqrt(3))) < 2.0


def test_paths_for_the_configured_workloads():
    """The classifier's decision for the benchmark workloads and the near-field
    test geometries: every benchmark configuration stays on the second-order
    paths; the reference's unit-test geometry takes the exact path."""
    c, tol, emax = _const("kNfBoundC"), _const("kNfPhaseTol"), _const("kExactMaxPhase")

    def path(E_ev, r, detz):
        k = 2 * np.pi / (1.24 / E_ev)
        rho2 = (r / detz) ** 2
        t = c * k * r ** 3 / detz ** 2
        if not (rho2 <= 1 / 16 and t <= emax):
            return "reject"
        return "second-order" if t <= tol else "exact"

    # fcc 12 nm cube (half-diagonal 10.4 nm) at 0.2 m, 8 keV; spheres of 10-25 nm at 0.1 m, 6.4 keV
    assert path(8000, 0.0104, 2e5) == "second-order"
    for r in (0.01, 0.015, 0.025):
        assert path(6400, r, 1e5) == "second-order"
    assert path(100, 10.0, 1000.0) == "exact"    # sphere(100, 100, 10) at 1000 um
    assert path(8000, 1.0, 1e4) == "exact"       # 1 um at 1 cm
    assert path(100, 100.0, 1000.0) == "reject"  # 100 um at 1000 um
