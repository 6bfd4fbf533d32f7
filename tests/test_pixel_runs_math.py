"""The geometry behind the split forward's pixel runs, on the CPU.

A run of 4 pixels along a detector row shares one FP64 phase taken at the
run's middle; pixel i adds the FP32 offset D_i . r with
D_i = -k (d_hat_i - d_hat_base).  An image uses runs only when
k * run_span * |r|max <= 1 rad, where run_span (computed by the library's
host code from the detector rotation, pixel size and distance) must bound
|d_hat_i - d_hat_base| for every run of the detector.  These tests restate
run_span and check that bound over random detector tilts and offsets, and
check the decomposition of the phase against the per-pixel FP64 phase.
"""

import numpy as np
import pytest

import oracle


def _run_span(rot, pixelsize, detz):
    # half a run (1.5 pixels along the row direction c1) over the distance of
    # the detector plane {px c0 + py c1 + detz c2} from the origin
    c0, c1, c2 = rot[:, 0], rot[:, 1], rot[:, 2]
    n = np.cross(c0, c1)
    h = abs(detz * np.dot(c2, n)) / np.linalg.norm(n)
    return 1.5 * abs(pixelsize) * np.linalg.norm(c1) / h


def _pixels(nx, ny, pixelsize, detz, rot, off, fiy=None):
    ix, iy = np.meshgrid(np.arange(nx, dtype=np.float64), np.arange(ny, dtype=np.float64), indexing="ij")
    if fiy is not None:
        iy = fiy
    px = (ix - nx * 0.5) * pixelsize + off[0]
    py = (iy - ny * 0.5) * pixelsize + off[1]
    pz = np.full_like(px, detz)
    d = np.stack([px, py, pz], -1) @ rot.T
    return d / np.linalg.norm(d, axis=-1, keepdims=True)


@pytest.mark.parametrize("seed", range(6))
def test_run_span_bounds_every_run(seed):
    g = np.random.default_rng(seed)
    nx, ny = 24, 32
    pixelsize = g.uniform(20.0, 200.0)
    detz = g.uniform(2e4, 2e5)
    angles = (g.uniform(-0.4, 0.4), g.uniform(-np.pi, np.pi))
    off = tuple(g.uniform(-3e4, 3e4, 2))
    rot = np.asarray(oracle.rotation(angles[0], angles[1], 0), dtype=np.float64)
    span = _run_span(rot, pixelsize, detz)
    dhat = _pixels(nx, ny, pixelsize, detz, rot, off)
    # middle of each aligned run of 4 pixels along a row
    iy_mid = np.repeat(np.arange(0, ny, 4, dtype=np.float64) + 1.5, 4)[None, :].repeat(nx, 0)
    base = _pixels(nx, ny, pixelsize, detz, rot, off, fiy=iy_mid)
    worst = np.linalg.norm(dhat - base, axis=-1).max()
    assert worst <= span * (1 + 1e-12), (worst, span)
    assert worst >= 0.5 * span  # the bound is not loose by more than the paraxial factor


def test_run_offsets_reproduce_the_per_pixel_phase():
    """phi_i = phi_base + D_i . r with D_i and r rounded to FP32 and the dot
    product in FP32: within 2e-7 rad of the FP64 phase when |D_i . r| <= 1."""
    g = np.random.default_rng(7)
    k = 2 * np.pi / (1.24 / 6400.0)
    pixelsize, detz = 75.0, 1e5
    rot = np.eye(3)
    nx, ny = 8, 16
    dhat = _pixels(nx, ny, pixelsize, detz, rot, (0.0, 0.0))
    iy_mid = np.repeat(np.arange(0, ny, 4, dtype=np.float64) + 1.5, 4)[None, :].repeat(nx, 0)
    base = _pixels(nx, ny, pixelsize, detz, rot, (0.0, 0.0), fiy=iy_mid)
    span = _run_span(rot, pixelsize, detz)
    rmax = 1.0 / (k * span)  # the largest object the runs accept
    r = g.normal(size=(500, 3))
    r *= (rmax * g.uniform(0, 1, (500, 1)) ** (1 / 3)) / np.linalg.norm(r, axis=1, keepdims=True)
    phi_pix = -k * (dhat.reshape(-1, 3) @ r.T)            # -k d_hat . r, FP64
    phi_base = -k * (base.reshape(-1, 3) @ r.T)
    D = (-k * (dhat - base)).reshape(-1, 3).astype(np.float32)
    off32 = (D[:, None, :] * r.astype(np.float32)[None, :, :]).sum(-1, dtype=np.float32)
    assert np.abs(off32).max() <= 1.0 + 1e-6
    err = np.abs((phi_base + off32.astype(np.float64)) - phi_pix)
    assert err.max() < 2e-7, err.max()
