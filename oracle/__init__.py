"""ORACLE — test infrastructure only.

CPU restatement of the reference's emitter-wavefield direct sum (plain C in
``wavefield_oracle.c``, built into ``liboracle.so`` by ``oracle/Makefile``) with a
numpy/ctypes front end.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it, and only as the checker or as the
timed CPU baseline; the ``idi_b200`` package never imports it.

Parity of this restatement with the reference itself is pinned by
``tests/test_oracle.py`` (executes the reference's numba code through
``oracle/refshim.py`` where the reference tree is present) and by the committed
fixtures in ``tests/golden/`` (produced by ``tests/golden/make_golden.py`` from
the reference's own ``cpu.simulate`` / ``time.simulate``).
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

NF = 1
SCALE = 2
SECONDORDER = 4
ACCURATE = 8


class OrcGeom(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("pixelsize", ctypes.c_double),
        ("detz", ctypes.c_double),
        ("k", ctypes.c_double),
        ("offx", ctypes.c_double),
        ("offy", ctypes.c_double),
        ("rot", ctypes.c_double * 9),
        ("has_rot", ctypes.c_int32),
    ]


def build(force: bool = False) -> str:
    srcs = [os.path.join(_HERE, f) for f in ("wavefield_oracle.c", "detector_oracle.c", "emitters_oracle.c",
                                              "qcorr_oracle.c", "philox_oracle.h")]
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < max(map(os.path.getmtime, srcs)):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        d = ctypes.c_double
        vp = ctypes.c_void_p
        L.orc_wavefield.argtypes = [P(OrcGeom), ctypes.c_int, vp, vp, ctypes.c_int64, vp]
        L.orc_wavefield.restype = None
        L.orc_adjoint.argtypes = [P(OrcGeom), ctypes.c_int, vp, vp, ctypes.c_int64, vp, vp, vp, vp, vp]
        L.orc_adjoint.restype = d
        L.orc_time_image.argtypes = [P(OrcGeom), ctypes.c_int, vp, vp, ctypes.c_int64, d, d, vp]
        L.orc_time_image.restype = None
        L.orc_time_image_digest.argtypes = [P(OrcGeom), ctypes.c_int, vp, vp, ctypes.c_int64, d, d, vp, vp, vp]
        L.orc_time_image_digest.restype = None
        L.orc_time_order.argtypes = [P(OrcGeom), ctypes.c_int, vp, vp, ctypes.c_int64, d,
                                     ctypes.c_int, ctypes.c_int, vp]
        L.orc_time_order.restype = None
        L.orc_time_keys.argtypes = [P(OrcGeom), ctypes.c_int, vp, vp, ctypes.c_int64, d,
                                    ctypes.c_int, ctypes.c_int, vp, vp, vp]
        L.orc_time_keys.restype = None
        u64 = ctypes.c_uint64
        L.orc_philox4x64.argtypes = [vp, vp, vp]
        L.orc_philox4x64.restype = None
        L.orc_uniforms.argtypes = [u64, u64, u64, u64, u64, ctypes.c_int64, vp]
        L.orc_uniforms.restype = None
        L.orc_image_sum.argtypes = [vp, ctypes.c_int64]
        L.orc_image_sum.restype = d
        L.orc_photons.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, d, u64, u64, u64, u64, vp, vp]
        L.orc_photons.restype = None
        L.orc_chargesharing.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, d, d, u64, u64, u64,
                                        u64, vp, vp, vp]
        L.orc_chargesharing.restype = None
        L.orc_emit.argtypes = [ctypes.c_int, ctypes.c_int32, ctypes.c_int64, d, vp, vp, d, d, vp, ctypes.c_int,
                               u64, u64, u64, u64, vp]
        L.orc_emit.restype = None
        L.orc_site_rotation.argtypes = [ctypes.c_int, vp, vp, u64, u64, u64, u64, vp]
        L.orc_site_rotation.restype = None
        L.orc_emit_sites.argtypes = [vp, ctypes.c_int64, ctypes.c_int32, ctypes.c_int64, ctypes.c_int, vp, vp,
                                     ctypes.c_int, vp, vp, ctypes.c_int, u64, u64, u64, u64, vp, vp]
        L.orc_emit_sites.restype = None
        L.orc_site_weights.argtypes = [vp, ctypes.c_int64, vp, vp, vp, vp]
        L.orc_site_weights.restype = None
        i32 = ctypes.c_int32
        L.orc_qcorr_radial.argtypes = [vp, vp, i32, i32, i32, i32, vp]
        L.orc_qcorr_radial.restype = None
        L.orc_qcorr_3d.argtypes = [vp, vp, i32, i32, i32, i32, i32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                   vp]
        L.orc_qcorr_3d.restype = None
        _lib = L
    return _lib


def rotation(alpha, beta, gamma):
    """Restatement of ``idi/util/__init__.py:348-372`` (yaw-pitch-roll matrix)."""
    cosa, cosb, cosg = math.cos(alpha), math.cos(beta), math.cos(gamma)
    sina, sinb, sing = math.sin(alpha), math.sin(beta), math.sin(gamma)
    return np.array(
        [
            [cosb * cosg, sina * sinb * cosg - cosa * sing, cosa * sinb * cosg + sina * sing],
            [cosb * sing, sina * sinb * sing + cosa * cosg, cosa * sinb * sing - sina * cosg],
            [-sinb, sina * cosb, cosa * cosb],
        ]
    )


def flags_from_settings(settings: str) -> int:
    f = 0
    if "nf" in settings:
        f |= NF
    if "scale" in settings:
        f |= SCALE
    if "secondorder" in settings:
        f |= SECONDORDER
    return f


def geometry(Ndet, pixelsize, detz, k, detangles=(0, 0), detoffset=(0, 0)) -> OrcGeom:
    if np.size(Ndet) == 1:
        Ndet = [int(np.ravel([Ndet])[0])] * 2
    g = OrcGeom()
    g.nx, g.ny = int(Ndet[0]), int(Ndet[1])
    g.pixelsize, g.detz, g.k = float(pixelsize), float(detz), float(k)
    g.offx, g.offy = float(detoffset[0]), float(detoffset[1])
    if np.any(detangles):
        M = rotation(detangles[0], detangles[1], 0)
        g.has_rot = 1
    else:
        M = np.eye(3)
        g.has_rot = 0
    for i, v in enumerate(M.ravel()):
        g.rot[i] = float(v)
    return g


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def wavefield(g: OrcGeom, flags: int, atoms, amp=None) -> np.ndarray:
    """One image: complex128 (nx, ny) field, following ``cpu.py:73-107``."""
    atoms = _c(atoms)
    assert atoms.ndim == 2 and atoms.shape[1] == 4
    out = np.empty((g.nx, g.ny), np.complex128)
    a = None if amp is None else _c(amp)
    lib().orc_wavefield(ctypes.byref(g), int(flags), atoms.ctypes.data,
                        None if a is None else a.ctypes.data, atoms.shape[0], out.ctypes.data)
    return out


def adjoint(g: OrcGeom, flags: int, atoms, amp, E, target):
    """FP64 gradients of L = sum (|E|^2 - target)^2; returns (loss, dpos, dpsi, damp)."""
    atoms = _c(atoms)
    n = atoms.shape[0]
    E = np.ascontiguousarray(E, np.complex128)
    T = _c(target)
    a = None if amp is None else _c(amp)
    gpos = np.zeros((n, 3))
    gpsi = np.zeros(n)
    gamp = np.zeros(n)
    loss = lib().orc_adjoint(ctypes.byref(g), int(flags), atoms.ctypes.data,
                             None if a is None else a.ctypes.data, n, E.ctypes.data, T.ctypes.data,
                             gpos.ctypes.data, gpsi.ctypes.data, gamp.ctypes.data)
    return loss, gpos, gpsi, gamp


def time_image(g: OrcGeom, flags: int, atoms, times, c, tau) -> np.ndarray:
    """Time-dependent intensity (nx, ny), following ``time.py:48-98``."""
    atoms = _c(atoms)
    times = _c(times)
    out = np.empty((g.nx, g.ny), np.float64)
    lib().orc_time_image(ctypes.byref(g), int(flags), atoms.ctypes.data, times.ctypes.data,
                         atoms.shape[0], float(c), float(tau), out.ctypes.data)
    return out


DIGEST_BASE = 0x9E3779B97F4A7C15


def order_digest(order) -> int:
    """sum_m (order[m] + 1) B^m mod 2^64: the per-pixel order digest of
    ``time_image_digest`` (python, for small cases)."""
    h, pw, mask = 0, 1, (1 << 64) - 1
    for j in np.asarray(order, dtype=np.int64):
        h = (h + (int(j) + 1) * pw) & mask
        pw = (pw * DIGEST_BASE) & mask
    return h


def time_image_digest(g: OrcGeom, flags: int, atoms, times, c, tau):
    """``time_image`` plus, per pixel, the digest of the sorted emitter order
    (``order_digest``) and the number of equal neighbouring keys (ties)."""
    atoms = _c(atoms)
    times = _c(times)
    out = np.empty((g.nx, g.ny), np.float64)
    dig = np.empty((g.nx, g.ny), np.uint64)
    ties = np.empty((g.nx, g.ny), np.int64)
    lib().orc_time_image_digest(ctypes.byref(g), int(flags), atoms.ctypes.data, times.ctypes.data,
                                atoms.shape[0], float(c), float(tau), out.ctypes.data, dig.ctypes.data,
                                ties.ctypes.data)
    return out, dig, ties


def time_order(g: OrcGeom, flags: int, atoms, times, c, ix, iy) -> np.ndarray:
    atoms = _c(atoms)
    times = _c(times)
    order = np.empty(atoms.shape[0], np.int64)
    lib().orc_time_order(ctypes.byref(g), int(flags), atoms.ctypes.data, times.ctypes.data,
                         atoms.shape[0], float(c), int(ix), int(iy), order.ctypes.data)
    return order


def time_keys(g: OrcGeom, flags: int, atoms, times, c, ix, iy):
    atoms = _c(atoms)
    times = _c(times)
    n = atoms.shape[0]
    t = np.empty(n)
    er = np.empty(n)
    ei = np.empty(n)
    lib().orc_time_keys(ctypes.byref(g), int(flags), atoms.ctypes.data, times.ctypes.data, n,
                        float(c), int(ix), int(iy), t.ctypes.data, er.ctypes.data, ei.ctypes.data)
    return t, er + 1j * ei


def intensity_metrics(I, I_ref, floor=1e-3):
    """Error statistics used by every parity test and by the bench record.

    Per-pixel relative error is ill-conditioned at speckle minima, so two
    figures are reported: the max of |dI|/I_ref over pixels with
    I_ref >= floor * mean(I_ref), and the max of |dI|/mean(I_ref) over all
    pixels; plus the 50/99/99.99 percentiles of |dI|/I_ref over the masked set.
    """
    I = np.asarray(I, np.float64)
    I_ref = np.asarray(I_ref, np.float64)
    mean = float(np.mean(I_ref))
    d = np.abs(I - I_ref)
    mask = I_ref >= floor * mean
    rel = d[mask] / I_ref[mask]
    return {
        "max_rel_masked": float(rel.max()) if rel.size else 0.0,
        "max_rel_to_mean": float(d.max() / mean) if mean > 0 else float(d.max()),
        "p50": float(np.percentile(rel, 50)) if rel.size else 0.0,
        "p99": float(np.percentile(rel, 99)) if rel.size else 0.0,
        "p9999": float(np.percentile(rel, 99.99)) if rel.size else 0.0,
        "masked_fraction": float(mask.mean()),
        "floor": floor,
    }


# ---------------------------------------------------------------------------
# detector stage (detector_oracle.c)
# ---------------------------------------------------------------------------
def philox4x64(counter, key) -> np.ndarray:
    """One Philox4x64-10 block: four uint64 words for a 4-word counter and 2-word key."""
    c = _c(np.asarray(counter, dtype=np.uint64), np.uint64)
    k = _c(np.asarray(key, dtype=np.uint64), np.uint64)
    out = np.empty(4, np.uint64)
    lib().orc_philox4x64(c.ctypes.data, k.ctypes.data, out.ctypes.data)
    return out


def uniforms(c1, c2, c3, key, n) -> np.ndarray:
    """First n uniform doubles of the stream with counter (0, c1, c2, c3)."""
    out = np.empty(int(n), np.float64)
    lib().orc_uniforms(int(c1), int(c2), int(c3), int(key[0]), int(key[1]), int(n), out.ctypes.data)
    return out


def image_sum(img) -> float:
    """Sum of one image in the device's fixed reduction tree."""
    a = _c(np.ravel(img))
    return float(lib().orc_image_sum(a.ctypes.data, a.size))


def photons(probs, n_photons, key, stream=0, return_rates=False, first_image=0):
    """Poisson counts (float64) of ``probs`` (..., nx, ny) restating common.py:11-23
    with the device's per-pixel streams; optionally also the rates."""
    p = _c(probs)
    shape = p.shape
    npix = shape[-1] * shape[-2]
    B = int(p.size // npix)
    counts = np.empty(p.size, np.float64)
    rates = np.empty(p.size, np.float64) if return_rates else None
    lib().orc_photons(p.ctypes.data, B, npix, float(n_photons), int(key[0]), int(key[1]), int(stream),
                      int(first_image), counts.ctypes.data, rates.ctypes.data if rates is not None else None)
    counts = counts.reshape(shape)
    return (counts, rates.reshape(shape)) if return_rates else counts


def chargesharing(counts, s, ns=0.0, key=(0, 0), stream=0, positions=None, scales=None, first_image=0) -> np.ndarray:
    """Charge sharing of integer counts (..., nx, ny), restating the scatter loop of
    common.py:49-67; photon offsets injected (``positions``, ``scales``) or drawn
    from the device's streams."""
    c = _c(np.asarray(counts).astype(np.int64), np.int64)
    shape = c.shape
    nx, ny = shape[-2], shape[-1]
    B = int(c.size // (nx * ny))
    out = np.empty(c.size, np.float64)
    pos = _c(positions) if positions is not None else None
    sc = _c(scales) if scales is not None else None
    lib().orc_chargesharing(c.ctypes.data, B, nx, ny, float(s), float(ns), int(key[0]), int(key[1]), int(stream),
                            int(first_image), pos.ctypes.data if pos is not None else None, sc.ctypes.data if sc is not None else None,
                            out.ctypes.data)
    return out.reshape(shape)


# ---------------------------------------------------------------------------
# emitter sources (emitters_oracle.c)
# ---------------------------------------------------------------------------
EMIT_KINDS = {"sphere": 0, "gnorm": 1, "foil": 2}


def _v3(x, pad):
    a = np.atleast_1d(np.asarray(x, np.float64)).ravel()
    if a.size == 1:
        a = np.repeat(a, 3)
    return _c(np.concatenate([a[:3], np.full(max(0, 3 - a.size), pad)]))


def emit(kind, n_images, n, key, stream=0, first_image=0, r=0.0, fwhm=1.0, rho=2.0, depth=0.0,
         attenuation=np.inf, rot=None, random_phase=True) -> np.ndarray:
    """(n_images * n, 4) rows of the sphere / gnorm / foil sources."""
    out = np.empty((int(n_images) * int(n), 4))
    f, g = _v3(fwhm, 1.0), _v3(rho, 2.0)
    M = _c(np.eye(3) if rot is None else np.asarray(rot, np.float64).reshape(3, 3))
    lib().orc_emit(EMIT_KINDS[kind], int(n_images), int(n), float(r), f.ctypes.data, g.ctypes.data, float(depth),
                   float(attenuation), M.ctypes.data, int(bool(random_phase)), int(key[0]), int(key[1]), int(stream),
                   int(first_image), out.ctypes.data)
    return out


def site_rotation(orientation, key, stream=0, image=0, axis=(0, 0, 1), rot=None) -> np.ndarray:
    M = np.empty(9)
    ax = _c(np.asarray(axis, np.float64))
    R = _c(np.eye(3) if rot is None else np.asarray(rot, np.float64).reshape(3, 3))
    lib().orc_site_rotation(int(orientation), ax.ctypes.data, R.ctypes.data, int(key[0]), int(key[1]), int(stream),
                            int(image), M.ctypes.data)
    return M.reshape(3, 3)


def emit_sites(sites, n_images, n, key, stream=0, first_image=0, weighted=False, fwhm=1.0, rho=2.0, orientation=0,
               axis=(0, 0, 1), rot=None, random_phase=True):
    """(rows (n_images * n, 4), selected site index per row) of the lattice-site subsample."""
    s = _c(sites)
    out = np.empty((int(n_images) * int(n), 4))
    sel = np.empty(int(n_images) * int(n), np.int64)
    f, g = _v3(fwhm, 1.0), _v3(rho, 2.0)
    ax = _c(np.asarray(axis, np.float64))
    R = _c(np.eye(3) if rot is None else np.asarray(rot, np.float64).reshape(3, 3))
    lib().orc_emit_sites(s.ctypes.data, s.shape[0], int(n_images), int(n), int(bool(weighted)), f.ctypes.data,
                         g.ctypes.data, int(orientation), ax.ctypes.data, R.ctypes.data, int(bool(random_phase)),
                         int(key[0]), int(key[1]), int(stream), int(first_image), out.ctypes.data, sel.ctypes.data)
    return out, sel


def site_weights(sites, fwhm, rho=2.0, rot=None) -> np.ndarray:
    s = _c(sites)
    w = np.empty(s.shape[0])
    f, g = _v3(fwhm, 1.0), _v3(rho, 2.0)
    R = _c(np.eye(3) if rot is None else np.asarray(rot, np.float64).reshape(3, 3))
    lib().orc_site_weights(s.ctypes.data, s.shape[0], R.ctypes.data, f.ctypes.data, g.ctypes.data, w.ctypes.data)
    return w


# ---------------------------------------------------------------------------
# direct q-space correlators (qcorr_oracle.c)
# ---------------------------------------------------------------------------
def qcorr_radial(q, images, qmax) -> np.ndarray:
    """(B, qmax) radial correlation; q (nr*nc, 4) float32, images (B, nr, nc)."""
    qq = _c(q, np.float32)
    im = _c(images, np.float32)
    if im.ndim == 2:
        im = im[None]
    B, nr, nc = im.shape
    out = np.empty((B, int(qmax)))
    lib().orc_qcorr_radial(qq.ctypes.data, im.ctypes.data, B, nr, nc, int(qmax), out.ctypes.data)
    return out


def qcorr_3d(zd, images, qmax, maxdqz, xcenter, ycenter, z) -> np.ndarray:
    """(B, 2 maxdqz, 2 qmax, 2 qmax) 3d correlation; zd (nr, nc) float32."""
    zz = _c(zd, np.float32)
    im = _c(images, np.float32)
    if im.ndim == 2:
        im = im[None]
    B, nr, nc = im.shape
    out = np.empty((B, 2 * int(maxdqz), 2 * int(qmax), 2 * int(qmax)))
    lib().orc_qcorr_3d(zz.ctypes.data, im.ctypes.data, B, nr, nc, int(qmax), int(maxdqz), float(xcenter),
                       float(ycenter), float(z), out.ctypes.data)
    return out
