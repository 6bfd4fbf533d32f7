"""Emitter sources with the reference's duck-typed simobject contract
(``idi/simulation/simobj.py:26-66``): ``.N``, ``.E``, ``.k = 2 pi / (1.24 / E)``,
``.get2() -> (pos (N,3), phase (N,1))``, ``.get() -> (N,4)``,
``rndPos`` / ``rndPhase`` switches.

Host sources (numpy draws, seedable through ``rng``): :class:`sphere` and
:class:`fixed` (injected positions/phases).

Device sources (drawn on the GPU by ``idiwf_emitters`` straight into the
forward's input rows, so the simulate loops never stage emitters through the
host): :class:`gnorm`, :class:`gauss`, :class:`crystal` with :class:`sc`,
:class:`fcc`, :class:`hcp`, :class:`cuso4`, and :class:`foil`, with the
reference's constructors.  ``device_batch(n_images)`` returns the
(n_images * N, 4) rows of the next images; ``get2()`` draws one image on the
device and returns it as numpy arrays.  Every source takes ``seed``; image i
of a source draws the same numbers however the images are batched.
:class:`sphere` draws on the device too when ``ondevice = True``.
"""

from __future__ import annotations

from warnings import warn

import numpy as np
import torch

from .. import _native as nat
from . import _core

__all__ = ["simobj", "sphere", "fixed", "gnorm", "gauss", "crystal", "sc", "fcc", "hcp", "cuso4", "foil"]


class simobj:
    ondevice = False

    def __init__(self, E, N, rng=None):
        self.E = E
        self.rndPhase = True
        self.rndPos = True
        self._N = int(N)
        self._pos = None
        self.rng = rng if rng is not None else np.random.default_rng()

    @property
    def N(self):
        return self._N

    @property
    def k(self):
        return 2 * np.pi / (1.24 / self.E)

    def updatePos(self):
        raise NotImplementedError

    def get2(self):
        if self.rndPos or self._pos is None:
            self._pos = None
            self.updatePos()
        if self.rndPhase:
            phase = self.rng.uniform(0, 2 * np.pi, (self.N, 1))
        else:
            phase = np.zeros((self.N, 1), self._pos.dtype)
        return self._pos, phase

    def get(self):
        ret = np.empty((self.N, 4), order="C")
        np.concatenate(self.get2(), -1, out=ret)
        return ret


class _DeviceDraws:
    """Device generation shared by the sources: a Philox key from the seed,
    one stream per source, and an image counter so image i always draws the
    same numbers.  ``rndPos = False`` keeps the first image's positions."""

    def _init_device(self, seed):
        if seed is None:
            seed = int(np.random.randint(2**63))
        self._key = tuple(int(x) for x in np.random.SeedSequence(int(seed)).generate_state(2, np.uint64))
        self._next_image = 0
        self._held = None  # device positions kept while rndPos is False

    def _desc(self, device):
        """(idiwf_emitters_desc, tensor to keep alive) of one image's draw."""
        raise NotImplementedError

    def device_batch(self, n_images, device=None, out=None):
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        n_images = int(n_images)
        first = self._next_image
        self._next_image += n_images
        if self.rndPos:
            self._held = None
            desc, keep = self._desc(dev)
            desc.random_phase = int(bool(self.rndPhase))
            return _core.emitters(desc, n_images, self.N, self._key, 0, first, dev, out, check=True, keep=keep)
        if self._held is None or self._held.device != dev:
            desc, keep = self._desc(dev)
            desc.random_phase = 0
            self._held = _core.emitters(desc, 1, self.N, self._key, 0, first, dev, check=True,
                                        keep=keep)[:, :3].contiguous()
        desc = _core.emitters_desc(nat.EMIT_FIXED, random_phase=self.rndPhase, sites=self._held)
        return _core.emitters(desc, n_images, self.N, self._key, 0, first, dev, out, keep=self._held)

    def _device_get2(self):
        a = self.device_batch(1).cpu().numpy()
        return np.ascontiguousarray(a[:, :3]), np.ascontiguousarray(a[:, 3:])


class sphere(simobj, _DeviceDraws):
    """N emitters uniform in a ball of radius r (the reference's ``sphere``,
    ``idi/simulation/simobj.py:119-130``).  Host draws from ``rng``; with
    ``ondevice = True`` (or ``device_batch``) the GPU draws them."""

    def __init__(self, E, N, r, rng=None, seed=None):
        self.r = r
        super().__init__(E, N, rng)
        self._init_device(seed if seed is not None else int(self.rng.integers(2**63)))

    def updatePos(self):
        rng = self.rng
        t = rng.uniform(-1, 1, self.N)
        p = rng.uniform(0, 2 * np.pi, self.N)
        u = self.r * rng.uniform(0, 1, self.N) ** (1 / 3)
        s = np.sqrt(1 - t ** 2)
        self._pos = np.stack([u * t, u * s * np.sin(p), u * s * np.cos(p)], -1)

    def _desc(self, device):
        return _core.emitters_desc(nat.EMIT_SPHERE, r=self.r), None

    def get2(self):
        return self._device_get2() if self.ondevice else super().get2()


class fixed(simobj):
    """Fixed positions; phases injected (one row per image, cycled) or random."""

    def __init__(self, E, pos, phases=None, rng=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        super().__init__(E, pos.shape[0], rng)
        self._fixed = pos
        self.rndPos = False
        self._phases = None if phases is None else np.atleast_2d(np.asarray(phases, dtype=np.float64))
        self._i = 0

    def updatePos(self):
        self._pos = self._fixed

    def get2(self):
        self._pos = self._fixed
        if self._phases is None:
            return super().get2()
        ph = self._phases[self._i % len(self._phases)].reshape(self.N, 1)
        self._i += 1
        return self._pos, ph


class _DeviceSource(simobj, _DeviceDraws):
    ondevice = True

    def __init__(self, E, N, seed=None):
        super().__init__(E, N)
        self._init_device(seed)

    def get2(self):
        return self._device_get2()

    def updatePos(self):
        self._held = None


def _rotmatrix(rotangles):
    return _core.rotation(*[float(a) for a in rotangles]) if np.any(rotangles) else None


class gnorm(_DeviceSource):
    """A generalised-normal shaped volume (``idi/simulation/simobj.py:154-176``):
    per axis Gaussian with ``fwhm`` for ``rho == 2``, flatter for larger rho;
    ``fwhm`` and ``rho`` scalars or per axis; positions rotated by ``rotangles``."""

    def __init__(self, E, N, fwhm, rho=2, rotangles=(0, 0, 0), seed=None):
        self.fwhm, self.rho = np.array(fwhm), np.array(rho)
        self._rot = _rotmatrix(rotangles)
        super().__init__(E, N, seed)

    def _desc(self, device):
        return _core.emitters_desc(nat.EMIT_GNORM, fwhm=self.fwhm, rho=self.rho, rot=self._rot), None


class gauss(gnorm):
    """A Gaussian shaped volume (``idi/simulation/simobj.py:178-184``)."""

    def __init__(self, E, N, fwhm, seed=None):
        super().__init__(E, N, fwhm, 2, seed=seed)


class crystal(_DeviceSource):
    """A crystal: ``N`` of the sites of ``repeats`` unit cells, drawn without
    replacement per image (``idi/simulation/simobj.py:357-497``); with ``fwhm``
    the draw is weighted by the generalised-normal envelope of width ``fwhm``
    and shape ``rho``; ``rndOrientation`` True (uniform) or an axis (random
    angle about it) rotates the crystal per image.  The sites are built on
    the host; the per-image rotation, weights and selection run on the GPU."""

    def __init__(self, E, lconst, langle, unitcell, N, repeats=None, rotangles=(0, 0, 0), fwhm=None, rho=2,
                 seed=None):
        if fwhm is not None:
            cosa, cosb, cosc = np.cos(np.array(langle))
            sina, sinb, sinc = np.sin(np.array(langle))
            cell_extent = np.array([1, sinc, np.sqrt(sinb ** 2 - ((cosa - cosb * cosc) / sinc) ** 2)]) * np.array(lconst)
            needed = np.ceil(2 * np.array(fwhm) / cell_extent).astype(int)
            if repeats is not None:
                if np.any(needed > repeats):
                    warn("Number of repeats small for choosen fwhm")
            else:
                repeats = needed
        if repeats is None:
            repeats = 3 * [int(np.rint((N / len(unitcell)) ** (1 / 3.0)))]
        if np.prod(repeats) * len(unitcell) < N:
            warn("Number of atoms high for atoms in focus")
        allpos = crystal._lattice(lconst, langle, unitcell, np.broadcast_to(repeats, (3,)))
        self._rot = _rotmatrix(rotangles)
        if self._rot is not None:
            allpos = np.matmul(self._rot, allpos.T, order="F").T
        self._allpos = allpos
        self._sites = None
        self.rndOrientation = False
        self.fwhm = None if fwhm is None else np.array(fwhm)
        self.rho = np.array(2) if rho is None else np.array(rho)
        super().__init__(E, N, seed)

    @staticmethod
    def _lattice(lconst, langle, unitcell, repeats):
        """Lattice sites, centred, as float32 (the reference's ``crystal._lattice``
        arithmetic, ``simobj.py:417-443`` with sigma = 0: the unit cell in the
        lattice basis, then translations along basis vectors 0, 1, 2 added in
        float32, the last axis outermost)."""
        cosa, cosb, cosc = np.cos(np.array(langle))
        sina, sinb, sinc = np.sin(np.array(langle))
        c2 = (cosa - cosb * cosc) / sinc
        basis = np.array([[1, 0, 0], [cosc, sinc, 0], [cosb, c2, np.sqrt(sinb ** 2 - c2 ** 2)]]) * np.expand_dims(lconst, 1)
        cell = np.dot(unitcell, basis).astype(np.float32)
        shifts = [np.stack([(basis[j] * k).astype(np.float32) for k in range(int(repeats[j]))]) for j in range(3)]
        grid = ((cell[None, None, None, :, :] + shifts[0][None, None, :, None, :])
                + shifts[1][None, :, None, None, :]) + shifts[2][:, None, None, None, :]
        sites = grid.reshape(-1, 3)
        return sites - (np.min(sites, axis=0) + np.max(sites, axis=0)) / 2.0

    def _desc(self, device):
        if self._sites is None or self._sites.device != device:
            self._sites = torch.from_numpy(np.ascontiguousarray(self._allpos, dtype=np.float64)).to(device)
        orient = nat.ORIENT_FIXED
        axis = (0.0, 0.0, 1.0)
        if np.any(self.rndOrientation):
            if np.size(self.rndOrientation) == 3:
                orient, axis = nat.ORIENT_AXIS, tuple(np.asarray(self.rndOrientation, np.float64))
            else:
                orient = nat.ORIENT_RANDOM
        rot = self._rot if (orient != nat.ORIENT_FIXED and self._rot is not None) else None
        weighted = self.fwhm is not None
        desc = _core.emitters_desc(nat.EMIT_SITES, orientation=orient, axis=axis, rot=rot, weighted=weighted,
                                   fwhm=self.fwhm if weighted else 1.0, rho=self.rho, sites=self._sites)
        return desc, self._sites


class sc(crystal):
    """Simple cubic crystal (``idi/simulation/simobj.py:499-508``)."""

    def __init__(self, E, N, a, repeats=None, rotangles=(0, 0, 0), fwhm=None, rho=None, seed=None):
        super().__init__(E, [a, a, a], np.array([90, 90, 90]) * np.pi / 180.0, [[0, 0, 0]], N, repeats, rotangles,
                         fwhm, rho, seed)


class fcc(crystal):
    """Face-centred cubic crystal (``idi/simulation/simobj.py:511-520``)."""

    def __init__(self, E, N, a, repeats=None, rotangles=(0, 0, 0), fwhm=None, rho=None, seed=None):
        cell = [[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]
        super().__init__(E, [a, a, a], np.array([90, 90, 90]) * np.pi / 180.0, cell, N, repeats, rotangles, fwhm,
                         rho, seed)


class hcp(crystal):
    """Hexagonal close-packed crystal (``idi/simulation/simobj.py:523-532``)."""

    def __init__(self, E, N, a, repeats=None, rotangles=(0, 0, 0), fwhm=None, rho=None, seed=None):
        cell = [[0, 0, 0], [1.0 / 3, 2.0 / 3, 1.0 / 2]]
        super().__init__(E, [a, a, 1.633 * a], np.array([90, 90, 120]) * np.pi / 180.0, cell, N, repeats, rotangles,
                         fwhm, rho, seed)


class cuso4(crystal):
    """CuSO4 lattice with its fixed lattice constants (``idi/simulation/simobj.py:535-545``)."""

    def __init__(self, N, E, repeats=None, rotangles=(0, 0, 0), fwhm=None, rho=None, seed=None):
        cell = [[0, 0, 0], [0.5, 0.5, 0]]
        lconst = np.array([6.141, 10.736, 5.986]) * 1e-4
        langle = np.array([82.27, 107.43, 102.67]) * np.pi / 180.0
        super().__init__(E, lconst, langle, cell, N, repeats, rotangles, fwhm, rho, seed)


class foil(_DeviceSource):
    """A foil (``idi/simulation/simobj.py:703-776``): in-plane generalised normal
    of width ``fwhm`` and shape ``rho``, depth uniform through the foil or
    truncated-exponential with ``attenuationlength``, tilted by ``rotangles``;
    N follows from the excitation density as in the reference."""

    def __init__(self, E, excitation, thickness, fwhm, attenuationlength=np.inf, rho=(2, 2), rotangles=(0, 0, 0),
                 seed=None):
        from math import exp, log

        from scipy.special import gamma

        self._rotmatrix = _core.rotation(*[float(a) for a in rotangles])
        self._rotangles = rotangles
        self._thickness = thickness
        self._attenuationlength = attenuationlength
        self._fwhm = (fwhm * np.array((1, 1)))[:, None]
        self._rho = (rho * np.array((1, 1)))[:, None]
        path = thickness / self._rotmatrix[-1, -1]
        depth_factor = path if np.isinf(attenuationlength) else (
            attenuationlength - attenuationlength / exp(path / attenuationlength))
        N = int(np.prod(self._fwhm * gamma(1 + 1 / self._rho) * log(2) ** (-1 / self._rho)) * depth_factor * excitation)
        super().__init__(E, N, seed)

    def _desc(self, device):
        return _core.emitters_desc(nat.EMIT_FOIL, fwhm=self._fwhm.ravel(), rho=self._rho.ravel(),
                                   depth=self._thickness / self._rotmatrix[-1, -1],
                                   attenuation=self._attenuationlength, rot=self._rotmatrix), None

    @property
    def fwhm(self):
        return self._fwhm.ravel()

    @property
    def thickness(self):
        return self._thickness

    @property
    def rho(self):
        return self._rho.ravel()

    @property
    def attenuationlength(self):
        return self._attenuationlength

    @property
    def rotangles(self):
        return self._rotangles
