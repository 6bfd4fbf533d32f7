"""Emitter sources with the reference's duck-typed simobject contract
(``idi/simulation/simobj.py:26-66``): ``.N``, ``.E``, ``.k = 2 pi / (1.24 / E)``,
``.get2() -> (pos (N,3), phase (N,1))``, ``.get() -> (N,4)``,
``rndPos`` / ``rndPhase`` switches.

Only the contract and two sources are provided: :class:`sphere` (uniform in a
ball, seedable) and :class:`fixed` (injected positions/phases, e.g. for
reproducible benchmarks).  The reference's other geometry generators are host
code outside the direct-sum path; any object with this contract works.
"""

from __future__ import annotations

import numpy as np

__all__ = ["simobj", "sphere", "fixed"]


class simobj:
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


class sphere(simobj):
    """N emitters uniform in a ball of radius r (the reference's ``sphere``)."""

    def __init__(self, E, N, r, rng=None):
        self.r = r
        super().__init__(E, N, rng)

    def updatePos(self):
        rng = self.rng
        t = rng.uniform(-1, 1, self.N)
        p = rng.uniform(0, 2 * np.pi, self.N)
        u = self.r * rng.uniform(0, 1, self.N) ** (1 / 3)
        s = np.sqrt(1 - t ** 2)
        self._pos = np.stack([u * t, u * s * np.sin(p), u * s * np.cos(p)], -1)


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
