"""Drop-in for ``idi.simulation.cutime`` / ``idi.simulation.time``: the
time-dependent direct sum (``idi/simulation/cutime.py:9-193``,
``idi/simulation/time.py:48-122``).

The whole computation runs in FP64 on the GPU (the reference's
``double|single|mixed`` precision substrings and ``threads`` are accepted and
ignored: there is one precision, and the kernel sorts each pixel on chip).
Emission times are drawn as the reference draws them,
``np.random.randn(N) * (pulsewidth / 2.35)`` after ``simobject.get()``, unless
``times=`` injects them.  Far field follows ``time.py``; ``"nf"`` follows the
near-field arrival time of ``simtime.cu:58-79``.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _core

__all__ = ["simulate", "simulate_gen"]


def simulate(
    simobject,
    Ndet,
    pixelsize,
    detz,
    k,
    c,
    tau,
    pulsewidth,
    detangles=(0, 0),
    settings="mixed",
    threads=None,
    *args,
    times=None,
    returngpu=False,
    device=None,
    **kwargs,
):
    """Time-dependent intensity, float64 (Nx, Ny) (``idi/simulation/time.py:48-98``)."""
    flags, _, _ = _core.parse_settings(settings)
    flags &= ~_core.nat.SECONDORDER
    Ndet = _core.ndet_pair(Ndet)
    geom = _core.make_geom(Ndet, pixelsize, detz, k, detangles, (0, 0), flags)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    data = np.ascontiguousarray(simobject.get(), dtype=np.float64)
    if times is None:
        times = np.random.randn(simobject.N) * (pulsewidth / 2.35)
    d_atoms = torch.from_numpy(data).to(dev)
    d_times = torch.from_numpy(np.ascontiguousarray(times, dtype=np.float64)).to(dev)
    out = _core.time_forward(d_atoms, d_times, geom, c, tau)
    if returngpu:
        return out
    return out.cpu().numpy()


def simulate_gen(
    simobject,
    Ndet,
    pixelsize,
    detz,
    k,
    c,
    tau,
    pulsewidth,
    detangles=(0, 0),
    settings="mixed",
    threads=None,
    maximg=np.inf,
    *args,
    **kwargs,
):
    """Generator over :func:`simulate` (``idi/simulation/cutime.py:142-193``)."""
    i = 0
    while i < maximg:
        yield simulate(simobject, Ndet, pixelsize, detz, k, c, tau, pulsewidth, detangles, settings, threads,
                       *args, **kwargs)
        i += 1
