"""Drop-in for ``idi.simulation.cuda`` (and ``idi.simulation.cpu``):
``simulate`` / ``simulate_gen`` with the reference's argument layout
(``idi/simulation/cuda.py:16-202``, ``idi/simulation/cpu.py:112-212``).

Differences from the reference, all additive:

* ``settings`` also accepts ``"split"`` (split-precision kernel, complex128
  output).  ``"single"`` runs the split-precision kernel with complex64 output
  (more accurate and faster than the reference's all-FP32 ``wfkernelf``);
  ``"double"`` (the default) runs the all-FP64 kernel, which reproduces the
  reference CPU kernel's rounding sequence.
* ``amplitudes=``: per-emitter amplitudes, shape (N,) for every image or
  (Nimg, N); float32 or float64.
* ``batch=``: images per GPU launch for ``simulate_gen`` (``simulate``
  batches automatically); ``device=``: CUDA device.
* ``returngpu=True`` yields/returns torch CUDA tensors (there is no cupy).
"""

from __future__ import annotations

import numpy as np
import torch

from .. import _native as nat
from . import _core

__all__ = ["simulate", "simulate_gen"]

# output bytes per launch in simulate(): bounds device memory for large Nimg
_MAX_OUT_BYTES = 1 << 30


def _setup(simobject, Ndet, pixelsize, detz, k, settings, detangles, detoffset, default="double"):
    if k is None:
        k = simobject.k
    flags, precision, c64 = _core.parse_settings(settings, default)
    Ndet = _core.ndet_pair(Ndet)
    geom = _core.make_geom(Ndet, pixelsize, detz, k, detangles, detoffset, flags)
    out_kind = nat.OUT_C64 if c64 else nat.OUT_C128
    return Ndet, geom, precision, out_kind


def _amplitude_rows(amplitudes, n_img, N, start):
    if amplitudes is None:
        return None
    a = np.asarray(amplitudes)
    if a.ndim == 1:
        if a.shape[0] != N:
            raise ValueError("amplitudes must have N entries")
        return np.tile(a, n_img)
    if a.shape[1] != N:
        raise ValueError("amplitudes must be (N,) or (Nimg, N)")
    return a[start:start + n_img].reshape(-1)


class _Stager:
    """Pinned host staging of emitter blocks and their upload."""

    def __init__(self, N, max_imgs, device):
        self.N = N
        self.device = device
        self.host = torch.empty((max_imgs * N, 4), dtype=torch.float64, pin_memory=True)
        self.hnp = self.host.numpy()

    def fill(self, simobject, n_img):
        N = self.N
        for i in range(n_img):
            pos, ph = simobject.get2()
            self.hnp[i * N:(i + 1) * N, :3] = pos
            self.hnp[i * N:(i + 1) * N, 3:] = np.reshape(ph, (N, 1))
        return self.host[: n_img * N].to(self.device, non_blocking=True)


def _upload_amps(rows, device):
    if rows is None:
        return None
    t = torch.from_numpy(np.ascontiguousarray(rows))
    if t.dtype not in (torch.float32, torch.float64):
        t = t.to(torch.float64)
    return t.to(device)


def simulate_gen(
    simobject,
    Ndet,
    pixelsize,
    detz,
    k=None,
    settings="double",
    maximg=np.inf,
    detangles=(0, 0),
    detoffset=(0, 0),
    returngpu=False,
    *args,
    amplitudes=None,
    batch=1,
    device=None,
    **kwargs,
):
    """Generator of simulated wavefields (complex (Nx, Ny) per image).

    Parameters follow ``idi/simulation/cuda.py:16-50``: ``simobject`` with
    ``.N``, ``.k`` and ``.get2()``; ``Ndet`` pixels; ``pixelsize``/``detz`` in
    the simobject's length unit; ``k`` (default ``simobject.k``); ``settings``
    substrings ``double|single|split``, ``nf``, ``scale``, ``secondorder``;
    ``maximg`` images; ``detangles`` (theta, phi); ``detoffset`` (x, y);
    ``returngpu`` yields CUDA tensors instead of numpy arrays.
    """
    Ndet, geom, precision, out_kind = _setup(simobject, Ndet, pixelsize, detz, k, settings, detangles, detoffset)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    N = int(simobject.N)
    batch = max(1, int(batch))
    stager = _Stager(N, batch, dev)

    def _gen():
        count = 0
        while count < maximg:
            nb = int(min(batch, maximg - count)) if np.isfinite(maximg) else batch
            d_atoms = stager.fill(simobject, nb)
            amps = _upload_amps(_amplitude_rows(amplitudes, nb, N, count), dev)
            offsets = np.arange(nb + 1, dtype=np.int64) * N
            E = _core.forward(d_atoms, offsets, geom, precision, out_kind, amplitudes=amps)
            if not returngpu:
                E = E.cpu().numpy()
            for i in range(nb):
                yield E[i]
            count += nb

    return _gen()


def simulate(
    Nimg,
    simobject,
    Ndet,
    pixelsize,
    detz,
    k=None,
    settings="double",
    verbose=True,
    detangles=(0, 0),
    detoffset=(0, 0),
    returngpu=False,
    *args,
    amplitudes=None,
    device=None,
    **kwargs,
):
    """``Nimg`` simulated wavefields, complex128 array (Nimg, Nx, Ny).

    Mirrors ``idi/simulation/cuda.py:141-202``: images are drawn from
    ``simobject.get2()`` in order; all images of a chunk run in one
    persistent GPU launch.  Ctrl-C returns the images finished so far.
    """
    Ndet, geom, precision, out_kind = _setup(simobject, Ndet, pixelsize, detz, k, settings, detangles, detoffset)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    N = int(simobject.N)
    Nimg = int(Nimg)
    per_img = Ndet[0] * Ndet[1] * 16
    chunk = int(max(1, min(Nimg, _MAX_OUT_BYTES // max(per_img, 1))))
    stager = _Stager(N, chunk, dev)
    if returngpu:
        result = torch.empty((Nimg, Ndet[0], Ndet[1]), dtype=torch.complex128, device=dev)
    else:
        result = np.empty((Nimg, Ndet[0], Ndet[1]), np.complex128)
    done = 0
    try:
        while done < Nimg:
            nb = min(chunk, Nimg - done)
            d_atoms = stager.fill(simobject, nb)
            amps = _upload_amps(_amplitude_rows(amplitudes, nb, N, done), dev)
            offsets = np.arange(nb + 1, dtype=np.int64) * N
            E = _core.forward(d_atoms, offsets, geom, precision, out_kind, amplitudes=amps)
            if returngpu:
                result[done:done + nb] = E
            else:
                result[done:done + nb] = E.cpu().numpy()
            done += nb
            if verbose:
                print(done, end=". ", flush=True)
        return result
    except KeyboardInterrupt:
        if verbose:
            print("Interrupted")
        return result[:done]


def simulate_batch(
    images,
    Ndet,
    pixelsize,
    detz,
    k,
    settings="split",
    detangles=(0, 0),
    detoffset=(0, 0),
    amplitudes=None,
    out="field",
    config=None,
):
    """Batched uneven images in one persistent launch (no reference counterpart).

    ``images``: list of (N_i, 4) arrays/tensors [x, y, z, phase].
    ``amplitudes``: optional list of (N_i,) arrays.  ``out``: ``"field"``
    (complex) or ``"intensity"`` (float64).  Returns a CUDA tensor
    (B, Nx, Ny).  For repeated launches of the same batch shape use
    :class:`idi_b200.simulation.batch.BatchPlan`, which captures the launch in
    a CUDA graph.
    """
    flags, precision, c64 = _core.parse_settings(settings, "split")
    geom = _core.make_geom(Ndet, pixelsize, detz, k, detangles, detoffset, flags)
    dev = torch.device("cuda", torch.cuda.current_device())
    rows = [torch.as_tensor(np.asarray(a) if not isinstance(a, torch.Tensor) else a, dtype=torch.float64)
            for a in images]
    offsets = np.concatenate([[0], np.cumsum([r.shape[0] for r in rows])]).astype(np.int64)
    atoms = torch.cat([r.reshape(-1, 4) for r in rows]).to(dev).contiguous()
    amps = None
    if amplitudes is not None:
        amps = torch.cat([torch.as_tensor(np.asarray(a)) for a in amplitudes]).to(dev)
    if out == "intensity":
        kind = nat.OUT_I64
    else:
        kind = nat.OUT_C64 if c64 else nat.OUT_C128
    return _core.forward(atoms, offsets, geom, precision, kind, amplitudes=amps, config=config)
