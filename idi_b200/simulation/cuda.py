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

__all__ = ["simulate", "simulate_gen", "simulate_photons", "simulate_to_npz"]

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


_PINNED = {}


def _pinned(key, nbytes):
    """Cached pinned host buffer (grow-only), reused across calls."""
    buf = _PINNED.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(int(nbytes), dtype=torch.uint8, pin_memory=True)
        _PINNED[key] = buf
    return buf


class _Stager:
    """Pinned host staging of emitter blocks and their upload (sources whose
    ``ondevice`` is set draw on the GPU instead).  With a `key`, the pinned
    buffer comes from a cache reused across calls."""

    def __init__(self, N, max_imgs, device, key=None):
        self.N = N
        self.device = device
        self.max_imgs = max_imgs
        self.key = key
        self.host = None

    def _alloc(self):
        N, m = self.N, self.max_imgs
        if self.key is None:
            self.host = torch.empty((m * N, 4), dtype=torch.float64, pin_memory=True)
        else:
            raw = _pinned(self.key, m * N * 32)
            self.host = raw[: m * N * 32].view(torch.float64).view(m * N, 4)
        self.hnp = self.host.numpy()

    def fill(self, simobject, n_img):
        if getattr(simobject, "ondevice", False):
            # the source draws straight into device memory (idiwf_emitters)
            return simobject.device_batch(n_img, self.device)
        if self.host is None:
            self._alloc()
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

    errors = _core.ErrorWord(dev)

    def _gen():
        count = 0
        while count < maximg:
            nb = int(min(batch, maximg - count)) if np.isfinite(maximg) else batch
            d_atoms = stager.fill(simobject, nb)
            amps = _upload_amps(_amplitude_rows(amplitudes, nb, N, count), dev)
            offsets = np.arange(nb + 1, dtype=np.int64) * N
            E = _core.forward(d_atoms, offsets, geom, precision, out_kind, amplitudes=amps, errors=errors)
            errors.check()  # device-side errors of this batch (synchronises)
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
    ``simobject.get2()`` in order and run in batched persistent launches.
    With host output, the images are processed in up to eight chunks whose
    device-to-host copies (into pinned staging, on a second stream) overlap
    the next chunk's kernel.  Ctrl-C returns the images finished so far.
    Device-side errors (split-precision emitters out of range, a near-field
    geometry outside the split range) raise ``IdiwfError`` once all images are
    done.
    """
    Ndet, geom, precision, out_kind = _setup(simobject, Ndet, pixelsize, detz, k, settings, detangles, detoffset)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    N = int(simobject.N)
    Nimg = int(Nimg)
    npix = Ndet[0] * Ndet[1]
    elem = 8 if out_kind == nat.OUT_C64 else 16
    per_img = npix * elem
    cap = int(max(1, _MAX_OUT_BYTES // max(per_img, 1)))
    nchunks = _nchunks(per_img * Nimg, Nimg)
    chunk = int(max(1, min(cap, -(-Nimg // nchunks))))
    done = 0
    if returngpu:
        result = torch.empty((Nimg, Ndet[0], Ndet[1]), dtype=torch.complex128, device=dev)
        stager = _Stager(N, chunk, dev)
        errors = _core.ErrorWord(dev)
        try:
            while done < Nimg:
                nb = min(chunk, Nimg - done)
                d_atoms = stager.fill(simobject, nb)
                amps = _upload_amps(_amplitude_rows(amplitudes, nb, N, done), dev)
                offsets = np.arange(nb + 1, dtype=np.int64) * N
                result[done:done + nb] = _core.forward(d_atoms, offsets, geom, precision, out_kind, amplitudes=amps,
                                                       errors=errors)
                done += nb
                if verbose:
                    print(done, end=". ", flush=True)
            errors.check()
            return result
        except KeyboardInterrupt:
            if verbose:
                print("Interrupted")
            return result[:done]

    dtype = torch.complex64 if out_kind == nat.OUT_C64 else torch.complex128
    return _pipelined(Nimg, simobject, N, Ndet, chunk, dev, geom, precision, out_kind, dtype, amplitudes, verbose,
                      np.complex128)


def _nchunks(out_bytes, Nimg):
    """Chunks of the host-output pipeline: enough to overlap the copies with
    the kernels, and the more the larger the output, since the first chunk's
    upload and the last chunk's copies are not overlapped."""
    if out_bytes >= (256 << 20) and Nimg >= 8:
        return 8
    if out_bytes >= (64 << 20) and Nimg >= 4:
        return 4
    return 1


def _prefault(a):
    """Touch one byte per 4 KiB page of a fresh host array, so that the page
    faults happen now (while the GPU computes) and not in the copy of the
    last chunk, which nothing overlaps."""
    flat = a.reshape(-1).view(np.uint8)
    flat[::4096] = 0


def _pipelined(Nimg, simobject, N, Ndet, chunk, dev, geom, precision, out_kind, out_dtype, amplitudes, verbose,
               result_dtype, post=None, sink=None):
    """Chunked device pipeline with host output: chunk i's device-to-host copy
    (pinned staging, second stream) overlaps chunk i+1's emitter upload and
    kernels.  ``post(field_or_intensity, first_image, slot)`` runs further device
    work on a chunk and returns the tensor to copy back (default: the forward
    output).  With ``sink(first_image, array)`` every chunk goes to the sink
    (which must consume it before returning) instead of into one result array,
    and the images finished are counted instead.  Ctrl-C returns the images
    finished so far."""
    result = None
    compute = torch.cuda.current_stream(dev)
    copy = torch.cuda.Stream(dev)
    stagers = [_Stager(N, chunk, dev, ("sim_in", dev.index, i)) for i in range(2)]
    d_out = [torch.empty((chunk, Ndet[0], Ndet[1]), dtype=out_dtype, device=dev) for _ in range(2)]
    h_out = [None, None]
    ev_done = [torch.cuda.Event(), torch.cuda.Event()]
    ev_copied = [torch.cuda.Event(), torch.cuda.Event()]
    ev_h2d = [None, None]
    pending = None  # (slot, start, count) of the chunk whose copy is in flight
    done = 0

    finished = [0]
    errors = _core.ErrorWord(dev)

    def _collect(ps, pstart, pn):
        ev_copied[ps].synchronize()
        if sink is not None:
            sink(pstart, h_out[ps][:pn].numpy())
        elif result.dtype == h_out[ps].numpy().dtype:
            # torch's CPU copy runs on several threads; the last chunk's copy
            # is on the critical path
            torch.from_numpy(result[pstart:pstart + pn]).copy_(h_out[ps][:pn])
        else:
            result[pstart:pstart + pn] = h_out[ps][:pn].numpy()
        finished[0] = pstart + pn
        if verbose:
            print(pstart + pn, end=". ", flush=True)

    try:
        i = 0
        while done < Nimg:
            slot = i & 1
            nb = min(chunk, Nimg - done)
            if ev_h2d[slot] is not None:
                ev_h2d[slot].synchronize()  # staging buffer free again
            d_atoms = stagers[slot].fill(simobject, nb)
            ev_h2d[slot] = torch.cuda.Event()
            ev_h2d[slot].record(compute)
            amps = _upload_amps(_amplitude_rows(amplitudes, nb, N, done), dev)
            offsets = np.arange(nb + 1, dtype=np.int64) * N
            compute.wait_event(ev_copied[slot])  # device buffers of this slot copied out
            _core.forward(d_atoms, offsets, geom, precision, out_kind, amplitudes=amps, out=d_out[slot][:nb],
                          errors=errors)
            src = d_out[slot][:nb] if post is None else post(d_out[slot][:nb], done, slot)
            if h_out[slot] is None:
                per = src[0].numel() * src.element_size()
                raw = _pinned(("sim_out", dev.index, slot), chunk * per)
                h_out[slot] = raw[: chunk * per].view(src.dtype).view((chunk,) + tuple(src.shape[1:]))
            if result is None and sink is None:
                result = np.empty((Nimg,) + tuple(src.shape[1:]), result_dtype)
            ev_done[slot].record(compute)
            copy.wait_event(ev_done[slot])
            with torch.cuda.stream(copy):
                h_out[slot][:nb].copy_(src, non_blocking=True)
            ev_copied[slot].record(copy)
            if i == 0 and result is not None and Nimg > nb:
                _prefault(result)  # overlaps the first chunk's kernels
            if pending is not None:
                _collect(*pending)
            pending = (slot, done, nb)
            done += nb
            i += 1
        _collect(*pending)
        errors.check()
        return finished[0] if sink is not None else result
    except KeyboardInterrupt:
        if verbose:
            print("Interrupted")
        torch.cuda.synchronize(dev)
        if sink is not None:
            return finished[0]
        if result is None:
            return np.empty((0, Ndet[0], Ndet[1]), result_dtype)
        return result[: pending[1] if pending else 0]


def simulate_to_npz(
    outfile,
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
    *args,
    extra=None,
    compress=True,
    amplitudes=None,
    device=None,
    **kwargs,
):
    """``Nimg`` intensity images |E|^2 written to ``outfile`` as the ``.npz``
    of ``scripts/idi_sim.py:86-88``: array ``result`` (Nimg, Nx, Ny) float64,
    plus the arrays of ``extra`` (e.g. the run's settings).  The intensities
    are formed on the device (8 bytes per pixel cross PCIe instead of 16) and
    streamed into the archive chunk by chunk, so host memory holds two chunks,
    not the run.  Arguments as :func:`simulate`.  Returns the number of
    images written (fewer after Ctrl-C, in which case the file is incomplete
    and raises on close)."""
    from .output import NpzStream

    Ndet, geom, precision, _ = _setup(simobject, Ndet, pixelsize, detz, k, settings, detangles, detoffset)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    N = int(simobject.N)
    Nimg = int(Nimg)
    per_img = Ndet[0] * Ndet[1] * 8
    cap = int(max(1, _MAX_OUT_BYTES // max(per_img, 1)))
    nchunks = _nchunks(per_img * Nimg, Nimg)
    chunk = int(max(1, min(cap, -(-Nimg // nchunks))))
    with NpzStream(outfile, compress=compress) as npz:
        member = npz.array("result", (Nimg, Ndet[0], Ndet[1]), np.float64)
        done = _pipelined(Nimg, simobject, N, Ndet, chunk, dev, geom, precision, nat.OUT_I64, torch.float64,
                          amplitudes, verbose, np.float64, sink=lambda first, a: member.write(a))
        npz.close_array()
        for name, value in (extra or {}).items():
            npz.add(name, value)
    return done


def simulate_photons(
    Nimg,
    simobject,
    Ndet,
    pixelsize,
    detz,
    Nphotons,
    k=None,
    settings="double",
    verbose=True,
    detangles=(0, 0),
    detoffset=(0, 0),
    returngpu=False,
    *args,
    dtype=np.uint32,
    rng=None,
    chargesharing=None,
    amplitudes=None,
    device=None,
    **kwargs,
):
    """``Nimg`` photon-count images from one device pipeline: direct sum,
    ``|E|^2``, Poisson photons with ``Nphotons`` expected per image
    (:func:`idi_b200.simulation.common.randomphotons`) and, with
    ``chargesharing=(s, ns)``, charge sharing.  The intensities never leave the
    GPU; only the counts are copied back.

    Replaces the reference's two-step ``randomphotons(np.abs(simulate(...))**2,
    Nphotons)`` (``scripts/idi_simrecon.py:38-45``).  Arguments as
    :func:`simulate`; ``dtype`` is the count type (float64 with charge
    sharing); ``rng`` as :func:`~idi_b200.simulation.common.randomphotons`.
    Image i draws from the same streams however the images are chunked.
    """
    from . import common

    Ndet, geom, precision, out_kind = _setup(simobject, Ndet, pixelsize, detz, k, settings, detangles, detoffset)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    N = int(simobject.N)
    Nimg = int(Nimg)
    npix = Ndet[0] * Ndet[1]
    key, stream = common._key_stream(rng)
    tdt, nd = common._count_dtype(dtype)
    if chargesharing is not None:
        cs_s, cs_ns = (tuple(chargesharing) + (0.0,))[:2]
        final = torch.float64
    else:
        final = tdt
    cap = int(max(1, _MAX_OUT_BYTES // max(npix * 16, 1)))
    nchunks = _nchunks(npix * 8 * Nimg, Nimg)
    chunk = int(max(1, min(cap, -(-Nimg // nchunks))))
    counts = [None, None]
    shared = [None, None]

    def post(intensity, first, slot):
        nb = intensity.shape[0]
        if counts[slot] is None:
            counts[slot] = torch.empty((chunk, Ndet[0], Ndet[1]), dtype=tdt, device=dev)
        c = _core.photons(intensity, Nphotons, key, stream, dtype=tdt, out=counts[slot][:nb], first_image=first)
        if chargesharing is None:
            return c
        if shared[slot] is None:
            shared[slot] = torch.empty((chunk, Ndet[0], Ndet[1]), dtype=torch.float64, device=dev)
        return _core.chargesharing(c, cs_s, cs_ns, key, stream, out=shared[slot][:nb], first_image=first)

    if returngpu:
        result = torch.empty((Nimg, Ndet[0], Ndet[1]), dtype=final, device=dev)
        stager = _Stager(N, chunk, dev)
        d_int = torch.empty((chunk, Ndet[0], Ndet[1]), dtype=torch.float64, device=dev)
        errors = _core.ErrorWord(dev)
        done = 0
        while done < Nimg:
            nb = min(chunk, Nimg - done)
            d_atoms = stager.fill(simobject, nb)
            amps = _upload_amps(_amplitude_rows(amplitudes, nb, N, done), dev)
            offsets = np.arange(nb + 1, dtype=np.int64) * N
            _core.forward(d_atoms, offsets, geom, precision, nat.OUT_I64, amplitudes=amps, out=d_int[:nb],
                          errors=errors)
            result[done:done + nb] = post(d_int[:nb], done, 0)
            done += nb
        errors.check()
        _core.workspace_error(dev, "photons")
        return result
    res_np = torch.empty(0, dtype=final).numpy().dtype
    out = _pipelined(Nimg, simobject, N, Ndet, chunk, dev, geom, precision, nat.OUT_I64, torch.float64, amplitudes,
                     verbose, res_np, post=post)
    _core.workspace_error(dev, "photons")
    if nd is not None and chargesharing is None and out.dtype != nd:
        out = out.astype(nd)
    return out


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
    errors = _core.ErrorWord(dev)
    res = _core.forward(atoms, offsets, geom, precision, kind, amplitudes=amps, config=config, errors=errors)
    errors.check()
    return res
