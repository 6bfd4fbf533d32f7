"""Differentiable intensities: a hand-written adjoint direct sum behind
``torch.autograd.Function`` (no reference counterpart).

    I = intensity(pos, phase, amplitudes, Ndet=..., pixelsize=..., detz=..., k=..., settings="nf")
    loss = ((I - target) ** 2).sum()
    loss.backward()        # pos.grad, phase.grad, amplitudes.grad

Forward and adjoint both run the split-precision kernels (FP64 phase in
turns, FP32 sincos and sums).  Device-side errors of both (a near-field
geometry outside the split range, emitters out of range) raise at the end of
the backward pass.  ``pos`` (N,3) and ``phase`` (N,) are float64
CUDA tensors; ``amplitudes`` (N,) float32/float64 or None.  Several images
with uneven emitter counts can be stacked with ``offsets``.
"""

from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from .. import _native as nat
from . import _core

__all__ = ["intensity", "WavefieldIntensity"]


class WavefieldIntensity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, phase, amplitudes, geom, offsets):
        atoms = torch.cat([pos.detach().to(torch.float64), phase.detach().to(torch.float64).reshape(-1, 1)], 1)
        atoms = atoms.contiguous()
        amps = None if amplitudes is None else amplitudes.detach().contiguous()
        errors = _core.ErrorWord(atoms.device)
        E = _core.forward(atoms, offsets, geom, nat.SPLIT, nat.OUT_C128, amplitudes=amps, errors=errors)
        I = E.real.square() + E.imag.square()
        ctx.errors = errors
        ctx.geom = geom
        ctx.offsets = offsets
        ctx.has_amp = amps is not None
        ctx.amp_dtype = None if amps is None else amps.dtype
        if amps is None:
            ctx.save_for_backward(atoms, E)
        else:
            ctx.save_for_backward(atoms, E, amps)
        return I

    @staticmethod
    def backward(ctx, grad_I):
        saved = ctx.saved_tensors
        atoms, E = saved[0], saved[1]
        amps = saved[2] if ctx.has_amp else None
        want_amp = bool(ctx.needs_input_grad[2])
        ga, gamp = _core.backward(atoms, ctx.offsets, ctx.geom, E, grad_I.contiguous().to(torch.float64), amps,
                                  want_amp=want_amp, errors=ctx.errors)
        # device-side errors of the forward and the adjoint (one synchronisation per step)
        ctx.errors.check()
        gpos = ga[:, :3] if ctx.needs_input_grad[0] else None
        gphase = ga[:, 3] if ctx.needs_input_grad[1] else None
        gamp_out = gamp.to(ctx.amp_dtype) if (want_amp and gamp is not None) else None
        return gpos, gphase, gamp_out, None, None


def intensity(
    pos: torch.Tensor,
    phase: torch.Tensor,
    amplitudes: Optional[torch.Tensor] = None,
    *,
    Ndet,
    pixelsize,
    detz,
    k,
    settings: str = "nf",
    detangles=(0, 0),
    detoffset=(0, 0),
    offsets=None,
) -> torch.Tensor:
    """Differentiable |E|^2, float64 (B, Nx, Ny); B = 1 unless ``offsets`` is given."""
    flags, _, _ = _core.parse_settings(settings)
    geom = _core.make_geom(Ndet, pixelsize, detz, k, detangles, detoffset, flags)
    if offsets is None:
        offsets = np.array([0, pos.shape[0]], dtype=np.int64)
    offsets = np.asarray(offsets, dtype=np.int64)
    return WavefieldIntensity.apply(pos, phase, amplitudes, geom, offsets)
