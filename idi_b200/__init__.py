"""idi_b200 — B200 (sm_100a) emitter-wavefield direct sum with the call
signatures of fzimmermann89/idi's ``idi.simulation`` backends.

    from idi_b200 import simulation as sim
    E = sim.cuda.simulate(Nimg, simobject, Ndet, pixelsize, detz, k, settings="nf split")

The compute runs in hand-written CUDA kernels (``idi_b200/csrc``) behind the C
ABI of ``include/idiwf.h``; PyTorch provides device memory and streams.
"""

__version__ = "0.1.0"
__all__ = ["simulation"]

from . import simulation  # noqa: E402
