"""Reference-compatible simulation API (``idi.simulation`` layout).

``cuda`` replaces ``idi.simulation.cuda`` (and ``cpu``), ``cutime`` replaces
``idi.simulation.cutime`` (and ``time``), ``common`` replaces
``idi.simulation.common`` (photon sampling, charge sharing);
``auto``/``autotime`` point at them
as in ``idi/simulation/__init__.py:7-31``.  There is no CPU fallback: the
compute calls need the CUDA library and a GPU.
"""

__all__ = ["cuda", "cutime", "time", "cpu", "auto", "autotime", "simobj", "autograd", "batch", "common"]

from . import _core, autograd, batch, common, cuda, cutime, simobj  # noqa: E402

auto = cuda
cpu = cuda
autotime = cutime
time = cutime
