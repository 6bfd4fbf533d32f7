"""Reference-compatible reconstruction API (``idi.reconstruction`` layout) for
the direct q-space correlators on the GPU.

``cucorrad`` replaces ``idi.reconstruction.cucorrad`` (radial correlation),
``cucor`` replaces ``idi.reconstruction.cucor`` (3d correlation), ``cusimple``
replaces ``idi.reconstruction.cusimple`` (FFT autocorrelation);
``qcorrad`` / ``qcor`` / ``simple`` point at them as
``idi/reconstruction/__init__.py:34-48`` does when CUDA is available.  There
is no CPU fallback.
"""

__all__ = ["cucor", "cucorrad", "cusimple", "qcor", "qcorrad", "simple"]

from . import cucor, cucorrad, cusimple  # noqa: E402

qcor = cucor
qcorrad = cucorrad
simple = cusimple
