"""Reference-compatible reconstruction API (``idi.reconstruction`` layout) for
the direct q-space correlators on the GPU.

``cucorrad`` replaces ``idi.reconstruction.cucorrad`` (radial correlation),
``cucor`` replaces ``idi.reconstruction.cucor`` (3d correlation);
``qcorrad`` / ``qcor`` point at them as ``idi/reconstruction/__init__.py:34-48``
does when CUDA is available.  There is no CPU fallback.
"""

__all__ = ["cucor", "cucorrad", "qcor", "qcorrad"]

from . import cucor, cucorrad  # noqa: E402

qcor = cucor
qcorrad = cucorrad
