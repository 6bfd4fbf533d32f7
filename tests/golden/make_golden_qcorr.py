"""Generate ``qcorr_ref.npz``: outputs of the reference's own GPU correlators
``idi/reconstruction/cucorrad.py`` and ``cucor.py`` on small seeded images.

    python tests/golden/make_golden_qcorr.py

The reference kernels are numba-CUDA code; they run here, unmodified, under
numba's CUDA simulator (``NUMBA_ENABLE_CUDASIM=1``, set before numba is
imported, which is why this is a script of its own).  The simulator swaps the
module-level ``cuda`` name for its per-thread stand-in but not the
``_numba.cuda`` attribute path the kernels also use, so each loaded module's
``_numba`` global is replaced by a proxy that forwards ``.cuda`` to the
module's (swapped) ``cuda`` global and everything else to numba.

The simulator runs the kernels' FP32 arithmetic as numpy float32 operations,
one rounding each, and reports out-of-bounds writes: ``cucor`` writes bins
past the end of its array for some geometries (a row of dqz = +maxdqz), so
the 3d cases use geometries where every bin is inside.

Needs the reference tree (``IDI_REFERENCE``, or ``oracle.refshim.REF_ROOT``).
"""

from __future__ import annotations

import importlib.util
import os
import sys

os.environ["NUMBA_ENABLE_CUDASIM"] = "1"

import numba  # noqa: E402
import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import refshim  # noqa: E402

REF = refshim.REF_ROOT

RADIAL_CASES = [
    # name, shape, z, maxq, xcenter, ycenter
    ("rad_12x10", (12, 10), 40.0, 15, None, None),
    ("rad_14x16_centre", (14, 16), 25.0, 20, 5.5, 7.0),
]
CUBE_CASES = [
    ("cube_16x16", (16, 16), 40.0, 32, None, None),
    ("cube_10x14_centre", (10, 14), 30.0, 40, 4.0, 8.0),
]


class _NumbaProxy:
    def __init__(self, globs):
        self._g = globs

    def __getattr__(self, name):
        if name == "cuda":
            return self._g["cuda"]
        return getattr(numba, name)


def _load(name):
    spec = importlib.util.spec_from_file_location(f"idiref_{name}", os.path.join(REF, "idi", "reconstruction",
                                                                                   f"{name}.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.__dict__["_numba"] = _NumbaProxy(mod.__dict__)
    return mod


def main():
    if not os.path.isdir(REF):
        raise SystemExit("reference tree not available")
    rad, cube = _load("cucorrad"), _load("cucor")
    out = {}
    for i, (name, shape, z, maxq, xc, yc) in enumerate(RADIAL_CASES):
        img = np.random.Generator(np.random.Philox(8000 + i)).uniform(0, 1, shape)
        with rad.corrfunction(shape, z, maxq, xc, yc) as f:
            res = f(img)
        out[f"{name}__image"] = img
        out[f"{name}__meta"] = np.array([z, maxq, np.nan if xc is None else xc, np.nan if yc is None else yc])
        out[f"{name}__out"] = np.asarray(res)
        print(name, "done", flush=True)
    for i, (name, shape, z, maxq, xc, yc) in enumerate(CUBE_CASES):
        img = np.random.Generator(np.random.Philox(8100 + i)).uniform(0, 1, shape)
        with cube.corrfunction(shape, z, maxq, xc, yc) as f:
            res = f(img)
        out[f"{name}__image"] = img
        out[f"{name}__meta"] = np.array([z, maxq, np.nan if xc is None else xc, np.nan if yc is None else yc])
        out[f"{name}__out"] = np.asarray(res)
        print(name, "done", flush=True)
    np.savez_compressed(os.path.join(HERE, "qcorr_ref.npz"), **out)


if __name__ == "__main__":
    sys.exit(main())
