"""Speed of the oracle's C port against the reference's own numba CPU kernel.

    python oracle/compare_cpu_speed.py [threads]

Test infrastructure: runs where the reference tree is present (it cannot
travel to other machines), on the small CPU configuration (2,000 emitters in
a 10 nm sphere, 256x256 pixels of 75 um at 0.1 m, 6.4 keV), near and far
field, 4 images.  The reference's ``cpu.simulate`` (idi/simulation/cpu.py:
112-156, numba, loaded through ``refshim``) and the oracle's
``wavefield`` (OpenMP) each use ``threads`` host threads on the same cores;
prints pairs/s for both, their ratio, and the largest field difference (0 in
the near field: the port reproduces numba's rounding bit for bit).  The
benchmark's reference arm times the port, so a ratio above 1 means that arm
is faster than the reference's own code would be on the same host.
"""

from __future__ import annotations

import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
if __name__ == "__main__":
    threads = sys.argv[1] if len(sys.argv) > 1 else str(os.cpu_count())
    os.environ["NUMBA_NUM_THREADS"] = threads
    os.environ["OMP_NUM_THREADS"] = threads
sys.path.insert(0, os.path.dirname(HERE))

import numpy as np  # noqa: E402

import oracle  # noqa: E402
from oracle import refshim  # noqa: E402


def main():
    ref = refshim.load()
    g = np.random.Generator(np.random.Philox(5))
    n, nimg, ndet = 2000, 4, 256
    t = g.uniform(-1, 1, n)
    p = g.uniform(0, 2 * np.pi, n)
    u = 0.01 * g.uniform(0, 1, n) ** (1 / 3)
    s = np.sqrt(1 - t * t)
    pos = np.stack([u * t, u * s * np.sin(p), u * s * np.cos(p)], -1)
    ph = g.uniform(0, 2 * np.pi, (nimg, n))
    k = 2 * np.pi / (1.24 / 6400.0)
    pairs = nimg * n * ndet * ndet
    og = oracle.geometry(ndet, 75.0, 1e5, k)
    rows = [np.ascontiguousarray(np.concatenate([pos, ph[i][:, None]], 1)) for i in range(nimg)]
    for settings, flags in (("nf", oracle.NF), ("", 0)):
        ref.cpu.simulate(1, refshim.InjectedObject(6400.0, pos, ph), ndet, 75.0, 1e5, k, settings=settings)
        t0 = time.perf_counter()
        r = ref.cpu.simulate(nimg, refshim.InjectedObject(6400.0, pos, ph), ndet, 75.0, 1e5, k, settings=settings)
        t_numba = time.perf_counter() - t0
        oracle.wavefield(og, flags, rows[0])
        t0 = time.perf_counter()
        o = [oracle.wavefield(og, flags, a) for a in rows]
        t_port = time.perf_counter() - t0
        diff = max(float(np.abs(o[i] - r[i]).max()) for i in range(nimg))
        print(f"{settings or 'far field'}: reference numba {pairs / t_numba:.3e} pairs/s, C port "
              f"{pairs / t_port:.3e} pairs/s, port/numba {t_numba / t_port:.2f}, max |dE| {diff:.1e} "
              f"({os.environ.get('NUMBA_NUM_THREADS')} threads)")


if __name__ == "__main__":
    main()
