"""Streaming ``.npz`` output for simulation results (the ``np.savez_compressed``
of ``scripts/idi_sim.py:86-88``), written chunk by chunk as the device
pipeline delivers images, so a run never holds all of its images in host
memory.  The files are ordinary ``.npz`` archives: ``numpy.load`` reads them.

The HDF5 writers of the reference (``idi/util/h5util.py``) need ``h5py``,
which this image does not have; they are not provided.
"""

from __future__ import annotations

import zipfile

import numpy as np

__all__ = ["NpzStream"]


class _Member:
    """One ``.npy`` member of the archive, filled along axis 0."""

    def __init__(self, zf, name, shape, dtype):
        self.shape = tuple(int(s) for s in shape)
        self.dtype = np.dtype(dtype)
        self._rows = 0
        self._fp = zf.open(name + ".npy", "w", force_zip64=True)
        header = {"descr": np.lib.format.dtype_to_descr(self.dtype), "fortran_order": False, "shape": self.shape}
        np.lib.format.write_array_header_2_0(self._fp, header)

    def write(self, chunk):
        a = np.ascontiguousarray(chunk, dtype=self.dtype)
        if a.shape[1:] != self.shape[1:]:
            raise ValueError(f"chunk shape {a.shape} does not fit {self.shape}")
        if self._rows + a.shape[0] > self.shape[0]:
            raise ValueError("more rows than the array was declared with")
        self._fp.write(a.tobytes())
        self._rows += a.shape[0]

    def close(self):
        self._fp.close()
        if self._rows != self.shape[0]:
            raise ValueError(f"array declared with {self.shape[0]} rows received {self._rows}")


class NpzStream:
    """A ``.npz`` archive written member by member: ``array(name, shape, dtype)``
    opens a member that receives its rows in chunks (``write``) and must be
    closed before the next; ``add(name, value)`` stores a whole array."""

    def __init__(self, path, compress=True):
        self._zf = zipfile.ZipFile(path, "w", compression=zipfile.ZIP_DEFLATED if compress else zipfile.ZIP_STORED,
                                   allowZip64=True)
        self._open = None

    def array(self, name, shape, dtype) -> _Member:
        if self._open is not None:
            raise RuntimeError("close the open array first")
        self._open = _Member(self._zf, name, shape, dtype)
        return self._open

    def close_array(self):
        if self._open is not None:
            m, self._open = self._open, None
            m.close()

    def add(self, name, value):
        self.close_array()
        with self._zf.open(name + ".npy", "w", force_zip64=True) as fp:
            np.lib.format.write_array(fp, np.asanyarray(value), allow_pickle=True)

    def close(self):
        try:
            self.close_array()
        finally:
            self._zf.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
