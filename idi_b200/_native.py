"""ctypes binding of the in-tree CUDA library ``idi_b200/_lib/libidiwf.so``.

The library is the product: every simulation call in this package goes
through it.  There is no CPU fallback.  If the shared object is missing the
import of :mod:`idi_b200.simulation` still works (so that documentation and
host-side helpers can be used without a GPU), but every compute call raises
:class:`NativeLibraryMissing`.  Build it with ``python -m idi_b200.build`` (or
``__graft_entry__.build()``).

Signatures mirror ``include/idiwf.h``.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libidiwf.so")

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CUDA = 2
ERR_WORKSPACE = 3
ERR_TIMEOUT = 4
ERR_UNSUPPORTED = 5

NF = 1
SCALE = 2
SECONDORDER = 4
ACCURATE = 8

DOUBLE = 0
SPLIT = 1

OUT_C128 = 0
OUT_C64 = 1
OUT_I64 = 2
OUT_I32 = 3

F64 = 0
F32 = 1
I32 = 2
U32 = 3
I64 = 4

EMIT_SPHERE = 0
EMIT_GNORM = 1
EMIT_FOIL = 2
EMIT_SITES = 3
EMIT_FIXED = 4
ORIENT_FIXED = 0
ORIENT_RANDOM = 1
ORIENT_AXIS = 2

# every symbol include/idiwf.h declares
EXPORTED = (
    "idiwf_forward_workspace_size",
    "idiwf_forward",
    "idiwf_forward_cta_times",
    "idiwf_forward_noalloc",
    "idiwf_forward_noalloc_error",
    "idiwf_backward_workspace_size",
    "idiwf_backward",
    "idiwf_time_max_emitters",
    "idiwf_time_workspace_size",
    "idiwf_time_forward",
    "idiwf_time_forward_digest",
    "idiwf_time_order",
    "idiwf_photons_workspace_size",
    "idiwf_photons",
    "idiwf_chargesharing_workspace_size",
    "idiwf_chargesharing",
    "idiwf_emitters_workspace_size",
    "idiwf_emitters",
    "idiwf_qcorr_workspace_size",
    "idiwf_qcorr_radial",
    "idiwf_qcorr_3d",
    "idiwf_power_spectrum",
    "idiwf_corr_crop",
    "idiwf_welford_update",
    "idiwf_fft_autocorr_workspace_size",
    "idiwf_fft_autocorr",
    "idiwf_fft_autocorr_1d_workspace_size",
    "idiwf_fft_autocorr_1d",
    "idiwf_tune",
    "idiwf_workspace_error",
    "idiwf_microbench",
    "idiwf_last_error_string",
    "idiwf_version",
)


class NativeLibraryMissing(RuntimeError):
    pass


class IdiwfError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"idiwf status {status}: {message}")
        self.status = status


class Geom(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("has_rot", ctypes.c_int32),
        ("pixelsize", ctypes.c_double),
        ("detz", ctypes.c_double),
        ("k", ctypes.c_double),
        ("offset", ctypes.c_double * 2),
        ("rot", ctypes.c_double * 9),
    ]


class Config(ctypes.Structure):
    _fields_ = [
        ("threads", ctypes.c_int32),
        ("pixels_per_thread", ctypes.c_int32),
        ("emitters_per_tile", ctypes.c_int32),
        ("ctas_per_sm", ctypes.c_int32),
        ("pixel_groups", ctypes.c_int32),
    ]


class Batch(ctypes.Structure):
    _fields_ = [
        ("n_images", ctypes.c_int32),
        ("amp_dtype", ctypes.c_int32),
        ("offsets", ctypes.POINTER(ctypes.c_int64)),
        ("atoms", ctypes.c_void_p),
        ("amplitudes", ctypes.c_void_p),
    ]


class Rng(ctypes.Structure):
    _fields_ = [
        ("key", ctypes.c_uint64 * 2),
        ("stream", ctypes.c_uint64),
        ("first_image", ctypes.c_uint64),
    ]


class EmittersDesc(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("random_phase", ctypes.c_int32),
        ("orientation", ctypes.c_int32),
        ("weighted", ctypes.c_int32),
        ("r", ctypes.c_double),
        ("fwhm", ctypes.c_double * 3),
        ("rho", ctypes.c_double * 3),
        ("depth", ctypes.c_double),
        ("attenuation", ctypes.c_double),
        ("rot", ctypes.c_double * 9),
        ("axis", ctypes.c_double * 3),
        ("sites", ctypes.c_void_p),
        ("n_sites", ctypes.c_int64),
    ]


_lib = None


def load():
    """Load the library (once) and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NativeLibraryMissing(
            f"{LIB_PATH} is missing: the CUDA library has not been built "
            "(run `python -m idi_b200.build`); there is no CPU fallback"
        )
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    st = ctypes.c_int32
    L.idiwf_forward_workspace_size.argtypes = [P(Geom), P(Batch), ctypes.c_int32, P(Config)]
    L.idiwf_forward_workspace_size.restype = ctypes.c_size_t
    L.idiwf_forward.argtypes = [P(Geom), P(Batch), ctypes.c_int32, ctypes.c_int32, vp, vp, ctypes.c_size_t,
                                P(Config), vp]
    L.idiwf_forward.restype = st
    L.idiwf_forward_noalloc.argtypes = [P(Geom), P(Batch), ctypes.c_int32, vp, vp]
    L.idiwf_forward_noalloc.restype = st
    L.idiwf_forward_noalloc_error.argtypes = [vp]
    L.idiwf_forward_noalloc_error.restype = st
    L.idiwf_forward_cta_times.argtypes = [vp, P(ctypes.c_uint64), ctypes.c_int32, P(ctypes.c_int32), vp]
    L.idiwf_forward_cta_times.restype = st
    L.idiwf_backward_workspace_size.argtypes = [P(Geom), P(Batch), P(Config)]
    L.idiwf_backward_workspace_size.restype = ctypes.c_size_t
    L.idiwf_backward.argtypes = [P(Geom), P(Batch), vp, vp, vp, vp, vp, ctypes.c_size_t, P(Config), vp]
    L.idiwf_backward.restype = st
    L.idiwf_time_max_emitters.argtypes = []
    L.idiwf_time_max_emitters.restype = ctypes.c_int64
    L.idiwf_time_workspace_size.argtypes = [P(Geom), ctypes.c_int64]
    L.idiwf_time_workspace_size.restype = ctypes.c_size_t
    L.idiwf_time_forward.argtypes = [P(Geom), vp, vp, ctypes.c_int64, ctypes.c_double, ctypes.c_double, vp, vp,
                                     ctypes.c_size_t, vp]
    L.idiwf_time_forward.restype = st
    L.idiwf_time_forward_digest.argtypes = [P(Geom), vp, vp, ctypes.c_int64, ctypes.c_double, ctypes.c_double, vp,
                                            vp, vp, ctypes.c_size_t, vp]
    L.idiwf_time_forward_digest.restype = st
    L.idiwf_time_order.argtypes = [P(Geom), vp, vp, ctypes.c_int64, ctypes.c_double, ctypes.c_int32,
                                   ctypes.c_int32, vp, vp, vp, ctypes.c_size_t, vp]
    L.idiwf_time_order.restype = st
    L.idiwf_photons_workspace_size.argtypes = [ctypes.c_int32, ctypes.c_int64]
    L.idiwf_photons_workspace_size.restype = ctypes.c_size_t
    L.idiwf_photons.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, P(Rng), vp,
                                ctypes.c_int32, vp, ctypes.c_size_t, vp]
    L.idiwf_photons.restype = st
    L.idiwf_chargesharing_workspace_size.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    L.idiwf_chargesharing_workspace_size.restype = ctypes.c_size_t
    L.idiwf_chargesharing.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                      ctypes.c_double, ctypes.c_double, P(Rng), vp, vp, ctypes.c_int64, vp, vp,
                                      ctypes.c_size_t, vp]
    L.idiwf_chargesharing.restype = st
    L.idiwf_emitters_workspace_size.argtypes = [P(EmittersDesc), ctypes.c_int32, ctypes.c_int64]
    L.idiwf_emitters_workspace_size.restype = ctypes.c_size_t
    L.idiwf_emitters.argtypes = [P(EmittersDesc), ctypes.c_int32, ctypes.c_int64, P(Rng), vp, vp, ctypes.c_size_t, vp]
    L.idiwf_emitters.restype = st
    L.idiwf_qcorr_workspace_size.argtypes = [ctypes.c_int32, ctypes.c_int32]
    L.idiwf_qcorr_workspace_size.restype = ctypes.c_size_t
    L.idiwf_qcorr_radial.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, vp, vp,
                                     ctypes.c_size_t, vp]
    L.idiwf_qcorr_radial.restype = st
    L.idiwf_qcorr_3d.argtypes = [vp, vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                 ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_float, vp, vp,
                                 ctypes.c_size_t, vp]
    L.idiwf_qcorr_3d.restype = st
    L.idiwf_power_spectrum.argtypes = [vp, ctypes.c_int64, ctypes.c_int32, vp]
    L.idiwf_power_spectrum.restype = st
    L.idiwf_corr_crop.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, P(ctypes.c_int32),
                                  P(ctypes.c_int32), vp, ctypes.c_int32, ctypes.c_double, vp, vp]
    L.idiwf_corr_crop.restype = st
    L.idiwf_welford_update.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.c_int64, vp]
    L.idiwf_welford_update.restype = st
    L.idiwf_fft_autocorr_workspace_size.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    L.idiwf_fft_autocorr_workspace_size.restype = ctypes.c_size_t
    L.idiwf_fft_autocorr.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, vp,
                                     ctypes.c_int32, ctypes.c_double, vp, vp, ctypes.c_size_t, vp]
    L.idiwf_fft_autocorr.restype = st
    L.idiwf_fft_autocorr_1d_workspace_size.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_int32]
    L.idiwf_fft_autocorr_1d_workspace_size.restype = ctypes.c_size_t
    L.idiwf_fft_autocorr_1d.argtypes = [vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, vp, ctypes.c_int32,
                                        ctypes.c_double, vp, vp, ctypes.c_size_t, vp]
    L.idiwf_fft_autocorr_1d.restype = st
    L.idiwf_tune.argtypes = [P(Geom), P(Batch), ctypes.c_int32, ctypes.c_int32, vp, vp, ctypes.c_size_t, vp,
                             P(Config)]
    L.idiwf_tune.restype = st
    L.idiwf_workspace_error.argtypes = [vp, vp]
    L.idiwf_workspace_error.restype = st
    L.idiwf_microbench.argtypes = [ctypes.c_int32, vp, vp, P(ctypes.c_double)]
    L.idiwf_microbench.restype = st
    L.idiwf_last_error_string.argtypes = []
    L.idiwf_last_error_string.restype = ctypes.c_char_p
    L.idiwf_version.argtypes = []
    L.idiwf_version.restype = ctypes.c_int32
    _lib = L
    return L


def check(status):
    if status != OK:
        msg = load().idiwf_last_error_string().decode(errors="replace")
        raise IdiwfError(status, msg)
