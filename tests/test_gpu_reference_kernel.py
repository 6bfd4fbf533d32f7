"""The reference's own GPU kernel (idi/simulation/sim.cu wfkerneld / wfkernelf,
compiled from the reference tree for sm_100a into oracle/_ref by
`make -C oracle ref`, settings "nf", no 1/r): checked against the oracle and
timed beside this library's kernels on the same inputs.  Skipped where
oracle/_ref was not built.

The reference kernel takes the detector geometry as float32 scalars
(idi/simulation/cuda.py:95-106), so its agreement with the FP64 oracle is
limited by the float32 pixel coordinates; the check is a coarse sanity bound.
"""

import ctypes
import os

import numpy as np
import pytest
import torch

import oracle
from idi_b200 import _native as nat
from idi_b200.simulation import _core
from tests.helpers import K64, atoms, rng, sphere

pytestmark = pytest.mark.gpu

REF_LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "libref_wf.so")


@pytest.fixture(scope="module")
def reflib():
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref/libref_wf.so not built")
    L = ctypes.CDLL(REF_LIB)
    L.ref_wf_launch.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_float] * 5 + \
                               [ctypes.c_int] * 3 + [ctypes.c_void_p]
    L.ref_wf_launch.restype = ctypes.c_int
    return L


def _time(fn, reps=3):
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e30
    for _ in range(reps):
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def test_reference_gpu_kernel_vs_oracle_and_timing(reflib):
    g0 = rng(2027)
    n, nd = 20000, 256
    at = atoms(sphere(g0, n, 0.01), g0.uniform(0, 2 * np.pi, n))
    d_at = torch.from_numpy(at).cuda()
    out = torch.empty((nd, nd), dtype=torch.complex128, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def ref_fp64():
        st = reflib.ref_wf_launch(0, out.data_ptr(), d_at.data_ptr(), 0.0, 0.0, 1e5, 75.0, K64, nd, nd, n, stream)
        assert st == 0

    ms_ref = _time(ref_fp64)
    E_ref = out.cpu().numpy()
    og = oracle.geometry(nd, 75.0, 1e5, K64)
    sub = (slice(0, 256, 17), slice(0, 256, 13))
    truth = np.abs(oracle.wavefield(og, oracle.NF, at)[sub]) ** 2
    # float32 k puts up to ~0.5 rad of constant phase per pixel into the
    # reference's fields; intensities are unaffected by it
    err = np.abs(np.abs(E_ref[sub]) ** 2 - truth).max() / truth.mean()
    assert err < 1e-2

    geom = _core.make_geom(nd, 75.0, 1e5, K64, flags=nat.NF)
    ms_d = _time(lambda: _core.forward(d_at, [0, n], geom, nat.DOUBLE, nat.OUT_C128))
    ms_s = _time(lambda: _core.forward(d_at, [0, n], geom, nat.SPLIT, nat.OUT_C128))
    pairs = n * nd * nd
    print(f"\nemitter-pixel pairs/s, 20k emitters x 256x256, near field: reference wfkerneld (sm_100a) "
          f"{pairs / ms_ref * 1e3:.3g}; idiwf double {pairs / ms_d * 1e3:.3g}; idiwf split {pairs / ms_s * 1e3:.3g}")
    assert ms_s < ms_ref
