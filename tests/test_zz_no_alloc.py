"""The allocation-free forward entry point, called through the C ABI.

idiwf_forward_noalloc exists for callers that cannot allocate device memory
or hand the library a workspace (code running inside another framework's
memory pool or allocator hooks, or plug-ins whose host forbids device
allocation).  It keeps its scratch in a static 16 MiB device array.  This
test checks it against the regular entry point (idiwf_forward, split
precision, caller workspace) on the same inputs, on two calls in a row with
different inputs, so that state left in the shared scratch by the first call
cannot leak into the second.

The file name sorts last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""

import ctypes

import numpy as np
import pytest
import torch

from idi_b200 import _native as nat
from idi_b200.simulation import _core
from tests.helpers import K64, atoms, rel_field_err, rng, sphere

pytestmark = pytest.mark.gpu

# split-precision tolerance used by the forward parity tests (field error
# relative to the rms field); both entry points run the same kernel
SPLIT_FIELD = 2e-5


def _noalloc(lib, geom, at, offsets, out_kind=nat.OUT_C128, amplitudes=None):
    off = np.ascontiguousarray(np.asarray(offsets, np.int64))
    b = nat.Batch()
    b.n_images = off.size - 1
    b.offsets = off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    b.atoms = ctypes.c_void_p(at.data_ptr())
    b.amplitudes = None if amplitudes is None else ctypes.c_void_p(amplitudes.data_ptr())
    b.amp_dtype = nat.F32 if amplitudes is not None and amplitudes.dtype == torch.float32 else nat.F64
    dtype = {nat.OUT_C128: torch.complex128, nat.OUT_I64: torch.float64}[out_kind]
    out = torch.empty((b.n_images, geom.nx, geom.ny), dtype=dtype, device=at.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = lib.idiwf_forward_noalloc(ctypes.byref(geom), ctypes.byref(b), out_kind, ctypes.c_void_p(out.data_ptr()),
                                   stream)
    return st, out


def test_noalloc_forward_matches_workspace_forward_twice():
    lib = nat.load()
    g0 = rng(4242)
    geom = _core.make_geom([61, 47], 75.0, 1e5, K64, (0.02, -0.01), (30.0, 10.0), nat.NF)
    results = []
    for call, counts in enumerate(([3000, 0, 1234], [777, 5000])):
        imgs = [atoms(sphere(g0, c, 0.012), g0.uniform(0, 2 * np.pi, c)) for c in counts]
        at = torch.from_numpy(np.ascontiguousarray(np.concatenate(imgs))).cuda()
        amp = torch.from_numpy(g0.uniform(0.5, 1.5, sum(counts)).astype(np.float32)).cuda()
        off = np.concatenate([[0], np.cumsum(counts)])
        st, E = _noalloc(lib, geom, at, off, amplitudes=amp)
        assert st == nat.OK, lib.idiwf_last_error_string()
        ref = _core.forward(at, off, geom, nat.SPLIT, nat.OUT_C128, amplitudes=amp)
        torch.cuda.synchronize()
        E = E.cpu().numpy()
        ref = ref.cpu().numpy()
        for b, c in enumerate(counts):
            if c == 0:
                assert np.all(E[b] == 0)
            else:
                assert rel_field_err(E[b], ref[b]) <= SPLIT_FIELD, (call, b)
        results.append(E)
    assert results[0].shape != results[1].shape


def test_noalloc_intensity_output_and_size_limit():
    lib = nat.load()
    g0 = rng(4343)
    geom = _core.make_geom([32, 32], 75.0, 1e5, K64, flags=nat.NF)
    n = 2000
    at = torch.from_numpy(atoms(sphere(g0, n, 0.01), g0.uniform(0, 2 * np.pi, n))).cuda()
    st, I = _noalloc(lib, geom, at, [0, n], out_kind=nat.OUT_I64)
    assert st == nat.OK
    ref = _core.forward(at, [0, n], geom, nat.SPLIT, nat.OUT_I64)
    torch.cuda.synchronize()
    # The regular entry point splits this small detector's work over emitter
    # chunks and adds the chunk sums in FP64; the allocation-free one sums in
    # one pass.  The field tolerance above, |dE| <= SPLIT_FIELD * E_rms, bounds
    # the intensity difference by 2 |E| |dE|.
    I, ref = I.cpu().numpy(), ref.cpu().numpy()
    bound = 2 * SPLIT_FIELD * np.sqrt(ref) * np.sqrt(ref.mean())
    assert np.all(np.abs(I - ref) <= bound), float(np.max(np.abs(I - ref) / bound))
    # beyond the static scratch: rejected on the host with a clear message
    big = torch.zeros((330000, 4), dtype=torch.float64, device="cuda")
    st, _ = _noalloc(lib, geom, big, [0, 330000])
    assert st == nat.ERR_UNSUPPORTED
    assert b"16 MiB" in lib.idiwf_last_error_string()
