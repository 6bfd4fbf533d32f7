"""The allocation-free forward entry point, called through the C ABI.

idiwf_forward_noalloc exists for callers that cannot allocate device memory
or hand the library a workspace (code running inside another framework's
memory pool or allocator hooks, or plug-ins whose host forbids device
allocation).  It keeps its scratch in a static 16 MiB device array.  These
tests check it against the regular entry point (idiwf_forward, split
precision, caller workspace) and against the FP64 oracle on the same inputs,
on two calls in a row with different inputs, so that state left in the shared
scratch by the first call cannot leak into the second; on a batch whose
images take the pixel-run, per-pixel and exact near-field kernels in one
call; and the device-side errors read back with idiwf_forward_noalloc_error.

The file name sorts last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""

import ctypes

import numpy as np
import pytest
import torch

import oracle
from idi_b200 import _native as nat
from idi_b200.simulation import _core
from tests.helpers import K64, atoms, rel_field_err, rng, sphere

pytestmark = pytest.mark.gpu

# split-precision tolerances used by the forward parity tests: field error
# relative to the rms field, and relative intensity over pixels with
# I >= 1e-3 <I>; both entry points run the same kernels
SPLIT_FIELD = 2e-5
SPLIT_REL_MASKED = 1e-4


def _vs_oracle(E, og, flags, at, amp, what):
    ref = oracle.wavefield(og, flags, at, amp)
    assert rel_field_err(E, ref) <= SPLIT_FIELD, (what, rel_field_err(E, ref))
    m = oracle.intensity_metrics(np.abs(E) ** 2, np.abs(ref) ** 2)
    assert m["max_rel_masked"] <= SPLIT_REL_MASKED, (what, m)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


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
    og = oracle.geometry([61, 47], 75.0, 1e5, K64, (0.02, -0.01), (30.0, 10.0))
    results = []
    for call, counts in enumerate(([3000, 0, 1234], [777, 5000])):
        imgs = [atoms(sphere(g0, c, 0.012), g0.uniform(0, 2 * np.pi, c)) for c in counts]
        at_np = np.ascontiguousarray(np.concatenate(imgs))
        at = torch.from_numpy(at_np).cuda()
        amp_np = g0.uniform(0.5, 1.5, sum(counts)).astype(np.float32)
        amp = torch.from_numpy(amp_np).cuda()
        off = np.concatenate([[0], np.cumsum(counts)])
        st, E = _noalloc(lib, geom, at, off, amplitudes=amp)
        assert st == nat.OK, lib.idiwf_last_error_string()
        assert lib.idiwf_forward_noalloc_error(_stream()) == nat.OK
        ref = _core.forward(at, off, geom, nat.SPLIT, nat.OUT_C128, amplitudes=amp)
        torch.cuda.synchronize()
        E = E.cpu().numpy()
        ref = ref.cpu().numpy()
        for b, c in enumerate(counts):
            if c == 0:
                assert np.all(E[b] == 0)
            else:
                assert rel_field_err(E[b], ref[b]) <= SPLIT_FIELD, (call, b)
                _vs_oracle(E[b], og, oracle.NF, at_np[off[b]:off[b + 1]], amp_np[off[b]:off[b + 1]].astype(np.float64),
                           (call, b))
        results.append(E)
    assert results[0].shape != results[1].shape


def test_noalloc_all_split_paths_in_one_call():
    """8 keV, 10 um pixels at 1 cm (ny a multiple of the pixel run): a 10 nm
    sphere takes the pixel-run kernel, a 50 nm sphere (beyond the run bound,
    inside the second-order bound) the per-pixel kernel and a 1 um object the
    exact near-field kernel, with an empty image between them -- all in one
    call and its shared work counters, twice in a row."""
    lib = nat.load()
    g0 = rng(4545)
    k = 2 * np.pi / (1.24 / 8000.0)
    geom = _core.make_geom([40, 32], 10.0, 1e4, k, flags=nat.NF)
    og = oracle.geometry([40, 32], 10.0, 1e4, k)
    for call in range(2):
        counts = [1800, 0, 1100, 700]
        radii = [0.01, 0.0, 0.05, 1.0]
        imgs = [atoms(sphere(g0, c, r), g0.uniform(0, 2 * np.pi, c)) for c, r in zip(counts, radii)]
        at_np = np.ascontiguousarray(np.concatenate(imgs))
        at = torch.from_numpy(at_np).cuda()
        off = np.concatenate([[0], np.cumsum(counts)])
        st, E = _noalloc(lib, geom, at, off)
        assert st == nat.OK, lib.idiwf_last_error_string()
        assert lib.idiwf_forward_noalloc_error(_stream()) == nat.OK
        ref = _core.forward(at, off, geom, nat.SPLIT, nat.OUT_C128)
        torch.cuda.synchronize()
        E, ref = E.cpu().numpy(), ref.cpu().numpy()
        assert np.all(E[1] == 0)
        for b in (0, 2, 3):
            assert rel_field_err(E[b], ref[b]) <= SPLIT_FIELD, (call, b)
            _vs_oracle(E[b], og, oracle.NF, imgs[b], None, (call, b))


def test_noalloc_device_errors_are_read_back():
    """Emitters beyond the split phase range, and a near-field image outside
    the split kernels' range, are reported by idiwf_forward_noalloc_error;
    the next clean call clears the word."""
    lib = nat.load()
    geom = _core.make_geom([8, 8], 75.0, 1e5, K64, flags=nat.NF)
    at = torch.zeros((4, 4), dtype=torch.float64, device="cuda")
    at[0, 0] = 1e4
    st, _ = _noalloc(lib, geom, at, [0, 4])
    assert st == nat.OK
    assert lib.idiwf_forward_noalloc_error(_stream()) == nat.ERR_UNSUPPORTED
    assert b"phase range" in lib.idiwf_last_error_string()
    at[0, 0] = 0.0
    st, _ = _noalloc(lib, geom, at, [0, 4])
    assert st == nat.OK and lib.idiwf_forward_noalloc_error(_stream()) == nat.OK
    # a 100 um sphere at 1000 um, 100 eV: remainder ~100 rad, outside the split range
    g0 = rng(4646)
    far = _core.make_geom(4, 10.0, 1000.0, 2 * np.pi / (1.24 / 100.0), flags=nat.NF)
    big = torch.from_numpy(atoms(sphere(g0, 64, 100.0), g0.uniform(0, 2 * np.pi, 64))).cuda()
    st, _ = _noalloc(lib, far, big, [0, 64])
    assert st == nat.OK
    assert lib.idiwf_forward_noalloc_error(_stream()) == nat.ERR_UNSUPPORTED
    assert b"near-field" in lib.idiwf_last_error_string()


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
