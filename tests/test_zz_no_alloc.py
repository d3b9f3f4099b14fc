"""ctb_fbp_noalloc: the FBP entry point for callers that cannot allocate device
memory (a caller-owned memory pool, a real-time loop that must not wait on an
allocator, a host whose allocator is not cudaMalloc). It keeps every
intermediate in the library's static device array; the caller only passes the
input sinograms and the output volume.

Checked here through the C ABI against the context-based ctb_fbp_d on the same
inputs, on two calls in a row with different geometry and filter (the second
must not see the first call's leftovers), within the parity tolerance of the
GPU tests. This file is collected last so that a failure here leaves every
other GPU test already run.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
import qtctreconstruction_b200 as ctb

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
MAX_ABS = 1e-4


def _sinograms(n, depth, na, nd, seed):
    rng = np.random.default_rng(seed)
    vol = np.zeros((depth, n, n), np.float32)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    for z in range(depth):
        for _ in range(4):
            cx, cy = rng.uniform(0.3 * n, 0.7 * n, 2)
            a, b = rng.uniform(0.05 * n, 0.2 * n, 2)
            vol[z][((xx - cx) / a) ** 2 + ((yy - cy) / b) ** 2 <= 1.0] += np.float32(rng.uniform(0.1, 1.0))
    return np.stack([O.sinogram_f32(vol[z], na, nd)[0] for z in range(depth)])


def test_fbp_noalloc_matches_fbp_d_twice():
    import torch
    lib = ctb.library()
    lib.ctb_fbp_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_void_p]
    stream = torch.cuda.Stream()
    cases = [(96, 3, 120, ctb.odd_detector_count(96), ctb.FilterType.Ramp, 5),
             (64, 4, 90, ctb.odd_detector_count(64), ctb.FilterType.Hann, 6)]
    with ctb.B200Backend(0) as be:
        be.set_stream(stream.cuda_stream)
        for n, depth, na, nd, kind, seed in cases:
            sinos = torch.from_numpy(_sinograms(n, depth, na, nd, seed)).cuda()
            ref = torch.zeros((depth, n, n), dtype=torch.float32, device="cuda")
            out = torch.full((depth, n, n), float("nan"), dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            be.fbp_d(sinos.data_ptr(), depth, na, nd, n, int(kind), ref.data_ptr())
            be.synchronize()
            st = lib.ctb_fbp_noalloc(ctypes.c_void_p(sinos.data_ptr()), depth, na, nd, None, n, int(kind),
                                     ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
            assert st == 0, lib.ctb_status_string(st)
            a, r = out.cpu().numpy(), ref.cpu().numpy()
            assert np.all(np.isfinite(a))
            assert O.rel_l2(a, r) <= REL_L2
            assert O.max_abs_rel(a, r) <= MAX_ABS


def test_fbp_noalloc_rejects_oversize():
    lib = ctb.library()
    lib.ctb_fbp_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_void_p]
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    assert lib.ctb_fbp_noalloc(dummy, 5, 90, 91, None, 64, 0, dummy, None) == 4       # depth > 4
    assert lib.ctb_fbp_noalloc(dummy, 1, 4096, 91, None, 64, 0, dummy, None) == 4     # angles > 2048
    assert lib.ctb_fbp_noalloc(dummy, 1, 1440, 4000, None, 64, 0, dummy, None) == 4   # conv length > 8192
