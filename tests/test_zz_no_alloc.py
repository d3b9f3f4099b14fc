"""ctb_fbp_noalloc: the FBP entry point for callers that cannot allocate device
memory (a caller-owned memory pool, a real-time loop that must not wait on an
allocator, a host whose allocator is not cudaMalloc). It keeps every
intermediate in the library's static device array; the caller only passes the
input sinograms and the output volume.

Checked here through the C ABI on calls in a row with different geometry,
angles and filter (a later call must not see an earlier call's leftovers):
against the oracle (SerialBackend's float path at rel-L2 <= 1e-5, max-abs <=
1e-4 * max|f|, or, where the output is larger and SerialBackend's own float
rounding approaches that bar, against the FP64 rerun at the same tolerance),
and against the context-based ctb_fbp_d on the same inputs. The cases include
explicit non-uniform angles and an output larger than the detector, which
exercise the per-angle edge-tap decisions, and the largest angle count the
static array holds for a geometry; one more angle must be refused. This file
is collected last so that a failure here leaves every other GPU test already
run.
"""
import concurrent.futures as cf
import ctypes
import math

import numpy as np
import pytest

import oracle as O
import qtctreconstruction_b200 as ctb

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
MAX_ABS = 1e-4

# The static array: 16 MiB, of which the filtered rows get what the fixed
# tables leave, in float4 bins: the error word (256 B), 2048 angles of degrees
# (4 B) and trig (24 B), the spectrum of an 8192-long convolution (8 B each)
# and the FFT twiddle tables of that length (15 (8192/8 - 1) + 4096 complex
# values, rounded up to 256 B); the packed copies the shorter lengths add fit
# in the same room.
_TW_BYTES = (8 * (15 * (8192 // 8 - 1) + 8192 // 2) + 255) // 256 * 256
FILT_CAPACITY = ((16 << 20) - (256 + 4 * 2048 + 24 * 2048 + 8 * 8192 + _TW_BYTES)) // 16


def _pitch(bins, n_out):
    """Filtered-row pitch (float4 bins) of the backprojector's layout for
    this detector and output size: guard bins either side of square_bins so
    that every staged window of every tile shape lies inside the row."""
    sq, _, _ = ctb.pad_geometry(bins)
    r = n_out // 2
    n_pad = (n_out + 63) // 64 * 64
    m = max(r, n_pad - 1 - r)
    reach = m * math.sqrt(2.0) + 3.0
    dc = sq // 2
    left = math.ceil(reach + 2.0 - dc)
    right = math.ceil(dc + reach + 76 + 2.0 - sq)
    return max(left, 0) + sq + max(right, 0)


def _declare():
    lib = ctb.library()
    lib.ctb_fbp_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_void_p]
    return lib


def _sinograms(n_img, depth, na, nd, seed, angles=None):
    rng = np.random.default_rng(seed)
    vol = np.zeros((depth, n_img, n_img), np.float32)
    yy, xx = np.mgrid[0:n_img, 0:n_img].astype(np.float64)
    for z in range(depth):
        for _ in range(4):
            cx, cy = rng.uniform(0.3 * n_img, 0.7 * n_img, 2)
            a, b = rng.uniform(0.05 * n_img, 0.2 * n_img, 2)
            vol[z][((xx - cx) / a) ** 2 + ((yy - cy) / b) ** 2 <= 1.0] += np.float32(rng.uniform(0.1, 1.0))
    if angles is None:
        return np.stack([O.sinogram_f32(vol[z], na, nd)[0] for z in range(depth)])
    return np.stack([O.sinogram_f64(vol[z], na, nd, angles)[0].astype(np.float32) for z in range(depth)])


def _oracle(sinos, angles, n_out, kind, f64):
    def one(z):
        if f64:
            return O.reconstruct_slice_f64(sinos[z].astype(np.float64), angles, n_out, kind)
        return O.reconstruct_slice_f32(sinos[z], angles, n_out, kind)
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        return np.stack(list(ex.map(one, range(sinos.shape[0]))))


# (image n, output size, depth, angles, filter, explicit angles, seed, oracle)
CASES = [(96, 96, 3, 120, ctb.FilterType.Ramp, False, 5, "serial"),
         (64, 64, 4, 90, ctb.FilterType.Hann, False, 6, "serial"),
         (48, 112, 2, 75, ctb.FilterType.SheppLogan, True, 7, "serial"),   # output > detector, explicit angles
         (128, 320, 2, None, ctb.FilterType.Cosine, True, 8, "fp64")]     # angle count at the array's limit


def test_fbp_noalloc_against_oracle_and_fbp_d():
    import torch
    lib = _declare()
    stream = torch.cuda.Stream()
    with ctb.B200Backend(0) as be:
        be.set_stream(stream.cuda_stream)
        for n_img, n, depth, na, kind, explicit, seed, ref_kind in CASES:
            nd = ctb.odd_detector_count(n_img)
            if na is None:
                na = FILT_CAPACITY // _pitch(nd, n)
                assert na <= 2048
            rng = np.random.default_rng(seed)
            angles = (np.sort(rng.uniform(0.0, 180.0, na)).astype(np.float32) if explicit
                      else O.uniform_angles_deg(na))
            sinos_h = _sinograms(n_img, depth, na, nd, seed, angles if explicit else None)
            sinos = torch.from_numpy(sinos_h).cuda()
            ref = torch.zeros((depth, n, n), dtype=torch.float32, device="cuda")
            out = torch.full((depth, n, n), float("nan"), dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            be.fbp_d(sinos.data_ptr(), depth, na, nd, n, int(kind), ref.data_ptr(),
                     angles_deg=angles if explicit else None)
            be.synchronize()
            ang_ptr = angles.ctypes.data if explicit else None
            st = lib.ctb_fbp_noalloc(ctypes.c_void_p(sinos.data_ptr()), depth, na, nd, ang_ptr, n, int(kind),
                                     ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
            assert st == 0, lib.ctb_status_string(st)
            a, r = out.cpu().numpy(), ref.cpu().numpy()
            assert np.all(np.isfinite(a))
            assert O.rel_l2(a, r) <= REL_L2
            assert O.max_abs_rel(a, r) <= MAX_ABS
            orc = _oracle(sinos_h, angles, n, int(kind), ref_kind == "fp64")
            for z in range(depth):
                assert O.rel_l2(a[z], orc[z]) <= REL_L2, (n, na, z, O.rel_l2(a[z], orc[z]))
                assert O.max_abs_rel(a[z], orc[z]) <= MAX_ABS, (n, na, z, O.max_abs_rel(a[z], orc[z]))


def test_fbp_noalloc_rejects_oversize_and_bad_filter():
    lib = _declare()
    dummy = ctypes.c_void_p(16)  # never dereferenced: the argument checks come first
    assert lib.ctb_fbp_noalloc(dummy, 5, 90, 91, None, 64, 0, dummy, None) == 4       # depth > 4
    assert lib.ctb_fbp_noalloc(dummy, 1, 4096, 91, None, 64, 0, dummy, None) == 4     # angles > 2048
    assert lib.ctb_fbp_noalloc(dummy, 1, 1440, 4000, None, 64, 0, dummy, None) == 4   # conv length > 8192
    # angles and convolution length within their limits, filtered rows not
    assert _pitch(91, 2048) * 2000 > FILT_CAPACITY
    assert lib.ctb_fbp_noalloc(dummy, 1, 2000, 91, None, 2048, 0, dummy, None) == 4
    nd, n = ctb.odd_detector_count(128), 320
    na_max = FILT_CAPACITY // _pitch(nd, n)
    assert lib.ctb_fbp_noalloc(dummy, 1, na_max + 1, nd, None, n, 0, dummy, None) == 4
    # filter ids outside CTB_FILTER_RAMP .. CTB_FILTER_BARTLETT are invalid, as for ctb_fbp_d
    assert lib.ctb_fbp_noalloc(dummy, 1, 90, 91, None, 64, 6, dummy, None) == 1
    assert lib.ctb_fbp_noalloc(dummy, 1, 90, 91, None, 64, -1, dummy, None) == 1
