"""The reference CUDA backend's conventions (CTB_CONVENTION_CUDA) on the GPU.

Checked against outputs of the reference's own CUDA backend
(tests/golden/cuda_conv.npz, written by tests/golden/make_cuda_golden.py from
CUDABackend.cu) and against the FP64 restatement of those conventions in the
oracle, which the CPU tests pin to the same fixtures. Tolerance: rel-L2 <= 1e-5
and max-abs <= 1e-4 * max|f|, as the Serial-convention parity tests; the
reference itself computes in float with cuFFT.
"""
import os

import numpy as np
import pytest

import oracle as O
import qtctreconstruction_b200 as ctb
from qtctreconstruction_b200 import FilterType, ReconstructionParams

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
MAX_ABS = 1e-4
CASES = ["ramp64", "shepp96", "hann128_even", "hamming80", "cosine48", "bartlett72"]


@pytest.fixture(scope="module")
def cg():
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "cuda_conv.npz"))


@pytest.fixture
def cuda_be(backend):
    backend.set_convention(ctb.CONVENTION_CUDA)
    yield backend
    backend.set_convention(ctb.CONVENTION_SERIAL)


def _close(a, ref):
    assert O.rel_l2(a, ref) <= REL_L2, O.rel_l2(a, ref)
    assert O.max_abs_rel(a, ref) <= MAX_ABS, O.max_abs_rel(a, ref)


@pytest.mark.parametrize("case", CASES)
def test_sinogram_matches_cuda_backend(cuda_be, cg, case):
    n, na, nd, kind = (int(v) for v in cg[f"{case}_meta"])
    s = cuda_be.computeSinogram(cg[f"{case}_slice"], na, nd)
    np.testing.assert_array_equal(np.float32([s.original_min_hu, s.original_max_hu]), cg[f"{case}_minmax"])
    _close(s.data, cg[f"{case}_sino"])
    f64, _, _ = O.cc_sinogram_f64(cg[f"{case}_slice"], na, nd)
    _close(s.data, f64)


@pytest.mark.parametrize("case", CASES)
def test_slice_matches_cuda_backend(cuda_be, cg, case):
    n, na, nd, kind = (int(v) for v in cg[f"{case}_meta"])
    lo, hi = (float(v) for v in cg[f"{case}_minmax"])
    ang = ctb.uniform_angles_deg(na)
    sino = ctb.Sinogram(data=cg[f"{case}_sino"], angles_deg=ang, original_min_hu=lo, original_max_hu=hi)
    rec = cuda_be.reconstructSlice(sino, n, ReconstructionParams(FilterType(kind), na))
    _close(rec, cg[f"{case}_recon"])
    _close(rec, O.cc_reconstruct_slice_f64(cg[f"{case}_sino"], ang, n, kind, lo, hi))


def test_volume_matches_cuda_backend(cuda_be, cg):
    n, depth, na, kind = (int(v) for v in cg["volume_meta"])
    out = cuda_be.reconstructVolume(cg["volume_in"], ReconstructionParams(FilterType(kind), na))
    _close(out, cg["volume_out"])
    _close(out, O.cc_reconstruct_volume_f64(cg["volume_in"], na, kind))


def test_larger_slice_against_fp64(cuda_be):
    rng = np.random.default_rng(5)
    n, na, nd = 256, 300, 363
    s = np.zeros((n, n), np.float32)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    for _ in range(6):
        cx, cy = rng.uniform(0.3 * n, 0.7 * n, 2)
        a, b = rng.uniform(0.05 * n, 0.2 * n, 2)
        s[((xx - cx) / a) ** 2 + ((yy - cy) / b) ** 2 <= 1.0] += np.float32(rng.uniform(100, 900))
    sino = cuda_be.computeSinogram(s, na, nd)
    f64, ang, mm = O.cc_sinogram_f64(s, na, nd)
    _close(sino.data, f64)
    rec = cuda_be.reconstructSlice(sino, n, ReconstructionParams(FilterType.SheppLogan, na))
    _close(rec, O.cc_reconstruct_slice_f64(sino.data, ang, n, int(FilterType.SheppLogan), *mm))


def test_convention_switch_leaves_serial_unchanged(backend, golden):
    n, na, nd, kind = (int(v) for v in golden["cfg_like_meta"])
    a = backend.computeSinogram(golden["cfg_like_slice"], na, nd).data
    backend.set_convention(ctb.CONVENTION_CUDA)
    backend.computeSinogram(golden["cfg_like_slice"], na, nd)
    backend.set_convention(ctb.CONVENTION_SERIAL)
    np.testing.assert_array_equal(backend.computeSinogram(golden["cfg_like_slice"], na, nd).data, a)
    with pytest.raises(ctb.CtbError):
        backend.set_convention(5)


def test_non_square_sinogram_against_fp64(cuda_be):
    rng = np.random.default_rng(8)
    w, h, na, nd = 90, 52, 70, 107
    s = np.zeros((h, w), np.float32)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    for _ in range(4):
        cx, cy = rng.uniform(0.3 * w, 0.7 * w), rng.uniform(0.3 * h, 0.7 * h)
        s[((xx - cx) / 9.0) ** 2 + ((yy - cy) / 6.0) ** 2 <= 1.0] += np.float32(rng.uniform(50, 500))
    sino = cuda_be.computeSinogram(s, na, nd)
    f64, _, _ = O.cc_sinogram_f64(s, na, nd)
    _close(sino.data, f64)
