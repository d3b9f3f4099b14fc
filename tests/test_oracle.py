"""The oracle itself: pinned against the reference's own outputs (CPU only).

The float restatement must reproduce SerialBackend bit for bit on every golden
case; the FP64 rerun must sit within the float path's known error.
"""
import os

import numpy as np
import pytest

import oracle as O
from oracle import reference as R


def test_filters_bit_exact(golden):
    for L in (64, 128, 1024):
        for kind in range(6):
            np.testing.assert_array_equal(O.filter_f32(L, kind), golden[f"filter_L{L}_k{kind}"])


def test_filter_f64_close_to_f32(golden):
    for kind in range(6):
        H32 = golden[f"filter_L1024_k{kind}"]
        H64 = O.filter_f64(1024, kind)
        assert O.rel_l2(H32, H64) < 1e-6


def test_ramp_spectrum_shape():
    # Ram-Lak: H[k] ~ 2k/L away from the lowest bins (|k|/L ramp of the analytic filter)
    L = 1024
    H = O.filter_f64(L, O.RAMP)
    k = np.arange(L // 2 + 1)
    mid = slice(8, L // 2 - 8)
    assert H[0] == 0.0
    assert np.max(np.abs(H[mid] - 2.0 * k[mid] / L)) < 2e-3


@pytest.mark.parametrize("case", ["cfg_like", "native_nd", "odd_n", "neg_min_zero_bg", "constant",
                                  "zeros", "hu_like", "bartlett_small_nd"])
def test_serial_restatement_bit_exact(golden, case):
    n, na, nd, kind = (int(v) for v in golden[f"{case}_meta"])
    sl = golden[f"{case}_slice"]
    sino, ang, mm = O.sinogram_f32(sl, na, nd)
    np.testing.assert_array_equal(sino, golden[f"{case}_sino"])
    np.testing.assert_array_equal(ang, golden[f"{case}_angles"])
    np.testing.assert_array_equal(mm, golden[f"{case}_minmax"])
    rec = O.reconstruct_slice_f32(sino, ang, n, kind)
    np.testing.assert_array_equal(rec, golden[f"{case}_recon"])


@pytest.mark.parametrize("case", ["cfg_like", "odd_n", "neg_min_zero_bg", "hu_like"])
def test_fp64_rerun_within_float_error(golden, case):
    n, na, nd, kind = (int(v) for v in golden[f"{case}_meta"])
    sl = golden[f"{case}_slice"]
    s64, _ = O.sinogram_f64(sl, na, nd)
    r64 = O.reconstruct_slice_f64(s64, golden[f"{case}_angles"], n, kind)
    r32 = golden[f"{case}_recon"]
    assert O.rel_l2(r32, r64) < 2e-5
    assert O.max_abs_rel(r32, r64) < 5e-5


def test_volume_restatement_bit_exact(golden):
    vol = golden["volume_in"]
    na, kind = (int(v) for v in golden["volume_meta"])
    out = O.reconstruct_volume_f32(vol, na, vol.shape[1], kind)
    np.testing.assert_array_equal(out, golden["volume_serial"])


def test_generator3d_restatement_bit_exact(golden):
    nx, ny, nz, n_ell, seed = (int(v) for v in golden["gen3d_meta"])
    vol = O.generator3d(nx, ny, nz, float(golden["gen3d_radius"][0]), n_ell, seed)
    np.testing.assert_array_equal(vol, golden["gen3d_vol"])


def test_point_cloud_restatement(golden):
    pts = O.point_cloud(golden["gen3d_vol"], float(golden["pc_threshold"][0]))
    np.testing.assert_array_equal(pts, golden["pc_points"])


def test_phantom_sum_properties():
    # one axis-aligned sphere of radius 0.5 at the origin, density 2
    p = np.zeros(16, np.float32)
    p[3], p[7], p[11] = 1.0, 1.0, 1.0
    p[12:15] = 1.0 / 0.25
    p[15] = 2.0
    v = O.phantom_sum(p, 20, 20, 20)
    X = (2 * np.arange(20) - 19) / 20.0
    r2 = X[None, None, :] ** 2 + X[None, :, None] ** 2 + X[:, None, None] ** 2
    assert np.all(v[r2 <= 0.249] == 2.0)
    assert np.all(v[r2 >= 0.251] == 0.0)


@pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")
def test_reference_build_matches_golden(golden):
    # the reference library that generated the fixtures still reproduces them
    sl = golden["cfg_like_slice"]
    n, na, nd, kind = (int(v) for v in golden["cfg_like_meta"])
    sino, ang, mm = R.compute_sinogram(R.SERIAL, sl, na, nd)
    np.testing.assert_array_equal(sino, golden["cfg_like_sino"])
    rec = R.reconstruct_slice(R.SERIAL, sino, ang, n, kind, mm[0], mm[1])
    np.testing.assert_array_equal(rec, golden["cfg_like_recon"])


@pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")
def test_openmp_fbp_matches_serial_fbp_on_same_sinogram(golden):
    # the reference's two FBP implementations share the filter + BP math; only
    # OpenMP's reconstructSlice denormalises (OpenMPBackend.cpp:37-59)
    sl = golden["cfg_like_slice"]
    n, na, nd, kind = (int(v) for v in golden["cfg_like_meta"])
    sino, ang, mm = R.compute_sinogram(R.SERIAL, sl, na, nd)
    ser = R.reconstruct_slice(R.SERIAL, sino, ang, n, kind, mm[0], mm[1])
    omp = R.reconstruct_slice(R.OPENMP, sino, ang, n, kind, 0.0, 1.0)  # span 1, min 0: identity
    assert O.rel_l2(omp, ser) < 1e-6


# ------------------------------------------- the CUDA backend's conventions
CUDA_CASES = ["ramp64", "shepp96", "hann128_even", "hamming80", "cosine48", "bartlett72"]


@pytest.fixture(scope="module")
def cuda_golden():
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "cuda_conv.npz"))


@pytest.mark.parametrize("case", CUDA_CASES)
def test_cuda_convention_oracle_pinned(cuda_golden, case):
    """The FP64 restatement of CUDABackend against outputs of CUDABackend itself
    (float arithmetic and cuFFT on the GPU): sinograms to 2e-6, reconstructions
    to 1e-5 rel-L2."""
    g = cuda_golden
    n, na, nd, kind = (int(v) for v in g[f"{case}_meta"])
    sino, ang, mm = O.cc_sinogram_f64(g[f"{case}_slice"], na, nd)
    np.testing.assert_array_equal(mm, g[f"{case}_minmax"])
    assert O.rel_l2(sino, g[f"{case}_sino"]) <= 2e-6
    rec = O.cc_reconstruct_slice_f64(g[f"{case}_sino"], ang, n, kind, *g[f"{case}_minmax"])
    assert O.rel_l2(rec, g[f"{case}_recon"]) <= 1e-5
    assert O.max_abs_rel(rec, g[f"{case}_recon"]) <= 1e-5


def test_cuda_convention_volume_pinned(cuda_golden):
    g = cuda_golden
    n, depth, na, kind = (int(v) for v in g["volume_meta"])
    out = O.cc_reconstruct_volume_f64(g["volume_in"], na, kind)
    assert O.rel_l2(out, g["volume_out"]) <= 1e-5
