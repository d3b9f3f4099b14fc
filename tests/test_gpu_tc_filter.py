"""The tensor-core filter option (CTB_FILTER_MODE_TC_BF16X3) on the GPU.

The option computes the same linear operator as the FFT path (the reference's
ramp filter with its dropped Nyquist bin) as a Toeplitz-matrix product on the
tcgen05 tensor cores with both factors split into three BF16 terms (six
products, about 24 significant bits). It is held to the product's gate,
rel-L2 <= 1e-5 and max-abs <= 1e-4 * max|f| against the FP64 rerun of
SerialBackend, like the FFT path.
"""
import numpy as np
import pytest

import oracle as O
import qtctreconstruction_b200 as ctb
from qtctreconstruction_b200 import FilterType, ReconstructionParams

pytestmark = pytest.mark.gpu

TC_REL_L2 = 1e-5
TC_MAX_ABS = 1e-4


def _slice(rng, n, k):
    s = np.zeros((n, n), np.float32)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    for _ in range(k):
        cx, cy = rng.uniform(0.25 * n, 0.75 * n, 2)
        a, b = rng.uniform(0.05 * n, 0.25 * n, 2)
        s[((xx - cx) / a) ** 2 + ((yy - cy) / b) ** 2 <= 1.0] += np.float32(rng.uniform(-0.3, 1.0))
    return s


@pytest.fixture
def tc_backend(backend):
    backend.set_filter_mode(ctb.FILTER_MODE_TC_BF16X3)
    yield backend
    backend.set_filter_mode(ctb.FILTER_MODE_FFT)


@pytest.mark.parametrize("n,na,kind", [(64, 90, FilterType.Ramp), (128, 180, FilterType.SheppLogan),
                                        (256, 200, FilterType.Hann), (96, 150, FilterType.Hamming),
                                        (48, 61, FilterType.Cosine), (80, 100, FilterType.Bartlett)])
def test_tc_slice_against_fp64(backend, n, na, kind):
    rng = np.random.default_rng(n + na)
    nd = ctb.odd_detector_count(n)
    sino, ang, _ = O.sinogram_f32(_slice(rng, n, 5), na, nd)
    s = ctb.Sinogram(data=sino, angles_deg=ang)
    p = ReconstructionParams(kind, na)
    fft = backend.reconstructSlice(s, n, p)
    backend.set_filter_mode(ctb.FILTER_MODE_TC_BF16X3)
    try:
        tc = backend.reconstructSlice(s, n, p)
    finally:
        backend.set_filter_mode(ctb.FILTER_MODE_FFT)
    f64 = O.reconstruct_slice_f64(sino, ang, n, int(kind))
    assert np.all(np.isfinite(tc))
    e_tc, e_fft = O.rel_l2(tc, f64), O.rel_l2(fft, f64)
    assert e_tc <= TC_REL_L2, (e_tc, e_fft)
    assert O.max_abs_rel(tc, f64) <= TC_MAX_ABS
    assert e_fft <= TC_REL_L2


def test_tc_volume_from_sinograms_matches_fft(backend):
    rng = np.random.default_rng(7)
    n, depth, na = 160, 6, 211  # depth not a multiple of 4; explicit angles
    nd = ctb.odd_detector_count(n)
    ang = np.sort(rng.uniform(0, 180, na)).astype(np.float32)
    sinos = np.stack([O.sinogram_f64(_slice(rng, n, 4), na, nd, ang)[0].astype(np.float32) for _ in range(depth)])
    p = ReconstructionParams(FilterType.SheppLogan, na)
    ref = backend.reconstructVolumeFromSinograms(sinos, ang, p, denorm=ctb.Denorm.SERIAL)
    backend.set_filter_mode(ctb.FILTER_MODE_TC_BF16X3)
    try:
        tc = backend.reconstructVolumeFromSinograms(sinos, ang, p, denorm=ctb.Denorm.SERIAL)
    finally:
        backend.set_filter_mode(ctb.FILTER_MODE_FFT)
    for z in range(depth):
        assert O.rel_l2(tc[z], ref[z]) <= TC_REL_L2


def test_tc_reconstruct_volume_against_serial(tc_backend):
    rng = np.random.default_rng(8)
    n, depth, na = 96, 5, 128
    vol = np.stack([_slice(rng, n, 3) for _ in range(depth)])
    out = tc_backend.reconstructVolume(vol, ReconstructionParams(FilterType.Hann, na), detector_bins=n)
    ser = O.reconstruct_volume_f32(vol, na, n, O.HANN)
    assert O.rel_l2(out, ser) <= TC_REL_L2


def test_mode_switch_restores_fft_bit_for_bit(backend):
    rng = np.random.default_rng(9)
    n, na = 128, 120
    nd = ctb.odd_detector_count(n)
    sino, ang, _ = O.sinogram_f32(_slice(rng, n, 4), na, nd)
    s = ctb.Sinogram(data=sino, angles_deg=ang)
    p = ReconstructionParams(FilterType.Ramp, na)
    a = backend.reconstructSlice(s, n, p)
    backend.set_filter_mode(ctb.FILTER_MODE_TC_BF16X3)
    backend.reconstructSlice(s, n, p)
    backend.set_filter_mode(ctb.FILTER_MODE_FFT)
    np.testing.assert_array_equal(backend.reconstructSlice(s, n, p), a)
    with pytest.raises(ctb.CtbError):
        backend.set_filter_mode(7)
