"""GPU parity: the CUDA path through the C ABI against the oracle.

Tolerances (floating point): rel-L2 <= 1e-5 and max-abs <= 1e-4 * max|f|
against SerialBackend (the reference's float path, bit-identical to the float
oracle and to the golden fixtures); against the FP64 rerun the GPU must be at
least as accurate as SerialBackend itself. Phantoms and point clouds are
bit-exact.
"""
import numpy as np
import pytest

import oracle as O
import qtctreconstruction_b200 as ctb
from qtctreconstruction_b200 import FilterType, ReconstructionParams, Denorm

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
MAX_ABS = 1e-4

CASES = ["cfg_like", "native_nd", "odd_n", "neg_min_zero_bg", "constant", "zeros", "hu_like",
         "bartlett_small_nd"]


def _close(a, ref, rel=REL_L2, mx=MAX_ABS):
    assert O.rel_l2(a, ref) <= rel, O.rel_l2(a, ref)
    assert O.max_abs_rel(a, ref) <= mx, O.max_abs_rel(a, ref)


def ellipse_slice(rng, n, k):
    s = np.zeros((n, n), np.float32)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    for _ in range(k):
        cx, cy = rng.uniform(0.25 * n, 0.75 * n, 2)
        a, b = rng.uniform(0.05 * n, 0.25 * n, 2)
        t = rng.uniform(0, np.pi)
        u = (xx - cx) * np.cos(t) + (yy - cy) * np.sin(t)
        v = -(xx - cx) * np.sin(t) + (yy - cy) * np.cos(t)
        s[(u / a) ** 2 + (v / b) ** 2 <= 1.0] += np.float32(rng.uniform(-0.3, 1.0))
    return s


# ------------------------------------------------------------------ forward
@pytest.mark.parametrize("case", CASES)
def test_sinogram_matches_serial(backend, golden, case):
    n, na, nd, kind = (int(v) for v in golden[f"{case}_meta"])
    sino = backend.computeSinogram(golden[f"{case}_slice"], na, nd)
    ref = golden[f"{case}_sino"]
    np.testing.assert_array_equal(sino.angles_deg, golden[f"{case}_angles"])
    assert sino.original_min_hu == golden[f"{case}_minmax"][0]
    assert sino.original_max_hu == golden[f"{case}_minmax"][1]
    _close(sino.data, ref, rel=2e-6, mx=2e-6)


def test_sinogram_vs_fp64_more_accurate_than_serial(backend):
    rng = np.random.default_rng(3)
    n, na = 96, 128
    nd = ctb.odd_detector_count(n)
    sl = ellipse_slice(rng, n, 6)
    gpu = backend.computeSinogram(sl, na, nd).data
    ser, _, _ = O.sinogram_f32(sl, na, nd)
    s64, _ = O.sinogram_f64(sl, na, nd)
    assert O.rel_l2(gpu, s64) <= O.rel_l2(ser, s64) * 1.01 + 1e-7
    assert O.rel_l2(gpu, s64) < 5e-7


# ---------------------------------------------------------------------- FBP
@pytest.mark.parametrize("case", CASES)
def test_reconstruct_slice_matches_serial(backend, golden, case):
    n, na, nd, kind = (int(v) for v in golden[f"{case}_meta"])
    sino = ctb.Sinogram(golden[f"{case}_sino"], golden[f"{case}_angles"])
    rec = backend.reconstructSlice(sino, n, ReconstructionParams(FilterType(kind), na))
    _close(rec, golden[f"{case}_recon"])


@pytest.mark.parametrize("kind", list(FilterType))
def test_all_filters_against_fp64(backend, kind):
    rng = np.random.default_rng(int(kind) + 10)
    n, na = 64, 90
    nd = ctb.odd_detector_count(n)
    sl = ellipse_slice(rng, n, 5)
    s32, ang, _ = O.sinogram_f32(sl, na, nd)
    ser = O.reconstruct_slice_f32(s32, ang, n, int(kind))
    r64 = O.reconstruct_slice_f64(s32.astype(np.float64), ang, n, int(kind))
    gpu = backend.reconstructSlice(ctb.Sinogram(s32, ang), n, ReconstructionParams(kind, na))
    _close(gpu, ser)
    # at least as accurate as the reference's float path
    assert O.rel_l2(gpu, r64) <= max(O.rel_l2(ser, r64), 1e-6)


def test_filtered_rows_through_delta(backend):
    # a single impulse per row reconstructs to the filter kernel's backprojection:
    # compare against the float oracle on a small detector with many angles
    n, na, nd = 40, 64, 57
    sino = np.zeros((na, nd), np.float32)
    sino[:, nd // 2] = 1.0
    ang = O.uniform_angles_deg(na)
    gpu = backend.reconstructSlice(ctb.Sinogram(sino, ang), n, ReconstructionParams(FilterType.Ramp, na))
    ref = O.reconstruct_slice_f32(sino, ang, n, O.RAMP)
    _close(gpu, ref)


def test_nonuniform_angles(backend):
    rng = np.random.default_rng(5)
    n, na = 48, 77
    nd = ctb.odd_detector_count(n)
    sl = ellipse_slice(rng, n, 4)
    ang = np.sort(rng.uniform(0, 180, na)).astype(np.float32)
    s64, _ = O.sinogram_f64(sl, na, nd, ang)
    s32 = s64.astype(np.float32)
    ser = O.reconstruct_slice_f32(s32, ang, n, O.HANN)
    gpu = backend.reconstructSlice(ctb.Sinogram(s32, ang), n, ReconstructionParams(FilterType.Hann, na))
    _close(gpu, ser)


@pytest.mark.parametrize("n,na,nd", [(33, 50, 47), (100, 37, 141), (65, 2100, 93), (20, 16, 11),
                                     (128, 180, 183), (256, 90, 363), (1768, 24, 2501)])
def test_reconstruct_slice_shapes(backend, n, na, nd):
    # odd sizes, sizes off the 32-voxel tile grid, > 2048 angles, detector
    # narrower than the image (taps outside the detector are skipped), and
    # convolution lengths 64 ... 8192 (the last one the scalar FFT kernel)
    # (at n = 1768 SerialBackend's own float result is 1.5e-4 from the FP64
    # rerun, so there the gate is the FP64 rerun, which the GPU must also meet
    # at least as well as SerialBackend does)
    rng = np.random.default_rng(n * 1000 + na)
    sl = ellipse_slice(rng, n, 4)
    s32, ang, _ = O.sinogram_f32(sl, na, nd)
    ser = O.reconstruct_slice_f32(s32, ang, n, O.SHEPP_LOGAN)
    gpu = backend.reconstructSlice(ctb.Sinogram(s32, ang), n, ReconstructionParams(FilterType.SheppLogan, na))
    if n <= 256:
        _close(gpu, ser)
    else:
        f64 = O.reconstruct_slice_f64(s32.astype(np.float64), ang, n, O.SHEPP_LOGAN)
        _close(gpu, f64)
        assert O.rel_l2(gpu, f64) <= O.rel_l2(ser, f64)


def test_output_size_larger_than_detector(backend):
    # output_size > bins: many taps fall outside the detector (SerialBackend.cpp:236)
    rng = np.random.default_rng(9)
    sl = ellipse_slice(rng, 24, 3)
    s32, ang, _ = O.sinogram_f32(sl, 40, 25)
    ser = O.reconstruct_slice_f32(s32, ang, 70, O.RAMP)
    gpu = backend.reconstructSlice(ctb.Sinogram(s32, ang), 70, ReconstructionParams(FilterType.Ramp, 40))
    _close(gpu, ser)


# ------------------------------------------------------------------ volumes
def test_reconstruct_volume_matches_serial_golden(backend, golden):
    vol = golden["volume_in"]
    na, kind = (int(v) for v in golden["volume_meta"])
    out = backend.reconstructVolume(vol, ReconstructionParams(FilterType(kind), na))
    ref = golden["volume_serial"]
    for z in range(vol.shape[0]):
        if z == 3:  # constant slice: min everywhere (span 0 -> recon 0)
            np.testing.assert_array_equal(out[z], ref[z])
        elif z == 2:  # all zeros: the reference output is exactly 0
            np.testing.assert_array_equal(out[z], ref[z])
        else:
            _close(out[z], ref[z])


def test_reconstruct_volume_config1_parity(backend):
    """128^3 phantom of 10 ellipsoids, 180 angles, odd Nd = 183, Ram-Lak."""
    n, nz, na = 128, 128, 180
    nd = ctb.odd_detector_count(n)
    p = ctb.phantom_params(1, 10)
    vol = backend.phantom(p, n, n, nz)
    np.testing.assert_array_equal(vol, O.phantom_sum(p, n, n, nz))
    out = backend.reconstructVolume(vol, ReconstructionParams(FilterType.Ramp, na), detector_bins=nd)
    ser = O.reconstruct_volume_f32(vol, na, nd, O.RAMP)
    _close(out, ser)
    zs = [10, 40, 64, 100]
    r64 = O.reconstruct_volume_f64(vol[zs], na, nd, O.RAMP)
    e_gpu = O.rel_l2(out[zs], r64)
    e_ser = O.rel_l2(ser[zs], r64)
    assert e_gpu <= e_ser, (e_gpu, e_ser)


def test_depth_not_multiple_of_four(backend):
    rng = np.random.default_rng(11)
    n, na = 40, 60
    nd = ctb.odd_detector_count(n)
    vol = np.stack([ellipse_slice(rng, n, 3) for _ in range(5)])
    out = backend.reconstructVolume(vol, ReconstructionParams(FilterType.Hann, na), detector_bins=nd)
    ser = O.reconstruct_volume_f32(vol, na, nd, O.HANN)
    _close(out, ser)


def test_sparse_slices_nonzero_box(backend):
    """The projector walks only the box of non-zero pixels of each 8-slice
    group: small blobs in corners (one reaching the edge detector bins),
    empty groups, a group whose box covers one slice only, and a raw value
    equal to the slice minimum (normalised to zero) outside a blob."""
    n, na = 64, 90
    nd = ctb.odd_detector_count(n)
    vol = np.zeros((20, n, n), np.float32)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)

    def blob(z, cx, cy, r, v):
        vol[z][((xx - cx) ** 2 + (yy - cy) ** 2) <= r * r] += np.float32(v)

    blob(1, 6, 5, 4, 0.8)     # top-left corner: reaches bin 0 near 45 degrees
    blob(2, 58, 60, 3, 1.5)   # bottom-right corner, same 8-slice group
    blob(9, 32, 20, 6, -0.4)  # the blob is the minimum: every pixel normalises to zero
    vol[12] = -2.0            # background at the minimum: normalises to zero
    blob(12, 40, 40, 5, 3.0)
    blob(19, 2, 61, 2, 0.3)   # last (partial) group, one slice, corner
    out = backend.reconstructVolume(vol, ReconstructionParams(FilterType.SheppLogan, na), detector_bins=nd)
    ser = O.reconstruct_volume_f32(vol, na, nd, O.SHEPP_LOGAN)
    scale = float(np.abs(ser).max())
    live = [z for z in range(vol.shape[0]) if vol[z].any()]
    r64 = O.reconstruct_volume_f64(vol[live], na, nd, O.SHEPP_LOGAN)
    for z in range(vol.shape[0]):
        if z not in live:
            # the reference gives exact zeros; the filter transforms two slices
            # as one complex row, so a zero slice paired with a non-zero one
            # carries rounding crosstalk of ~1e-8 of the volume's scale
            assert np.abs(out[z]).max() <= 1e-7 * scale, (z, np.abs(out[z]).max(), scale)
        else:
            # small blobs far from the centre: SerialBackend's own float error
            # (s in float at |s - centre| ~ 40) reaches 4e-5 here, so the bar is
            # the FP64 rerun: at least as accurate as SerialBackend
            e_gpu = O.rel_l2(out[z], r64[live.index(z)])
            e_ser = O.rel_l2(ser[z], r64[live.index(z)])
            assert e_gpu <= e_ser + 1e-7, (z, e_gpu, e_ser)


def test_forward_bounds_off_walks_whole_image(backend):
    """With the non-zero bounds off the projector walks the whole image: the
    same sinograms up to rounding (the walk's chunk starts move), both within
    the parity bar against SerialBackend."""
    rng = np.random.default_rng(21)
    n, na = 72, 100
    nd = ctb.odd_detector_count(n)
    sl = np.zeros((n, n), np.float32)
    sl[10:40, 20:50] = ellipse_slice(rng, 30, 3)
    ref, _, _ = O.sinogram_f32(sl, na, nd)
    on = backend.computeSinogram(sl, na, nd).data
    try:
        backend.set_forward_bounds(False)
        off = backend.computeSinogram(sl, na, nd).data
    finally:
        backend.set_forward_bounds(True)
    s64, _ = O.sinogram_f64(sl, na, nd)
    for g in (on, off):
        _close(g, ref)
        # off-centre pixels: SerialBackend's own float error dominates, so
        # the bar is the FP64 rerun
        assert O.rel_l2(g, s64) <= O.rel_l2(ref, s64) + 1e-8
    assert O.rel_l2(on, off) <= 1e-6


@pytest.mark.parametrize("denorm", [Denorm.NONE, Denorm.SERIAL, Denorm.OPENMP, Denorm.CUDA])
def test_from_sinograms(backend, golden, denorm):
    sinos, ang = golden["fromsino_in"], golden["fromsino_angles"]
    kind = int(golden["fromsino_meta"][0])
    out = backend.reconstructVolumeFromSinograms(sinos, ang, ReconstructionParams(FilterType(kind), len(ang)),
                                                 denorm=denorm)
    nz, na, bins = sinos.shape
    for z in range(nz):
        rec = O.reconstruct_slice_f32(sinos[z], ang, bins, kind)
        lo, hi = float(sinos[z].min()), float(sinos[z].max())
        span = np.float32(hi) - np.float32(lo)
        if denorm == Denorm.SERIAL:
            rec = rec * (np.float32(1.0) if span <= 0 else span) + np.float32(lo)
        elif denorm == Denorm.OPENMP:
            rec = np.full_like(rec, lo) if span <= 0 else rec * span + np.float32(lo)
        elif denorm == Denorm.CUDA:
            rec = rec * span + np.float32(lo) if span > 0 else rec
        if denorm == Denorm.NONE:
            np.testing.assert_allclose(out[z], golden["fromsino_serial"][z], rtol=0, atol=1e-4 * max(
                1e-30, np.abs(golden["fromsino_serial"][z]).max()))
        if np.abs(rec).max() > 0:
            _close(out[z], rec)
        else:
            np.testing.assert_array_equal(out[z], rec)


# ----------------------------------------------------------------- phantoms
@pytest.mark.parametrize("shape", [(16, 16, 16), (33, 20, 7), (64, 64, 48), (128, 96, 120)])
def test_phantom_sum_bit_exact(backend, shape):
    nx, ny, nz = shape
    p = ctb.phantom_params(42, 24)
    np.testing.assert_array_equal(backend.phantom(p, nx, ny, nz), O.phantom_sum(p, nx, ny, nz))


def test_generator3d_bit_exact(backend, golden):
    nx, ny, nz, n_ell, seed = (int(v) for v in golden["gen3d_meta"])
    vol = backend.generator3d(nx, ny, nz, float(golden["gen3d_radius"][0]), n_ell, seed)
    np.testing.assert_array_equal(vol, golden["gen3d_vol"])
    big = backend.generator3d(64, 48, 40, 50.0, 120, 42)
    np.testing.assert_array_equal(big, O.generator3d(64, 48, 40, 50.0, 120, 42))


def test_point_cloud(backend, golden):
    pts = backend.extractPointCloud(golden["gen3d_vol"], float(golden["pc_threshold"][0]))
    np.testing.assert_array_equal(pts, golden["pc_points"])
    empty = backend.extractPointCloud(golden["gen3d_vol"], 1e9)
    assert empty.shape == (0, 4)


# ------------------------------------------------------------ empty inputs
def test_empty_inputs_return_empty(backend):
    s = backend.computeSinogram(np.zeros((0, 0), np.float32), 10, 10)
    assert s.data.size == 0
    r = backend.reconstructSlice(ctb.Sinogram(np.zeros((0, 0), np.float32), np.zeros(0, np.float32)), 16,
                                 ReconstructionParams())
    assert r.size == 0


@pytest.mark.parametrize("n,depth", [(96, 50), (40, 260)])
def test_host_volume_pipeline_equals_device_path(backend, n, depth):
    """ctb_reconstruct_volume streams slabs (copies overlapped with compute;
    at depth 260 the schedule tapers at both ends and ends on a partial
    8-slice group); the result must equal ctb_reconstruct_volume_d on the
    whole volume bit for bit."""
    import torch
    rng = np.random.default_rng(17)
    na = 120
    nd = ctb.odd_detector_count(n)
    vol = np.stack([ellipse_slice(rng, n, 3) for _ in range(depth)])
    host = backend.reconstructVolume(vol, ReconstructionParams(FilterType.SheppLogan, na), detector_bins=nd)
    d_vol = torch.from_numpy(vol).cuda()
    d_out = torch.empty_like(d_vol)
    backend.reconstruct_volume_d(d_vol.data_ptr(), n, depth, na, nd, int(FilterType.SheppLogan), d_out.data_ptr())
    backend.synchronize()
    np.testing.assert_array_equal(host, d_out.cpu().numpy())
    ser = O.reconstruct_volume_f32(vol[:6], na, nd, O.SHEPP_LOGAN)
    _close(host[:6], ser)


@pytest.mark.parametrize("w,h", [(80, 48), (37, 101)])
def test_sinogram_non_square_slice(backend, w, h):
    """computeSinogram takes any width x height (SerialBackend.cpp:59-136):
    the walked axis and its transposed copy differ in length."""
    rng = np.random.default_rng(w * h)
    sl = np.zeros((h, w), np.float32)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    for _ in range(4):
        cx, cy = rng.uniform(0.3 * w, 0.7 * w), rng.uniform(0.3 * h, 0.7 * h)
        a, b = rng.uniform(0.05, 0.2) * w, rng.uniform(0.05, 0.2) * h
        sl[((xx - cx) / a) ** 2 + ((yy - cy) / b) ** 2 <= 1.0] += np.float32(rng.uniform(0.2, 1.0))
    na, nd = 90, ctb.odd_detector_count(max(w, h))
    gpu = backend.computeSinogram(sl, na, nd)
    ref, ang, mm = O.sinogram_f32(sl, na, nd)
    _close(gpu.data, ref)
    assert (gpu.original_min_hu, gpu.original_max_hu) == (mm[0], mm[1])
    f64, _ = O.sinogram_f64(sl, na, nd, ang)
    assert O.rel_l2(gpu.data, f64) <= O.rel_l2(ref, f64)  # at least as accurate as SerialBackend


def test_angles_outside_half_turn_and_single_angle(backend):
    rng = np.random.default_rng(21)
    n = 64
    nd = ctb.odd_detector_count(n)
    sl = ellipse_slice(rng, n, 4)
    for ang in (np.sort(rng.uniform(-90, 300, 61)).astype(np.float32), np.float32([37.5])):
        s64, _ = O.sinogram_f64(sl, len(ang), nd, ang)
        s32 = s64.astype(np.float32)
        ser = O.reconstruct_slice_f32(s32, ang, n, O.RAMP)
        gpu = backend.reconstructSlice(ctb.Sinogram(s32, ang), n, ReconstructionParams(FilterType.Ramp, len(ang)))
        _close(gpu, ser)
