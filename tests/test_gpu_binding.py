"""The reference-side C++ binding on the GPU (GPU).

ct::B200Backend (qtctreconstruction_b200/binding), built against the
reference's own IReconstructionBackend.h / CTTypes.h, is driven through
virtual calls on ct::IReconstructionBackend with the reference's containers
(Buffer2D, Volume, Sinogram), as the reference's controller calls a backend
(CtReconstructionController.cpp:1002,1146,1240). Its results are held to the
golden fixtures that SerialBackend itself wrote: sinograms and slices within
the parity tolerance (rel-L2 <= 1e-5, max-abs <= 1e-4 * max|f|; sinograms
2e-6), reconstructVolume and reconstructVolumeFromSinograms within the same
tolerance, the point cloud bit for bit. The binding library is built on the
build machine (it needs the reference's headers) and travels with the tree.
"""
import numpy as np
import pytest

import binding_lib as B  # noqa: E402  (tests/ is on sys.path under pytest)
import oracle as O

pytestmark = pytest.mark.gpu

CASES = ["cfg_like", "native_nd", "odd_n", "neg_min_zero_bg", "constant", "zeros", "hu_like",
         "bartlett_small_nd"]


def _close(a, ref, rel=1e-5, mx=1e-4):
    assert O.rel_l2(a, ref) <= rel, O.rel_l2(a, ref)
    assert O.max_abs_rel(a, ref) <= mx, O.max_abs_rel(a, ref)


@pytest.fixture(scope="module")
def be():
    L = B.load()
    assert L is not None, f"{B.LIB} was not built (make -C qtctreconstruction_b200/binding)"
    h = L.b200be_create(0)
    assert h and L.b200be_is_available(h) == 1
    yield L, h
    L.b200be_destroy(h)


@pytest.mark.parametrize("case", CASES)
def test_compute_sinogram_and_reconstruct_slice(be, golden, case):
    L, h = be
    n, na, nd, kind = (int(v) for v in golden[f"{case}_meta"])
    sl = np.ascontiguousarray(golden[f"{case}_slice"], np.float32)
    sino = np.zeros((na, nd), np.float32)
    ang, mm = np.zeros(na, np.float32), np.zeros(2, np.float32)
    assert L.b200be_compute_sinogram(h, sl, sl.shape[1], sl.shape[0], na, nd, sino, ang, mm) == 0
    np.testing.assert_array_equal(ang, golden[f"{case}_angles"])
    np.testing.assert_array_equal(mm, golden[f"{case}_minmax"])
    _close(sino, golden[f"{case}_sino"], rel=2e-6, mx=2e-6)
    assert L.b200be_last_sinogram_ms(h) > 0.0
    gs = np.ascontiguousarray(golden[f"{case}_sino"], np.float32)
    ga = np.ascontiguousarray(golden[f"{case}_angles"], np.float32)
    rec = np.zeros((n, n), np.float32)
    assert L.b200be_reconstruct_slice(h, gs, na, nd, ga.ctypes.data, n, kind, 0.0, 0.0, rec) == 0
    _close(rec, golden[f"{case}_recon"])


def test_reconstruct_volume(be, golden):
    L, h = be
    vol = np.ascontiguousarray(golden["volume_in"], np.float32)
    na, kind = (int(v) for v in golden["volume_meta"])
    nz, n, _ = vol.shape
    out = np.zeros_like(vol)
    seen = np.full(nz, -1, np.int32)
    assert L.b200be_reconstruct_volume(h, vol, n, nz, na, kind, out, seen.ctypes.data) == 0
    np.testing.assert_array_equal(seen, np.arange(nz))  # the callback saw every slice, in order
    ref = golden["volume_serial"]
    for z in range(nz):
        if np.abs(ref[z]).max() == 0 or z == 3:
            np.testing.assert_array_equal(out[z], ref[z])
        else:
            _close(out[z], ref[z])


def test_reconstruct_from_sinograms(be, golden):
    L, h = be
    sinos = np.ascontiguousarray(golden["fromsino_in"], np.float32)
    ang = np.ascontiguousarray(golden["fromsino_angles"], np.float32)
    kind = int(golden["fromsino_meta"][0])
    nz, na, bins = sinos.shape
    out = np.zeros((nz, bins, bins), np.float32)
    assert L.b200be_reconstruct_from_sinograms(h, sinos, nz, na, bins, ang, kind, out) == 0
    ref = golden["fromsino_serial"]
    for z in range(nz):
        np.testing.assert_allclose(out[z], ref[z], rtol=0, atol=1e-4 * max(1e-30, np.abs(ref[z]).max()))
    assert L.b200be_last_reconstruction_ms(h) > 0.0


def test_extract_point_cloud(be, golden):
    L, h = be
    vol = np.ascontiguousarray(golden["gen3d_vol"], np.float32)
    nz, ny, nx = vol.shape
    thr = float(golden["pc_threshold"][0])
    total = L.b200be_extract_point_cloud(h, vol, nx, ny, nz, thr, None, 0)
    ref = golden["pc_points"]
    assert total == ref.shape[0]
    pts = np.zeros((total, 4), np.float32)
    assert L.b200be_extract_point_cloud(h, vol, nx, ny, nz, thr, pts.ctypes.data, total) == total
    np.testing.assert_array_equal(pts, ref)
