"""Accuracy at the benchmark sizes against the FP64 rerun (GPU).

The parity tests hold small cases to SerialBackend's float path. At n = 512
and above that bar no longer applies: SerialBackend's own float result drifts
from the exact algorithm as n grows (about 3e-5 rel-L2 at 512), so a result
can be closer to the FP64 rerun than SerialBackend is and still differ from
it by more than 1e-5. The gate here is the one stated for the product:
rel-L2 <= 1e-5 and max-abs <= 1e-4 * max|f| against the FP64 rerun of
SerialBackend's reconstructVolume (SerialBackend.cpp:261-318), per checked
slice, with the float path's own error reported beside it.

* 512^3, 32 ellipsoids, 720 angles, 725 bins, Shepp-Logan (the benchmark
  volume): the device-resident call and the host-buffer call (which streams
  slabs of slices through copy and compute streams) must agree bit for bit
  over the whole volume, and the slices on both sides of the first and last
  slab boundaries of the host schedule (8, 24, 7 x 64, 24, 8 slices), the
  middle and the ends are checked against FP64.
* 1024^2 x 256, 64 ellipsoids, 1440 angles, 1449 bins, Hann (the precision
  workload), FFT filter: two central slices against FP64.
"""
import concurrent.futures as cf

import numpy as np
import pytest

import oracle as O
import qtctreconstruction_b200 as ctb
from qtctreconstruction_b200 import FilterType, ReconstructionParams

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
MAX_ABS = 1e-4


def _oracle_slices(vol, zs, na, nd, kind):
    """FP64 rerun and float SerialBackend restatement of each slice in zs
    (slices are independent), computed in threads."""
    def one(z, f64):
        v = np.ascontiguousarray(vol[z:z + 1])
        return (O.reconstruct_volume_f64 if f64 else O.reconstruct_volume_f32)(v, na, nd, kind)[0]
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        f64 = list(ex.map(lambda z: one(z, True), zs))
        f32 = list(ex.map(lambda z: one(z, False), zs))
    return f64, f32


def _device_volume(backend, torch, vol_host, na, nd, kind):
    nz, n, _ = vol_host.shape
    d_vol = torch.from_numpy(vol_host).cuda()
    d_out = torch.full_like(d_vol, float("nan"))
    backend.reconstruct_volume_d(d_vol.data_ptr(), n, nz, na, nd, int(kind), d_out.data_ptr())
    backend.synchronize()
    return d_out.cpu().numpy()


def _gate(out, zs, f64, f32):
    worst = []
    for z, ref, flt in zip(zs, f64, f32):
        e, m = O.rel_l2(out[z], ref), O.max_abs_rel(out[z], ref)
        worst.append((e, m, O.rel_l2(flt, ref), z))
        assert e <= REL_L2, f"slice {z}: rel-L2 vs FP64 {e:.3e} (float SerialBackend {O.rel_l2(flt, ref):.3e})"
        assert m <= MAX_ABS, f"slice {z}: max-abs vs FP64 {m:.3e}"
    return max(worst)


def test_config2_512cubed_720_angles_shepp_logan_vs_fp64(backend):
    import torch
    n, nz, na, kind = 512, 512, 720, FilterType.SheppLogan
    nd = ctb.odd_detector_count(n)
    assert nd == 725
    vol = backend.phantom(ctb.phantom_params(2, 32), n, n, nz)
    dev = _device_volume(backend, torch, vol, na, nd, kind)
    host = backend.reconstructVolume(vol, ReconstructionParams(kind, na), detector_bins=nd)
    assert np.isfinite(dev).all()
    np.testing.assert_array_equal(host, dev)
    zs = [0, 7, 8, 31, 32, 95, 96, 255, 256, 479, 480, 503, 504, 511]
    f64, f32 = _oracle_slices(vol, zs, na, nd, int(kind))
    e, m, serial, z = _gate(dev, zs, f64, f32)
    print(f"512^3 x 720: worst slice {z}: rel-L2 {e:.2e}, max-abs {m:.2e} vs FP64 "
          f"(float SerialBackend {serial:.2e})")


def test_config3_1024sq_256_slices_1440_angles_hann_fft_vs_fp64(backend):
    import torch
    n, nz, na, kind = 1024, 256, 1440, FilterType.Hann
    nd = ctb.odd_detector_count(n)
    assert nd == 1449
    backend.set_filter_mode(ctb.FILTER_MODE_FFT)
    params = ctb.phantom_params(3, 64)
    vol = backend.phantom(params, n, n, nz)
    dev = _device_volume(backend, torch, vol, na, nd, kind)
    assert np.isfinite(dev).all()
    zs = [nz // 2 - 1, nz // 2]
    f64, f32 = _oracle_slices(vol, zs, na, nd, int(kind))
    e, m, serial, z = _gate(dev, zs, f64, f32)
    print(f"1024^2 x 256 x 1440: worst slice {z}: rel-L2 {e:.2e}, max-abs {m:.2e} vs FP64 "
          f"(float SerialBackend {serial:.2e})")
