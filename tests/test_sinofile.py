"""The consumer sinogram format (NPY (depth, num_angles, bins) float32 +
<name>.meta.json), host side: round trips through the library, files written
the way the reference's exporter writes them (CtReconstructionController.cpp:
1353-1482; its NPY header FileIO.cpp:53-148) and by numpy, and the reader's
fallbacks (no sidecar, wrong angle count, missing min/max), as the reference's
importer applies them (CtReconstructionController.cpp:1494-1616)."""
import json
import os

import numpy as np
import pytest

import qtctreconstruction_b200 as ctb


def _reference_style_npy(path, arr):
    """The reference's writer: NPY 1.0, its own header text, padded to 16."""
    z, y, x = arr.shape
    hdr = "{'descr': '<f4', 'fortran_order': False, 'shape': (%d, %d, %d), }" % (z, y, x)
    n = len(hdr) + 1
    while (10 + n) % 16:
        n += 1
    hdr = hdr + " " * (n - len(hdr) - 1) + "\n"
    with open(path, "wb") as f:
        f.write(b"\x93NUMPY\x01\x00" + len(hdr).to_bytes(2, "little") + hdr.encode() + arr.astype("<f4").tobytes())


def _reference_style_meta(path, depth, na, bins, lo, hi, spacing=1.0):
    step = np.float32(180.0) / np.float32(na)
    meta = {"version": 1, "depth": depth, "num_angles": na, "detector_bins": bins,
            "detector_spacing_mm": spacing, "original_min_hu": lo, "original_max_hu": hi,
            "angles_deg": [float(step * np.float32(a)) for a in range(na)]}
    with open(path[:-4] + ".meta.json", "w") as f:
        json.dump(meta, f, indent=4)


def test_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    s = rng.standard_normal((3, 17, 25)).astype(np.float32)
    ang = np.sort(rng.uniform(0, 180, 17)).astype(np.float32)
    p = str(tmp_path / "sino.npy")
    ctb.save_sinogram_file(p, s, ang, spacing_mm=0.5, min_hu=-1000.0, max_hu=2500.5)
    got, a, meta = ctb.load_sinogram_file(p)
    np.testing.assert_array_equal(got, s)
    np.testing.assert_array_equal(a, ang)
    assert meta == {"detector_spacing_mm": 0.5, "original_min_hu": -1000.0, "original_max_hu": 2500.5}
    # numpy reads the library's NPY, and the sidecar is plain JSON
    np.testing.assert_array_equal(np.load(p), s)
    m = json.load(open(str(tmp_path / "sino.meta.json")))
    assert (m["depth"], m["num_angles"], m["detector_bins"], m["version"]) == (3, 17, 25, 1)
    np.testing.assert_array_equal(np.float32(m["angles_deg"]), ang)


def test_reads_reference_writer(tmp_path):
    rng = np.random.default_rng(1)
    s = rng.uniform(-5, 5, (2, 9, 11)).astype(np.float32)
    p = str(tmp_path / "ref.npy")
    _reference_style_npy(p, s)
    _reference_style_meta(p, 2, 9, 11, -1000.0, 1200.0, 1.0)
    got, a, meta = ctb.load_sinogram_file(p)
    np.testing.assert_array_equal(got, s)
    np.testing.assert_array_equal(a, ctb.uniform_angles_deg(9))
    assert meta["original_min_hu"] == -1000.0 and meta["original_max_hu"] == 1200.0


def test_numpy_writer_and_fallbacks(tmp_path):
    rng = np.random.default_rng(2)
    s = rng.uniform(-3, 7, (4, 6, 5)).astype(np.float32)
    p = str(tmp_path / "np.npy")
    np.save(p, s)
    got, a, meta = ctb.load_sinogram_file(p)  # no sidecar: uniform angles, min/max from data
    np.testing.assert_array_equal(got, s)
    np.testing.assert_array_equal(a, ctb.uniform_angles_deg(6))
    assert meta == {"detector_spacing_mm": 1.0, "original_min_hu": float(s.min()), "original_max_hu": float(s.max())}
    with open(p[:-4] + ".meta.json", "w") as f:  # wrong angle count, no min/max
        json.dump({"angles_deg": [1.0, 2.0], "detector_spacing_mm": 2.0}, f)
    _, a, meta = ctb.load_sinogram_file(p)
    np.testing.assert_array_equal(a, ctb.uniform_angles_deg(6))
    assert meta["detector_spacing_mm"] == 2.0 and meta["original_max_hu"] == float(s.max())


def test_rejects_other_formats(tmp_path):
    p = str(tmp_path / "d.npy")
    np.save(p, np.zeros((2, 3, 4), np.float64))
    with pytest.raises(ctb.CtbError):
        ctb.load_sinogram_file(p)
    np.save(p, np.zeros((3, 4), np.float32))
    with pytest.raises(ctb.CtbError):
        ctb.load_sinogram_file(p)
    with pytest.raises(ctb.CtbError):
        ctb.load_sinogram_file(str(tmp_path / "missing.npy"))
