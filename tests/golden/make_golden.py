"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs the unmodified QtCTReconstruction CPU backends (oracle/_ref/libctref.so,
built by ``make -C oracle`` from the reference sources) on small seeded inputs
and stores inputs and outputs in ``serial_small.npz``. The committed fixtures
pin the oracle restatement and the GPU path where the reference tree is
absent. Re-run with ``python tests/golden/make_golden.py`` after rebuilding the
reference library; the inputs are deterministic.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from oracle import reference as R  # noqa: E402


def ellipse_slice(rng, n, k, background=0.0):
    """k random ellipses (summed) on a constant background."""
    s = np.full((n, n), background, np.float32)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    for _ in range(k):
        cx, cy = rng.uniform(0.2 * n, 0.8 * n, 2)
        a, b = rng.uniform(0.06 * n, 0.3 * n, 2)
        t = rng.uniform(0, np.pi)
        d = np.float32(rng.uniform(-0.3, 1.0))
        u = (xx - cx) * np.cos(t) + (yy - cy) * np.sin(t)
        v = -(xx - cx) * np.sin(t) + (yy - cy) * np.cos(t)
        s[(u / a) ** 2 + (v / b) ** 2 <= 1.0] += d
    return s


def main():
    if not R.available():
        raise SystemExit("oracle/_ref/libctref.so missing: run `make -C oracle` with the reference tree")
    rng = np.random.default_rng(20261203)
    out = {}

    # FilterDesign::createFilter for every filter type at three FFT sizes.
    for L in (64, 128, 1024):
        for kind in range(6):
            out[f"filter_L{L}_k{kind}"] = R.create_filter(L, kind)

    # Single-slice cases: (name, n, na, nd, filter, slice)
    cases = [
        ("cfg_like", 32, 45, O.odd_detector_count(32), O.RAMP, ellipse_slice(rng, 32, 5)),
        ("native_nd", 24, 30, 24, O.SHEPP_LOGAN, ellipse_slice(rng, 24, 4, background=0.0) + 0.25),
        ("odd_n", 17, 16, 25, O.HANN, ellipse_slice(rng, 17, 3)),
        ("neg_min_zero_bg", 28, 36, O.odd_detector_count(28), O.SHEPP_LOGAN,
         ellipse_slice(rng, 28, 6) - np.float32(0.0)),
        ("constant", 16, 12, 23, O.RAMP, np.full((16, 16), 0.7, np.float32)),
        ("zeros", 16, 12, 23, O.HAMMING, np.zeros((16, 16), np.float32)),
        ("hu_like", 20, 24, 29, O.COSINE,
         (ellipse_slice(rng, 20, 4) * 1000.0 - 1000.0).astype(np.float32)),
        ("bartlett_small_nd", 20, 18, 11, O.BARTLETT, ellipse_slice(rng, 20, 4)),
    ]
    names = []
    for name, n, na, nd, kind, sl in cases:
        sino, ang, mm = R.compute_sinogram(R.SERIAL, sl, na, nd)
        rec = R.reconstruct_slice(R.SERIAL, sino, ang, n, kind, mm[0], mm[1])
        omp_rec = R.reconstruct_slice(R.OPENMP, sino, ang, n, kind, mm[0], mm[1])
        out[f"{name}_slice"] = sl
        out[f"{name}_meta"] = np.array([n, na, nd, kind], np.int64)
        out[f"{name}_sino"] = sino
        out[f"{name}_angles"] = ang
        out[f"{name}_minmax"] = mm
        out[f"{name}_recon"] = rec
        out[f"{name}_omp_recon"] = omp_rec
        names.append(name)
    out["slice_cases"] = np.array(names)

    # reconstructVolume (detector_bins = width inside the reference).
    vol = np.stack([ellipse_slice(rng, 20, 4), ellipse_slice(rng, 20, 3) * 3.0,
                    np.zeros((20, 20), np.float32), np.full((20, 20), -2.0, np.float32)])
    out["volume_in"] = vol
    out["volume_meta"] = np.array([24, O.SHEPP_LOGAN], np.int64)
    out["volume_serial"] = R.reconstruct_volume(R.SERIAL, vol, 24, O.SHEPP_LOGAN)

    # reconstructVolumeFromSinograms: default per-slice implementation of the interface.
    sinos = np.stack([R.compute_sinogram(R.SERIAL, vol[z], 24, 29)[0] for z in range(vol.shape[0])])
    ang = O.uniform_angles_deg(24)
    out["fromsino_in"] = sinos
    out["fromsino_angles"] = ang
    out["fromsino_meta"] = np.array([O.HANN], np.int64)
    out["fromsino_serial"] = R.reconstruct_from_sinograms(R.SERIAL, sinos, ang, O.HANN)

    # Generator3DCPU with default tissue parameters, a small grid.
    out["gen3d_meta"] = np.array([24, 20, 16, 40, 7], np.int64)  # nx, ny, nz, n_ell, seed
    out["gen3d_radius"] = np.array([50.0], np.float32)
    out["gen3d_vol"] = R.generator3d(24, 20, 16, 50.0, 40, 7)

    # extractPointCloud on the generated volume.
    out["pc_threshold"] = np.array([100.0], np.float32)
    out["pc_points"] = R.extract_point_cloud(R.SERIAL, out["gen3d_vol"], 100.0)

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "serial_small.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {os.path.getsize(path)} bytes, {len(out)} arrays")


if __name__ == "__main__":
    main()
