"""Write tests/golden/cuda_conv.npz: outputs of the reference's own CUDA backend
(CUDABackend.cu, built from its sources by oracle/Makefile into
oracle/_ref/libctref_cuda.so) on seeded inputs. They pin the oracle's
restatement of that backend's conventions (ray-march forward projector with
(nd-1)/2 detector centre, Nyquist-keeping filter, backprojection with
(N-1)/2 and (sq-1)/2 centres and per-tap bounds, denormalisation when
max > min). Needs a GPU; run once:

    python tests/golden/make_cuda_golden.py tests/golden/cuda_conv.npz
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
F32 = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def lib():
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libctref_cuda.so"))
    i, f = ctypes.c_int, ctypes.c_float
    L.cref_compute_sinogram.argtypes = [F32, i, i, i, i, F32, F32]
    L.cref_reconstruct_slice.argtypes = [F32, i, i, F32, i, i, f, f, F32]
    L.cref_reconstruct_volume.argtypes = [F32, i, i, i, i, F32]
    return L


def ellipse_slice(rng, n, k, background):
    s = np.full((n, n), background, np.float32)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    for _ in range(k):
        cx, cy = rng.uniform(0.25 * n, 0.75 * n, 2)
        a, b = rng.uniform(0.06 * n, 0.25 * n, 2)
        t = rng.uniform(0, np.pi)
        u = (xx - cx) * np.cos(t) + (yy - cy) * np.sin(t)
        v = -(xx - cx) * np.sin(t) + (yy - cy) * np.cos(t)
        s[(u / a) ** 2 + (v / b) ** 2 <= 1.0] += np.float32(rng.uniform(50.0, 900.0))
    return s


# (name, n, angles, detector bins, filter, background)
CASES = [("ramp64", 64, 90, 91, 0, 0.0), ("shepp96", 96, 120, 137, 1, -1000.0),
         ("hann128_even", 128, 180, 128, 4, 0.0), ("hamming80", 80, 100, 113, 2, -200.0),
         ("cosine48", 48, 61, 69, 3, 0.0), ("bartlett72", 72, 80, 103, 5, -50.0)]


def main(out_path):
    L = lib()
    rng = np.random.default_rng(2026)
    res = {}
    for name, n, na, nd, kind, bg in CASES:
        sl = ellipse_slice(rng, n, 5, bg)
        sino = np.zeros((na, nd), np.float32)
        mm = np.zeros(2, np.float32)
        assert L.cref_compute_sinogram(sl, n, n, na, nd, sino, mm) == 0
        ang = (np.float32(180.0) / np.float32(na)) * np.arange(na, dtype=np.float32)
        rec = np.zeros((n, n), np.float32)
        assert L.cref_reconstruct_slice(sino, na, nd, ang, n, kind, float(mm[0]), float(mm[1]), rec) == 0
        res[f"{name}_slice"], res[f"{name}_sino"], res[f"{name}_minmax"] = sl, sino, mm
        res[f"{name}_recon"], res[f"{name}_meta"] = rec, np.array([n, na, nd, kind], np.int32)
    n, depth, na, kind = 64, 3, 90, 1
    vol = np.stack([ellipse_slice(rng, n, 4, 0.0) for _ in range(depth)])
    out = np.zeros_like(vol)
    assert L.cref_reconstruct_volume(vol, n, depth, na, kind, out) == 0
    res["volume_in"], res["volume_out"], res["volume_meta"] = vol, out, np.array([n, depth, na, kind], np.int32)
    np.savez_compressed(out_path, **res)
    print("wrote", out_path, len(res), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "cuda_conv.npz"))
