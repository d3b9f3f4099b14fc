"""TEST INFRASTRUCTURE — the CPU oracle for the B200 FBP backend.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import this package, and only as
the checker or the timed CPU baseline; the product path never calls it.

Two native libraries are wrapped here:

* ``libctoracle.so`` (built from ``ct_oracle.cpp``): a restatement of
  QtCTReconstruction's ``SerialBackend`` path in float (bit-for-bit the
  reference's arithmetic) and in double precision (the "FP64 rerun").
* ``_ref/libctref*.so`` (built by ``Makefile`` from the unmodified reference
  sources): the reference's own ``SerialBackend``, ``OpenMPBackend``,
  ``FilterDesign`` and ``Generator3DCPU``. Present when the reference tree was
  available at build time; the loader returns ``None`` otherwise.

Filter ids follow ``ReconstructionParams::FilterType`` (CTTypes.h:151):
0 Ramp, 1 Shepp-Logan, 2 Hamming, 3 Cosine, 4 Hann, 5 Bartlett.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_F32P = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")

RAMP, SHEPP_LOGAN, HAMMING, COSINE, HANN, BARTLETT = range(6)

# Generator3D::Params defaults (Generator3D.h:16-34): soft tissue, then bone.
GENERATOR3D_TISSUE = np.array(
    [-20.0, 45.0, 3.0, 10.0, 0.0, 0.0, 0.0, 1.0,
     200.0, 1000.0, 2.0, 8.0, 1.0, 0.7, 0.9, 0.15], dtype=np.float32)


def build() -> None:
    """Build libctoracle.so (and oracle/_ref when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "-j8"], check=True)


def _load(name: str):
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        return None
    return ctypes.CDLL(path)


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load("libctoracle.so")
        if _lib is None:
            build()
            _lib = _load("libctoracle.so")
        _declare_oracle(_lib)
    return _lib


def _declare_oracle(L):
    i, f, p = ctypes.c_int, ctypes.c_float, ctypes.c_void_p
    L.orc_filter_f32.argtypes = [i, i, _F32P]
    L.orc_filter_f64.argtypes = [i, i, _F64P]
    L.orc_pad_geometry.argtypes = [i, ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(i)]
    L.orc_sinogram_f32.argtypes = [_F32P, i, i, i, i, _F32P, _F32P, _F32P]
    L.orc_sinogram_f64.argtypes = [_F32P, i, i, i, i, _F32P, _F64P, _F64P]
    L.orc_reconstruct_slice_f32.argtypes = [_F32P, i, i, _F32P, i, i, _F32P]
    L.orc_reconstruct_slice_f64.argtypes = [_F64P, i, i, _F32P, i, i, _F64P]
    L.orc_filter_rows_f32.argtypes = [_F32P, i, i, i, _F32P]
    L.orc_filter_rows_f64.argtypes = [_F64P, i, i, i, _F64P]
    L.orc_backproject_f64.argtypes = [_F64P, i, i, _F32P, i, _F64P]
    L.orc_reconstruct_volume_f32.argtypes = [_F32P, i, i, i, i, i, _F32P]
    L.orc_reconstruct_volume_f64.argtypes = [_F32P, i, i, i, i, i, _F64P]
    L.orc_phantom_params.argtypes = [ctypes.c_uint64, i, _F32P]
    L.orc_phantom_sum.argtypes = [_F32P, i, i, i, i, _F32P]
    L.orc_phantom_sum_slab.argtypes = [_F32P, i, i, i, i, i, i, _F32P]
    L.orc_generator3d.argtypes = [i, i, i, f, i, ctypes.c_uint, _F32P, _F32P]
    L.orc_point_cloud.argtypes = [_F32P, i, i, i, f, p, ctypes.c_longlong,
                                  ctypes.POINTER(ctypes.c_longlong)]
    L.orc_cc_sinogram_f64.argtypes = [_F32P, i, i, i, i, ctypes.c_double, _F32P, _F64P, _F32P]
    L.orc_cc_reconstruct_slice_f64.argtypes = [_F64P, i, i, _F32P, i, i, f, f, _F64P]
    L.orc_cc_reconstruct_volume_f64.argtypes = [_F32P, i, i, i, i, _F64P]


def _ok(rc: int, what: str):
    if rc != 0:
        raise ValueError(f"oracle {what} rejected its arguments (status {rc})")


# ----------------------------------------------------------------- geometry
def odd_detector_count(n: int) -> int:
    """ceil(sqrt(2) * n) rounded up to an odd number of detector bins."""
    nd = math.ceil(math.sqrt(2.0) * n)
    return nd + 1 if nd % 2 == 0 else nd


def pad_geometry(bins: int):
    """(square_bins, pad_before, fft_size) of reconstructSlice (SerialBackend.cpp:152-163)."""
    sq, pad, L = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _ok(lib().orc_pad_geometry(bins, ctypes.byref(sq), ctypes.byref(pad), ctypes.byref(L)), "pad_geometry")
    return sq.value, pad.value, L.value


def uniform_angles_deg(na: int) -> np.ndarray:
    """180/na * a in float arithmetic, as SerialBackend stores them."""
    step = np.float32(180.0) / np.float32(na)
    return (step * np.arange(na, dtype=np.float32)).astype(np.float32)


# ------------------------------------------------------------------ filters
def filter_f32(L: int, kind: int) -> np.ndarray:
    H = np.zeros(L // 2 + 1, np.float32)
    _ok(lib().orc_filter_f32(L, kind, H), "filter_f32")
    return H


def filter_f64(L: int, kind: int) -> np.ndarray:
    H = np.zeros(L // 2 + 1, np.float64)
    _ok(lib().orc_filter_f64(L, kind, H), "filter_f64")
    return H


# ------------------------------------------------------------ forward / FBP
def sinogram_f32(slice2d: np.ndarray, na: int, nd: int):
    s = np.ascontiguousarray(slice2d, np.float32)
    h, w = s.shape
    sino = np.zeros((na, nd), np.float32)
    ang = np.zeros(na, np.float32)
    mm = np.zeros(2, np.float32)
    _ok(lib().orc_sinogram_f32(s, w, h, na, nd, sino, ang, mm), "sinogram_f32")
    return sino, ang, mm


def sinogram_f64(slice2d: np.ndarray, na: int, nd: int, angles_deg=None):
    s = np.ascontiguousarray(slice2d, np.float32)
    h, w = s.shape
    ang = uniform_angles_deg(na) if angles_deg is None else np.ascontiguousarray(angles_deg, np.float32)
    sino = np.zeros((na, nd), np.float64)
    mm = np.zeros(2, np.float64)
    _ok(lib().orc_sinogram_f64(s, w, h, na, nd, ang, sino, mm), "sinogram_f64")
    return sino, mm


def filter_rows_f32(sino: np.ndarray, kind: int) -> np.ndarray:
    s = np.ascontiguousarray(sino, np.float32)
    na, nd = s.shape
    sq, _, _ = pad_geometry(nd)
    out = np.zeros((na, sq), np.float32)
    _ok(lib().orc_filter_rows_f32(s, na, nd, kind, out), "filter_rows_f32")
    return out


def filter_rows_f64(sino: np.ndarray, kind: int) -> np.ndarray:
    s = np.ascontiguousarray(sino, np.float64)
    na, nd = s.shape
    sq, _, _ = pad_geometry(nd)
    out = np.zeros((na, sq), np.float64)
    _ok(lib().orc_filter_rows_f64(s, na, nd, kind, out), "filter_rows_f64")
    return out


def backproject_f64(filt: np.ndarray, angles_deg, n_out: int) -> np.ndarray:
    f = np.ascontiguousarray(filt, np.float64)
    na, sq = f.shape
    out = np.zeros((n_out, n_out), np.float64)
    _ok(lib().orc_backproject_f64(f, na, sq, np.ascontiguousarray(angles_deg, np.float32), n_out, out),
        "backproject_f64")
    return out


def reconstruct_slice_f32(sino: np.ndarray, angles_deg, n_out: int, kind: int) -> np.ndarray:
    s = np.ascontiguousarray(sino, np.float32)
    na, nd = s.shape
    out = np.zeros((n_out, n_out), np.float32)
    _ok(lib().orc_reconstruct_slice_f32(s, na, nd, np.ascontiguousarray(angles_deg, np.float32),
                                        n_out, kind, out), "reconstruct_slice_f32")
    return out


def reconstruct_slice_f64(sino: np.ndarray, angles_deg, n_out: int, kind: int) -> np.ndarray:
    s = np.ascontiguousarray(sino, np.float64)
    na, nd = s.shape
    out = np.zeros((n_out, n_out), np.float64)
    _ok(lib().orc_reconstruct_slice_f64(s, na, nd, np.ascontiguousarray(angles_deg, np.float32),
                                        n_out, kind, out), "reconstruct_slice_f64")
    return out


def reconstruct_volume_f32(vol: np.ndarray, na: int, nd: int, kind: int) -> np.ndarray:
    v = np.ascontiguousarray(vol, np.float32)
    nz, n, n2 = v.shape
    assert n == n2
    out = np.zeros_like(v)
    _ok(lib().orc_reconstruct_volume_f32(v, n, nz, na, nd, kind, out), "reconstruct_volume_f32")
    return out


def reconstruct_volume_f64(vol: np.ndarray, na: int, nd: int, kind: int) -> np.ndarray:
    v = np.ascontiguousarray(vol, np.float32)
    nz, n, n2 = v.shape
    assert n == n2
    out = np.zeros(v.shape, np.float64)
    _ok(lib().orc_reconstruct_volume_f64(v, n, nz, na, nd, kind, out), "reconstruct_volume_f64")
    return out


# ----------------------------------------------------------------- phantoms
def phantom_params(seed: int, count: int) -> np.ndarray:
    """Ellipsoid records (count, 16) float32 of the seeded benchmark phantom."""
    p = np.zeros(max(count, 1) * 16, np.float32)
    _ok(lib().orc_phantom_params(seed, count, p), "phantom_params")
    return p[: count * 16].reshape(count, 16)


def phantom_sum(params: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    p = np.ascontiguousarray(params, np.float32).reshape(-1)
    k = p.size // 16
    vol = np.zeros((nz, ny, nx), np.float32)
    _ok(lib().orc_phantom_sum(p, k, nx, ny, nz, vol), "phantom_sum")
    return vol


def phantom_sum_slab(params: np.ndarray, nx: int, ny: int, nz: int, z0: int, nzs: int) -> np.ndarray:
    """Slices [z0, z0+nzs) of phantom_sum(params, nx, ny, nz)."""
    p = np.ascontiguousarray(params, np.float32).reshape(-1)
    vol = np.zeros((nzs, ny, nx), np.float32)
    _ok(lib().orc_phantom_sum_slab(p, p.size // 16, nx, ny, nz, z0, nzs, vol), "phantom_sum_slab")
    return vol


def generator3d(nx: int, ny: int, nz: int, radius_mm=50.0, n_ell=120, seed=42, tissue=None):
    t = GENERATOR3D_TISSUE if tissue is None else np.ascontiguousarray(tissue, np.float32)
    vol = np.zeros((nz, ny, nx), np.float32)
    _ok(lib().orc_generator3d(nx, ny, nz, radius_mm, n_ell, seed, t, vol), "generator3d")
    return vol


def point_cloud(vol: np.ndarray, thr: float) -> np.ndarray:
    v = np.ascontiguousarray(vol, np.float32)
    nz, ny, nx = v.shape
    cnt = ctypes.c_longlong()
    _ok(lib().orc_point_cloud(v, nx, ny, nz, thr, None, 0, ctypes.byref(cnt)), "point_cloud")
    pts = np.zeros((cnt.value, 4), np.float32)
    if cnt.value:
        _ok(lib().orc_point_cloud(v, nx, ny, nz, thr, pts.ctypes.data, cnt.value, ctypes.byref(cnt)),
            "point_cloud")
    return pts


# ------------------------------------------------------- error measures
# ------------------------------------------- the CUDA backend's conventions
def cc_sinogram_f64(slice2d: np.ndarray, na: int, nd: int, det_center=None, angles_deg=None):
    """CUDABackend::computeSinogram restated in FP64 (ray march, bilinear,
    every pixel normalised; detector centre (nd - 1) / 2 unless given).
    Returns (sino[na][nd] f64, angles, minmax)."""
    s = np.ascontiguousarray(slice2d, np.float32)
    h, w = s.shape
    ang = uniform_angles_deg(na) if angles_deg is None else np.ascontiguousarray(angles_deg, np.float32)
    out = np.zeros((na, nd), np.float64)
    mm = np.zeros(2, np.float32)
    dc = 0.5 * (nd - 1) if det_center is None else float(det_center)
    _ok(lib().orc_cc_sinogram_f64(s, w, h, na, nd, dc, ang, out, mm), "cc_sinogram_f64")
    return out, ang, mm


def cc_reconstruct_slice_f64(sino: np.ndarray, angles_deg, n_out: int, kind: int, min_hu=0.0, max_hu=0.0):
    """CUDABackend::reconstructSlice restated in FP64 (Nyquist kept, (N-1)/2 and
    (sq-1)/2 centres, per-tap bounds, denormalised when max_hu > min_hu)."""
    s = np.ascontiguousarray(sino, np.float64)
    na, nd = s.shape
    out = np.zeros((n_out, n_out), np.float64)
    _ok(lib().orc_cc_reconstruct_slice_f64(s, na, nd, np.ascontiguousarray(angles_deg, np.float32), n_out, kind,
                                          float(min_hu), float(max_hu), out), "cc_reconstruct_slice_f64")
    return out


def cc_reconstruct_volume_f64(vol: np.ndarray, na: int, kind: int) -> np.ndarray:
    """CUDABackend::reconstructVolume restated in FP64 (nd = n, detector centre floor(n / 2))."""
    v = np.ascontiguousarray(vol, np.float32)
    depth, n, _ = v.shape
    out = np.zeros(v.shape, np.float64)
    _ok(lib().orc_cc_reconstruct_volume_f64(v, n, depth, na, kind, out), "cc_reconstruct_volume_f64")
    return out


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (d if d > 0 else 1.0))


def max_abs_rel(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    m = np.max(np.abs(b)) if b.size else 0.0
    return float(np.max(np.abs(a - b)) / (m if m > 0 else 1.0)) if a.size else 0.0


from . import reference  # noqa: E402  (the reference-build wrapper)
