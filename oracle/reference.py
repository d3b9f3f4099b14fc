"""TEST INFRASTRUCTURE — ctypes wrapper over oracle/_ref/libctref*.so, the
reference's own CPU backends compiled from its unmodified sources.

``available()`` is False when the libraries were never built (the reference
tree was absent at build time); callers skip or fall back to the restatement.
``timing_lib()`` picks the widest-ISA timing build the host CPU supports.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref")
_F32P = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
SERIAL, OPENMP = 0, 1
_cache: dict = {}


def _cpu_flags() -> set:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def _declare(L):
    i, f, p = ctypes.c_int, ctypes.c_float, ctypes.c_void_p
    L.ref_set_threads.argtypes = [i]
    L.ref_max_threads.restype = i
    L.ref_compute_sinogram.argtypes = [i, _F32P, i, i, i, i, _F32P, _F32P, _F32P]
    L.ref_reconstruct_slice.argtypes = [i, _F32P, i, i, _F32P, f, f, i, i, _F32P]
    L.ref_reconstruct_volume.argtypes = [i, _F32P, i, i, i, i, _F32P, ctypes.POINTER(ctypes.c_double)]
    L.ref_reconstruct_from_sinograms.argtypes = [i, _F32P, i, i, i, _F32P, i, _F32P]
    L.ref_extract_point_cloud.argtypes = [i, _F32P, i, i, i, f, p, ctypes.c_longlong,
                                          ctypes.POINTER(ctypes.c_longlong)]
    L.ref_create_filter.argtypes = [i, i, _F32P]
    L.ref_generator3d.argtypes = [i, i, i, f, i, ctypes.c_uint, _F32P, _F32P]
    return L


def _open(name: str):
    if name not in _cache:
        path = os.path.join(HERE, name)
        _cache[name] = _declare(ctypes.CDLL(path)) if os.path.exists(path) else None
    return _cache[name]


def available() -> bool:
    return parity_lib() is not None


def parity_lib():
    """-O2 baseline-ISA build: bit-comparable with the float restatement."""
    return _open("libctref.so")


def timing_lib():
    """-O3 build for the widest ISA this CPU runs (the timed CPU baseline)."""
    flags = _cpu_flags()
    if {"avx512f", "avx512bw", "avx512vl", "avx512dq", "avx512cd"} <= flags:
        lib = _open("libctref_v4.so")
        if lib is not None:
            return lib, "x86-64-v4"
    if {"avx2", "fma", "bmi2"} <= flags:
        lib = _open("libctref_v3.so")
        if lib is not None:
            return lib, "x86-64-v3"
    return parity_lib(), "x86-64"


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference {what} returned status {rc}")


def compute_sinogram(which: int, slice2d, na: int, nd: int, lib=None):
    L = lib or parity_lib()
    s = np.ascontiguousarray(slice2d, np.float32)
    h, w = s.shape
    sino = np.zeros((na, nd), np.float32)
    ang = np.zeros(na, np.float32)
    mm = np.zeros(2, np.float32)
    _check(L.ref_compute_sinogram(which, s, w, h, na, nd, sino, ang, mm), "computeSinogram")
    return sino, ang, mm


def reconstruct_slice(which: int, sino, angles_deg, n_out: int, kind: int,
                      min_hu=0.0, max_hu=1.0, lib=None):
    L = lib or parity_lib()
    s = np.ascontiguousarray(sino, np.float32)
    na, nd = s.shape
    out = np.zeros((n_out, n_out), np.float32)
    _check(L.ref_reconstruct_slice(which, s, na, nd, np.ascontiguousarray(angles_deg, np.float32),
                                   min_hu, max_hu, n_out, kind, out), "reconstructSlice")
    return out


def reconstruct_volume(which: int, vol, na: int, kind: int, lib=None):
    L = lib or parity_lib()
    v = np.ascontiguousarray(vol, np.float32)
    nz, n, _ = v.shape
    out = np.zeros_like(v)
    ms = ctypes.c_double()
    _check(L.ref_reconstruct_volume(which, v, n, nz, na, kind, out, ctypes.byref(ms)),
           "reconstructVolume")
    return out


def reconstruct_from_sinograms(which: int, sinos, angles_deg, kind: int, lib=None):
    L = lib or parity_lib()
    s = np.ascontiguousarray(sinos, np.float32)
    nz, na, bins = s.shape
    out = np.zeros((nz, bins, bins), np.float32)
    _check(L.ref_reconstruct_from_sinograms(which, s, nz, na, bins,
                                            np.ascontiguousarray(angles_deg, np.float32), kind, out),
           "reconstructVolumeFromSinograms")
    return out


def extract_point_cloud(which: int, vol, thr: float, lib=None):
    L = lib or parity_lib()
    v = np.ascontiguousarray(vol, np.float32)
    nz, ny, nx = v.shape
    cnt = ctypes.c_longlong()
    _check(L.ref_extract_point_cloud(which, v, nx, ny, nz, thr, None, 0, ctypes.byref(cnt)),
           "extractPointCloud")
    pts = np.zeros((cnt.value, 4), np.float32)
    if cnt.value:
        _check(L.ref_extract_point_cloud(which, v, nx, ny, nz, thr, pts.ctypes.data, cnt.value,
                                         ctypes.byref(cnt)), "extractPointCloud")
    return pts


def create_filter(L_fft: int, kind: int, lib=None):
    L = lib or parity_lib()
    H = np.zeros(L_fft // 2 + 1, np.float32)
    _check(L.ref_create_filter(L_fft, kind, H), "createFilter")
    return H


def generator3d(nx, ny, nz, radius_mm=50.0, n_ell=120, seed=42, tissue=None, lib=None):
    from . import GENERATOR3D_TISSUE
    L = lib or parity_lib()
    t = GENERATOR3D_TISSUE if tissue is None else np.ascontiguousarray(tissue, np.float32)
    vol = np.zeros((nz, ny, nx), np.float32)
    _check(L.ref_generator3d(nx, ny, nz, radius_mm, n_ell, seed, t, vol), "generateBrainHU")
    return vol
