"""qtctreconstruction_b200 — B200-native backend for QtCTReconstruction's FBP path.

The compute path is ``libctb200.so`` (hand-written sm_100a CUDA kernels behind
the C ABI declared in ``include/ctb200.h``). This module loads it with ctypes
and mirrors the reference's ``ct::IReconstructionBackend`` interface
(IReconstructionBackend.h:10-55) with the same method names, argument meaning
and result units, so code written against the reference's backends reads the
same here. There is no CPU fallback: if the library or an sm_100 GPU is
missing, construction raises.

Conventions (the reference's SerialBackend): slices are ``[y][x]`` float32,
volumes ``[z][y][x]``, sinograms ``[angle][bin]``; uniform angles are
``180/na * a`` degrees in float; filter ids follow
``ReconstructionParams::FilterType``.
"""
from __future__ import annotations

import ctypes
import enum
import os
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
# CTB200_LIB selects another build of the library (e.g. a tuning variant)
LIB_PATH = os.environ.get("CTB200_LIB", os.path.join(PKG, "libctb200.so"))


class FilterType(enum.IntEnum):
    """ReconstructionParams::FilterType (CTTypes.h:151)."""
    Ramp = 0
    SheppLogan = 1
    Hamming = 2
    Cosine = 3
    Hann = 4
    Bartlett = 5


class Denorm(enum.IntEnum):
    """Output units of a reconstruction from sinograms (ctb_denorm)."""
    NONE = 0     # normalised units (SerialBackend::reconstructSlice)
    SERIAL = 1   # x * (span <= 0 ? 1 : span) + min  (SerialBackend.cpp:297-304)
    OPENMP = 2   # x * span + min, min if span <= 0  (OpenMPBackend.cpp:37-59)
    CUDA = 3     # x * span + min if span > 0, else x  (CUDABackend.cu:676-681)


@dataclass
class ReconstructionParams:
    """ReconstructionParams (CTTypes.h:150-156)."""
    filter: FilterType = FilterType.SheppLogan
    num_angles: int = 180
    zero_padding: bool = True  # never read by the reference either


@dataclass
class Sinogram:
    """Sinogram (CTTypes.h:131-137): data is [angle][bin] (height=angles, width=bins)."""
    data: np.ndarray
    angles_deg: np.ndarray
    detector_spacing_mm: float = 1.0
    original_min_hu: float = 0.0
    original_max_hu: float = 0.0


class CtbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"ctb status {status}: {message}")
        self.status = status


_lib = None
_F32P = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


class FbpJob(ctypes.Structure):
    """ctb_fbp_job: one job of a batch (device pointers, host angle list or None)."""
    _fields_ = [("sino", ctypes.c_void_p), ("depth", ctypes.c_int), ("num_angles", ctypes.c_int),
                ("bins", ctypes.c_int), ("angles_deg", ctypes.c_void_p), ("output_size", ctypes.c_int),
                ("filter", ctypes.c_int), ("out", ctypes.c_void_p)]


class ServerConfig(ctypes.Structure):
    """ctb_server_config."""
    _fields_ = [("device", ctypes.c_int), ("memory_budget", ctypes.c_size_t), ("max_batch", ctypes.c_int),
                ("copy_threads", ctypes.c_int), ("staging_bytes", ctypes.c_size_t), ("fault_every", ctypes.c_int)]


class Request(ctypes.Structure):
    """ctb_request."""
    _fields_ = [("sino", ctypes.c_void_p), ("depth", ctypes.c_int), ("num_angles", ctypes.c_int),
                ("bins", ctypes.c_int), ("angles_deg", ctypes.c_void_p), ("output_size", ctypes.c_int),
                ("filter", ctypes.c_int), ("out", ctypes.c_void_p), ("flags", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    """ctb_server_stats."""
    _fields_ = [(k, ctypes.c_uint64) for k in ("submitted", "completed", "failed", "cancelled", "rejected",
                                                "batches")] + \
               [(k, ctypes.c_double) for k in ("mean_batch", "p50_ms", "p99_ms", "max_ms", "volumes_per_s",
                                               "updates_per_s")] + \
               [("memory_budget", ctypes.c_size_t), ("memory_peak", ctypes.c_size_t)]


STATUS_OK, STATUS_INVALID, STATUS_CUDA, STATUS_OOM, STATUS_UNSUPPORTED = 0, 1, 2, 3, 4  # ctb_status
STATUS_NO_DEVICE, STATUS_TIMEOUT, STATUS_CANCELLED, STATUS_NOT_FOUND, STATUS_BUSY = 5, 6, 7, 8, 9
REQ_DEVICE = 1     # CTB_REQ_DEVICE
CONVENTION_SERIAL = 0       # CTB_CONVENTION_SERIAL
CONVENTION_CUDA = 1         # CTB_CONVENTION_CUDA
FILTER_MODE_FFT = 0         # CTB_FILTER_MODE_FFT
FILTER_MODE_TC_BF16X3 = 1   # CTB_FILTER_MODE_TC_BF16X3
BATCH_GRAPH = 1    # CTB_BATCH_GRAPH
BATCH_PER_JOB = 2  # CTB_BATCH_PER_JOB
BATCH_PERSISTENT = 4  # CTB_BATCH_PERSISTENT


def library() -> ctypes.CDLL:
    """Load libctb200.so (raises if it was never built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m qtctreconstruction_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def _declare(L):
    i, f, p, u64 = ctypes.c_int, ctypes.c_float, ctypes.c_void_p, ctypes.c_uint64
    P = ctypes.POINTER
    L.ctb_create.argtypes = [P(p), i]
    L.ctb_destroy.argtypes = [p]
    L.ctb_destroy.restype = None
    L.ctb_last_error.argtypes = [p]
    L.ctb_last_error.restype = ctypes.c_char_p
    L.ctb_status_string.argtypes = [i]
    L.ctb_status_string.restype = ctypes.c_char_p
    L.ctb_set_stream.argtypes = [p, p]
    L.ctb_synchronize.argtypes = [p]
    L.ctb_last_sinogram_ms.argtypes = [p]
    L.ctb_last_sinogram_ms.restype = ctypes.c_double
    L.ctb_last_reconstruction_ms.argtypes = [p]
    L.ctb_last_reconstruction_ms.restype = ctypes.c_double
    L.ctb_last_phantom_ms.argtypes = [p]
    L.ctb_last_phantom_ms.restype = ctypes.c_double
    L.ctb_launch_count.argtypes = [p]
    L.ctb_launch_count.restype = u64
    L.ctb_pad_geometry.argtypes = [i, P(i), P(i), P(i)]
    L.ctb_filter_response.argtypes = [i, i, _F32P]
    L.ctb_compute_sinogram.argtypes = [p, p, i, i, i, i, p, p, p]
    L.ctb_reconstruct_slice.argtypes = [p, p, i, i, p, i, i, p]
    L.ctb_reconstruct_slice_hu.argtypes = [p, p, i, i, p, i, i, f, f, p]
    L.ctb_set_convention.argtypes = [p, i]
    L.ctb_reconstruct_volume.argtypes = [p, p, i, i, i, i, i, p]
    L.ctb_reconstruct_from_sinograms.argtypes = [p, p, i, i, i, p, i, i, p]
    L.ctb_forward_d.argtypes = [p, p, i, i, i, i, p, p, p]
    L.ctb_fbp_d.argtypes = [p, p, i, i, i, p, i, i, p, i, p]
    L.ctb_reconstruct_volume_d.argtypes = [p, p, i, i, i, i, i, p]
    L.ctb_phantom_params.argtypes = [u64, i, _F32P]
    L.ctb_phantom_sum_d.argtypes = [p, _F32P, i, i, i, i, p]
    L.ctb_phantom_sum.argtypes = [p, _F32P, i, i, i, i, p]
    L.ctb_generator3d.argtypes = [p, i, i, i, f, i, ctypes.c_uint32, _F32P, p]
    L.ctb_extract_point_cloud.argtypes = [p, p, i, i, i, f, p, ctypes.c_int64, P(ctypes.c_int64)]
    L.ctb_set_profiling.argtypes = [p, i]
    L.ctb_set_filter_mode.argtypes = [p, i]
    L.ctb_set_forward_bounds.argtypes = [p, i]
    L.ctb_set_bp_shape.argtypes = [p, i]
    L.ctb_bp_shape_info.argtypes = [i, P(i), P(i), P(i), P(i)]
    L.ctb_bp_shape_for.argtypes = [p, i, i, i, P(i)]
    L.ctb_set_autotune.argtypes = [p, i]
    L.ctb_autotune_table.argtypes = [p, P(i), i, P(i)]
    L.ctb_autotune_load.argtypes = [p, P(i), i]
    L.ctb_sinogram_file_shape.argtypes = [ctypes.c_char_p, P(i), P(i), P(i)]
    L.ctb_load_sinogram_file.argtypes = [ctypes.c_char_p, p, p, p]
    L.ctb_save_sinogram_file.argtypes = [ctypes.c_char_p, p, i, i, i, p, f, f, f]
    L.ctb_filter_kernel_ms.argtypes = [p, i, P(ctypes.c_double)]
    L.ctb_stage_times.argtypes = [p, i, P(ctypes.c_double)]
    L.ctb_probe_smem_bandwidth.argtypes = [p, P(ctypes.c_double)]
    L.ctb_selftest_bounded_wait.argtypes = [p, ctypes.c_uint]
    L.ctb_set_fault_injection.argtypes = [p, i]
    L.ctb_batch_create.argtypes = [p, P(FbpJob), i, i, P(p)]
    L.ctb_batch_run.argtypes = [p]
    L.ctb_batch_info.argtypes = [p, P(i), P(ctypes.c_double), P(ctypes.c_size_t)]
    L.ctb_batch_destroy.argtypes = [p]
    L.ctb_batch_destroy.restype = None
    L.ctb_fbp_batch_d.argtypes = [p, P(FbpJob), i]
    L.ctb_fbp.argtypes = [p, p, i, i, i, p, i, i, p]
    L.ctb_server_create.argtypes = [P(ServerConfig), P(p)]
    L.ctb_server_submit.argtypes = [p, P(Request), P(u64)]
    L.ctb_server_poll.argtypes = [p, u64]
    L.ctb_server_wait.argtypes = [p, u64, ctypes.c_double]
    L.ctb_server_cancel.argtypes = [p, u64]
    L.ctb_server_release.argtypes = [p, u64]
    L.ctb_server_get_stats.argtypes = [p, P(ServerStats)]
    L.ctb_server_destroy.argtypes = [p]
    L.ctb_server_destroy.restype = None
    sz = ctypes.c_size_t
    L.ctb_arena_create.argtypes = [sz, P(p)]
    L.ctb_arena_alloc.argtypes = [p, sz, P(sz)]
    L.ctb_arena_free.argtypes = [p, sz]
    L.ctb_arena_stats.argtypes = [p, P(sz), P(sz), P(sz)]
    L.ctb_arena_destroy.argtypes = [p]
    L.ctb_arena_destroy.restype = None


# ----------------------------------------------------------------- helpers
def bp_shape_info(variant: int):
    """(tile_x, tile_y, voxels_per_thread, angles_per_chunk) of a backprojection tile shape."""
    v = [ctypes.c_int() for _ in range(4)]
    st = library().ctb_bp_shape_info(variant, *[ctypes.byref(x) for x in v])
    if st:
        raise CtbError(st, "bp_shape_info")
    return tuple(x.value for x in v)


def pad_geometry(bins: int):
    """(square_bins, pad_before, fft_size) of reconstructSlice (SerialBackend.cpp:152-163)."""
    sq, pad, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    st = library().ctb_pad_geometry(bins, ctypes.byref(sq), ctypes.byref(pad), ctypes.byref(n))
    if st:
        raise CtbError(st, "pad_geometry")
    return sq.value, pad.value, n.value


def filter_response(fft_size: int, kind: int) -> np.ndarray:
    """FilterDesign::createFilter evaluated in double precision (fft_size/2+1 floats)."""
    H = np.zeros(fft_size // 2 + 1, np.float32)
    st = library().ctb_filter_response(fft_size, int(kind), H)
    if st:
        raise CtbError(st, "filter_response")
    return H


def uniform_angles_deg(na: int) -> np.ndarray:
    step = np.float32(180.0) / np.float32(na)
    return (step * np.arange(na, dtype=np.float32)).astype(np.float32)


def odd_detector_count(n: int) -> int:
    """ceil(sqrt(2) * n) rounded up to an odd number (the benchmark detector)."""
    import math
    nd = math.ceil(math.sqrt(2.0) * n)
    return nd + 1 if nd % 2 == 0 else nd


def phantom_params(seed: int, count: int) -> np.ndarray:
    """Benchmark phantom ellipsoids: (count, 16) float32 records."""
    p = np.zeros(max(count, 1) * 16, np.float32)
    st = library().ctb_phantom_params(seed, count, p)
    if st:
        raise CtbError(st, "phantom_params")
    return p[: count * 16].reshape(count, 16)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


# ------------------------------------------------------------ sinogram files
def load_sinogram_file(path: str):
    """Read a sinogram stack written in the reference's consumer format
    (NPY (depth, num_angles, bins) float32 + optional <name>.meta.json):
    returns (sinos, angles_deg, {"detector_spacing_mm", "original_min_hu",
    "original_max_hu"}) with the reference's fallbacks for missing keys."""
    L = library()
    d, a, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    st = L.ctb_sinogram_file_shape(os.fsencode(path), ctypes.byref(d), ctypes.byref(a), ctypes.byref(b))
    if st:
        raise CtbError(st, f"cannot read {path}")
    sinos = np.empty((d.value, a.value, b.value), np.float32)
    ang = np.empty(a.value, np.float32)
    meta = np.empty(3, np.float32)
    st = L.ctb_load_sinogram_file(os.fsencode(path), sinos.ctypes.data, ang.ctypes.data, meta.ctypes.data)
    if st:
        raise CtbError(st, f"cannot read {path}")
    return sinos, ang, {"detector_spacing_mm": float(meta[0]), "original_min_hu": float(meta[1]),
                        "original_max_hu": float(meta[2])}


def save_sinogram_file(path: str, sinos, angles_deg=None, spacing_mm: float = 1.0, min_hu=None, max_hu=None):
    """Write sinograms[depth][num_angles][bins] in the consumer format (min/max
    default to the data's)."""
    s = _f32(sinos)
    if s.ndim != 3:
        raise ValueError("sinograms must be (depth, num_angles, bins)")
    ang = None if angles_deg is None else _f32(angles_deg)
    lo = float(s.min()) if min_hu is None else float(min_hu)
    hi = float(s.max()) if max_hu is None else float(max_hu)
    st = library().ctb_save_sinogram_file(os.fsencode(path), s.ctypes.data, *s.shape,
                                          None if ang is None else ang.ctypes.data, spacing_mm, lo, hi)
    if st:
        raise CtbError(st, f"cannot write {path}")


# ----------------------------------------------------------------- backend
class B200Backend:
    """ct::IReconstructionBackend on one B200 (the new backend type)."""

    def __init__(self, device: int = 0):
        L = library()
        h = ctypes.c_void_p()
        st = L.ctb_create(ctypes.byref(h), device)
        if st:
            raise CtbError(st, L.ctb_status_string(st).decode())
        self._lib = L
        self._h = h
        self.device = device

    # -- lifecycle -------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.ctb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int, what: str):
        if st:
            msg = self._lib.ctb_last_error(self._h).decode()
            raise CtbError(st, f"{what}: {msg or self._lib.ctb_status_string(st).decode()}")

    @property
    def handle(self):
        return self._h

    # -- IReconstructionBackend ------------------------------------------
    def name(self) -> str:
        return "B200 (CUDA sm_100a)"

    def isAvailable(self) -> bool:
        return self._h is not None

    def computeSinogram(self, slice2d, num_angles: int, detector_bins: int,
                        use_parallel: bool = True) -> Sinogram:
        """SerialBackend::computeSinogram (SerialBackend.cpp:59-136)."""
        s = _f32(slice2d)
        if s.ndim != 2 or s.size == 0 or num_angles <= 0 or detector_bins <= 0:
            return Sinogram(np.zeros((0, 0), np.float32), np.zeros(0, np.float32))
        h, w = s.shape
        sino = np.zeros((num_angles, detector_bins), np.float32)
        ang = np.zeros(num_angles, np.float32)
        mm = np.zeros(2, np.float32)
        self._check(self._lib.ctb_compute_sinogram(self._h, _ptr(s), w, h, num_angles, detector_bins,
                                                   _ptr(sino), _ptr(ang), _ptr(mm)), "computeSinogram")
        return Sinogram(sino, ang, 1.0, float(mm[0]), float(mm[1]))

    def reconstructSlice(self, sinogram: Sinogram, output_size: int,
                         params: ReconstructionParams) -> np.ndarray:
        """IReconstructionBackend::reconstructSlice: SerialBackend's normalised units
        (SerialBackend.cpp:142-255), or with the CUDA convention the CUDA backend's
        denormalisation by the sinogram's original_min_hu/max_hu (CUDABackend.cu:676-681)."""
        d = _f32(sinogram.data)
        if d.ndim != 2 or d.size == 0 or output_size <= 0:
            return np.zeros((0, 0), np.float32)
        na, nd = d.shape
        ang = _f32(sinogram.angles_deg)
        out = np.zeros((output_size, output_size), np.float32)
        self._check(self._lib.ctb_reconstruct_slice_hu(self._h, _ptr(d), na, nd, _ptr(ang), output_size,
                                                       int(params.filter), float(sinogram.original_min_hu),
                                                       float(sinogram.original_max_hu), _ptr(out)),
                    "reconstructSlice")
        return out

    def reconstructVolume(self, volume, params: ReconstructionParams,
                          onSliceDone: Optional[Callable[[int, np.ndarray], None]] = None,
                          detector_bins: Optional[int] = None) -> np.ndarray:
        """SerialBackend::reconstructVolume (SerialBackend.cpp:261-318).

        The reference projects onto detector_bins = width; pass detector_bins
        to use another detector (the benchmark uses odd ceil(sqrt(2) n)).
        """
        v = _f32(volume)
        if v.size == 0:
            return np.zeros((0, 0, 0), np.float32)
        nz, n, n2 = v.shape
        if n != n2:
            raise ValueError("reconstructVolume needs square slices")
        nd = n if detector_bins is None else int(detector_bins)
        out = np.zeros_like(v)
        self._check(self._lib.ctb_reconstruct_volume(self._h, _ptr(v), n, nz, int(params.num_angles), nd,
                                                     int(params.filter), _ptr(out)), "reconstructVolume")
        if onSliceDone:
            for z in range(nz):
                onSliceDone(z, out[z])
        return out

    def reconstructVolumeFromSinograms(self, sinograms, angles_deg, params: ReconstructionParams,
                                       onSliceDone: Optional[Callable[[int, np.ndarray], None]] = None,
                                       denorm: Denorm = Denorm.NONE) -> np.ndarray:
        """IReconstructionBackend::reconstructVolumeFromSinograms (IReconstructionBackend.h:39-44).

        The default (Denorm.NONE) stores reconstructSlice's normalised units,
        as the interface's default per-slice loop does with SerialBackend.
        """
        s = _f32(sinograms)
        if s.size == 0:
            return np.zeros((0, 0, 0), np.float32)
        nz, na, bins = s.shape
        ang = _f32(angles_deg)
        out = np.zeros((nz, bins, bins), np.float32)
        self._check(self._lib.ctb_reconstruct_from_sinograms(self._h, _ptr(s), nz, na, bins, _ptr(ang),
                                                             int(params.filter), int(denorm), _ptr(out)),
                    "reconstructVolumeFromSinograms")
        if onSliceDone:
            for z in range(nz):
                onSliceDone(z, out[z])
        return out

    def extractPointCloud(self, vol, threshold: float) -> np.ndarray:
        """Points (x, y, z, hu) with hu > threshold, index coordinates, z/y/x order."""
        v = _f32(vol)
        if v.size == 0:
            return np.zeros((0, 4), np.float32)
        nz, ny, nx = v.shape
        cnt = ctypes.c_int64()
        self._check(self._lib.ctb_extract_point_cloud(self._h, _ptr(v), nx, ny, nz, float(threshold), None, 0,
                                                      ctypes.byref(cnt)), "extractPointCloud")
        pts = np.zeros((cnt.value, 4), np.float32)
        if cnt.value:
            self._check(self._lib.ctb_extract_point_cloud(self._h, _ptr(v), nx, ny, nz, float(threshold),
                                                          _ptr(pts), cnt.value, ctypes.byref(cnt)),
                        "extractPointCloud")
        return pts

    def lastSinogramTimeMs(self) -> float:
        return float(self._lib.ctb_last_sinogram_ms(self._h))

    def last_phantom_ms(self) -> float:
        """Device time of the last summed-ellipsoid phantom kernel."""
        return float(self._lib.ctb_last_phantom_ms(self._h))

    def lastReconstructionTimeMs(self) -> float:
        return float(self._lib.ctb_last_reconstruction_ms(self._h))

    # -- phantoms ----------------------------------------------------------
    def phantom(self, params: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
        p = _f32(params).reshape(-1)
        vol = np.zeros((nz, ny, nx), np.float32)
        self._check(self._lib.ctb_phantom_sum(self._h, p, p.size // 16, nx, ny, nz, _ptr(vol)), "phantom")
        return vol

    def generator3d(self, nx: int, ny: int, nz: int, radius_mm=50.0, count=120, seed=42,
                    tissue=None) -> np.ndarray:
        """Generator3D::generateBrainHU (Generator3DCPU.cpp:94-117) on the GPU."""
        t = _f32(tissue if tissue is not None else GENERATOR3D_TISSUE)
        vol = np.zeros((nz, ny, nx), np.float32)
        self._check(self._lib.ctb_generator3d(self._h, nx, ny, nz, float(radius_mm), int(count), int(seed), t,
                                              _ptr(vol)), "generator3d")
        return vol

    # -- device-resident entry points (torch tensors or raw pointers) -------
    def set_stream(self, stream_handle: int):
        self._check(self._lib.ctb_set_stream(self._h, ctypes.c_void_p(stream_handle)), "set_stream")

    def synchronize(self):
        self._check(self._lib.ctb_synchronize(self._h), "synchronize")

    def launch_count(self) -> int:
        return int(self._lib.ctb_launch_count(self._h))

    def forward_d(self, d_vol: int, n: int, depth: int, na: int, nd: int, d_sino: int, d_stats: int,
                  angles_deg=None):
        ang = None if angles_deg is None else _f32(angles_deg)
        self._check(self._lib.ctb_forward_d(self._h, ctypes.c_void_p(d_vol), n, depth, na, nd,
                                            None if ang is None else _ptr(ang), ctypes.c_void_p(d_sino),
                                            ctypes.c_void_p(d_stats)), "forward_d")

    def fbp_d(self, d_sino: int, depth: int, na: int, bins: int, output_size: int, kind: int,
              d_out: int, d_stats: int = 0, denorm: Denorm = Denorm.NONE, angles_deg=None):
        ang = None if angles_deg is None else _f32(angles_deg)
        self._check(self._lib.ctb_fbp_d(self._h, ctypes.c_void_p(d_sino), depth, na, bins,
                                        None if ang is None else _ptr(ang), output_size, int(kind),
                                        ctypes.c_void_p(d_stats) if d_stats else None, int(denorm),
                                        ctypes.c_void_p(d_out)), "fbp_d")

    def reconstruct_volume_host(self, host_vol: int, n: int, depth: int, na: int, nd: int, kind: int,
                                host_out: int):
        """reconstructVolume through the host-buffer C ABI call on raw (e.g. pinned) pointers."""
        self._check(self._lib.ctb_reconstruct_volume(self._h, ctypes.c_void_p(host_vol), n, depth, na, nd,
                                                     int(kind), ctypes.c_void_p(host_out)), "reconstructVolume")

    def set_convention(self, convention: int):
        """CONVENTION_SERIAL (default, SerialBackend) or CONVENTION_CUDA (the reference CUDA backend)."""
        self._check(self._lib.ctb_set_convention(self._h, int(convention)), "set_convention")

    def set_forward_bounds(self, enable: bool):
        """Forward projector walks only the bounding box, centred disc and
        8-row-band column ranges of each 8-slice group's non-zero pixels
        (default True; the other pixels
        are exact zero contributions). False walks the whole image, with the
        same results, for timing comparisons."""
        self._check(self._lib.ctb_set_forward_bounds(self._h, 1 if enable else 0), "set_forward_bounds")

    def set_filter_mode(self, mode: int):
        """FILTER_MODE_FFT (default) or FILTER_MODE_TC_BF16X3 (tensor-core Toeplitz product)."""
        self._check(self._lib.ctb_set_filter_mode(self._h, int(mode)), "set_filter_mode")

    def set_bp_shape(self, variant: int):
        """Force a backprojection tile shape (0..5, see bp_shape_info); -1 = automatic."""
        self._check(self._lib.ctb_set_bp_shape(self._h, int(variant)), "set_bp_shape")

    def bp_shape_for(self, output_size: int, depth: int, num_angles: int) -> int:
        v = ctypes.c_int()
        self._check(self._lib.ctb_bp_shape_for(self._h, output_size, depth, num_angles, ctypes.byref(v)),
                    "bp_shape_for")
        return v.value

    def set_autotune(self, enable: bool = True):
        self._check(self._lib.ctb_set_autotune(self._h, int(bool(enable))), "set_autotune")

    def autotune_table(self):
        """[(n bucket, angle bucket, depth bucket, shape), ...] of the tuned buckets."""
        n = ctypes.c_int()
        self._check(self._lib.ctb_autotune_table(self._h, None, 0, ctypes.byref(n)), "autotune_table")
        buf = (ctypes.c_int * (4 * max(n.value, 1)))()
        self._check(self._lib.ctb_autotune_table(self._h, buf, n.value, ctypes.byref(n)), "autotune_table")
        return [tuple(buf[4 * k:4 * k + 4]) for k in range(n.value)]

    def autotune_load(self, entries):
        flat = [int(x) for e in entries for x in e]
        buf = (ctypes.c_int * max(len(flat), 1))(*flat)
        self._check(self._lib.ctb_autotune_load(self._h, buf, len(flat) // 4), "autotune_load")

    def set_profiling(self, enable: bool = True):
        self._check(self._lib.ctb_set_profiling(self._h, int(bool(enable))), "set_profiling")

    def stage_times(self, back: int = 0):
        """Device ms of {stats+normalise, forward, filter, backprojection} of a profiled call."""
        t = (ctypes.c_double * 4)()
        self._check(self._lib.ctb_stage_times(self._h, back, t), "stage_times")
        return list(t)

    def filter_kernel_ms(self, back: int = 0) -> float:
        """Device ms of the filter's main kernel in a profiled volume call."""
        t = ctypes.c_double()
        self._check(self._lib.ctb_filter_kernel_ms(self._h, back, ctypes.byref(t)), "filter_kernel_ms")
        return t.value

    def probe_smem_bandwidth(self) -> float:
        g = ctypes.c_double()
        self._check(self._lib.ctb_probe_smem_bandwidth(self._h, ctypes.byref(g)), "probe_smem_bandwidth")
        return g.value

    def selftest_bounded_wait(self, limit_us: int) -> int:
        """Run the device timeout path on purpose (ctb_selftest_bounded_wait):
        a wait of at most limit_us microseconds on a barrier nothing completes.
        Returns the raw status, STATUS_TIMEOUT when the wait gave up as it should."""
        return int(self._lib.ctb_selftest_bounded_wait(self._h, int(limit_us)))

    def set_fault_injection(self, slab: int):
        """Test hook: ctb_reconstruct_volume fails after queuing slab `slab` (-1 = off)."""
        self._check(self._lib.ctb_set_fault_injection(self._h, int(slab)), "set_fault_injection")

    def reconstruct_volume_d(self, d_vol: int, n: int, depth: int, na: int, nd: int, kind: int, d_out: int):
        self._check(self._lib.ctb_reconstruct_volume_d(self._h, ctypes.c_void_p(d_vol), n, depth, na, nd,
                                                       int(kind), ctypes.c_void_p(d_out)), "reconstruct_volume_d")

    def _jobs(self, jobs):
        """ctypes array of FbpJob from dicts {sino, depth, num_angles, bins, output_size, filter,
        out[, angles_deg]} (device pointers as ints); keeps angle arrays alive on the array."""
        arr = (FbpJob * len(jobs))()
        keep = []
        for k, j in enumerate(jobs):
            ang = j.get("angles_deg")
            ap = None
            if ang is not None:
                a = _f32(ang)
                keep.append(a)
                ap = a.ctypes.data
            arr[k] = FbpJob(j["sino"], j["depth"], j["num_angles"], j["bins"], ap, j["output_size"],
                            int(j["filter"]), j["out"])
        arr._keep = keep
        return arr

    def fbp(self, sinos, output_size: int, kind: int, angles_deg=None) -> np.ndarray:
        """Plain one-request-per-call FBP on host arrays (ctb_fbp): sinos[depth][na][bins] ->
        [depth][output_size]^2 in normalised units."""
        s = _f32(sinos)
        depth, na, bins = s.shape
        out = np.empty((depth, output_size, output_size), np.float32)
        ang = None if angles_deg is None else _f32(angles_deg)
        self._check(self._lib.ctb_fbp(self._h, s.ctypes.data, depth, na, bins, None if ang is None else ang.ctypes.data,
                                      output_size, int(kind), out.ctypes.data), "fbp")
        return out

    def fbp_host_ptr(self, host_sino: int, depth: int, na: int, bins: int, output_size: int, kind: int,
                     host_out: int):
        """ctb_fbp on raw host pointers (e.g. preallocated buffers)."""
        self._check(self._lib.ctb_fbp(self._h, ctypes.c_void_p(host_sino), depth, na, bins, None, output_size,
                                      int(kind), ctypes.c_void_p(host_out)), "fbp")

    def fbp_batch_d(self, jobs):
        """Filter + backproject many device jobs in one batch (ctb_fbp_batch_d); synchronous."""
        arr = self._jobs(jobs)
        self._check(self._lib.ctb_fbp_batch_d(self._h, arr, len(jobs)), "fbp_batch_d")

    def batch(self, jobs, flags: int = 0) -> "Batch":
        return Batch(self, jobs, flags)

    def phantom_d(self, params: np.ndarray, nx: int, ny: int, nz: int, d_vol: int):
        p = _f32(params).reshape(-1)
        self._check(self._lib.ctb_phantom_sum_d(self._h, p, p.size // 16, nx, ny, nz, ctypes.c_void_p(d_vol)),
                    "phantom_d")


class Batch:
    """A planned batch (ctb_batch_create); run() enqueues it on the backend's stream."""

    def __init__(self, backend: B200Backend, jobs, flags: int = 0):
        self._be = backend
        self._lib = backend._lib
        arr = backend._jobs(jobs)
        h = ctypes.c_void_p()
        backend._check(self._lib.ctb_batch_create(backend.handle, arr, len(jobs), int(flags), ctypes.byref(h)),
                       "batch_create")
        self._h = h

    def run(self):
        self._be._check(self._lib.ctb_batch_run(self._h), "batch_run")

    def info(self):
        """(kernel launches per run, voxel-angle updates, device bytes)."""
        n, u, b = ctypes.c_int(), ctypes.c_double(), ctypes.c_size_t()
        self._be._check(self._lib.ctb_batch_info(self._h, ctypes.byref(n), ctypes.byref(u), ctypes.byref(b)),
                        "batch_info")
        return n.value, u.value, b.value

    def close(self):
        if self._h:
            self._lib.ctb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Server:
    """The serving loop (ctb_server_*): submit FBP requests at any time, they are
    admitted against the device memory budget and run in continuous batches.

    Host requests: ``submit(sino[depth][na][bins], output_size, filter)``; the
    result array is returned by ``result(id)`` once the request is done.
    Device requests: ``submit_device(d_sino, depth, na, bins, output_size,
    filter, d_out)`` with device pointers."""

    def __init__(self, device: int = 0, memory_budget: int = 0, max_batch: int = 0, copy_threads: int = 0,
                 staging_bytes: int = 0, fault_every: int = 0):
        self._lib = library()
        cfg = ServerConfig(device, memory_budget, max_batch, copy_threads, staging_bytes, fault_every)
        h = ctypes.c_void_p()
        st = self._lib.ctb_server_create(ctypes.byref(cfg), ctypes.byref(h))
        if st:
            raise CtbError(st, "ctb_server_create: " + self._lib.ctb_status_string(st).decode())
        self._h = h
        self._keep = {}

    def _submit(self, req: Request, keep) -> int:
        rid = ctypes.c_uint64()
        st = self._lib.ctb_server_submit(self._h, ctypes.byref(req), ctypes.byref(rid))
        if st:
            raise CtbError(st, "ctb_server_submit: " + self._lib.ctb_status_string(st).decode())
        self._keep[rid.value] = keep
        return rid.value

    def submit(self, sino, output_size: int, kind: int, angles_deg=None, out=None) -> int:
        s = _f32(sino)
        depth, na, bins = s.shape
        o = np.empty((depth, output_size, output_size), np.float32) if out is None else out
        ang = None if angles_deg is None else _f32(angles_deg)
        req = Request(s.ctypes.data, depth, na, bins, None if ang is None else ang.ctypes.data, output_size,
                      int(kind), o.ctypes.data, 0)
        return self._submit(req, (s, o, ang))

    def submit_device(self, d_sino: int, depth: int, na: int, bins: int, output_size: int, kind: int,
                      d_out: int, angles_deg=None) -> int:
        ang = None if angles_deg is None else _f32(angles_deg)
        req = Request(d_sino, depth, na, bins, None if ang is None else ang.ctypes.data, output_size, int(kind),
                      d_out, REQ_DEVICE)
        return self._submit(req, (None, None, ang))

    def poll(self, rid: int) -> int:
        return int(self._lib.ctb_server_poll(self._h, rid))

    def wait(self, rid: int, timeout_ms: float = -1.0) -> int:
        return int(self._lib.ctb_server_wait(self._h, rid, float(timeout_ms)))

    def cancel(self, rid: int) -> int:
        return int(self._lib.ctb_server_cancel(self._h, rid))

    def result(self, rid: int, timeout_ms: float = -1.0):
        """Wait for a host request and return its output array (raises on failure)."""
        st = self.wait(rid, timeout_ms)
        if st:
            raise CtbError(st, self._lib.ctb_status_string(st).decode())
        return self._keep[rid][1]

    def release(self, rid: int) -> int:
        st = int(self._lib.ctb_server_release(self._h, rid))
        if st == 0:
            self._keep.pop(rid, None)
        return st

    def stats(self) -> dict:
        s = ServerStats()
        st = self._lib.ctb_server_get_stats(self._h, ctypes.byref(s))
        if st:
            raise CtbError(st, "ctb_server_get_stats")
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ctb_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Arena:
    """The server's admission allocator (ctb_arena_*): host bookkeeping only."""

    def __init__(self, capacity: int):
        self._lib = library()
        h = ctypes.c_void_p()
        st = self._lib.ctb_arena_create(capacity, ctypes.byref(h))
        if st:
            raise CtbError(st, "ctb_arena_create")
        self._h = h

    def alloc(self, nbytes: int):
        """Offset of a new block, or None when nothing fits."""
        off = ctypes.c_size_t()
        st = self._lib.ctb_arena_alloc(self._h, nbytes, ctypes.byref(off))
        return None if st else off.value

    def free(self, offset: int) -> bool:
        return self._lib.ctb_arena_free(self._h, offset) == 0

    def stats(self):
        """(used, peak, largest free range) in bytes."""
        u, p, l = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
        self._lib.ctb_arena_stats(self._h, ctypes.byref(u), ctypes.byref(p), ctypes.byref(l))
        return u.value, p.value, l.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ctb_arena_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# Generator3D::Params defaults (Generator3D.h:16-34): soft tissue, then bone.
GENERATOR3D_TISSUE = np.array(
    [-20.0, 45.0, 3.0, 10.0, 0.0, 0.0, 0.0, 1.0,
     200.0, 1000.0, 2.0, 8.0, 1.0, 0.7, 0.9, 0.15], dtype=np.float32)

__all__ = ["CONVENTION_SERIAL", "CONVENTION_CUDA", "bp_shape_info", "load_sinogram_file", "save_sinogram_file", "FILTER_MODE_FFT", "FILTER_MODE_TC_BF16X3", "B200Backend", "Batch", "Server", "Arena", "ServerConfig", "Request", "ServerStats", "REQ_DEVICE", "FbpJob", "BATCH_GRAPH", "BATCH_PER_JOB", "BATCH_PERSISTENT", "FilterType", "Denorm", "ReconstructionParams", "Sinogram", "CtbError",
           "library", "pad_geometry", "filter_response", "uniform_angles_deg", "odd_detector_count",
           "phantom_params", "GENERATOR3D_TISSUE", "LIB_PATH"]
