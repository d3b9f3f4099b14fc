"""ctypes access to the reference-side C++ binding (qtctreconstruction_b200/
binding: ct::B200Backend behind ct::IReconstructionBackend) through its C
entry b200backend_capi.cpp. The library is built by the binding's Makefile
against the reference's own interface headers; `build()` runs that recipe,
`load()` opens the result (None when it was never built)."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINDING = os.path.join(ROOT, "qtctreconstruction_b200", "binding")
LIB = os.path.join(BINDING, "_build", "libb200backend.so")
_F32P = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def reference_dir():
    """The reference source directory: $QTCT_REFERENCE_DIR, else a checkout
    named `reference` beside the repository root (the Makefile's default)."""
    d = os.environ.get("QTCT_REFERENCE_DIR") or os.path.join(os.path.dirname(ROOT), "reference",
                                                              "QtCTReconstruction")
    return d if os.path.exists(os.path.join(d, "IReconstructionBackend.h")) else None


def make(target: str = "all"):
    ref = reference_dir()
    return subprocess.run(["make", "-s", "-C", BINDING, target, f"REF={ref}"], capture_output=True, text=True)


def load():
    if not os.path.exists(LIB):
        return None
    L = ctypes.CDLL(LIB)
    i, f, p, d = ctypes.c_int, ctypes.c_float, ctypes.c_void_p, ctypes.c_double
    L.b200be_create.argtypes = [i]
    L.b200be_create.restype = p
    L.b200be_destroy.argtypes = [p]
    L.b200be_destroy.restype = None
    L.b200be_is_available.argtypes = [p]
    L.b200be_name.argtypes = [p, ctypes.c_char_p, i]
    L.b200be_last_status.argtypes = [p]
    L.b200be_compute_sinogram.argtypes = [p, _F32P, i, i, i, i, _F32P, _F32P, _F32P]
    L.b200be_reconstruct_slice.argtypes = [p, _F32P, i, i, p, i, i, f, f, _F32P]
    L.b200be_reconstruct_volume.argtypes = [p, _F32P, i, i, i, i, _F32P, p]
    L.b200be_reconstruct_from_sinograms.argtypes = [p, _F32P, i, i, i, _F32P, i, _F32P]
    L.b200be_extract_point_cloud.argtypes = [p, _F32P, i, i, i, f, p, ctypes.c_longlong]
    L.b200be_extract_point_cloud.restype = ctypes.c_longlong
    L.b200be_last_sinogram_ms.argtypes = [p]
    L.b200be_last_sinogram_ms.restype = d
    L.b200be_last_reconstruction_ms.argtypes = [p]
    L.b200be_last_reconstruction_ms.restype = d
    return L
