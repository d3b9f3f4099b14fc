"""The reference-side C++ binding (CPU).

ct::B200Backend (qtctreconstruction_b200/binding) is the class a maintainer
adds to QtCTReconstruction. Here it is compiled against the reference's own
IReconstructionBackend.h and CTTypes.h (IReconstructionBackend.h:10-55), with
warnings as errors for the binding's own code, so a drift between include/ctb200.h,
the binding and the reference interface fails the build; then linked and
loaded, and driven on this machine without a GPU, where the interface's
contract is isAvailable() == false and empty results (SerialBackend.cpp:64,148).
Skipped only when the reference tree is absent.
"""
import numpy as np
import pytest

import binding_lib as B  # noqa: E402  (tests/ is on sys.path under pytest)


@pytest.fixture(scope="module")
def ref():
    d = B.reference_dir()
    if d is None:
        pytest.skip("reference source tree not present (set QTCT_REFERENCE_DIR)")
    return d


def test_binding_compiles_against_reference_interface(ref):
    r = B.make("check")
    assert r.returncode == 0, r.stdout + r.stderr


def test_binding_links_and_reports_unavailable_without_gpu(ref):
    import torch
    r = B.make("all")
    assert r.returncode == 0, r.stdout + r.stderr
    L = B.load()
    assert L is not None
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU test covers the available backend")
    h = L.b200be_create(0)
    assert h
    try:
        assert L.b200be_is_available(h) == 0
        import ctypes
        buf = ctypes.create_string_buffer(64)
        assert L.b200be_name(h, buf, 64) > 0 and buf.value.startswith(b"B200")
        sl = np.ones((8, 8), np.float32)
        sino = np.zeros((4, 13), np.float32)
        ang, mm = np.zeros(4, np.float32), np.zeros(2, np.float32)
        assert L.b200be_compute_sinogram(h, sl, 8, 8, 4, 13, sino, ang, mm) == 1  # empty Sinogram
        out = np.zeros((8, 8), np.float32)
        assert L.b200be_reconstruct_slice(h, sino, 4, 13, None, 8, 0, 0.0, 0.0, out) == 1
        assert L.b200be_last_sinogram_ms(h) == 0.0
    finally:
        L.b200be_destroy(h)
