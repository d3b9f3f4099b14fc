"""The C ABI boundary: libctb200.so loads, exports every symbol declared in
include/ctb200.h, and its host-side logic behaves without a GPU (CPU only)."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O
import qtctreconstruction_b200 as ctb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if name.endswith(".h"):
            text = open(os.path.join(ROOT, "include", name)).read()
            syms |= set(re.findall(r"\b(ctb_[a-z0-9_]+)\s*\(", text))
    return sorted(syms)


def test_library_exports_every_declared_symbol():
    lib = ctb.library()
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_library_is_built_for_sm100a():
    # the shared object embeds an sm_100a cubin: the arch string is in its ELF notes
    data = open(ctb.LIB_PATH, "rb").read()
    assert b"sm_100a" in data


def test_pad_geometry_matches_reference_formula():
    for bins in (11, 23, 91, 183, 725, 1087, 1449):
        assert ctb.pad_geometry(bins) == O.pad_geometry(bins)


@pytest.mark.parametrize("kind", range(6))
def test_filter_response_is_fp64_accurate(kind):
    for L in (64, 1024, 4096):
        H = ctb.filter_response(L, kind)
        H64 = O.filter_f64(L, kind)
        assert np.max(np.abs(H - H64)) <= 2e-7 * max(1.0, np.max(np.abs(H64)))
        # and within the float reference's own rounding of the same filter
        assert O.rel_l2(H, O.filter_f32(L, kind)) < 1e-6


def test_status_strings():
    lib = ctb.library()
    for s in range(10):
        assert lib.ctb_status_string(s)


def test_invalid_arguments_rejected_without_gpu():
    lib = ctb.library()
    assert lib.ctb_pad_geometry(0, None, None, None) == 1
    assert lib.ctb_filter_response(100, 0, np.zeros(51, np.float32)) == 1  # not a power of two
    assert lib.ctb_create(None, 0) == 1


def test_phantom_params_deterministic_and_in_range():
    a = ctb.phantom_params(7, 32)
    b = ctb.phantom_params(7, 32)
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, ctb.phantom_params(8, 32))
    c = a[:, 0:3]
    assert np.all(np.abs(c) <= 0.6)
    axes = 1.0 / np.sqrt(a[:, 12:15])
    assert np.all(axes >= 0.05 - 1e-6) and np.all(axes <= 0.4 + 1e-6)
    assert np.all(a[:, 15] >= -0.3) and np.all(a[:, 15] <= 1.0)
    for r in a[:, 3:12].reshape(-1, 3, 3):
        np.testing.assert_allclose(r @ r.T, np.eye(3), atol=1e-6)


def test_create_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = ctb.library()
    h = ctypes.c_void_p()
    assert lib.ctb_create(ctypes.byref(h), 0) == 5  # CTB_ERR_NO_DEVICE
    with pytest.raises(ctb.CtbError):
        ctb.B200Backend(0)


def test_cli_built_and_prints_usage():
    """The headless C++ CLI (qtctreconstruction_b200/bin/ctbench) links against the library."""
    import subprocess
    cli = os.path.join(ROOT, "qtctreconstruction_b200", "bin", "ctbench")
    assert os.path.exists(cli)
    r = subprocess.run([cli], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr
