"""Host logic of bench.py's forward-projector accounting (CPU).

`image_support` counts the pixels the forward projector must read: the
non-zero normalised pixels (raw != 0 and raw != the slice minimum; the others
contribute exact zeros) and the pixels of the per-8-slice-group bounding
boxes of those. The forward roofline's algorithmic bytes are built on the
first count, so it is checked here against a direct count.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def _direct(vol):
    nz = vol.shape[0]
    nnz, walked = 0, 0
    for g in range(0, nz, 8):
        masks = []
        for z in range(g, min(g + 8, nz)):
            lo = vol[z].min()
            m = (vol[z] != 0) & (vol[z] != lo)
            nnz += int(m.sum())
            masks.append(m)
        u = np.any(masks, axis=0)
        ys, xs = np.nonzero(u)
        if ys.size:
            walked += (ys.max() - ys.min() + 1) * (xs.max() - xs.min() + 1) * len(masks)
    return nnz, walked


def test_image_support_small_cases():
    v = np.zeros((10, 6, 6), np.float32)
    v[1, 2:4, 1:3] = 1.0           # 4 pixels, box 2 x 2 in group 0 (8 slices)
    v[9, 0, 5] = -1.0              # the slice minimum: normalises to zero
    v[9, 1, 1] = 2.0               # 1 pixel, box 1 x 1 in group 1 (2 slices)
    assert bench.image_support(v) == (5, 4 * 8 + 1 * 2)
    assert bench.image_support(np.zeros((3, 5, 5), np.float32)) == (0, 0)


def test_image_support_random_against_direct_count():
    rng = np.random.default_rng(2)
    v = np.zeros((21, 40, 33), np.float32)
    for z in range(21):
        if z % 5 == 3:
            continue  # empty slices
        y0, x0 = rng.integers(0, 30), rng.integers(0, 25)
        v[z, y0:y0 + 8, x0:x0 + 6] = rng.uniform(-1, 1, (8, 6)).astype(np.float32)
        if z % 4 == 0:
            v[z] = np.where(v[z] == 0, v[z].min(), v[z])  # background at the minimum
    assert bench.image_support(v) == _direct(v)


def test_oracle_phantom_params_equal_library_bit_for_bit():
    """The timed CPU baseline draws the benchmark phantom from the oracle's
    restatement of the seeded parameter draw, so that it never loads the
    product library; both must give the same records bit for bit."""
    import oracle as O
    import qtctreconstruction_b200 as ctb
    for seed, count in [(1, 10), (2, 32), (3, 64), (4, 24), (5, 1), (2**40 + 17, 9), (7, 0)]:
        a = O.phantom_params(seed, count)
        b = ctb.phantom_params(seed, count)
        assert a.shape == b.shape == (count, 16)
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))


def test_reference_arm_loads_no_product_library():
    """bench.py --impl reference runs the reference's CPU path only: after it,
    no shared object of the product package is mapped into the process."""
    import subprocess
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--config', 'small', "
            "'--steps', '1', '--warmup', '0', '--ref-slices', '1']; "
            "import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "assert 'libctb200' not in maps, 'product library loaded'; "
            "assert 'qtctreconstruction_b200' not in sys.modules, 'product package imported'")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
    import json
    d = json.loads(line)
    assert d["impl"] == "reference" and d["value"] > 0


def test_accuracy_slices_straddle_the_host_schedule_ends():
    """The bench's FP64 check covers both sides of the first and last slab
    boundaries of the 512-slice host schedule (8, 24, 7 x 64, 24, 8)."""
    zs = bench.accuracy_slices(512, 512)
    for b in (8, 32, 96, 480, 504):
        assert b - 1 in zs and b in zs, b
    assert 0 in zs and 511 in zs and 255 in zs and 256 in zs
    assert zs == sorted(set(zs)) and all(0 <= z < 512 for z in zs)
