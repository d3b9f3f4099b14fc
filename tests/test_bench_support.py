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
