"""Backprojection tile shapes and the autotuner on the GPU.

Every compiled shape must meet the parity bar against the oracle on sizes
that are and are not multiples of its tile edges; the shapes that differ
only in angle-chunk size give identical bits; the automatic choice is a
function of the job alone; the autotuner times the shapes on the first job of
a size bucket, remembers the fastest, and its table can be exported and
loaded; results stay within the parity tolerance whichever shape runs.
"""
import numpy as np
import pytest

import oracle as O
import qtctreconstruction_b200 as ctb
from qtctreconstruction_b200 import FilterType

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5
MAX_ABS = 1e-4


def _job(rng, n, depth, na):
    nd = ctb.odd_detector_count(n)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    sl = []
    for _ in range(depth):
        s = np.zeros((n, n), np.float32)
        for _ in range(4):
            cx, cy = rng.uniform(0.3 * n, 0.7 * n, 2)
            a, b = rng.uniform(0.05 * n, 0.2 * n, 2)
            s[((xx - cx) / a) ** 2 + ((yy - cy) / b) ** 2 <= 1.0] += np.float32(rng.uniform(0.1, 1.0))
        sl.append(s)
    return np.stack([O.sinogram_f64(s, na, nd, O.uniform_angles_deg(na))[0].astype(np.float32) for s in sl])


def _fbp(backend, torch, sinos, n, kind):
    depth, na, nd = sinos.shape
    d_s = torch.from_numpy(sinos).cuda()
    d_o = torch.full((depth, n, n), float("nan"), dtype=torch.float32, device="cuda")
    backend.fbp_d(d_s.data_ptr(), depth, na, nd, n, int(kind), d_o.data_ptr())
    backend.synchronize()
    return d_o.cpu().numpy()


def test_shape_info():
    assert [ctb.bp_shape_info(v) for v in range(6)] == [(32, 32, 4, 32), (64, 32, 8, 32), (32, 16, 2, 32),
                                                        (16, 16, 1, 32), (32, 32, 4, 16), (32, 32, 4, 64)]
    with pytest.raises(ctb.CtbError):
        ctb.bp_shape_info(6)


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("n,depth,na", [(64, 5, 90), (97, 3, 120), (200, 6, 150)])
def test_every_shape_meets_parity(backend, variant, n, depth, na):
    import torch
    rng = np.random.default_rng(n * 7 + variant)
    sinos = _job(rng, n, depth, na)
    backend.set_bp_shape(variant)
    try:
        got = _fbp(backend, torch, sinos, n, FilterType.Hann)
    finally:
        backend.set_bp_shape(-1)
    assert np.all(np.isfinite(got))
    ang = O.uniform_angles_deg(na)
    for z in range(depth):
        ref = O.reconstruct_slice_f32(sinos[z], ang, n, int(FilterType.Hann))
        assert O.rel_l2(got[z], ref) <= REL_L2
        assert O.max_abs_rel(got[z], ref) <= MAX_ABS


@pytest.mark.parametrize("na", [17, 90, 150, 301])
def test_angle_chunk_size_does_not_change_bits(backend, na):
    """Shapes 4 and 5 are shape 0 with 16- and 64-angle chunks: every voxel
    sums its angles in the same order, so the outputs are identical, also
    when the angle count is not a multiple of the chunk."""
    import torch
    rng = np.random.default_rng(na)
    sinos = _job(rng, 96, 5, na)
    outs = []
    for v in (0, 4, 5):
        backend.set_bp_shape(v)
        try:
            outs.append(_fbp(backend, torch, sinos, 96, FilterType.SheppLogan))
        finally:
            backend.set_bp_shape(-1)
    np.testing.assert_array_equal(outs[1], outs[0])
    np.testing.assert_array_equal(outs[2], outs[0])


def test_default_shape_depends_on_size_only(backend):
    assert backend.bp_shape_for(512, 512, 720) == 0
    assert backend.bp_shape_for(128, 64, 201) == 0
    assert backend.bp_shape_for(64, 16, 101) == 3
    assert backend.bp_shape_for(128, 16, 201) == 2  # 16 tiles x 4 slice groups: over a quarter of the SMs


def test_autotune_table_round_trip(backend):
    import torch
    rng = np.random.default_rng(3)
    sinos = _job(rng, 160, 8, 200)
    backend.set_autotune(True)
    try:
        got = _fbp(backend, torch, sinos, 160, FilterType.Ramp)
        table = backend.autotune_table()
        assert len(table) >= 1 and all(0 <= e[3] < 4 for e in table)
        tuned = backend.bp_shape_for(160, 8, 200)
        assert (160 + 63) // 64 in [e[0] for e in table]
        again = _fbp(backend, torch, sinos, 160, FilterType.Ramp)  # no re-tuning: same shape, same bits
        np.testing.assert_array_equal(got, again)
        backend.autotune_load([(1, 1, 0, 3)])
        assert (1, 1, 0, 3) in backend.autotune_table()
    finally:
        backend.set_autotune(False)
    ang = O.uniform_angles_deg(200)
    for z in range(8):
        ref = O.reconstruct_slice_f32(sinos[z], ang, 160, int(FilterType.Ramp))
        assert O.rel_l2(got[z], ref) <= REL_L2
    assert tuned in range(6)
