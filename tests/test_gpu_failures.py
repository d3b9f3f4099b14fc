"""Failure paths on the GPU, made without a GPU fault (GPU).

* The device timeout path: every device-side wait of the kernels is bounded
  and a wait that gives up turns into CTB_ERR_TIMEOUT on the host (the
  reference prints or throws on device errors, CUDABackend.cu:37-43,
  HybridBackend.cu:44-65). ctb_selftest_bounded_wait makes one CTA wait on a
  barrier nothing completes, with no copy in flight, and a short time limit;
  the call must report the timeout, and the context must stay usable: a parity
  case passes right after it.
* A volume pipeline that fails half way (host-side fault injection after
  queuing a slab, earlier slabs' copies and kernels still in flight) must not
  return before all its queued work has finished: the slabs before the failure
  are complete in the caller's output buffer, nothing writes into that buffer
  after the call returned, and the next call on the context succeeds.
"""
import time

import numpy as np
import pytest

import oracle as O
import qtctreconstruction_b200 as ctb
from qtctreconstruction_b200 import FilterType, ReconstructionParams

pytestmark = pytest.mark.gpu


def _parity_case(backend):
    n, nz, na = 48, 3, 64
    nd = ctb.odd_detector_count(n)
    vol = backend.phantom(ctb.phantom_params(9, 6), n, n, nz)
    out = backend.reconstructVolume(vol, ReconstructionParams(FilterType.Ramp, na), detector_bins=nd)
    ref = O.reconstruct_volume_f32(vol, na, nd, O.RAMP)
    assert O.rel_l2(out, ref) <= 1e-5
    assert O.max_abs_rel(out, ref) <= 1e-4


def test_bounded_wait_times_out_and_context_survives(backend):
    _parity_case(backend)
    for limit_us in (1, 100, 20000):
        t0 = time.perf_counter()
        assert backend.selftest_bounded_wait(limit_us) == ctb.STATUS_TIMEOUT
        assert time.perf_counter() - t0 < 5.0
        assert "bounded device wait" in backend._lib.ctb_last_error(backend.handle).decode()
        backend.synchronize()  # the error word was cleared: nothing stale is reported
        _parity_case(backend)


def test_volume_pipeline_failure_returns_after_queued_work(backend):
    import torch
    n, nz, na = 192, 200, 96
    nd = ctb.odd_detector_count(n)
    vol = backend.phantom(ctb.phantom_params(21, 10), n, n, nz)
    hin = torch.from_numpy(vol).pin_memory()
    ref = torch.empty_like(hin).pin_memory()
    backend.reconstruct_volume_host(hin.data_ptr(), n, nz, na, nd, int(FilterType.SheppLogan), ref.data_ptr())
    ref = ref.numpy().copy()
    out = torch.full_like(hin, float("nan")).pin_memory()
    backend.set_fault_injection(3)
    try:
        with pytest.raises(ctb.CtbError) as ei:
            backend.reconstruct_volume_host(hin.data_ptr(), n, nz, na, nd, int(FilterType.SheppLogan),
                                            out.data_ptr())
        assert ei.value.status == ctb.STATUS_CUDA and "injected fault" in str(ei.value)
    finally:
        backend.set_fault_injection(-1)
    got = out.numpy()
    # slabs finished before the failure are in the output; copy the whole
    # buffer now, then plant a sentinel and check that no late copy overwrites it
    done = [z for z in range(nz) if np.isfinite(got[z]).all()]
    assert len(done) >= 8, "earlier slabs must have been copied out before the call returned"
    np.testing.assert_array_equal(got[done], ref[done])
    got[:] = 7.0
    time.sleep(0.2)
    assert (got == 7.0).all(), "the failed call left copies writing into the caller's buffer"
    # the context still works
    again = torch.empty_like(hin).pin_memory()
    backend.reconstruct_volume_host(hin.data_ptr(), n, nz, na, nd, int(FilterType.SheppLogan), again.data_ptr())
    np.testing.assert_array_equal(again.numpy(), ref)
