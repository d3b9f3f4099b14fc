"""The serving loop (ctb_server_*) on the GPU.

Each request's result must be the same alone and in the mix: every request of
a mixed stream (host and device-resident, uneven sizes, all filters, explicit
angle lists) is compared bit for bit with ctb_fbp_d on the same request alone,
and one request per stream with the oracle within the parity tolerance
(rel-L2 <= 1e-5, max-abs <= 1e-4 * max|f|). Also covered: admission under a
budget that holds only a few requests at once, rejection of a request larger
than the budget, cancellation, host-side fault injection (the other requests
are unaffected), statistics, and shutdown with work still queued.
"""
import numpy as np
import pytest

import oracle as O
import qtctreconstruction_b200 as ctb
from qtctreconstruction_b200 import FilterType

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]

REL_L2 = 1e-5
MAX_ABS = 1e-4
OK, OOM, CANCELLED, CUDA_ERR, NOT_FOUND, BUSY = 0, 3, 7, 2, 8, 9

SHAPES = [(64, 16, 101, FilterType.Ramp), (96, 5, 151, FilterType.SheppLogan), (128, 9, 201, FilterType.Hann),
          (33, 3, 52, FilterType.Ramp), (160, 4, 251, FilterType.Hamming), (64, 1, 17, FilterType.Bartlett),
          (200, 6, 314, FilterType.Cosine), (96, 7, 150, FilterType.Hann)]


def _requests(shapes, seed, explicit_every=3):
    rng = np.random.default_rng(seed)
    out = []
    for k, (n, depth, na, kind) in enumerate(shapes):
        nd = ctb.odd_detector_count(n)
        sino = rng.standard_normal((depth, na, nd)).astype(np.float32)
        ang = np.sort(rng.uniform(0, 180, na)).astype(np.float32) if k % explicit_every == 1 else None
        out.append(dict(sino=sino, n=n, kind=kind, angles=ang))
    return out


def _alone(backend, torch, rq):
    depth, na, nd = rq["sino"].shape
    d_sino = torch.from_numpy(rq["sino"]).cuda()
    out = torch.zeros((depth, rq["n"], rq["n"]), dtype=torch.float32, device="cuda")
    backend.fbp_d(d_sino.data_ptr(), depth, na, nd, rq["n"], int(rq["kind"]), out.data_ptr(),
                  angles_deg=rq["angles"])
    backend.synchronize()
    return out.cpu().numpy()


def test_mixed_stream_equals_alone(backend):
    import torch
    reqs = _requests(SHAPES * 2, 21)
    with ctb.Server(0, memory_budget=2 << 30, copy_threads=2) as srv:
        ids = [srv.submit(r["sino"], r["n"], r["kind"], angles_deg=r["angles"]) for r in reqs]
        outs = [srv.result(i) for i in ids]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["batches"] >= 1 and 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["volumes_per_s"] > 0 and st["memory_peak"] <= st["memory_budget"]
    for r, o in zip(reqs, outs):
        assert np.all(np.isfinite(o))
        np.testing.assert_array_equal(o, _alone(backend, torch, r))
    r, o = reqs[2], outs[2]
    for z in range(r["sino"].shape[0]):
        ref = O.reconstruct_slice_f32(r["sino"][z], r["angles"] if r["angles"] is not None
                                      else O.uniform_angles_deg(r["sino"].shape[1]), r["n"], int(r["kind"]))
        assert O.rel_l2(o[z], ref) <= REL_L2
        assert O.max_abs_rel(o[z], ref) <= MAX_ABS


def test_device_resident_requests(backend):
    import torch
    reqs = _requests(SHAPES[:5], 22)
    with ctb.Server(0, memory_budget=1 << 30) as srv:
        bufs, ids = [], []
        for r in reqs:
            depth, na, nd = r["sino"].shape
            d_s = torch.from_numpy(r["sino"]).cuda()
            d_o = torch.full((depth, r["n"], r["n"]), float("nan"), dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            bufs.append((d_s, d_o))
            ids.append(srv.submit_device(d_s.data_ptr(), depth, na, nd, r["n"], r["kind"], d_o.data_ptr(),
                                         angles_deg=r["angles"]))
        assert [srv.wait(i) for i in ids] == [OK] * len(ids)
    for r, (_, d_o) in zip(reqs, bufs):
        np.testing.assert_array_equal(d_o.cpu().numpy(), _alone(backend, torch, r))


def test_small_budget_admission_and_rejection(backend):
    import torch
    reqs = _requests([(128, 12, 201, FilterType.Ramp)] * 6, 23)
    one = 4 * 12 * (201 * ctb.odd_detector_count(128) + 128 * 128)  # sinograms + volume
    budget = 6 * one  # the filtered rows take about as much again: a few requests at a time
    with ctb.Server(0, memory_budget=budget, copy_threads=2) as srv:
        ids = [srv.submit(r["sino"], r["n"], r["kind"], angles_deg=r["angles"]) for r in reqs]
        outs = [srv.result(i) for i in ids]
        big = np.zeros((64, 400, ctb.odd_detector_count(256)), np.float32)
        with pytest.raises(ctb.CtbError) as e:
            srv.submit(big, 256, FilterType.Ramp)
        assert e.value.status == OOM
        st = srv.stats()
    assert st["rejected"] == 1 and st["completed"] == len(reqs)
    assert st["memory_peak"] <= budget
    for r, o in zip(reqs, outs):
        np.testing.assert_array_equal(o, _alone(backend, torch, r))


def test_cancel_and_release():
    reqs = _requests([(160, 16, 251, FilterType.Hann)] * 10, 24)
    # about 10.6 MB per request: one request at a time, the later ones still queued
    with ctb.Server(0, memory_budget=16 << 20, copy_threads=1) as srv:
        ids = [srv.submit(r["sino"], r["n"], r["kind"]) for r in reqs]
        for i in ids[5:]:
            assert srv.cancel(i) == OK
        status = [srv.wait(i) for i in ids]
        assert all(s in (OK, CANCELLED) for s in status)
        assert status.count(CANCELLED) >= 1
        assert srv.poll(10 ** 9) == NOT_FOUND
        assert srv.release(ids[0]) == OK and srv.poll(ids[0]) == NOT_FOUND
        st = srv.stats()
        assert st["completed"] + st["cancelled"] == len(reqs)


def test_fault_injection_isolated(backend):
    import torch
    reqs = _requests(SHAPES[:6], 25)
    with ctb.Server(0, memory_budget=1 << 30, fault_every=3) as srv:
        ids = [srv.submit(r["sino"], r["n"], r["kind"], angles_deg=r["angles"]) for r in reqs]
        status = [srv.wait(i) for i in ids]
        st = srv.stats()
        assert status == [OK, OK, CUDA_ERR, OK, OK, CUDA_ERR]
        assert st["failed"] == 2 and st["completed"] == 4
        for k, i in enumerate(ids):
            if status[k] == OK:
                np.testing.assert_array_equal(srv.result(i), _alone(backend, torch, reqs[k]))


def test_shutdown_with_queued_work():
    reqs = _requests([(192, 32, 301, FilterType.Ramp)] * 8, 26)
    srv = ctb.Server(0, memory_budget=512 << 20, copy_threads=1)
    ids = [srv.submit(r["sino"], r["n"], r["kind"]) for r in reqs]
    assert srv.wait(ids[0]) == OK
    srv.close()  # cancels what is still queued and returns


def test_concurrent_submitters(backend):
    """Requests submitted from several host threads at once all complete and
    each equals the request alone."""
    import threading

    import torch
    reqs = _requests(SHAPES * 2, 27)
    with ctb.Server(0, memory_budget=1 << 30, copy_threads=3) as srv:
        ids = [None] * len(reqs)

        def submit(k0):
            for k in range(k0, len(reqs), 4):
                r = reqs[k]
                ids[k] = srv.submit(r["sino"], r["n"], r["kind"], angles_deg=r["angles"])
        th = [threading.Thread(target=submit, args=(k,)) for k in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        outs = [srv.result(i) for i in ids]
    for r, o in zip(reqs, outs):
        np.testing.assert_array_equal(o, _alone(backend, torch, r))


def test_page_locked_host_requests_copy_directly(backend):
    """Requests in page-locked host memory are copied by the copy engines
    straight from and into the caller's buffers (no staging); results are
    the same as from pageable buffers and as the request alone."""
    import torch
    reqs = _requests(SHAPES, 23)
    with ctb.Server(0, memory_budget=2 << 30, copy_threads=2, staging_bytes=1 << 20) as srv:
        pinned, ids = [], []
        for r in reqs:
            depth, na, nd = r["sino"].shape
            hs = torch.from_numpy(r["sino"]).pin_memory()
            ho = torch.full((depth, r["n"], r["n"]), float("nan"), dtype=torch.float32).pin_memory()
            pinned.append((hs, ho))
            ids.append(srv.submit(hs.numpy(), r["n"], r["kind"], angles_deg=r["angles"], out=ho.numpy()))
        assert all(srv.wait(i) == OK for i in ids)
    for r, (_, ho) in zip(reqs, pinned):
        np.testing.assert_array_equal(ho.numpy(), _alone(backend, torch, r))


@pytest.mark.parametrize("depth", [3, 16, 17, 90, 200])
@pytest.mark.parametrize("pinned", [False, True])
def test_plain_fbp_pipeline_equals_device_path(backend, depth, pinned):
    """ctb_fbp streams the stack in slabs with copies on their own streams;
    the result equals ctb_fbp_d on the whole stack bit for bit, from pageable
    and from page-locked buffers, for one slab and for several (200 slices
    make 7 slabs)."""
    import torch
    rng = np.random.default_rng(depth)
    n, na = 72, 96
    nd = ctb.odd_detector_count(n)
    sino = rng.standard_normal((depth, na, nd)).astype(np.float32)
    ang = np.sort(rng.uniform(0, 180, na)).astype(np.float32) if depth % 2 else None
    ref = _alone(backend, torch, dict(sino=sino, n=n, kind=FilterType.SheppLogan, angles=ang))
    if pinned:
        hs = torch.from_numpy(sino).pin_memory()
        ho = torch.full((depth, n, n), float("nan"), dtype=torch.float32).pin_memory()
        backend._check(backend._lib.ctb_fbp(backend.handle, hs.data_ptr(), depth, na, nd,
                                            None if ang is None else ang.ctypes.data, n,
                                            int(FilterType.SheppLogan), ho.data_ptr()), "fbp")
        got = ho.numpy()
    else:
        got = backend.fbp(sino, n, FilterType.SheppLogan, angles_deg=ang)
    np.testing.assert_array_equal(got, ref)
    assert backend.lastReconstructionTimeMs() > 0.0
