"""The headless C++ CLI (qtctreconstruction_b200/bin/ctbench) on the GPU, and
the consumer path from a sinogram file.

`ctbench sinofile` reads sinograms + .meta.json (the reference's export
format), reconstructs them with reconstructVolumeFromSinograms semantics
(output size = bins, normalised units) and writes a volume NPY; the result
must equal the library called directly from Python on the same data, bit for
bit, and the oracle within the parity tolerance. `volume` and `serve` must run
and report sane figures.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle as O
import qtctreconstruction_b200 as ctb
from qtctreconstruction_b200 import FilterType, ReconstructionParams

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "qtctreconstruction_b200", "bin", "ctbench")


def _run(*args):
    r = subprocess.run([CLI, *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_cli_sinofile_matches_library_and_oracle(backend, tmp_path):
    rng = np.random.default_rng(4)
    n, depth, na = 96, 3, 120
    bins = ctb.odd_detector_count(n)
    ang = np.sort(rng.uniform(0, 180, na)).astype(np.float32)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    sl = []
    for _ in range(depth):
        s = np.zeros((n, n), np.float32)
        for _ in range(4):
            cx, cy = rng.uniform(0.3 * n, 0.7 * n, 2)
            a, b = rng.uniform(0.05 * n, 0.2 * n, 2)
            s[((xx - cx) / a) ** 2 + ((yy - cy) / b) ** 2 <= 1.0] += np.float32(rng.uniform(0.1, 1.0))
        sl.append(s)
    sinos = np.stack([O.sinogram_f64(s, na, bins, ang)[0].astype(np.float32) for s in sl])
    src = str(tmp_path / "scan.npy")
    ctb.save_sinogram_file(src, sinos, ang, spacing_mm=1.0)
    dst = str(tmp_path / "recon.npy")
    info = _run("sinofile", src, dst, "--filter", str(int(FilterType.SheppLogan)))
    assert (info["depth"], info["num_angles"], info["bins"]) == (depth, na, bins)
    got = np.load(dst)
    ref = backend.reconstructVolumeFromSinograms(sinos, ang, ReconstructionParams(FilterType.SheppLogan, na))
    np.testing.assert_array_equal(got, ref)
    for z in range(depth):
        ser = O.reconstruct_slice_f32(sinos[z], ang, bins, int(FilterType.SheppLogan))
        assert O.rel_l2(got[z], ser) <= 1e-5 and O.max_abs_rel(got[z], ser) <= 1e-4


def test_cli_volume_and_serve():
    v = _run("volume", "--n", "128", "--slices", "16", "--angles", "180", "--steps", "2", "--warmup", "1")
    assert v["value"] > 0 and v["ms_per_step"] > 0 and len(v["stage_ms"]) == 4
    t = _run("volume", "--n", "128", "--slices", "8", "--angles", "180", "--steps", "1", "--warmup", "1",
             "--filter-mode", "tc")
    assert t["filter_mode"] == "tc_bf16x3" and t["value"] > 0
    s = _run("serve", "--requests", "6", "--budget-gb", "4", "--copy-threads", "2")
    assert s["mode"] == "served" and s["volumes_per_s"] > 0 and s["p50_ms"] <= s["p99_ms"]
    p = _run("serve", "--requests", "4", "--plain")
    assert p["mode"] == "plain" and p["volumes_per_s"] > 0
