"""The forward projector's reads stay inside the image planes (CPU).

`k_forward` (csrc/forward_proj.cu) reads, at each walked row, the 32 pixels
of a window that starts at the crossing of its strip's lower bin edge, with
no clamp: the planes carry a zero border of kFwdGuard = 64 columns on each
side and kFwdRows = 16 rows below the image, and the row ranges it walks are
meant to keep every window within 50 columns of the image. This test replays
that index arithmetic on the host for many geometries, angles and non-zero
boxes (including the whole image, i.e. the bounds turned off) and checks every
column and row a lane can read:

* the per-strip set-up in FP64 (crossing q0, slopes, the row range where the
  strip comes within 2 columns of the box, narrowed by the disc test);
* chunks of 16 rows starting at multiples of 16 from the range's first row;
* per row the float32 crossing fq + pp * dqf, rounded by the 1.5 * 2^23
  addition as on the device, and lanes at columns cb + S * l, l < 32.

The half-chunk band skip only removes reads, so every row of every chunk is
checked.
"""
import math

import numpy as np
import pytest

GUARD = 64
ROWS = 16
LANES = 32
KREACH = 2.0
F32 = np.float32


def strip_bins(akq):
    return int(math.floor(31.5 * akq)) - 1


def prange(qa, qb, dq, idq, cl, ch, rl, rh):
    lo, hi = rl, rh
    if dq != 0.0:
        p = [(cl - KREACH - qa) * idq, (ch + KREACH - qa) * idq, (cl - KREACH - qb) * idq, (ch + KREACH - qb) * idq]
        lo = max(rl, int(math.floor(min(p))) - 1)
        hi = min(rh, int(math.ceil(max(p))) + 1)
    elif max(qa, qb) < cl - KREACH or min(qa, qb) > ch + KREACH:
        hi = -1
    return lo, hi


def windows(w, h, nd, deg, box, r4):
    """Yield (row, first column, last column, nq, np) of every window read."""
    t = deg / 180.0
    c, s = math.cos(math.pi * t), math.sin(math.pi * t)
    rows = abs(c) >= abs(s)
    kq, kp = (c, s) if rows else (s, c)
    akq = max(abs(kq), 0.7071)
    K = max(1, strip_bins(akq))
    np_, nq = (h, w) if rows else (w, h)
    cq = 0.5 * (nq - 1)
    cp = 0.5 * (np_ - 1)
    dcf = float(nd // 2)
    bx0, bx1, by0, by1 = box
    rl, rh = (by0, by1) if rows else (bx0, bx1)
    cl, ch = (bx0, bx1) if rows else (by0, by1)
    inv = 1.0 / kq
    dq = -kp * inv
    idq = 1.0 / dq if dq != 0.0 else 0.0
    dqf = F32(dq)
    neg = kq < 0.0
    for k in range((nd + K - 1) // K):
        b_lo = k * K - 1
        q0 = cq + (b_lo - dcf + cp * kp) * inv
        p_lo, p_hi = prange(q0, q0 + (K + 1) * inv, dq, idq, cl, ch, rl, rh)
        rad = 0.5 * math.sqrt(float(r4)) + 1.5
        u0 = b_lo - dcf
        u1 = u0 + K + 1
        a0, a1 = max(min(u0, u1), -rad), min(max(u0, u1), rad)
        if a0 > a1:
            continue
        m = 0.0 if (a0 <= 0.0 <= a1) else min(abs(a0), abs(a1))
        vm = math.sqrt(max(0.0, rad * rad - m * m))
        e0, e1, ev = a0 * kp, a1 * kp, vm * abs(kq)
        p_lo = max(p_lo, int(math.floor(cp + min(e0, e1) - ev)) - 2)
        p_hi = min(p_hi, int(math.ceil(cp + max(e0, e1) + ev)) + 2)
        p0 = p_lo & ~(ROWS - 1) if p_lo >= 0 else p_lo
        while p0 <= p_hi:
            qs = p0 * dq + q0
            base = math.floor(qs)
            fq = F32(qs - base)
            pp = np.arange(ROWS, dtype=F32)
            A = (pp * dqf + fq).astype(F32)
            tr = (A + F32(12582912.0)).astype(F32)
            cb = base + (tr - F32(12582912.0)).astype(np.int64)
            first = cb - (LANES - 1 if neg else 0)
            last = cb + (0 if neg else LANES - 1)
            yield p0, int(first.min()), int(last.max()), nq, np_
            p0 += ROWS


@pytest.mark.parametrize("seed", range(6))
def test_forward_windows_stay_in_the_zero_border(seed):
    rng = np.random.default_rng(seed)
    worst_lo, worst_hi = 0, 0
    for _ in range(40):
        w = int(rng.integers(8, 400))
        h = int(rng.integers(8, 400)) if rng.random() < 0.3 else w
        nd = int(rng.integers(3, 3 * max(w, h)))
        if rng.random() < 0.3:  # bounds off: the whole image and a disc through its corners
            box = (0, w - 1, 0, h - 1)
            r4 = (w - 1) ** 2 + (h - 1) ** 2
        else:
            x0, x1 = sorted(rng.integers(0, w, 2))
            y0, y1 = sorted(rng.integers(0, h, 2))
            box = (int(x0), int(x1), int(y0), int(y1))
            r4 = max((2 * x - w + 1) ** 2 + (2 * y - h + 1) ** 2 for x in (x0, x1) for y in (y0, y1))
        angles = list(rng.uniform(0.0, 180.0, 12)) + [0.0, 45.0, 90.0, 135.0, 179.75, 44.999, 45.001]
        for deg in angles:
            for p0, c_first, c_last, nq, np_ in windows(w, h, nd, float(deg), box, r4):
                assert p0 >= 0 and p0 + ROWS - 1 <= np_ - 1 + ROWS, (w, h, nd, deg, p0)
                assert c_first >= -50 and c_last <= nq - 1 + 50, (w, h, nd, deg, box, c_first, c_last, nq)
                worst_lo = min(worst_lo, c_first)
                worst_hi = max(worst_hi, c_last - (nq - 1))
    assert worst_lo >= -GUARD and worst_hi <= GUARD
