"""Exhaustive checks of two arithmetic facts the window kernel relies on
(setsm_b200/csrc/vll_split.cu, vll_window.cuh), in IEEE arithmetic on the
CPU:

* the FindPeakNcc top-two fold keeps the replaced maximum as
  q_result(dq_result(x)) -- x / 1000 in double, times 1000, rounded half
  away from zero -- which is x itself for every int16 x, so the fold needs
  no FP64 division;
* the box conversion takes a lane's first texel pair and its step as
  (n + 0.5) * r truncated, r an FP32 reciprocal of the pairs per row bp with
  a relative error of a few ulp (__fdividef): the quotient equals n // bp
  for every lane n <= 31, the step n = 32, and bp up to 4096;
* the target box, placed before the orientation is known, covers every
  rotated window (radius H + 2 around the centre texel);
* the fold in registers equals the reference's sequential fold with its
  re-quantisation on random peak sequences (ties and int16 extremes
  included)."""
import numpy as np


def c_round(v: np.ndarray) -> np.ndarray:
    """C's round(): halves away from zero."""
    return np.where(v >= 0, np.floor(v + 0.5), -np.floor(-v + 0.5))


def test_requantised_maximum_is_identity_on_int16():
    x = np.arange(-32768, 32768, dtype=np.float64)
    v = x / 1000.0                      # dq_result
    back = c_round(v * 1000.0)          # q_result before the short conversion
    assert np.array_equal(back, x)


def test_fp32_reciprocal_quotients_are_exact():
    bp = np.arange(1, 4097, dtype=np.float32)
    n = np.arange(0, 33, dtype=np.float32)[:, None]
    exact = (np.arange(0, 33)[:, None] // np.arange(1, 4097)[None, :])
    r0 = (np.float32(1.0) / bp).astype(np.float32)
    for k in range(-4, 5):               # the reciprocal off by up to 4 ulp either way
        r = r0
        step = np.inf if k > 0 else -np.inf
        for _ in range(abs(k)):
            r = np.nextafter(r, np.float32(step)).astype(np.float32)
        q = np.floor((n + np.float32(0.5)) * r[None, :]).astype(np.int64)
        assert np.array_equal(q, exact), k


def test_target_box_radius_holds_for_every_rotation():
    """The window kernel places the target box [centre - R, centre + R + 1]
    with R = H + 2 before it knows the rotation: every sample of a window
    rotated by any angle (FP32 positions, as the kernel computes them) reads
    texels floor(f) and floor(f) + 1 inside it, f the sample's position from
    the centre texel, whatever the centre's fraction."""
    for H in range(2, 8):
        R = H + 2
        rows, cols = np.meshgrid(np.arange(-H, H + 1), np.arange(-H, H + 1), indexing="ij")
        keep = rows * rows + cols * cols <= (H + 1) * (H + 1)
        row = rows[keep].astype(np.float32)
        col = cols[keep].astype(np.float32)
        ang = np.deg2rad(np.arange(0.0, 360.0, 0.25))
        c = np.cos(ang).astype(np.float32)[:, None]
        s = np.sin(ang).astype(np.float32)[:, None]
        for frac in (0.0, 0.25, 0.5, 0.75, np.nextafter(np.float32(1), np.float32(0))):
            tf = np.float32(frac)
            # the kernel: b = (-s, c) * row + tf, then f = (c, s) * col + b
            bx = (-s * row + tf).astype(np.float32)
            by = (c * row + tf).astype(np.float32)
            fx = (c * col + bx).astype(np.float32)
            fy = (s * col + by).astype(np.float32)
            for f in (fx, fy):
                lo = np.floor(f)
                assert lo.min() >= -R and lo.max() + 1 <= R + 1, (H, frac)


def _fold_reference(state, peaks):
    """FindPeakNcc's ordered top-two update as the reference states it: the
    replaced maximum re-quantised through dq_result / q_result."""
    r0, r1, r2, r3, r4 = state
    for q, h in peaks:
        if r4 < 10:
            r4 += 1
        if r0 < q:
            t1 = r0 / 1000.0
            t2 = r2
            r0, r2 = q, h
            q1 = int(c_round(np.float64(t1) * 1000.0))
            if r1 < q1:
                r1, r3 = q1, t2
        elif r1 < q:
            r1, r3 = q, h
    return r0, r1, r2, r3, r4


def _fold_kernel(state, peaks):
    """The window kernel's fold in registers (no re-quantisation)."""
    r0, r1, r2, r3, r4 = state
    for q, h in peaks:
        if r4 < 10:
            r4 += 1
        if r0 < q:
            if r1 < r0:
                r1, r3 = r0, r2
            r0, r2 = q, h
        elif r1 < q:
            r1, r3 = q, h
    return r0, r1, r2, r3, r4


def test_register_fold_equals_reference_fold():
    rng = np.random.default_rng(7)
    for trial in range(4000):
        n = int(rng.integers(0, 12))
        if trial % 3 == 0:   # ties and near-ties
            qs = rng.integers(-5, 6, size=n) + int(rng.integers(-1000, 1000))
        else:
            qs = rng.integers(-32768, 32768, size=n)
        peaks = [(int(q), float(h)) for q, h in zip(qs, rng.normal(0, 100, size=n))]
        start = (int(rng.choice([-32768, -1000, 0, 500, 32767])),
                 int(rng.choice([-32768, -1000, 0, 400, 32767])),
                 float(rng.normal()), float(rng.normal()), int(rng.integers(0, 11)))
        assert _fold_kernel(start, peaks) == _fold_reference(start, peaks), (start, peaks)
