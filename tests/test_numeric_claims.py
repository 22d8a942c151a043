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
  for every lane n <= 31, the step n = 32, and bp up to 4096."""
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
