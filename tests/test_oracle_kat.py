"""Known-answer tests of the oracle's building blocks, and the same answers
from the reference's own functions where the reference build is present.

The reference ships no tests or golden vectors; these answers follow from its
code:
* Correlate returns 1 for identical vectors, -1 for opposite ones and the -99
  sentinel for N <= 0 or a variance at or below 1e-8 (SubFunctions.cpp:974-1018).
* The result quantiser rounds half away from zero, the voxel quantiser
  truncates toward zero, both through a 32-bit integer (Template.hpp:964-993).
* The circular window of half-size H holds 45/25/9 (H=3), 109/45/25 (H=5),
  145/45/9 (H=6) and 193/77/25 (H=7) samples in its three nested
  sub-windows (SubFunctions.cpp:3281-3313 over setsm_code.cpp:6429-6453).
* The RPC projection clamps to [0, off + 1.2 * scale] and wraps longitudes
  that normalise beyond +-10 (CoordConversion.hpp:30-84).
"""
import numpy as np
import pytest

from oracle import oraclepy as op
from oracle import refpy
from tests import cases

WINDOW_COUNTS = {3: (45, 25, 9), 5: (109, 45, 25), 6: (145, 45, 9), 7: (193, 77, 25)}

need_ref = pytest.mark.skipif(not refpy.available(), reason="reference build not available")


@pytest.mark.parametrize("half", sorted(WINDOW_COUNTS))
def test_window_counts(half):
    assert op.window_counts(half) == WINDOW_COUNTS[half]


@need_ref
@pytest.mark.parametrize("half", [2, 3, 4, 5, 6, 7, 8])
def test_window_counts_match_reference(half):
    assert op.window_counts(half) == refpy.window_counts(half)


def _correlate_cases():
    rng = np.random.default_rng(11)
    a = rng.normal(size=49)
    out = [
        (a, a),                              # identical -> 1
        (a, -a),                             # opposite -> -1
        (np.full(9, 3.0), a[:9]),            # zero variance -> -99
        (a[:25], np.full(25, 7.0)),
        (a[:0], a[:0]),                      # N = 0 -> -99
        (a[:25], 2.0 * a[:25] + 5.0),        # affine -> 1
        (np.r_[1.0, 1.0 + 1e-4, 1.0], np.r_[0.0, 1.0, 2.0]),   # SumL2 ~ 6.7e-9 < 1e-8
        (np.r_[1.0, 1.0 + 2e-4, 1.0], np.r_[0.0, 1.0, 2.0]),   # SumL2 ~ 2.7e-8 > 1e-8
    ]
    for n in (9, 25, 45, 109, 193):
        out.append((rng.integers(1, 2048, n).astype(float), rng.integers(1, 2048, n).astype(float)))
    return out


def test_correlate_known_answers():
    c = _correlate_cases()
    assert op.correlate(*c[0]) == pytest.approx(1.0, abs=1e-15)
    assert op.correlate(*c[1]) == pytest.approx(-1.0, abs=1e-15)
    assert op.correlate(*c[2]) == -99.0
    assert op.correlate(*c[3]) == -99.0
    assert op.correlate(*c[4]) == -99.0
    assert op.correlate(*c[5]) == pytest.approx(1.0, abs=1e-15)
    assert op.correlate(*c[6]) == -99.0
    assert op.correlate(*c[7]) == pytest.approx(0.0, abs=1e-6)


def test_correlate_matches_numpy_pearson():
    for left, right in _correlate_cases()[8:]:
        expect = np.corrcoef(left, right)[0, 1]
        assert op.correlate(left, right) == pytest.approx(expect, abs=1e-12)


@need_ref
def test_correlate_bit_exact_with_reference():
    for left, right in _correlate_cases():
        assert op.correlate(left, right) == refpy.correlate(left, right)


def test_quantizers():
    # rounding (result / grid) vs truncation (voxel)
    assert op.quantize_result(0.4567) == 457 and op.quantize_voxel(0.4567) == 456
    assert op.quantize_result(-0.4567) == -457 and op.quantize_voxel(-0.4567) == -456
    assert op.quantize_result(0.0005) == 1 and op.quantize_result(-0.0005) == -1
    assert op.quantize_voxel(0.0009999) == 0 and op.quantize_voxel(-0.9999) == -999
    assert op.quantize_result(-1.0) == -1000 and op.quantize_voxel(-1.0) == -1000
    # AWNCC's "no peak" sentinel wraps through the 32-bit integer
    assert op.quantize_result(-100.0) == 31072   # (short)(int)-100000
    # NaN and out-of-range inputs give the integer-indefinite value's low half: 0
    assert op.quantize_result(float("nan")) == 0 and op.quantize_voxel(float("nan")) == 0
    assert op.quantize_voxel(1e12) == 0


@need_ref
def test_rpc_projection_and_clamp_match_reference():
    sc = cases.scene(3, 768)
    rng = np.random.default_rng(5)
    for ci in range(2):
        rpc = sc.rpcs[ci]
        n = 4000
        lon = rpc[2] + rpc[7] * rng.uniform(-1.6, 1.6, n)   # beyond the image: clamps
        lat = rpc[3] + rpc[8] * rng.uniform(-1.6, 1.6, n)
        hgt = rpc[4] + rpc[9] * rng.uniform(-1.5, 1.5, n)
        lon[:50] += 360.0   # normalised beyond +-10: wrapped back
        a = op.rpc_project(rpc, (0.3, -0.2), lon, lat, hgt)
        b = refpy.rpc_project(rpc, (0.3, -0.2), lon, lat, hgt)
        assert np.array_equal(a, b)
        # clamped to [0, off + 1.2 * scale] per axis (x = sample, y = line)
        assert a[:, 0].min() >= 0 and a[:, 1].min() >= 0
        assert a[:, 0].max() <= rpc[1] + 1.2 * rpc[6] + 1e-9
        assert a[:, 1].max() <= rpc[0] + 1.2 * rpc[5] + 1e-9
        assert (a[:, 0] == 0).any() or (a[:, 1] == 0).any()
