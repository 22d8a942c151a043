"""The bound the blunder_detection_TIN threshold band rests on
(vll_tinblunder.cu: sum_band): the sequential FP64 sum of m non-negative terms
(the reference's order, setsm_code.cpp:9257-9273) and a sum of the same terms
in any other order differ by at most 3 m u times the latter (u = 2^-53).
Checked here on the CPU against numpy's sequential (add.accumulate) and
pairwise (add.reduce) sums, including adversarial spreads of magnitude."""
import numpy as np
import pytest


def seq_sum(v):
    return float(np.add.accumulate(v)[-1]) if len(v) else 0.0


@pytest.mark.parametrize("seed", range(6))
def test_sequential_sum_inside_band(seed):
    rng = np.random.default_rng(seed)
    m = int(rng.integers(1, 300_000))
    kind = seed % 3
    if kind == 0:
        v = rng.uniform(0, 60, m)
    elif kind == 1:
        v = np.exp(rng.uniform(-40, 12, m))            # many magnitudes
    else:
        v = np.where(rng.random(m) < 0.001, 1e6, rng.uniform(0, 1e-3, m))   # rare giants
    for terms in (v, v * v):
        s_any = float(np.sum(terms[rng.permutation(m)]))
        s_seq = seq_sum(terms)
        e = s_any * (3.0 * m * 2.0 ** -53) * (1.0 + 2.0 ** -40)
        assert np.nextafter(s_any - e, -np.inf) <= s_seq <= np.nextafter(s_any + e, np.inf)


# ---- the threshold band of the library (host-only diagnostic) ----------------

import ctypes as C
import math


def ref_height_th(L, it, is_ra, gs, hint, sd, sd2, dh_count, hbin):
    """The reference's height threshold (setsm_code.cpp:9320-9418), in its
    operation order on Python floats (IEEE doubles, no contraction)."""
    check_dh = (3 <= L <= 4) or (L == 2 and it <= 4) or (L <= 1 and it <= 2)
    if L >= 1:
        gsd = gs
        if L >= 3 and gs < 2 ** (L - 1):
            gsd = float(2 ** (L - 1))
    else:
        gsd = 0.5
    h2 = gsd * 30 if is_ra else gsd * 10
    height_th = hint if hint < h2 else h2

    def up3():
        mean = sd / dh_count
        v = (sd2 - sd * sd / dh_count) / dh_count
        std = math.sqrt(v) if v >= 0 else float("nan")
        return mean + 3 * std
    if L >= 3:
        up = up3() if check_dh else height_th
        if up < height_th:
            height_th = height_th / 2.0 if up < height_th / 2.0 else up
        return height_th
    th80, total, found, t = 1000, 0, False, 0
    while t < len(hbin) and not found:
        total = (total + int(hbin[t])) & 0xFFFFFFFF
        if total / dh_count * 100.0 > 99:
            th80, found = t, True
        t += 1
    if not found:
        th80 = t - 1
    up = up3()
    height_th = up if up < th80 else float(th80)
    return 50.0 if height_th > 50 else height_th


def lib_band(L, it, is_ra, gs, hint, sd, sd2, m, dh_count, hbin, exact):
    from setsm_b200 import vll
    lo, hi = C.c_double(), C.c_double()
    hb = np.ascontiguousarray(hbin, dtype=np.uint32)
    rc = vll.load().vll_debug_tin_threshold(L, it, int(is_ra), gs, hint, sd, sd2, m, dh_count,
                                            hb.ctypes.data, len(hb), int(exact), C.byref(lo),
                                            C.byref(hi))
    assert rc == 0
    return lo.value, hi.value


def lib_available():
    try:
        from setsm_b200 import vll
        vll.load()
        return True
    except Exception:
        return False


def terms_for(rng, kind, m):
    if kind == 0:
        return rng.uniform(0, 40, m)
    if kind == 1:
        return np.abs(rng.normal(0, 3, m))
    if kind == 2:
        return np.full(m, rng.uniform(0.1, 30))            # variance ~ 0: cancellation
    if kind == 3:
        return np.where(rng.random(m) < 0.01, rng.uniform(100, 400, m), rng.uniform(0, 2, m))
    if kind == 4:
        return np.round(rng.uniform(0, 20, m), 1) + rng.normal(0, 1e-9, m).clip(0)
    # a tail at 45 above the 99th percentile: mean + 3 sd below it (the
    # threshold is up_3sigma itself below level 3)
    return np.where(rng.random(m) < 0.015, 45.0, rng.uniform(0, 5, m))


@pytest.mark.skipif(not lib_available(), reason="library not built")
@pytest.mark.parametrize("seed", range(60))
def test_threshold_band_holds_the_reference_threshold(seed):
    rng = np.random.default_rng(1000 + seed)
    L = int(rng.integers(0, 5))
    it = int(rng.integers(1, 6))
    is_ra = bool(rng.random() < 0.2)
    gs = float(rng.choice([2.0, 4.0, 8.0, 16.0]))
    hint = float(rng.uniform(5, 120))
    m = 3 * int(rng.integers(1, 60_000))
    v = terms_for(rng, seed % 6, m)
    sq = v * v
    sd_seq, sd2_seq = seq_sum(v), seq_sum(sq)
    perm = rng.permutation(m)
    sd_any, sd2_any = float(np.sum(v[perm])), float(np.sum(sq[perm]))
    hdiffcount = int(hint)
    iv = v.astype(np.uint32)
    hbin = np.bincount(iv[iv < hdiffcount], minlength=hdiffcount)[:hdiffcount]
    want = ref_height_th(L, it, is_ra, gs, hint, sd_seq, sd2_seq, m, hbin)
    # exact sums: the library's threshold is the reference's
    lo, hi = lib_band(L, it, is_ra, gs, hint, sd_seq, sd2_seq, m, m, hbin, True)
    assert lo == hi == want
    # sums in another order: the band holds the reference's threshold
    lo, hi = lib_band(L, it, is_ra, gs, hint, sd_any, sd2_any, m, m, hbin, False)
    assert lo <= want <= hi, (lo, want, hi)
    if seed % 6 != 2:   # away from the cancelling case the band is narrow
        assert hi - lo <= 1e-6 * max(1.0, abs(want))
