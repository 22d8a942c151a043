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
