"""The box conversion's lane arithmetic (convert_tile, setsm_b200/csrc/
vll_window.cuh), emulated for 32 lanes on the CPU for every box width and a
range of heights: two adjacent box texels per lane step, the lane's first
pair and its step from an FP32 reciprocal of the pairs per row.  Every box
texel [0, bw) of every row is written exactly once, every texel the windows
read ([0, bw] of a row) is examined for a zero intensity exactly once, and
no load reaches past texel bw of its row."""
import numpy as np
import pytest


def convert_lanes(bw: int, bh: int):
    bp = (bw + 1) >> 1
    n2 = bp * bh
    rbp = np.float32(1.0) / np.float32(bp)
    written, examined, max_read = {}, {}, -1
    for lane in range(32):
        by = int(np.floor(np.float32(np.float32(lane) + np.float32(0.5)) * rbp))
        bq = lane - by * bp
        dby = int(np.floor(np.float32(32.5) * rbp))
        dbq = 32 - dby * bp
        q = lane
        while q < n2:
            bx = 2 * bq
            two = bx + 1 < bw
            max_read = max(max_read, bx + 2 if two else bx + 1)
            end2 = two and bx + 2 == bw
            for t in range(3):
                if t < 2 or end2:
                    examined[(by, bx + t)] = examined.get((by, bx + t), 0) + 1
            written[(by, bx)] = written.get((by, bx), 0) + 1
            if two:
                written[(by, bx + 1)] = written.get((by, bx + 1), 0) + 1
            bq += dbq
            by += dby
            if bq >= bp:
                bq -= bp
                by += 1
            q += 32
    return written, examined, max_read


@pytest.mark.parametrize("bh", [1, 2, 7, 17, 33])
def test_pairs_cover_the_box_once(bh):
    for bw in range(1, 130):
        written, examined, max_read = convert_lanes(bw, bh)
        want_w = {(y, x) for y in range(bh) for x in range(bw)}
        want_e = {(y, x) for y in range(bh) for x in range(bw + 1)}
        assert set(written) == want_w and all(v == 1 for v in written.values()), bw
        assert set(examined) == want_e and all(v == 1 for v in examined.values()), bw
        assert max_read <= bw, bw
