"""Host logic of the serving loop (no GPU): request streams and HBM-budget
admission in arrival order."""
import numpy as np

from setsm_b200 import serving


class _Spec:
    image_size = 4096
    gsd = 0.5


class _Scene:
    spec = _Spec()


class _RS:
    def __init__(self, sid):
        self.sid = sid
        self.scene = _Scene()


def test_poisson_stream_shapes():
    scenes = [_RS(0), _RS(1)]
    reqs = serving.poisson_requests(2000, 200.0, scenes, seed=3, levels=(0, 1),
                                    templates=(11, 15))
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0)
    rate = len(reqs) / arr[-1]
    assert 170 < rate < 230                       # Poisson at ~200 / s
    sides = np.array([r.n for r in reqs])
    ks = np.array([r.k for r in reqs])
    assert sides.min() >= 8 and sides.max() <= 1024
    assert 8 <= ks.min() and ks.max() <= 512
    # log-uniform: about half the requests below the geometric mean
    assert 0.4 < np.mean(ks < np.sqrt(8 * 512)) < 0.6
    assert {r.sid for r in reqs} == {0, 1} and {r.level for r in reqs} == {0, 1}
    assert {r.template for r in reqs} == {11, 15}


def test_admission_respects_budget_in_arrival_order():
    reqs = [serving.TileRequest(rid=i, sid=0, level=0, template=11, n=n, spacing=2.0, k=64,
                                fx=0.5, fy=0.5, seed=i)
            for i, n in enumerate([256, 512, 128, 1024, 64])]
    sizes = [serving.request_bytes(r) for r in reqs]
    budget = sizes[0] + sizes[1] + sizes[2] // 2
    srv = serving.Server([], hbm_budget=budget)
    for r in reqs:
        srv.submit(r)
    # the first two fit; the third waits (arrival order is kept even though
    # later requests are small)
    assert [r.rid for r in srv.ready] == [0, 1]
    assert [r.rid for r in srv.waiting] == [2, 3, 4]
    assert srv.in_use <= budget
    # releasing memory admits the next ones in order
    with srv.lock:
        srv.ready.clear()
        srv.in_use -= sizes[0] + sizes[1]
        srv._admit_locked(0.0)
    assert [r.rid for r in srv.ready] == [2]      # request 3 (1024^2) does not fit next to it
    with srv.lock:
        srv.ready.clear()
        srv.in_use = 0.0
        srv._admit_locked(0.0)
    # an oversize request is admitted alone when nothing else holds memory
    assert [r.rid for r in srv.ready][0] == 3
