"""The autotuner's choice (setsm_b200/autotune.py) with a fake context: the
default tuning stays unless a candidate is at least 5 % faster, the choice is
applied and cached, and a cached choice is reused."""
from setsm_b200 import autotune


class FakeStats:
    def __init__(self, ms):
        self.kernel_ms = ms


class FakeCtx:
    """Batch time per tuning from a table; remembers the tuning applied."""

    def __init__(self, times):
        self.times = times
        self.tuning = None

    def set_tuning(self, **t):
        self.tuning = dict(t)

    def batch(self, levels):
        key = tuple(sorted(self.tuning.items()))
        return None, FakeStats(self.times.get(key, 100.0))


class Desc:
    template_size = 11
    pyramid_step = 0


def _key(t):
    return tuple(sorted(t.items()))


def test_default_kept_unless_clearly_faster(tmp_path, monkeypatch):
    monkeypatch.setattr(autotune, "gpu_key", lambda device=0: "fake")
    other = dict(blocks_per_sm=2, grab=1, box_margin=1.25)
    # 3 % faster: the default stays
    ctx = FakeCtx({_key(other): 97.0})
    r = autotune.tune(ctx, [(Desc(),)], path=str(tmp_path / "a.json"))
    assert r["tuning"] == autotune.DEFAULT and ctx.tuning == autotune.DEFAULT
    # 10 % faster: it is chosen, applied and cached
    ctx = FakeCtx({_key(other): 90.0})
    r = autotune.tune(ctx, [(Desc(),)], path=str(tmp_path / "b.json"))
    assert r["tuning"] == other and ctx.tuning == other
    ctx2 = FakeCtx({})
    r2 = autotune.tune(ctx2, [(Desc(),)], path=str(tmp_path / "b.json"))
    assert r2["tuning"] == other and ctx2.tuning == other
