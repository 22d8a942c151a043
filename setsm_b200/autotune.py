"""Launch autotuner of the split pipeline's persistent window kernel.

The window kernel's launch shape is a trade between occupancy, queue traffic
and shared-memory footprint, and the best point depends on the GPU, the window
sizes and the epipolar sweep of the scenes.  The tunable parameters
(``vll_tuning``, include/setsm_vll.h) are:

* ``blocks_per_sm`` -- CTAs of 4 warps per SM (0 = the occupancy maximum);
* ``grab``          -- nodes a warp takes per queue access (at most 32 are
                       used), i.e. the chunk of the queue a warp owns at a time;
* ``box_margin``    -- the per-warp shared-memory budget for the staged image
                       footprints over the swept-box estimate (larger boxes keep
                       rare wide footprints on the FP32 path, smaller ones raise
                       occupancy).

``tune`` times every candidate on a batch (the whole pipeline through
``vll_vertical_line_locus_batch``, CUDA events), keeps the fastest (the default
unless a candidate is at least 5 % faster), and caches
it in a JSON file keyed by GPU, SM count and the batch's window sizes and
pyramid levels.  Results never depend on the tuning (tests/test_gpu_batch.py).
"""
from __future__ import annotations

import itertools
import json
import os
import time

DEFAULT = {"blocks_per_sm": 0, "grab": 8, "box_margin": 1.1}

# a candidate replaces the default only when this much faster
MARGIN_TO_SWITCH = 0.05

CANDIDATES = [dict(blocks_per_sm=b, grab=g, box_margin=m)
              for b, g, m in itertools.product((0, 2), (1, 4, 8, 16, 32), (1.0, 1.1, 1.25))]


def cache_path() -> str:
    return os.environ.get("SETSM_VLL_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "setsm_b200",
                                       "tuning.json"))


def gpu_key(device: int = 0) -> str:
    import torch
    p = torch.cuda.get_device_properties(device)
    return f"{p.name}|sm{p.multi_processor_count}"


def batch_key(descs) -> str:
    """Window sizes and pyramid levels of a batch (what the tuning depends on)."""
    shape = sorted({(int(d.template_size), int(d.pyramid_step)) for d in descs})
    return ";".join(f"T{t}L{l}" for t, l in shape)


def load_cache(path: str | None = None) -> dict:
    path = path or cache_path()
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(cache: dict, path: str | None = None) -> None:
    path = path or cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def time_batch(ctx, levels, repeats: int = 2) -> float:
    """Best device time (ms) of `repeats` batch passes after one warm-up."""
    ctx.batch(levels)
    best = float("inf")
    for _ in range(repeats):
        _, st = ctx.batch(levels)
        best = min(best, float(st.kernel_ms))
    return best


def tune(ctx, levels, candidates=None, repeats: int = 2, path: str | None = None,
         device: int = 0, force: bool = False) -> dict:
    """Chooses the fastest tuning for `levels` (a batch as for Context.batch),
    applies it to `ctx` and caches it; a cached choice is reused unless
    `force`.  Returns {"tuning": ..., "ms": ..., "trials": [...]}."""
    key = gpu_key(device) + "|" + batch_key([lv[0] for lv in levels])
    cache = load_cache(path)
    if key in cache and not force:
        ctx.set_tuning(**cache[key]["tuning"])
        return cache[key]
    trials = []
    t0 = time.time()
    for c in candidates or CANDIDATES:
        ctx.set_tuning(**c)
        trials.append({"tuning": c, "ms": time_batch(ctx, levels, repeats)})
    best = min(trials, key=lambda t: t["ms"])
    # the default stays unless a candidate beats it clearly: single timings
    # on a sample of the work differ by a few percent from run to run
    default = next((t for t in trials if t["tuning"] == DEFAULT), None)
    if default is not None and best["ms"] > (1.0 - MARGIN_TO_SWITCH) * default["ms"]:
        best = default
    ctx.set_tuning(**best["tuning"])
    entry = {"tuning": best["tuning"], "ms": best["ms"], "trials": trials,
             "tuned_s": round(time.time() - t0, 2)}
    cache[key] = entry
    save_cache(cache, path)
    return entry


def apply_cached(ctx, descs, path: str | None = None, device: int = 0) -> dict | None:
    """Applies a cached tuning for a batch of these descriptors, if any."""
    key = gpu_key(device) + "|" + batch_key(descs)
    entry = load_cache(path).get(key)
    if entry:
        ctx.set_tuning(**entry["tuning"])
    return entry
