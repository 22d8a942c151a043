#!/usr/bin/env python
"""Benchmark of the vertical-line-locus hot path (node x height NCC evals/s).

Workload (default ``c2``): level-0 full scene -- a seeded synthetic 16384^2
uint16 stereo pair (pushbroom cameras, cubic RPCs), a 4096^2 grid at 2 m with
TIN-derived height ranges of 8-512 candidates at 0.5 m, matched with the 7x7
and 11x11 windows on the memory-tight route (inline first/second peak
selection).  One step = one VerticalLineLocus pass per window over the whole
grid.

* value: evals/s with inputs resident in HBM (device-pointer C ABI), K steps
  timed with CUDA events on the library's stream; max over ranks.
* e2e: the same metric through the host-buffer C ABI call
  (vll_vertical_line_locus) from pinned host memory, uploads and downloads
  inside the timed region.
* roofline: the window kernel's algorithmic bytes (8 B per window sample,
  2 orientation bytes, 4 B NCC out) per launch over its average duration.
* fp64_plain_gpu: the plain FP64 one-node-per-thread kernel on the same
  workload (untimed leg, CUDA events), with identical-peak and tie rates.
* cpu_baseline: the reference SETSM code (oracle/_ref, OpenMP, all host
  cores) on a bounded band of grid rows of the same workload.

``--impl reference`` times the reference CPU implementation alone (rank 0).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "node x height NCC evals/s"
UNIT = "evals/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        import tempfile
        try:
            fd, self.path = tempfile.mkstemp(prefix=f"clocks_gpu{self.index}_", suffix=".csv")
            self.f = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_setup(gpus: int):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(world, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------
# CPU reference leg
# ---------------------------------------------------------------------------
# The reference's VerticalLineLocus is timed on a band of grid rows in the
# middle of the grid holding at least this fraction of the nodes, per window.
REF_NODE_FRACTION = 0.01
# Image rows kept around a band's projected footprint: the rotated 11x11
# window (radius <= 9 px) plus the orientation window (6 px) and Sobel (1 px),
# with room to spare.
REF_FOOTPRINT_MARGIN = 48
# Rows discarded at each cut edge of a preprocessed crop: Sobel reads one row
# and the orientation window six rows past a pixel, so rows further than this
# from a cut are the full image's values.
REF_CROP_EDGE = 16

_EVAL_COUNTS = {}


def ref_band(wl, evals_budget: float = 5e6) -> tuple:
    """(first row, rows) of the reference band: >= REF_NODE_FRACTION of the
    nodes (plus one row), or more rows on grids where that is cheap."""
    from setsm_b200 import workloads
    H = wl.grid.height
    rows = max(int(math.ceil(H * REF_NODE_FRACTION)) + 1, workloads.rows_for_budget(wl, evals_budget))
    rows = min(H, rows)
    return (H - rows) // 2, rows


def band_footprint(wl, r0: int, rows: int) -> list:
    """Image-row range [y0, y1) of each image that the band's nodes can reach:
    every node projected at its minimum and maximum height, plus
    REF_FOOTPRINT_MARGIN rows."""
    import torch
    from setsm_b200 import synth
    W = wl.grid.width
    sl = slice(r0 * W, (r0 + rows) * W)
    wgs = torch.from_numpy(np.ascontiguousarray(wl.host["wgs"][sl]))
    n = wl.scene.spec.image_size
    out = []
    for ci in range(2):
        lines = []
        for f in ("minHeight", "maxHeight"):
            h = torch.from_numpy(wl.gp3[f][sl].astype(np.float64))
            _, line = synth.rpc_eval(wl.scene.rpcs[ci], wgs[:, 0], wgs[:, 1], h)
            lines.append(line)
        line = torch.cat(lines)
        y0 = max(0, int(math.floor(float(line.min()))) - REF_FOOTPRINT_MARGIN)
        y1 = min(n, int(math.ceil(float(line.max()))) + REF_FOOTPRINT_MARGIN)
        out.append((y0, y1))
    return out


def reference_planes(wl, footprints: list) -> dict:
    """Magnitude and orientation planes made by the reference's own
    MakeSobelMagnitudeImage and Orientation (SubFunctions.cpp:2418, :2473) on
    crops of the images around `footprints` (one [y0, y1) row range per
    image and band), written into zero full-size planes."""
    from oracle import refpy
    n = wl.scene.spec.image_size
    mags = [np.zeros((n, n), np.uint16) for _ in range(2)]
    oris = [np.zeros((n, n), np.uint8) for _ in range(2)]
    for fp in footprints:
        for ci, (y0, y1) in enumerate(fp):
            c0 = max(0, y0 - REF_CROP_EDGE)
            c1 = min(n, y1 + REF_CROP_EDGE)
            m, o = refpy.preprocess(wl.host["img"][ci][c0:c1], 15)
            mags[ci][y0:y1] = m[y0 - c0:y1 - c0]
            oris[ci][y0:y1] = o[y0 - c0:y1 - c0]
    return {"mag": mags, "ori": oris}


def band_evals(inp, key) -> int:
    """Evaluations (ComputeMultiNCC calls) of a band, counted once per band by
    the C restatement of the path on the identical inputs, outside any timed
    region (the reference's function returns no such count)."""
    if key not in _EVAL_COUNTS:
        from oracle import oraclepy
        oraclepy.set_threads(os.cpu_count() or 1)
        _EVAL_COUNTS[key] = int(oraclepy.vertical_line_locus(inp, inp.new_nccresult(),
                                                             want_evals=True)[1])
    return _EVAL_COUNTS[key]


class ReferenceLeg:
    """The reference SETSM code (oracle/_ref, OpenMP on every host core) on a
    band of grid rows of the workload, one band per window, with planes made by
    the reference's own preprocessing.  Nothing of this repository's GPU
    library runs here."""

    def __init__(self, wl, templates):
        from oracle import refpy
        self.ok = refpy.available()
        self.wl = wl
        self.templates = templates
        self.cores = os.cpu_count() or 1
        if not self.ok:
            return
        refpy.set_threads(self.cores)
        self.r0, self.rows = ref_band(wl)
        self.footprint = band_footprint(wl, self.r0, self.rows)
        t = time.perf_counter()
        self.planes = reference_planes(wl, [self.footprint])
        self.prep_s = time.perf_counter() - t
        self.inputs = {tm: wl.host_inputs(tm, rows=(self.r0, self.r0 + self.rows),
                                          planes=self.planes) for tm in templates}
        self.evals = {tm: band_evals(self.inputs[tm], (tm, self.r0, self.rows))
                      for tm in templates}
        self.last_ncc = {}

    def run(self, rows: int | None = None) -> dict:
        """One pass of every window over the band (or over its first `rows`
        rows, for untimed warm-ups); returns the measured sample."""
        from oracle import refpy
        from setsm_b200 import workloads
        if not self.ok:
            return {"value": None, "unit": UNIT, "cores": self.cores, "kind": "reference",
                    "sample": "reference build missing (oracle/_ref not built)"}
        total_evals, total_s, parts = 0, 0.0, []
        for tm in self.templates:
            inp = self.inputs[tm]
            if rows is not None:
                inp = self.wl.host_inputs(tm, rows=(self.r0, self.r0 + rows), planes=self.planes)
            ncc = inp.new_nccresult()
            t = time.perf_counter()
            refpy.vertical_line_locus(inp, ncc)
            dt = time.perf_counter() - t
            if rows is not None:
                continue
            self.last_ncc[tm] = ncc
            total_evals += self.evals[tm]
            total_s += dt
            parts.append(f"{self.rows} rows x {self.wl.grid.width} nodes "
                         f"({100.0 * self.rows / self.wl.grid.height:.2f} % of the grid), "
                         f"{workloads.WINDOW_OF_TEMPLATE[tm]}: {self.evals[tm]} evals in {dt:.2f} s")
        if rows is not None:
            return {}
        return {"value": total_evals / total_s, "unit": UNIT, "cores": self.cores,
                "kind": "reference", "sample": "; ".join(parts)}

    def parity(self, gpu_ncc: dict, gpu_planes: dict | None = None) -> dict:
        """The last band results against the GPU's whole-grid NCCresult of the
        same rows (every field), and the reference-made planes against the
        GPU-made ones over the band's footprint rows."""
        from tests.cases import field_mismatch
        W = self.wl.grid.width
        sl = slice(self.r0 * W, (self.r0 + self.rows) * W)
        out = {"rows": [self.r0, self.r0 + self.rows], "nodes": self.rows * W, "windows": {}}
        for tm in self.templates:
            from setsm_b200 import workloads
            a = self.last_ncc[tm]
            b = gpu_ncc[tm][sl]
            mism = field_mismatch(a, b)
            ran = a["check_height_change"] > 0
            dh = np.abs(a["result2"][ran].astype(np.float64) - b["result2"][ran].astype(np.float64))
            out["windows"][workloads.WINDOW_OF_TEMPLATE[tm]] = {
                "fields_mismatched": mism, "nodes_mismatched": int(sum(
                    np.count_nonzero(a[f] != b[f]) for f in a.dtype.names if f in mism)),
                "max_height_err_m": float(dh.max()) if dh.size else 0.0}
        if gpu_planes is not None:
            same = True
            for ci, (y0, y1) in enumerate(self.footprint):
                same &= bool(np.array_equal(self.planes["mag"][ci][y0:y1], gpu_planes["mag"][ci][y0:y1]))
                same &= bool(np.array_equal(self.planes["ori"][ci][y0:y1], gpu_planes["ori"][ci][y0:y1]))
            out["planes_identical_on_footprint"] = same
        return out


def run_reference_arm(args):
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    from setsm_b200 import workloads
    t0 = time.time()
    # the synthetic scene is generated with torch; this repository's GPU
    # library is not loaded in this process
    wl = workloads.build(args.config, None, device="cuda:0" if _cuda() else "cpu", seed=1)
    templates = workloads.CONFIGS[args.config]["templates"]
    leg = ReferenceLeg(wl, templates)
    log(f"workload built in {time.time() - t0:.1f} s; reference planes in "
        f"{getattr(leg, 'prep_s', 0.0):.1f} s; band rows {getattr(leg, 'rows', 0)}")
    for _ in range(args.warmup):
        leg.run(rows=2)
    vals = []
    cb = None
    t = time.perf_counter()
    for _ in range(args.steps):
        cb = leg.run()
        vals.append(cb["value"] or 0.0)
    elapsed = time.perf_counter() - t
    value = statistics.mean(vals) if vals else None
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": elapsed * 1e3 / max(1, args.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_block(args, wl),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cb["cores"], "kind": cb["kind"],
                         "sample": cb["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _cuda() -> bool:
    import torch
    return torch.cuda.is_available()


# DRAM bytes per evaluation of the window kernel measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum, a one-pass capture) on the
# full C2 launches: 4551.3 MB / 1993.23 M evaluations (7x7), 4633.3 MB /
# 1992.24 M (11x11).
DRAM_BYTES_PER_EVAL = {11: 4551.3e6 / 1993.23e6, 15: 4633.3e6 / 1992.24e6}


def traffic_per_launch(evals_step: dict, templates) -> float:
    return sum(evals_step[t] * DRAM_BYTES_PER_EVAL[t] for t in templates) / len(templates)


def config_block(args, wl) -> dict:
    from setsm_b200 import workloads
    cfg = workloads.CONFIGS[args.config]
    return {
        "workload": {
            "c2": "C2 level-0 full scene: 16384^2 uint16 stereo pair, 4096^2 grid at 2 m, "
                  "TIN ranges K=8-512 log-uniform at 0.5 m, 7x7 and 11x11 windows, "
                  "memory-tight route (inline peaks)",
            "c1": "C1: 2048^2 pair, 256^2 grid, 64 heights at 1 m, 7x7",
            "c2_small": "C2-like reduced: 4096^2 pair, 1024^2 grid, TIN K=8-512 at 0.5 m",
        }[args.config],
        "nodes": int(wl.n_nodes),
        "image": f"{cfg['image_size']}^2 uint16",
        "windows": [workloads.WINDOW_OF_TEMPLATE[t] for t in cfg["templates"]],
        "kernel": args.kernel,
        "l2": "inputs larger than L2 (images 2 x 1.25 GiB with magnitude and orientation)",
        "parallelism": f"replicas x{args.gpus} (independent scenes per GPU)",
    }


def slot_accuracy(ctx, wl, templates, r0: int, rows: int) -> dict:
    """Max |delta NCC| of the split kernel's FP32 window values against the
    FP64 kernel's, slot by slot, on a band of grid rows of the workload (the
    split pipeline settles every decision within its error band of 4e-6 in
    FP64, which is exact while this error stays below half the band)."""
    from setsm_b200 import workloads
    out = {}
    for t in templates:
        inp = wl.host_inputs(t, rows=(r0, r0 + rows))
        r32, off = ctx.debug_slot_rho(inp, inp.new_nccresult(), "split")
        r64, _ = ctx.debug_slot_rho(inp, inp.new_nccresult(), "plain")
        both = ~np.isnan(r32) & ~np.isnan(r64)
        err = np.abs(r32[both] - r64[both])
        out[workloads.WINDOW_OF_TEMPLATE[t]] = {
            "slots": int(both.sum()), "max_abs_dncc": float(err.max()) if err.size else 0.0,
            "p9999_abs_dncc": float(np.quantile(err, 0.9999)) if err.size else 0.0,
            "same_slots_evaluated": bool(np.array_equal(np.isnan(r32), np.isnan(r64))),
            "within_half_band": bool(err.size == 0 or err.max() < 2e-6)}
    out["rows"] = [r0, r0 + rows]
    return out


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    world, rank, local = dist_setup(args.gpus)
    import torch
    from setsm_b200 import abi, vll, workloads

    dev = torch.device("cuda", local)
    ctx = vll.Context(local)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    t0 = time.time()
    wl = workloads.build(args.config, ctx, device=f"cuda:{local}", seed=1 + rank)
    log(f"[rank {rank}] workload {args.config} built in {time.time() - t0:.1f} s "
        f"({wl.n_nodes} nodes)")
    templates = workloads.CONFIGS[args.config]["templates"]
    descs = {t: wl.device_desc(t) for t in templates}
    tuned = None
    if not args.no_tune:
        # autotune the window kernel's launch on a band of grid rows (cached
        # per GPU and window set; results do not depend on the tuning)
        from setsm_b200 import autotune
        ios = [wl.device_band_io(t, args.tune_rows) for t in templates]
        tuned = autotune.tune(ctx, ios, repeats=2)
        log(f"[rank {rank}] tuning {tuned['tuning']} ({tuned.get('tuned_s', 'cached')} s)")

    def one_step(kernel, stats=True):
        out = {}
        for t in templates:
            st = ctx.vertical_line_locus_device(descs[t], wl.d_gp3.data_ptr(), wl.d_ncc.data_ptr(),
                                                None, None, kernel, stats=stats)
            out[t] = st
        return out

    # warm-up (untimed)
    for _ in range(max(3, args.warmup)):
        ref_stats = one_step(args.kernel)
    evals_step = {t: ref_stats[t].evals for t in templates}
    # every window's whole-grid result, each from a cleared NCCresult array
    # (parity legs below compare against these)
    gpu_ncc = {}
    for t in templates:
        wl.d_ncc.zero_()
        torch.cuda.synchronize(dev)   # the library runs on its own stream
        ctx.vertical_line_locus_device(descs[t], wl.d_gp3.data_ptr(), wl.d_ncc.data_ptr(),
                                       None, None, args.kernel, stats=True)
        gpu_ncc[t] = workloads.ncc_host(wl)
    barrier(world)

    # ---- timed: resident inputs ----
    clocks = Clocks(local)
    clocks.start()
    launches0 = ctx.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    barrier(world)
    e0.record(stream)
    window_ms = {t: 0.0 for t in templates}
    rechecks = 0
    for _ in range(args.steps):
        st = one_step(args.kernel)
        for t in templates:
            window_ms[t] += st[t].window_ms
            rechecks += st[t].fp64_rechecks
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    clk = clocks.stop()
    elapsed_ms = e0.elapsed_time(e1)
    launches = ctx.launch_count() - launches0
    elapsed_ms = max_over_ranks(world, elapsed_ms)
    evals_total_rank = sum(evals_step.values()) * args.steps
    evals_total = sum_over_ranks(world, evals_total_rank)
    value = evals_total / (elapsed_ms / 1e3)

    # ---- roofline of the window kernel ----
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    alg_bytes = sum(evals_step[t] * workloads.BYTES_PER_EVAL[t] for t in templates)
    win_ms_per_step = sum(window_ms.values()) / args.steps
    achieved = alg_bytes / (win_ms_per_step / 1e3) / 1e9
    per_window = {workloads.WINDOW_OF_TEMPLATE[t]: {
        "evals": evals_step[t], "ms": window_ms[t] / args.steps,
        "gbs": evals_step[t] * workloads.BYTES_PER_EVAL[t] / (window_ms[t] / args.steps / 1e3) / 1e9,
        "evals_per_s": evals_step[t] / (window_ms[t] / args.steps / 1e3),
        "stage_ms": ref_stats[t].as_dict()["stage_ms"],
        "exact_nodes": ref_stats[t].exact_nodes, "fp64_nodes": ref_stats[t].fp64_nodes,
        "scan_rounds": ref_stats[t].scan_rounds, "fp64_rechecks": ref_stats[t].fp64_rechecks}
        for t in templates}

    # ---- e2e through the host-buffer C ABI (pinned host memory) ----
    e2e = None
    if not args.skip_e2e:
        host_inp = {t: wl.host_inputs(t) for t in templates}
        ncc_h = host_inp[templates[0]].new_nccresult()
        pinned_ncc = torch.empty(ncc_h.nbytes, dtype=torch.uint8, pin_memory=True).numpy()
        ncc_h = pinned_ncc.view(abi.NCCRESULT_DTYPE)
        for t in templates:   # warm
            ctx.vertical_line_locus(host_inp[t], ncc_h, None, args.kernel)
        img_bytes = sum(a.nbytes for k in ("img", "mag", "ori") for a in wl.host[k])
        grid_bytes = wl.host["wgs"].nbytes + wl.host["pts"].nbytes + wl.gp3.nbytes + ncc_h.nbytes
        h2d = len(templates) * (img_bytes + grid_bytes)
        d2h = len(templates) * ncc_h.nbytes
        torch.cuda.synchronize(dev)
        barrier(world)
        t_e2e = time.perf_counter()
        for _ in range(args.e2e_steps):
            for t in templates:
                ctx.vertical_line_locus(host_inp[t], ncc_h, None, args.kernel)
        e2e_ms = (time.perf_counter() - t_e2e) * 1e3
        e2e_ms = max_over_ranks(world, e2e_ms)
        e2e_val = sum_over_ranks(world, sum(evals_step.values()) * args.e2e_steps) / (e2e_ms / 1e3)
        e2e = {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "steps": args.e2e_steps,
               "timing": "host wall clock around synchronous C-ABI calls"}

    # ---- plain FP64 GPU drop-in on the same workload + parity ----
    fp64 = None
    if not args.skip_fp64 and rank == 0:
        from tests.cases import field_mismatch
        plain_ms, plain_evals = 0.0, 0
        mism, n_valid, n_same, n_ties = {}, 0, 0, 0
        for t in templates:
            wl.d_ncc.zero_()
            torch.cuda.synchronize(dev)
            e2 = torch.cuda.Event(enable_timing=True)
            e3 = torch.cuda.Event(enable_timing=True)
            e2.record(stream)
            st = ctx.vertical_line_locus_device(descs[t], wl.d_gp3.data_ptr(), wl.d_ncc.data_ptr(),
                                                None, None, "plain", stats=True)
            e3.record(stream)
            torch.cuda.synchronize(dev)
            plain_ms += e2.elapsed_time(e3)
            plain_evals += st.evals
            ncc_plain = workloads.ncc_host(wl)
            ncc_split = gpu_ncc[t]
            mism[workloads.WINDOW_OF_TEMPLATE[t]] = field_mismatch(ncc_plain, ncc_split)
            valid = (ncc_plain["check_height_change"] > 0) & (ncc_plain["result4"] > 0)
            same_h = (ncc_plain["result2"] == ncc_split["result2"]) & \
                     (ncc_plain["result0"] == ncc_split["result0"])
            n_valid += int(valid.sum())
            n_same += int((same_h & valid).sum())
            n_ties += int((valid & (ncc_plain["result0"] == ncc_plain["result1"])).sum())
        plain_rate = plain_evals / (plain_ms / 1e3)
        fp64 = {"value": plain_rate, "unit": UNIT, "ms_per_step": plain_ms,
                "speedup_split_vs_fp64": value / world / plain_rate,
                "mismatched_fields_per_window": mism,
                "identical_peak_rate": n_same / n_valid if n_valid else None,
                "tie_rate": n_ties / max(1, n_valid),
                "tie_note": "nodes whose two top peaks quantise to the same rho*1000 in the "
                            "FP64 kernel (the reference's own ties); their heights are identical too",
                "nodes_with_peaks": n_valid}

    # ---- FP32 window error against FP64, slot by slot, on a band of rows ----
    accuracy = None
    cpu = None
    leg = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        leg = ReferenceLeg(wl, templates)
        if leg.ok:
            accuracy = slot_accuracy(ctx, wl, templates, leg.r0, leg.rows)
            leg.run(rows=2)
            cpu = leg.run()
            cpu["parity_vs_gpu"] = leg.parity(gpu_ncc, {"mag": wl.host["mag"], "ori": wl.host["ori"]})
        else:
            cpu = leg.run()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": elapsed_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 window sums, f64 RPC and decisions", "data": "synthetic",
            "config": config_block(args, wl),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak,
                         "traffic": traffic_per_launch(evals_step, templates),
                         "traffic_unit": "bytes per window launch (mean of the step's windows)",
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                           "of the window kernel's full C2 launches (one-pass "
                                           "capture), per evaluation, times this step's "
                                           "evaluations",
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback",
                         "kernel": "window_kernel", "per_window": per_window},
            "e2e": e2e,
            "gpu_launches": int(launches),
            "tuning": tuned["tuning"] if tuned else None,
            "fp64_rechecks_per_step": rechecks / args.steps,
            "fp64_plain_gpu": fp64,
            "accuracy_vs_fp64": accuracy,
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    barrier(world)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# batched multi-level configurations (C3 ragged tiles, C4 pyramid)
# ---------------------------------------------------------------------------
def run_multi(args):
    """C3 / C4: the workload's levels matched in one pass of the split
    pipeline per window size (a CUDA graph each, vll_plan_run, replayed back
    to back) after the autotuner has chosen the window kernel's launch shape.
    A persistent window launch serves its levels at the footprint budget of
    the largest window among them, so the 7x7 and 11x11 levels of C4 go to
    two passes.  Reported beside it: the same levels as separate per-level
    split calls, and the plain FP64 kernel per level on a sample of levels
    (with identical-peak and tie rates)."""
    world, rank, local = dist_setup(args.gpus)
    import torch
    from setsm_b200 import abi, autotune, vll, workloads
    dev = torch.device("cuda", local)
    ctx = vll.Context(local)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    t0 = time.time()
    build = workloads.build_c3 if args.config == "c3" else workloads.build_c4
    mw = build(ctx, device=f"cuda:{local}", seed=1 + rank)
    log(f"[rank {rank}] workload {args.config}: {len(mw.levels)} levels, {mw.n_nodes} nodes, "
        f"built in {time.time() - t0:.1f} s")
    ios = mw.ios()
    # tune on a spread of levels holding about 1e9 height slots
    slots = [lv.slots(lv.host_desc_kwargs["step"]) for lv in mw.levels]
    stride = max(1, int(math.ceil(sum(slots) / 1e9)))
    tuned = autotune.tune(ctx, ios[::stride], repeats=2)
    log(f"[rank {rank}] tuning {tuned['tuning']} ({tuned.get('tuned_s', 'cached')} s)")
    groups = {}
    for i, lv in enumerate(mw.levels):
        groups.setdefault(lv.template, []).append(i)
    groups = list(groups.values())
    acc = np.zeros(len(ios), dtype=np.int64)
    evals_step = 0
    for g in groups:
        a, st0 = ctx.batch([ios[i] for i in g])
        acc[g] = a
        evals_step += int(st0.evals)
    plans = [(g, ctx.plan([ios[i] for i in g])) for g in groups]
    for _ in range(max(3, args.warmup)):
        for _, plan in plans:
            plan.run(wait=False)
    torch.cuda.synchronize(dev)
    barrier(world)
    clocks = Clocks(local)
    clocks.start()
    launches0 = ctx.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        for _, plan in plans:
            plan.run(wait=False)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    clk = clocks.stop()
    launches = ctx.launch_count() - launches0
    ms = max_over_ranks(world, e0.elapsed_time(e1))
    acc2 = np.zeros_like(acc)
    for g, plan in plans:
        acc2[g] = plan.run()[0]
    assert (acc2 == acc).all()
    value = sum_over_ranks(world, evals_step * args.steps) / (ms / 1e3)
    ncc_batch = [lv.d_ncc.cpu().numpy().view(abi.NCCRESULT_DTYPE).copy() for lv in mw.levels]
    # the same levels as separate split calls (one pipeline per level)
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    per_level = []
    for lv in mw.levels:
        stl = ctx.vertical_line_locus_device(lv.desc, lv.d_gp3.data_ptr(), lv.d_ncc.data_ptr(),
                                             None, None, "split", stats=True)
        per_level.append(stl)
    e3.record(stream)
    torch.cuda.synchronize(dev)
    per_level_ms = e2.elapsed_time(e3)
    # the separate calls' records against the batch's, level by level
    parity = {"levels": len(mw.levels), "nodes": int(mw.n_nodes), "fields_mismatched": {},
              "accessable_equal": all(int(per_level[i].accessable_grid) == int(acc[i])
                                      for i in range(len(mw.levels)))}
    for i, lv in enumerate(mw.levels):
        got = lv.d_ncc.cpu().numpy().view(abi.NCCRESULT_DTYPE)
        for k, v in cases_field_mismatch(got, ncc_batch[i]).items():
            parity["fields_mismatched"][k] = parity["fields_mismatched"].get(k, 0) + v
    level_rows = [{"level": lv.name, "nodes": int(lv.n_nodes), "evals": int(per_level[i].evals),
                   "accessable": int(acc[i])} for i, lv in enumerate(mw.levels)]
    # plain FP64 per level on a sample of levels (about 1e9 evaluations at most)
    fp64 = None
    if not args.skip_fp64 and rank == 0:
        order = sorted(range(len(mw.levels)), key=lambda i: mw.levels[i].n_nodes)
        sample, ev_s, ms_s, same, valid_n, ties = [], 0, 0.0, 0, 0, 0
        for i in order:
            lv = mw.levels[i]
            e4 = torch.cuda.Event(enable_timing=True)
            e5 = torch.cuda.Event(enable_timing=True)
            e4.record(stream)
            stp = ctx.vertical_line_locus_device(lv.desc, lv.d_gp3.data_ptr(), lv.d_ncc.data_ptr(),
                                                 None, None, "plain", stats=True)
            e5.record(stream)
            torch.cuda.synchronize(dev)
            ms_s += e4.elapsed_time(e5)
            ev_s += stp.evals
            nf = lv.d_ncc.cpu().numpy().view(abi.NCCRESULT_DTYPE)
            nb = ncc_batch[i]
            v = (nf["check_height_change"] > 0) & (nf["result4"] > 0)
            same += int(((nf["result2"] == nb["result2"]) & (nf["result0"] == nb["result0"]))[v].sum())
            valid_n += int(v.sum())
            ties += int((v & (nf["result0"] == nf["result1"])).sum())
            sample.append(lv.name)
            if ev_s >= args.fp64_evals:
                break
        fp64 = {"value": ev_s / (ms_s / 1e3), "unit": UNIT, "levels": sample,
                "evals": int(ev_s), "identical_peak_rate": same / max(1, valid_n),
                "tie_rate": ties / max(1, valid_n), "timing": "per-level launches, CUDA events"}
    if rank == 0:
        wins = sorted({lv.template for lv in mw.levels})
        alg = sum(workloads.BYTES_PER_EVAL[t] * 1.0 for t in wins) / len(wins)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 window sums, f64 RPC and decisions", "data": "synthetic",
            "config": {"workload": {
                "c3": "C3: 64 ragged stereo tiles (grids 128^2-2048^2 log-uniform at 2 m, images "
                      "4 px per node, convergence 20-40 deg, own DEM and TIN ranges K 8-512 at "
                      "0.5 m), 7x7, one persistent launch per step, CUDA graph",
                "c4": "C4: 5-level pyramid of a 16384^2 pair (9x9 sigma 1.5 downsample), grids "
                      "32 m -> 2 m, K 256 -> 16, each finer level's ranges +-3 sigma around the "
                      "previous level's matches (SelectMPs, TIN) interpolated at its nodes, "
                      "7x7 and 11x11 at every level, one persistent launch per window size "
                      "per step (two CUDA graphs replayed back to back)"}[args.config],
                "levels": len(mw.levels), "nodes": mw.n_nodes, "evals_per_step": evals_step,
                "tuning": tuned["tuning"], "l2": "inputs larger than L2",
                "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": evals_step * alg / (ms / args.steps / 1e3) / 1e9,
                         "peak": json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
                         if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else 6650.0,
                         "unit": "GB/s", "note": "whole pipeline time (graph replay), mean "
                                                 "algorithmic bytes per evaluation of the windows"},
            "per_level_split_calls": {"value": evals_step / (per_level_ms / 1e3), "unit": UNIT,
                                      "ms": per_level_ms},
            "levels": level_rows,
            "parity_batch_vs_calls": parity,
            "range_chain": mw.info or None,
            "gpu_launches": int(launches),
            "fp64_plain_gpu": fp64,
            "clocks": clk,
        }
        line["roofline"]["frac"] = line["roofline"]["achieved"] / line["roofline"]["peak"]
        print(json.dumps(line), flush=True)
    for _, plan in plans:
        plan.close()
    barrier(world)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# SGM aggregation (AWNCC with Pyramid_step <= SGM_py)
# ---------------------------------------------------------------------------
def run_sgm(args):
    """AWNCC with semi-global aggregation on the voxel route at level 0
    (SGM_py = 1): the reduced C2 scene (4096^2 pair, 1024^2 grid, TIN ranges),
    InitializeVoxel by the reference on the host (it stays the caller's in
    SETSM), VerticalLineLocus (split) and AWNCC on the GPU, against the
    reference's AWNCC with OpenMP on every host core; every NCCresult field is
    compared.  Metric: voxel slots aggregated per second."""
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import torch
    from oracle import refpy
    from setsm_b200 import vll, workloads
    from tests.cases import field_mismatch
    ctx = vll.Context(0)
    wl = workloads.build("c2_small", ctx, device="cuda:0", seed=1)
    inp = wl.host_inputs(11)
    inp.check_matching_rate = False
    inp.sgm_py = 1
    refpy.set_threads(os.cpu_count() or 1)
    ncc0 = inp.new_nccresult()
    gp3 = inp.gridpt3.copy()
    inp.gridpt3 = gp3
    vox0 = refpy.initialize_voxel(inp, ncc0, None)
    ncc = ncc0.copy()
    vox = vox0.copy()
    ctx.vertical_line_locus(inp, ncc, vox, "split")
    ncc_v, vox_v = ncc.copy(), vox.copy()
    times = []
    for _ in range(max(1, args.warmup)):
        n1 = ncc_v.copy()
        ctx.awncc(inp, n1, vox_v)
    for _ in range(args.steps):
        n1 = ncc_v.copy()
        t = time.perf_counter()
        st = ctx.awncc(inp, n1, vox_v)
        times.append((st.kernel_ms, (time.perf_counter() - t) * 1e3))
    slots = int(vox_v.size)
    dev_ms = statistics.median(t[0] for t in times)
    e2e_ms = statistics.median(t[1] for t in times)
    n_ref = ncc_v.copy()
    t = time.perf_counter()
    refpy.awncc(inp, n_ref, vox_v.copy())
    cpu_s = time.perf_counter() - t
    mism = field_mismatch(n1, n_ref)
    line = {
        "metric": "voxel slots aggregated/s (AWNCC with SGM)", "value": slots / (dev_ms / 1e3),
        "unit": "slots/s", "n_gpus": 1, "steps": args.steps, "warmup": max(1, args.warmup),
        "ms_per_step": dev_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 path costs, f64 arithmetic (the reference's)", "data": "synthetic",
        "config": {"workload": "SGM: reduced C2 scene (4096^2 pair, 1024^2 grid, TIN ranges "
                               "K 8-512 at 0.5 m), voxel route, level 0, 7x7, SGM_py = 1",
                   "nodes": int(wl.n_nodes), "slots": slots},
        "e2e": {"value": slots / (e2e_ms / 1e3), "unit": "slots/s",
                "timing": "host wall clock of vll_awncc_peaks (uploads voxels, downloads "
                          "NCCresult)"},
        "cpu_baseline": {"value": slots / cpu_s, "unit": "slots/s", "cores": os.cpu_count(),
                         "kind": "reference", "sample": f"whole grid, {cpu_s:.2f} s"},
        "parity_mismatch_fields": mism,
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    del torch


def run_variant(args):
    """The orthoimage-window variants on the reduced C2 scene (4096^2 pair at
    0.5 m, 1024^2 grid, node heights from the TIN estimate): seeddem =
    VerticalLineLocus_seeddem at level 0 (5 m template, 11x11 window);
    blunder = VerticalLineLocus_blunder with the blunder level 1 (the level-1
    pyramid built on the GPU) as in DecisionMPs' second call.  GPU: the C ABI
    on host buffers (device time of the raster + node kernels; e2e = host wall
    clock of the call with its copies); CPU: the reference's own function
    with OpenMP on every host core, on the whole grid; outputs compared.
    Metric: grid nodes per second."""
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import copy
    import ctypes as C
    import torch
    from oracle import refpy
    from setsm_b200 import abi, vll, workloads
    from tests.cases import field_mismatch
    ctx = vll.Context(0)
    wl = workloads.build("c2_small", ctx, device="cuda:0", seed=1)
    inp = wl.host_inputs(11)
    kind = args.config
    if kind == "blunder":
        n = wl.d_img[0].shape[0] // 2
        for ci, im in enumerate(inp.images):
            d_b = torch.empty((n, n), dtype=torch.int16, device="cuda:0")
            d_m = torch.empty_like(d_b)
            d_o = torch.empty((n, n), dtype=torch.uint8, device="cuda:0")
            ctx.pyramid_down_device(wl.d_img[ci].data_ptr(), 2 * n, 2 * n, d_b.data_ptr())
            ctx.preprocess_device(d_b.data_ptr(), n, n, d_m.data_ptr(), d_o.data_ptr())
            torch.cuda.synchronize()
            im.image_b = d_b.cpu().numpy().view(np.uint16)
            im.mag_b = d_m.cpu().numpy().view(np.uint16)
        inp.blunder_level = 1
    gp3_0 = inp.gridpt3.copy()

    ncc = np.zeros(inp.n, dtype=np.float32)

    def call():
        # a fresh copy of the UGRID (the calls update it in place), outside the clock
        inp.gridpt3 = gp3_0.copy()
        d = inp.desc()
        t = time.perf_counter()
        if kind == "seeddem":
            st = ctx.seeddem(inp)
        else:
            st = abi.Stats()
            ctx._check(vll.load().vll_vertical_line_locus_blunder(
                ctx._h, C.byref(d), inp.gridpt3.ctypes.data, 1, 0, ncc.ctypes.data, C.byref(st)))
        return st, (time.perf_counter() - t) * 1e3
    for _ in range(max(1, args.warmup)):
        call()
    clocks = Clocks(0)
    clocks.start()
    times = []
    for _ in range(args.steps):
        st, ms = call()
        times.append((st.kernel_ms, ms))
    clk = clocks.stop()
    got = inp.gridpt3.copy()
    dev_ms = statistics.median(t[0] for t in times)
    e2e_ms = statistics.median(t[1] for t in times)
    ref = copy.copy(inp)
    ref.gridpt3 = gp3_0.copy()
    refpy.set_threads(os.cpu_count() or 1)
    t = time.perf_counter()
    want = refpy.vll_seeddem(ref) if kind == "seeddem" else refpy.vll_blunder(ref, 1, False)
    cpu_s = time.perf_counter() - t
    parity = {"ugrid_field_mismatch": field_mismatch(got, ref.gridpt3)}
    if kind == "blunder":
        parity["ncc_float_identical_frac"] = float(np.mean(ncc.view(np.uint32)
                                                           == want.view(np.uint32)))
        parity["ncc_max_abs_diff"] = float(np.abs(ncc.astype(np.float64) - want).max())
        parity["ncc_max_ulps"] = int(np.abs(ncc.view(np.int32).astype(np.int64)
                                            - want.view(np.int32).astype(np.int64)).max())
    n = int(inp.n)
    name = {"seeddem": "VerticalLineLocus_seeddem, level 0, 5 m template (11x11 window)",
            "blunder": "VerticalLineLocus_blunder, blunder level 1, iteration 1"}[kind]
    line = {
        "metric": f"grid nodes/s ({kind})", "value": n / (dev_ms / 1e3), "unit": "nodes/s",
        "n_gpus": 1, "steps": args.steps, "warmup": max(1, args.warmup), "ms_per_step": dev_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (the reference's arithmetic)", "data": "synthetic",
        "config": {"workload": f"{name}: reduced C2 scene (4096^2 pair at 0.5 m, 1024^2 grid, "
                               "TIN height estimate)", "nodes": n},
        "e2e": {"value": n / (e2e_ms / 1e3), "unit": "nodes/s",
                "timing": "host wall clock of the C-ABI call on host buffers (image planes, "
                          "grid and UGRID copied in, UGRID and NCC copied out)"},
        "cpu_baseline": {"value": n / cpu_s, "unit": "nodes/s", "cores": os.cpu_count(),
                         "kind": "reference", "sample": f"whole grid, {cpu_s:.2f} s"},
        "gpu_launches": 2 * args.steps,
        "clocks": clk,
        "parity": parity,
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    del torch


def tin_workload(ctx):
    """The reduced C2 scene (4096^2 pair at 0.5 m, 1024^2 grid at 2 m) with
    matched points on 2 % of the grid nodes (60 % anchored, candidates off the
    truth by up to 25 m, height ranges +-40 m) and their Delaunay TIN.
    Returns (inputs, UGRID, points, triangles)."""
    from setsm_b200 import abi, workloads
    from tests.cases import delaunay
    wl = workloads.build("c2_small", ctx, device="cuda:0", seed=1)
    inp = wl.host_inputs(11)
    rng = np.random.default_rng(5)
    g0 = inp.gridpt3.copy()
    n = len(g0)
    sel = np.sort(rng.choice(n, size=int(0.02 * n), replace=False))
    truth = g0["Height"][sel].astype(np.float64)
    anchor = rng.random(len(sel)) < 0.6
    pts0 = np.zeros(len(sel), dtype=abi.POINT3_DTYPE)
    pts0["x"], pts0["y"] = inp.grid_pts[sel, 0], inp.grid_pts[sel, 1]
    pts0["z"] = np.where(anchor, truth, truth + rng.uniform(-25.0, 25.0, len(sel)))
    pts0["flag"] = 1
    g0["anchor_flag"] = 0
    g0["anchor_flag"][sel] = np.where(anchor, 1, 2)
    g0["minHeight"][sel] = np.floor(truth - 40.0).astype(np.int16)
    g0["maxHeight"][sel] = np.ceil(truth + 40.0).astype(np.int16)
    r = rng.random(n)
    g0["Matched_flag"] = np.where(r < 0.2, 0, np.where(r < 0.4, 4, 1))
    g0["Mean_ortho_ncc"] = rng.integers(-1000, 1000, n).astype(np.int16)
    return inp, g0, pts0, delaunay(pts0)


def run_tin_create(args):
    """TINCreate_list (SubFunctions.cpp:2768-2846) on matched points of the
    reduced C2 grid (1024^2 nodes at 2 m): 2 % of the nodes (21 k points, the
    TIN workload's) and 50 % of them (524 k points), snapped to the grid.
    GPU: vll_tin_create_device on resident points (CUDA events); e2e: the
    host-buffer call; CPU: the reference's own TINCreate_list; the triangle
    lists compared (identical, in order).  Metric: points per second."""
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import torch
    from oracle import refpy
    from setsm_b200 import abi, vll, workloads
    ctx = vll.Context(0)
    inp, _, pts21, _ = tin_workload(ctx)
    bound = np.asarray(inp.boundary, dtype=np.float64)
    res = float(inp.grid_resolution)
    rng = np.random.default_rng(9)
    sel = np.sort(rng.choice(inp.n, size=inp.n // 2, replace=False))
    pts_half = np.zeros(len(sel), dtype=abi.POINT3_DTYPE)
    pts_half["x"], pts_half["y"] = inp.grid_pts[sel, 0], inp.grid_pts[sel, 1]
    pts_half["z"] = inp.gridpt3["Height"][sel]
    pts_half["flag"] = 1
    rows = {}
    for name, pts in (("2%", pts21), ("50%", pts_half)):
        t = time.perf_counter()
        want = refpy.tin_create(pts, bound, res)
        cpu_s = time.perf_counter() - t
        d_pts = torch.from_numpy(pts.view(np.uint8).copy()).cuda()
        cap = 2 * len(pts) + 16
        d_tris = torch.zeros(cap * abi.TRI_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        for _ in range(max(3, args.warmup)):
            ctx.tin_create_device(d_pts.data_ptr(), len(pts), bound, res, d_tris.data_ptr(), cap)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            n = ctx.tin_create_device(d_pts.data_ptr(), len(pts), bound, res, d_tris.data_ptr(),
                                      cap)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        got = d_tris[:n * abi.TRI_DTYPE.itemsize].cpu().numpy().view(abi.TRI_DTYPE)
        t = time.perf_counter()
        for _ in range(args.steps):
            host = ctx.tin_create(pts, bound, res)
        e2e_ms = (time.perf_counter() - t) * 1e3 / args.steps
        rows[name] = {"points": int(len(pts)), "triangles": int(n), "device_ms": ms,
                      "points_per_s": len(pts) / (ms / 1e3), "e2e_ms": e2e_ms,
                      "cpu_reference_ms": cpu_s * 1e3,
                      "cpu_points_per_s": len(pts) / cpu_s,
                      "identical_to_reference": bool(got.tobytes() == want.tobytes() and
                                                     host.tobytes() == want.tobytes())}
    big = rows["50%"]
    line = {
        "metric": "points/s (TINCreate_list)", "value": big["points_per_s"], "unit": "points/s",
        "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup),
        "ms_per_step": big["device_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64 grid coordinates", "data": "synthetic",
        "config": {"workload": "matched points snapped to the reduced C2 grid (1024^2 nodes at "
                               "2 m): 2 % and 50 % of the nodes; value: the 50 % set"},
        "sets": rows,
        "e2e": {"value": big["points"] / (big["e2e_ms"] / 1e3), "unit": "points/s",
                "h2d_bytes_per_step": big["points"] * abi.POINT3_DTYPE.itemsize,
                "d2h_bytes_per_step": big["triangles"] * abi.TRI_DTYPE.itemsize},
        "cpu_baseline": {"value": big["cpu_points_per_s"], "unit": "points/s", "cores": 1,
                         "kind": "reference", "sample": "the same 50 % point set"},
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def run_height_range(args):
    """SetHeightRange (setsm_code.cpp:9851-10255) on the TIN workload of
    tin_workload (1024^2 grid, 21 k points, 41.8 k triangles), level 0,
    iteration 2, MPP 1.5.  GPU: the C ABI on host buffers (host wall clock of
    the call, copies included: the call waits); CPU: the reference's own
    SetHeightRange (mostly sequential); returned grids compared.  Metric:
    grid nodes per second."""
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import copy
    import torch
    from oracle import refpy
    from setsm_b200 import vll
    from tests.cases import field_mismatch
    ctx = vll.Context(0)
    inp, g0, pts, tris = tin_workload(ctx)
    it, mpp = 2, 1.5
    n = int(inp.n)
    d = inp.desc()
    d_pts = torch.from_numpy(pts.view(np.uint8).copy()).cuda()
    d_tris = torch.from_numpy(tris.view(np.uint8).copy()).cuda()
    d_g0 = torch.from_numpy(g0.view(np.uint8).copy()).cuda()
    d_g = torch.empty_like(d_g0)
    d_out = torch.empty(n * 20, dtype=torch.uint8, device="cuda:0")

    def dev_call():
        d_g.copy_(d_g0)
        torch.cuda.synchronize()
        t = time.perf_counter()
        ctx.set_height_range_device(d, d_pts.data_ptr(), len(pts), d_tris.data_ptr(), len(tris),
                                    d_g.data_ptr(), d_out.data_ptr(), it, mpp, False)
        return (time.perf_counter() - t) * 1e3
    for _ in range(max(1, args.warmup)):
        dev_call()
    dev_ms = statistics.median(dev_call() for _ in range(args.steps))

    def call():
        inp.gridpt3 = g0.copy()
        t = time.perf_counter()
        out, ext = ctx.set_height_range(inp, pts, tris, it, mpp, False)
        return (time.perf_counter() - t) * 1e3, out, ext
    for _ in range(max(1, args.warmup)):
        call()
    clocks = Clocks(0)
    clocks.start()
    times = []
    lc0 = vll.load().vll_launch_count(ctx._h)
    for _ in range(args.steps):
        ms, out, ext = call()
        times.append(ms)
    launches = vll.load().vll_launch_count(ctx._h) - lc0
    clk = clocks.stop()
    ms = statistics.median(times)
    ref = copy.copy(inp)
    ref.gridpt3 = g0.copy()
    refpy.set_threads(os.cpu_count() or 1)
    t = time.perf_counter()
    want, wext = refpy.set_height_range(ref, pts, tris, it, mpp, False)
    cpu_s = time.perf_counter() - t
    line = {
        "metric": "grid nodes/s (SetHeightRange)", "value": n / (dev_ms / 1e3), "unit": "nodes/s",
        "n_gpus": 1, "steps": args.steps, "warmup": max(1, args.warmup), "ms_per_step": dev_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (the reference's arithmetic)", "data": "synthetic",
        "config": {"workload": "SetHeightRange: 1024^2 grid at 2 m, 21 k matched points, "
                               "Delaunay TIN, level 0, iteration 2, MPP 1.5",
                   "nodes": n, "points": int(len(pts)), "triangles": int(len(tris))},
        "e2e": {"value": n / (ms / 1e3), "unit": "nodes/s",
                "timing": "host wall clock of vll_set_height_range on host buffers (copies "
                          "included; value: vll_set_height_range_device on resident data)"},
        "cpu_baseline": {"value": n / cpu_s, "unit": "nodes/s", "cores": os.cpu_count(),
                         "kind": "reference", "sample": f"whole grid, {cpu_s:.3f} s"},
        "gpu_launches": int(launches),
        "clocks": clk,
        "parity": {"result_field_mismatch": field_mismatch(out, want),
                   "extent_identical": ext == wext},
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    del torch


def run_tin_blunder(args):
    """blunder_detection_TIN (setsm_code.cpp:9158-9787) on the TIN workload of
    tin_workload (1024^2 grid, 21 k points, 41.8 k triangles) with point flags
    0 (10 % already 1) and an orthoimage NCC per node over [-1, 1], level 0,
    iteration 1, flag_blunder on, Hinterval 60.  value: the device entry
    point on resident buffers (host clock around the call, which waits; the
    count of calls whose threshold band made it re-run the point pass is
    reported);
    e2e: the host-buffer entry point (copies included); CPU: the reference's
    own blunder_detection_TIN with OpenMP on every host core.  Flags, the new
    blunder marks, UGRID, counts and extent compared.  Metric: matched points
    per second."""
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import copy
    import torch
    from oracle import refpy
    from setsm_b200 import vll
    from tests.cases import field_mismatch
    ctx = vll.Context(0)
    inp, g0, pts0, tris = tin_workload(ctx)
    rng = np.random.default_rng(23)
    pts0["flag"] = np.where(rng.random(len(pts0)) < 0.1, 1, 0)
    n = int(inp.n)
    oncc = np.where(rng.random(n) < 0.2, rng.uniform(-1.0, 0.3, n),
                    rng.uniform(0.3, 1.0, n)).astype(np.float32)
    it, fb, cbl, hint = 1, True, 1, 60.0
    d = inp.desc()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()
    d_pts0, d_tris, d_g0, d_o = dev(pts0), dev(tris), dev(g0), dev(oncc)
    d_pts, d_g = torch.empty_like(d_pts0), torch.empty_like(d_g0)
    d_det = torch.empty(len(pts0), dtype=torch.uint8, device="cuda:0")

    def dev_call():
        d_pts.copy_(d_pts0)
        d_g.copy_(d_g0)
        d_det.zero_()
        torch.cuda.synchronize()
        counts, zext = np.zeros(2, np.int64), np.array([1e5, -1e5])
        t = time.perf_counter()
        ctx.blunder_detection_tin_device(d, it, d_o.data_ptr(), fb, cbl, hint, d_pts.data_ptr(),
                                         d_det.data_ptr(), len(pts0), d_tris.data_ptr(),
                                         len(tris), d_g.data_ptr(), counts, zext)
        return (time.perf_counter() - t) * 1e3
    for _ in range(max(1, args.warmup)):
        dev_call()
    rr0 = vll.load().vll_tin_rerun_count(ctx._h)
    dev_ms = statistics.median(dev_call() for _ in range(args.steps))
    reruns = vll.load().vll_tin_rerun_count(ctx._h) - rr0

    def call():
        inp.gridpt3 = g0.copy()
        pts, det = pts0.copy(), np.zeros(len(pts0), np.uint8)
        counts, zext = np.zeros(2, np.int64), np.array([1e5, -1e5])
        t = time.perf_counter()
        ctx.blunder_detection_tin(inp, it, oncc, fb, cbl, hint, pts, det, tris, counts, zext)
        return (time.perf_counter() - t) * 1e3, (pts, det, inp.gridpt3, counts, zext)
    for _ in range(max(1, args.warmup)):
        call()
    clocks = Clocks(0)
    clocks.start()
    times = []
    lc0 = vll.load().vll_launch_count(ctx._h)
    for _ in range(args.steps):
        ms, got = call()
        times.append(ms)
    launches = vll.load().vll_launch_count(ctx._h) - lc0
    clk = clocks.stop()
    ms = statistics.median(times)
    ref = copy.copy(inp)
    ref.gridpt3 = g0.copy()
    r_pts, r_det = pts0.copy(), np.zeros(len(pts0), np.uint8)
    r_counts, r_zext = np.zeros(2, np.int64), np.array([1e5, -1e5])
    refpy.set_threads(os.cpu_count() or 1)
    t = time.perf_counter()
    refpy.blunder_detection_tin(ref, it, oncc, fb, cbl, hint, r_pts, r_det, tris, r_counts,
                                r_zext)
    cpu_s = time.perf_counter() - t
    pts, det, gp3, counts, zext = got
    npt = len(pts0)
    line = {
        "metric": "matched points/s (blunder_detection_TIN)", "value": npt / (dev_ms / 1e3),
        "unit": "points/s", "n_gpus": 1, "steps": args.steps, "warmup": max(1, args.warmup),
        "ms_per_step": dev_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (the reference's arithmetic)", "data": "synthetic",
        "config": {"workload": "blunder_detection_TIN: 1024^2 grid at 2 m, 21 k matched points, "
                               "Delaunay TIN, level 0, iteration 1, Hinterval 60",
                   "nodes": n, "points": npt, "triangles": int(len(tris))},
        "e2e": {"value": npt / (ms / 1e3), "unit": "points/s",
                "h2d_bytes_per_step": int(pts0.nbytes + tris.nbytes + oncc.nbytes + npt),
                "d2h_bytes_per_step": int(pts0.nbytes + npt + 9 * npt),
                "timing": "host wall clock of vll_blunder_detection_tin on host buffers (copies "
                          "included: points, triangles, the ortho NCC grid and the marks up; "
                          "points, marks and the anchor_flag writes down; value: "
                          "vll_blunder_detection_tin_device on resident data)"},
        "cpu_baseline": {"value": npt / cpu_s, "unit": "points/s", "cores": os.cpu_count(),
                         "kind": "reference", "sample": f"whole TIN, {cpu_s:.4f} s"},
        "gpu_launches": int(launches),
        "clocks": clk,
        "parity": {"flags_identical": bool(np.array_equal(pts["flag"], r_pts["flag"])),
                   "detected_identical": bool(np.array_equal(det, r_det)),
                   "gridpt3_field_mismatch": field_mismatch(gp3, ref.gridpt3),
                   "counts_identical": bool(np.array_equal(counts, r_counts)),
                   "extent_identical": bool(np.array_equal(zext, r_zext)),
                   "new_blunders": int(det.sum()),
                   "point_pass_reruns": f"{reruns} of {args.steps} timed device calls"},
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    del torch


def run_voxel_iter(args):
    """One matching iteration of the voxel route at level 0 with SGM
    (SGM_py = 1) on the reduced C2 scene (4096^2 pair, 1024^2 grid, TIN
    ranges, 7x7): InitializeVoxel -> VerticalLineLocus (split) -> AWNCC with
    semi-global aggregation.  value: the three calls on device-resident data
    (vll_initialize_voxel_device, vll_vertical_line_locus_device,
    vll_awncc_peaks_device; host clock around them, synchronized); e2e: the
    host-buffer entry points (copies included); CPU: the reference's own
    InitializeVoxel, VerticalLineLocus and AWNCC with OpenMP on every host core
    on the whole grid; the final NCCresult compared.  Metric: node x height
    evaluations per second of the iteration."""
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import copy
    import torch
    from oracle import refpy
    from setsm_b200 import abi, vll, workloads
    from tests.cases import field_mismatch
    ctx = vll.Context(0)
    wl = workloads.build("c2_small", ctx, device="cuda:0", seed=1)
    n = int(wl.n_nodes)
    d = wl.device_desc(11)
    d.check_matching_rate = 0
    d.sgm_py = 1
    d.iteration = 1
    g = wl.gp3
    hs = wl.cfg["height_step"]
    cap = int(((g["maxHeight"].astype(np.int64) - g["minHeight"].astype(np.int64) + 4) / hs
               + 4).clip(0).sum())
    d_gp3_0 = wl.d_gp3.clone()
    d_vox = torch.empty(cap * 4, dtype=torch.uint8, device="cuda:0")
    d_off = torch.empty(n + 1, dtype=torch.int64, device="cuda:0")
    gp3_p, ncc_p = wl.d_gp3.data_ptr(), wl.d_ncc.data_ptr()

    def device_step():
        wl.d_gp3.copy_(d_gp3_0)
        wl.d_ncc.zero_()
        torch.cuda.synchronize()
        t = time.perf_counter()
        ctx.initialize_voxel_device(d, gp3_p, ncc_p, None, d_vox.data_ptr(), cap,
                                    d_off.data_ptr())
        st = ctx.vertical_line_locus_device(d, gp3_p, ncc_p, d_vox.data_ptr(), d_off.data_ptr(),
                                            kernel="split", stats=True)
        ctx.awncc_device(d, gp3_p, ncc_p, d_vox.data_ptr(), d_off.data_ptr())
        torch.cuda.synchronize()
        return (time.perf_counter() - t) * 1e3, int(st.evals)
    for _ in range(max(1, args.warmup)):
        device_step()
    clocks = Clocks(0)
    clocks.start()
    times, evals = [], 0
    lc0 = vll.load().vll_launch_count(ctx._h)
    for _ in range(args.steps):
        ms, evals = device_step()
        times.append(ms)
    launches = vll.load().vll_launch_count(ctx._h) - lc0
    clk = clocks.stop()
    dev_ms = statistics.median(times)
    dev_ncc = wl.d_ncc.cpu().numpy().view(abi.NCCRESULT_DTYPE).copy()
    # host-buffer entry points (e2e): resident (image planes and grid arrays
    # sent once, the voxel packing kept on the device between the three
    # calls; records cross every call), and copying everything every call
    inp = wl.host_inputs(11)
    inp.check_matching_rate = False
    inp.sgm_py = 1
    g0 = inp.gridpt3.copy()
    e2e, e2e_copy = [], []
    ctx.set_residency(planes=True, voxels=True)
    for _ in range(max(1, args.warmup) + args.steps):
        inp.gridpt3 = g0.copy()
        ncc = inp.new_nccresult()
        ctx.resident_reset()
        t = time.perf_counter()
        ctx.initialize_voxel_resident(inp, ncc)
        ctx.vertical_line_locus(inp, ncc, None, "split")
        ctx.awncc(inp, ncc, None)
        e2e.append((time.perf_counter() - t) * 1e3)
    e2e = e2e[max(1, args.warmup):]
    ncc_resident = ncc.copy()
    ctx.set_residency()
    for _ in range(2):
        inp.gridpt3 = g0.copy()
        ncc = inp.new_nccresult()
        t = time.perf_counter()
        vox = ctx.initialize_voxel(inp, ncc, None)
        ctx.vertical_line_locus(inp, ncc, vox, "split")
        ctx.awncc(inp, ncc, vox)
        e2e_copy.append((time.perf_counter() - t) * 1e3)
    e2e_ms = statistics.median(e2e)
    e2e_copy_ms = min(e2e_copy)
    rec_bytes = n * (abi.UGRID_DTYPE.itemsize + abi.NCCRESULT_DTYPE.itemsize)
    ref = copy.copy(inp)
    ref.gridpt3 = g0.copy()
    ref_ncc = ref.new_nccresult()
    refpy.set_threads(os.cpu_count() or 1)
    t = time.perf_counter()
    rvox = refpy.initialize_voxel(ref, ref_ncc, None)
    refpy.vertical_line_locus(ref, ref_ncc, rvox)
    refpy.awncc(ref, ref_ncc, rvox)
    cpu_s = time.perf_counter() - t
    line = {
        "metric": "node x height evals/s (voxel-route iteration: InitializeVoxel + "
                  "VerticalLineLocus + AWNCC with SGM)",
        "value": evals / (dev_ms / 1e3), "unit": "evals/s", "n_gpus": 1, "steps": args.steps,
        "warmup": max(1, args.warmup), "ms_per_step": dev_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 window sums, f64 RPC and decisions (the reference's)", "data": "synthetic",
        "config": {"workload": "voxel-route iteration 1 at level 0, SGM_py 1: reduced C2 scene "
                               "(4096^2 pair, 1024^2 grid, TIN ranges K 8-512 at 0.5 m), 7x7",
                   "nodes": n, "evals": evals},
        "e2e": {"value": evals / (e2e_ms / 1e3), "unit": "evals/s", "steps": len(e2e),
                "h2d_bytes_per_step": int(3 * rec_bytes), "d2h_bytes_per_step": int(3 * rec_bytes),
                "timing": "host wall clock of vll_initialize_voxel + vll_vertical_line_locus + "
                          "vll_awncc_peaks on host buffers with residency (image planes and grid "
                          "arrays sent on the first call, voxel packing kept on the device; "
                          "UGRID and NCCresult up and down every call), median of the steps"},
        "e2e_copy_every_call": {"value": evals / (e2e_copy_ms / 1e3), "unit": "evals/s",
                                "timing": "the same calls without residency (planes, grid "
                                          "arrays and voxels up and voxels down every call)"},
        "cpu_baseline": {"value": evals / cpu_s, "unit": "evals/s", "cores": os.cpu_count(),
                         "kind": "reference", "sample": f"whole grid, {cpu_s:.1f} s"},
        "gpu_launches": int(launches),
        "clocks": clk,
        "parity": {"device_vs_reference": field_mismatch(dev_ncc, ref_ncc),
                   "host_api_vs_reference": field_mismatch(ncc, ref_ncc),
                   "resident_host_api_vs_reference": field_mismatch(ncc_resident, ref_ncc)},
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    del torch


def run_select_mps(args):
    """SelectMPs (setsm_code.cpp:8535-8895) on the reduced C2 scene: the
    peaks of the 7x7 memory-tight matching (split kernel) of its 1024^2 grid,
    level 0, iteration 1, its UGRID.  GPU: the C ABI on host buffers (host
    wall clock of the call, copies included: the call waits); CPU: the
    reference's SelectMPs (sequential); points and UGRID compared.  Metric:
    grid nodes per second (value: device-resident inputs)."""
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import copy
    import torch
    from oracle import refpy
    from setsm_b200 import vll, workloads
    from tests.cases import field_mismatch
    ctx = vll.Context(0)
    wl = workloads.build("c2_small", ctx, device="cuda:0", seed=1)
    inp = wl.host_inputs(11)
    ncc = inp.new_nccresult()
    ctx.vertical_line_locus(inp, ncc, None, "split")
    g0 = inp.gridpt3.copy()
    sel_args = (0.6, 0.2, 0.8, 0.7, 1, 1.5, 1, 10.0)
    # device-resident form: NCCresult, UGRID and grid points on the GPU
    n = int(inp.n)
    d = wl.device_desc(11)
    d_ncc = torch.from_numpy(ncc.view(np.uint8).copy()).cuda()
    d_g0 = torch.from_numpy(g0.view(np.uint8).copy()).cuda()
    d_g = torch.empty_like(d_g0)
    d_pts = torch.empty(n * 32, dtype=torch.uint8, device="cuda:0")

    def dev_call():
        d_g.copy_(d_g0)
        torch.cuda.synchronize()
        t = time.perf_counter()
        ctx.select_mps_device(d, d_ncc.data_ptr(), d_g.data_ptr(), d_pts.data_ptr(), n, *sel_args)
        return (time.perf_counter() - t) * 1e3
    for _ in range(max(1, args.warmup)):
        dev_call()
    dev_ms = statistics.median(dev_call() for _ in range(args.steps))

    def call():
        inp.gridpt3 = g0.copy()
        t = time.perf_counter()
        pts = ctx.select_mps(inp, ncc, *sel_args)
        return (time.perf_counter() - t) * 1e3, pts
    for _ in range(max(1, args.warmup)):
        call()
    clocks = Clocks(0)
    clocks.start()
    times = []
    lc0 = vll.load().vll_launch_count(ctx._h)
    for _ in range(args.steps):
        ms, pts = call()
        times.append(ms)
    launches = vll.load().vll_launch_count(ctx._h) - lc0
    clk = clocks.stop()
    ms = statistics.median(times)
    ref = copy.copy(inp)
    ref.gridpt3 = g0.copy()
    t = time.perf_counter()
    _, want = refpy.select_mps(ref, ncc, *sel_args)
    cpu_s = time.perf_counter() - t
    same = len(pts) == len(want) and all(np.array_equal(pts[f], want[f])
                                         for f in ("x", "y", "z", "flag"))
    line = {
        "metric": "grid nodes/s (SelectMPs)", "value": n / (dev_ms / 1e3), "unit": "nodes/s",
        "n_gpus": 1, "steps": args.steps, "warmup": max(1, args.warmup), "ms_per_step": dev_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (the reference's arithmetic)", "data": "synthetic",
        "config": {"workload": "SelectMPs: peaks of the 7x7 memory-tight matching of the reduced "
                               "C2 scene (1024^2 grid), level 0, iteration 1",
                   "nodes": n, "points": int(len(pts))},
        "e2e": {"value": n / (ms / 1e3), "unit": "nodes/s",
                "timing": "host wall clock of vll_select_mps on host buffers (copies included; "
                          "value: vll_select_mps_device on resident data, host clock)"},
        "cpu_baseline": {"value": n / cpu_s, "unit": "nodes/s", "cores": 1, "kind": "reference",
                         "sample": f"whole grid, {cpu_s:.3f} s (the reference's loop is serial)"},
        "gpu_launches": int(launches),
        "clocks": clk,
        "parity": {"points_identical": bool(same),
                   "ugrid_field_mismatch": field_mismatch(inp.gridpt3, ref.gridpt3)},
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    del torch


def run_ortho_tin(args):
    """Ortho_blunder (TIN-triangle orthoimage height search, setsm_code.cpp:
    8028-8533) on the reduced C2 scene (4096^2 pair at 0.5 m, 1024^2 grid at
    2 m): matched points on 2 % of the grid nodes (60 % anchored, candidates
    off the truth by up to 25 m, height ranges +-40 m), their Delaunay TIN,
    MPP 1.5.  GPU: the C ABI on host buffers, timed by the host wall clock of
    the call (each round ends by reading a flag, so the call waits for the GPU
    anyway); CPU: the
    reference's Ortho_blunder with OpenMP on every host core; outputs
    compared.  Metric: triangles per second (TIN triangles / call time)."""
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import copy
    import torch
    from oracle import refpy
    from setsm_b200 import vll
    from tests.cases import field_mismatch
    ctx = vll.Context(0)
    inp, g0, pts0, tris = tin_workload(ctx)
    mpp = 1.5

    def call():
        inp.gridpt3 = g0.copy()
        pts = pts0.copy()
        t = time.perf_counter()
        rounds = ctx.ortho_blunder(inp, mpp, pts, tris)
        return (time.perf_counter() - t) * 1e3, rounds, pts
    for _ in range(max(1, args.warmup)):
        call()
    clocks = Clocks(0)
    clocks.start()
    times = []
    lc0 = vll.load().vll_launch_count(ctx._h)
    for _ in range(args.steps):
        ms, rounds, pts = call()
        times.append(ms)
    launches = vll.load().vll_launch_count(ctx._h) - lc0
    clk = clocks.stop()
    ms = statistics.median(times)
    ref = copy.copy(inp)
    ref.gridpt3 = g0.copy()
    ref_pts = pts0.copy()
    refpy.set_threads(os.cpu_count() or 1)
    t = time.perf_counter()
    refpy.ortho_blunder(ref, mpp, ref_pts, tris.copy())
    cpu_s = time.perf_counter() - t
    same_pts = all(np.array_equal(pts[f], ref_pts[f]) for f in ("x", "y", "z", "flag"))
    line = {
        "metric": "TIN triangles/s (Ortho_blunder)", "value": len(tris) / (ms / 1e3),
        "unit": "triangles/s", "n_gpus": 1, "steps": args.steps, "warmup": max(1, args.warmup),
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (the reference's arithmetic)", "data": "synthetic",
        "config": {"workload": "Ortho_blunder: reduced C2 scene (4096^2 pair at 0.5 m, 1024^2 "
                               "grid at 2 m), points on 2% of the nodes, Delaunay TIN, MPP 1.5",
                   "points": int(len(pts0)), "triangles": int(len(tris)), "rounds": rounds},
        "e2e": {"value": len(tris) / (ms / 1e3), "unit": "triangles/s",
                "timing": "host wall clock of the C-ABI call on host buffers (the call waits "
                          "for a flag after every round, so device and e2e time coincide)"},
        "cpu_baseline": {"value": len(tris) / cpu_s, "unit": "triangles/s",
                         "cores": os.cpu_count(), "kind": "reference",
                         "sample": f"whole TIN, {cpu_s:.2f} s"},
        "gpu_launches": int(launches),
        "clocks": clk,
        "parity": {"points_identical": bool(same_pts),
                   "ugrid_field_mismatch": field_mismatch(inp.gridpt3, ref.gridpt3)},
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    del torch


# ---------------------------------------------------------------------------
# C5 serving
# ---------------------------------------------------------------------------
def run_c5(args):
    """C5: a Poisson stream of stereo-tile requests over resident scenes,
    served with continuous batching (setsm_b200/serving.py); p50 / p99
    latency from arrival to result on the host, and evals/s over the
    stream's makespan, beside sequential plain-FP64 processing of a sample."""
    world, rank, local = dist_setup(args.gpus)
    import torch
    from setsm_b200 import serving, vll
    dev = torch.device("cuda", local)
    ctx = vll.Context(local)
    t0 = time.time()
    scenes = [serving.make_resident_scene(ctx, sid, args.c5_image, 5, dev,
                                          seed=100 * (rank + 1) + sid)
              for sid in range(args.c5_scenes)]
    log(f"[rank {rank}] {len(scenes)} resident scenes built in {time.time() - t0:.1f} s "
        f"({torch.cuda.memory_allocated(dev) / 1e9:.1f} GB)")
    mix = dict(levels=(0, 1, 2, 3, 4), templates=(11, 15))
    warm = serving.poisson_requests(16, 200.0, scenes, seed=1000 + rank, **mix)
    serving.Server(scenes, device=local, hbm_budget=args.c5_budget * 1e9).run(warm, realtime=False)
    reqs = serving.poisson_requests(args.c5_requests, args.c5_rate, scenes, seed=7 + rank, **mix)
    clocks = Clocks(local)
    clocks.start()
    srv = serving.Server(scenes, device=local, hbm_budget=args.c5_budget * 1e9,
                         max_batch=args.c5_max_batch, n_workers=2)
    barrier(world)
    rep = srv.run(reqs, realtime=True)
    clk = clocks.stop()
    # the same mix below saturation: the rate scaled so that the offered load
    # is half of what the first run served, for steady-state latencies
    load = rep["offered_slots_per_s"] / max(rep["served_slots_per_s"], 1e-9)
    rate2 = args.c5_rate * min(1.0, 0.5 / max(load, 1e-9))
    n2 = max(50, min(args.c5_requests, int(rate2 * 60)))
    reqs2 = serving.poisson_requests(n2, rate2, scenes, seed=17 + rank, **mix)
    srv2 = serving.Server(scenes, device=local, hbm_budget=args.c5_budget * 1e9,
                          max_batch=args.c5_max_batch, n_workers=2)
    barrier(world)
    rep2 = srv2.run(reqs2, realtime=True)
    # sequential plain FP64 on a sample of the same requests
    by_sid = {rs.sid: rs for rs in scenes}
    ev, ms = 0, 0.0
    sample = reqs[: max(1, args.c5_fp64_sample)]
    for r in sample:
        ev0 = time.perf_counter()
        _, _, e = serving.run_alone(ctx, r, by_sid[r.sid], dev, kernel="plain")
        ms += (time.perf_counter() - ev0) * 1e3
        ev += e
    makespan = max_over_ranks(world, rep["makespan_s"])
    value = sum_over_ranks(world, rep["evals"]) / makespan
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": 1,
            "warmup": 1, "ms_per_step": makespan * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 window sums, f64 RPC and decisions", "data": "synthetic",
            "config": {"workload": f"C5 serving: Poisson {args.c5_rate:g} req/s, "
                                   f"{args.c5_requests} requests, grid 64^2-1024^2 and K 8-512 "
                                   f"log-uniform, pyramid levels 0-4 and 7x7 / 11x11 windows "
                                   f"drawn uniformly, {args.c5_scenes} resident "
                                   f"{args.c5_image}^2 pairs with 5-level pyramids, HBM budget "
                                   f"{args.c5_budget:g} GB, continuous batching on 2 streams",
                       "parallelism": f"replicas x{world}"},
            "serving": rep,
            "latency_ms": {"p50": rep["p50_ms"], "p99": rep["p99_ms"]},
            "offered_vs_served_slots_per_s": [rep["offered_slots_per_s"],
                                              rep["served_slots_per_s"]],
            "below_saturation": {"rate_req_per_s": rate2, "requests": n2,
                                 "offered_slots_per_s": rep2["offered_slots_per_s"],
                                 "served_slots_per_s": rep2["served_slots_per_s"],
                                 "evals_per_s": rep2["evals_per_s"],
                                 "latency_ms": {"p50": rep2["p50_ms"], "p99": rep2["p99_ms"]}},
            "fp64_plain_sequential": {"value": ev / (ms / 1e3), "unit": UNIT,
                                      "requests": len(sample),
                                      "timing": "host wall clock per request (synchronous)"},
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    barrier(world)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_shard(args):
    """One scene of the config split into grid-row bands, one per rank
    (strong scaling).  Every rank builds the same seeded scene, keeps only its
    band's image footprint (shard.footprint_of) on its GPU, matches its rows
    with each window, and the NCCresult bands are all-gathered with
    dist.all_gather_into_tensor (NCCL) after each call, so every rank holds
    the whole grid's records as a full call would leave them.  Rank 0 checks
    the gathered grid against the whole-grid call on the same scene."""
    world, rank, local = dist_setup(args.gpus)
    import torch
    from setsm_b200 import shard, vll, workloads

    dev = torch.device("cuda", local)
    ctx = vll.Context(local)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    t0 = time.time()
    wl = workloads.build(args.config, ctx, device=f"cuda:{local}", seed=1, keep_host=False)
    templates = workloads.CONFIGS[args.config]["templates"]
    W, Hg = wl.grid.width, wl.grid.height
    whole = {}
    if rank == 0:
        # the whole-grid call on the same scene (parity reference)
        for t in templates:
            wl.d_ncc.zero_()
            torch.cuda.synchronize(dev)
            st = ctx.vertical_line_locus_device(wl.device_desc(t), wl.d_gp3.data_ptr(),
                                                wl.d_ncc.data_ptr(), None, None, args.kernel,
                                                stats=True)
            whole[t] = (workloads.ncc_host(wl), int(st.accessable_grid))
    r0, r1 = shard.row_bands(Hg, world)[rank]
    band = wl.device_band(r0, r1)
    # the whole planes and the whole-grid record array are released: the
    # rank keeps its band's footprint
    wl.d_img, wl.d_mag, wl.d_ori = [], [], []
    wl.d_ncc = None
    torch.cuda.synchronize(dev)
    torch.cuda.empty_cache()
    descs = {t: band.desc(t) for t in templates}
    rows_max = max(b1 - b0 for b0, b1 in shard.row_bands(Hg, world))
    band_ncc = torch.zeros(max(1, rows_max * W) * shard.NCC_BYTES, dtype=torch.uint8, device=dev)
    log(f"[rank {rank}] band rows [{r0}, {r1}) of {Hg}, footprint planes "
        f"{band.image_bytes() / 2**20:.0f} MiB, built in {time.time() - t0:.1f} s")

    def one_step():
        # (the call's statistics carry Accessable_grid, as the whole-grid leg's do)
        out = {}
        with torch.cuda.stream(stream):
            for t in templates:
                st = ctx.vertical_line_locus_device(descs[t], band.d_gridpt3(),
                                                    band_ncc.data_ptr(), None, None,
                                                    args.kernel, stats=True)
                acc = int(st.accessable_grid)
                if world > 1:
                    full, acc = shard.gather_bands_tensor(band_ncc, acc, W, Hg, device=dev)
                else:
                    full = band_ncc
                out[t] = (st, full, acc)
        return out

    for _ in range(max(3, args.warmup)):
        warm = one_step()
    evals_rank = sum(warm[t][0].evals for t in templates)
    # parity: each window's gathered grid from a cleared band array
    parity = None
    for t in templates:
        band_ncc.zero_()
        torch.cuda.synchronize(dev)
        with torch.cuda.stream(stream):
            st = ctx.vertical_line_locus_device(descs[t], band.d_gridpt3(), band_ncc.data_ptr(),
                                                None, None, args.kernel, stats=True)
            acc = int(st.accessable_grid)
            if world > 1:
                full, acc = shard.gather_bands_tensor(band_ncc, acc, W, Hg, device=dev)
            else:
                full = band_ncc
        torch.cuda.synchronize(dev)
        if rank == 0:
            got = full[:W * Hg * shard.NCC_BYTES].cpu().numpy().view(whole[t][0].dtype)
            mism = cases_field_mismatch(got, whole[t][0])
            p = parity or {"nodes": int(W * Hg), "fields_mismatched": {}, "accessable_equal": True}
            for k, v in mism.items():
                p["fields_mismatched"][k] = p["fields_mismatched"].get(k, 0) + v
            p["accessable_equal"] = p["accessable_equal"] and acc == whole[t][1]
            parity = p
    barrier(world)

    clocks = Clocks(local)
    clocks.start()
    launches0 = ctx.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    barrier(world)
    e0.record(stream)
    for _ in range(args.steps):
        one_step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    clk = clocks.stop()
    ms = max_over_ranks(world, e0.elapsed_time(e1))
    launches = ctx.launch_count() - launches0
    evals_total = sum_over_ranks(world, evals_rank * args.steps)
    value = evals_total / (ms / 1e3)
    img_mib = max_over_ranks(world, band.image_bytes() / 2**20)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 window sums, f64 RPC and decisions", "data": "synthetic",
            "config": {"workload": config_block(args, wl)["workload"], "nodes": int(W * Hg),
                       "windows": [workloads.WINDOW_OF_TEMPLATE[t] for t in templates],
                       "kernel": args.kernel,
                       "l2": "inputs larger than L2 (band footprints of 16384^2 planes)",
                       "parallelism": f"row bands x{world}, NCCresult bands all-gathered "
                                      "(all_gather_into_tensor) after every call"},
            "shard": {"bands": [list(b) for b in shard.row_bands(Hg, world)],
                      "max_footprint_planes_mib": img_mib,
                      "parity_vs_whole_grid": parity},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    barrier(world)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_phase_cycles(args):
    """Where the window kernel's time goes, on the config's workload: the
    library built with the phase counters
    (setsm_b200/build.py build_phase_cycles) runs each window once after a
    warm-up, and the line gives per 32-slot group the warp cycles of each
    phase and their shares.  The counters add a clock read per phase, so the
    launch time is reported beside the uninstrumented library's."""
    import ctypes as C
    import torch
    from setsm_b200 import build as bld
    from setsm_b200 import vll, workloads
    names = ["tile_wait", "box_conversion", "node_setup", "geometry_and_tile_copies",
             "window_statistics", "peak_scan_and_writes", "node_end"]
    out = {}
    for lib in (bld.LIB, bld.LIB_PHASES):
        vll._lib = None
        vll.LIB_PATH = lib
        ctx = vll.Context(0)
        wl = workloads.build(args.config, ctx, device="cuda:0", seed=1, keep_host=False)
        torch.cuda.synchronize()
        L = C.CDLL(lib)
        for t in workloads.CONFIGS[args.config]["templates"]:
            d = wl.device_desc(t)
            ctx.vertical_line_locus_device(d, wl.d_gp3.data_ptr(), wl.d_ncc.data_ptr(), None,
                                           None, "split")
            buf = (C.c_ulonglong * 16)()
            if lib == bld.LIB_PHASES:
                L.vll_window_phase_cycles(buf, 1)
            wl.d_ncc.zero_()
            torch.cuda.synchronize()
            st = ctx.vertical_line_locus_device(d, wl.d_gp3.data_ptr(), wl.d_ncc.data_ptr(), None,
                                                None, "split", stats=True)
            w = out.setdefault(workloads.WINDOW_OF_TEMPLATE[t], {})
            if lib == bld.LIB:
                w["window_ms"] = st.window_ms
                continue
            L.vll_window_phase_cycles(buf, 1)
            groups, nodes = int(buf[8]), int(buf[9])
            tot = sum(buf[i] for i in range(7))
            w.update({"window_ms_instrumented": st.window_ms, "groups": groups, "nodes": nodes,
                      "cycles_per_group": {n: buf[i] / max(groups, 1) for i, n in enumerate(names)},
                      "share": {n: buf[i] / max(tot, 1) for i, n in enumerate(names)}})
        ctx.close()
        del wl
        torch.cuda.empty_cache()
    print(json.dumps({"metric": "window kernel warp cycles per 32-slot group, by phase",
                      "config": args.config, "windows": out}), flush=True)


def cases_field_mismatch(got, want) -> dict:
    """Mismatching records per NCCresult field (numpy structured arrays)."""
    out = {}
    for name in want.dtype.names:
        a, b = got[name], want[name]
        if a.dtype.kind == "f":
            n = int(np.count_nonzero(a.view(np.uint32 if a.itemsize == 4 else np.uint64) !=
                                     b.view(np.uint32 if b.itemsize == 4 else np.uint64)))
        else:
            n = int(np.count_nonzero(a != b))
        if n:
            out[name] = n
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2",
                    choices=["c1", "c2", "c2_small", "c3", "c4", "c5", "sgm", "seeddem",
                             "blunder", "ortho_tin", "height_range", "select_mps",
                             "voxel_iter", "tin_blunder", "tin_create"])
    ap.add_argument("--kernel", default="split", choices=["split", "plain"])
    ap.add_argument("--phase-cycles", action="store_true",
                    help="the window kernel's per-phase warp cycles on the config's scene "
                         "(the library built with the phase counters)")
    ap.add_argument("--shard", action="store_true",
                    help="one scene split into grid-row bands over the ranks (strong scaling)")
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="end-to-end steps of the default config (0: as many as --steps)")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--tune-rows", type=int, default=256)
    ap.add_argument("--fp64-evals", type=float, default=5e8,
                    help="evaluations of the plain FP64 comparison on multi-level configs")
    ap.add_argument("--c5-scenes", type=int, default=8)
    ap.add_argument("--c5-image", type=int, default=16384)
    ap.add_argument("--c5-requests", type=int, default=400)
    ap.add_argument("--c5-rate", type=float, default=200.0)
    ap.add_argument("--c5-budget", type=float, default=120.0, help="HBM budget, GB")
    ap.add_argument("--c5-max-batch", type=int, default=32)
    ap.add_argument("--c5-fp64-sample", type=int, default=8)
    args = ap.parse_args()
    if args.e2e_steps <= 0:
        args.e2e_steps = args.steps
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.phase_cycles:
        run_phase_cycles(args)
    elif args.shard:
        run_shard(args)
    elif args.config in ("c3", "c4"):
        run_multi(args)
    elif args.config == "c5":
        run_c5(args)
    elif args.config == "sgm":
        run_sgm(args)
    elif args.config in ("seeddem", "blunder"):
        run_variant(args)
    elif args.config == "ortho_tin":
        run_ortho_tin(args)
    elif args.config == "height_range":
        run_height_range(args)
    elif args.config == "select_mps":
        run_select_mps(args)
    elif args.config == "voxel_iter":
        run_voxel_iter(args)
    elif args.config == "tin_create":
        run_tin_create(args)
    elif args.config == "tin_blunder":
        run_tin_blunder(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
