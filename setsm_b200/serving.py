"""Serving loop: stereo-tile matching requests with continuous batching.

Scenes (pyramid planes of both images, RPCs) stay resident in HBM.  A request
asks for VerticalLineLocus (setsm_code.cpp:6049-6548) over a tile of one
resident scene: a grid of n x n nodes at some pyramid level, window size and
per-node height ranges.  The server

* admits arriving requests while their device memory (grid arrays, UGRID /
  NCCresult and the pipeline's per-slot scratch) fits the HBM budget, and
  keeps the rest waiting in arrival order;
* hands every idle worker the admitted requests that are ready -- up to
  ``max_batch`` of them -- as ONE batch: one pass of the split pipeline with a
  single persistent window launch over all the batch's (node, 32-slot) items
  (``vll_vertical_line_locus_batch``);
* runs ``n_workers`` workers, each with its own GPU context and stream, so a
  batch formed from requests that arrived while another batch was on the GPU
  runs concurrently with it; memory is released as batches finish, which
  admits further requests (continuous batching, not a queue alone).

A request's result is a function of its own inputs only: the same bits
alone, in any batch and under any tuning (tests/test_gpu_serving.py).
Latency is measured from a request's arrival to its result on the host.
"""
from __future__ import annotations

import math
import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import abi, level, synth, vll, workloads


@dataclass
class ResidentScene:
    """A stereo scene kept on the device: per level and camera the planes
    {img, mag, ori}, plus the RPCs and projection."""
    sid: int
    scene: synth.Scene
    planes: list                     # [level][camera] -> dict of device tensors
    sizes: list                      # [level] (height, width)


def make_resident_scene(ctx, sid: int, image_size: int, levels: int, device, seed: int,
                        convergence: float = 30.0) -> ResidentScene:
    cams = (synth.CameraSpec(convergence / 2, 0.7), synth.CameraSpec(-convergence / 2, -0.9))
    spec = synth.SceneSpec(seed=seed, image_size=image_size, cameras=cams)
    scene = synth.make_scene(spec, device=device, rows_per_chunk=512)
    pyr = [[scene.images[ci].contiguous()] for ci in range(2)]
    for ci in range(2):
        for _ in range(levels - 1):
            src = pyr[ci][-1]
            h, w = src.shape
            out = torch.empty((h // 2, w // 2), dtype=src.dtype, device=src.device)
            ctx.pyramid_down_device(src.data_ptr(), w, h, out.data_ptr())
            pyr[ci].append(out)
    planes = [[workloads._planes(ctx, pyr[ci][lv]) for ci in range(2)] for lv in range(levels)]
    scene.images = []
    torch.cuda.synchronize(device)
    return ResidentScene(sid=sid, scene=scene, planes=planes,
                         sizes=[tuple(planes[lv][0]["img"].shape) for lv in range(levels)])


@dataclass
class TileRequest:
    rid: int
    sid: int                 # resident scene
    level: int               # pyramid level
    template: int            # Template_size (11 -> 7x7 at level 0, 15 -> 11x11)
    n: int                   # grid side (nodes)
    spacing: float           # grid spacing (m)
    k: int                   # candidates per node (log-uniform spread applied per node)
    fx: float                # tile centre, fraction of the scene extent
    fy: float
    seed: int
    arrival: float = 0.0     # seconds from the start of the stream
    # filled by the server
    admitted: float = -1.0
    done: float = -1.0
    accessable: int = -1
    nccresult: np.ndarray | None = None
    batch_size: int = 0

    @property
    def n_nodes(self) -> int:
        return self.n * self.n


class _Materialized:
    """Device arrays of one request for the duration of its batch."""

    def __init__(self, req: TileRequest, rs: ResidentScene, device):
        sc = rs.scene
        spec = sc.spec
        L = req.level
        ext = spec.image_size * spec.gsd
        cx, cy = sc.center_xy
        half = 0.5 * req.n * req.spacing
        ox = cx - ext / 2 + half + req.fx * max(0.0, ext - 2 * half)
        oy = cy - ext / 2 + half + req.fy * max(0.0, ext - 2 * half)
        b = np.array([ox - half, oy - half, ox + half, oy + half])
        col = torch.arange(req.n, dtype=torch.float64, device=device)
        X = (b[0] + col[None, :] * req.spacing).expand(req.n, req.n).reshape(-1)
        Y = (b[1] + col[:, None] * req.spacing).expand(req.n, req.n).reshape(-1)
        lon, lat = synth.ps2wgs(sc.param, X, Y)
        truth = sc.dem_at(X, Y)
        step = workloads.height_step(L, spec.gsd)
        # per-node candidate counts log-uniform in [8, min(2k, 512)] and a
        # prior of truth + N(0, 3 m), drawn on the device from the request's
        # seed (the same request always gets the same ranges)
        gen = torch.Generator(device=device)
        gen.manual_seed(req.seed)
        n = req.n_nodes
        kmax = min(512.0, max(9.0, 2.0 * req.k))
        u = torch.rand(n, generator=gen, device=device, dtype=torch.float64)
        kk = torch.exp(math.log(8.0) + u * (math.log(kmax) - math.log(8.0)))
        centre = truth + 3.0 * torch.randn(n, generator=gen, device=device, dtype=torch.float64)
        span = torch.clamp(torch.round(kk * step), min=1.0)
        lo = torch.floor(centre - span / 2)
        hi = lo + span
        # UGRID records (20 bytes): Height f32 @0, minHeight @4, maxHeight @6,
        # Matched_flag u8 @16, the rest zero
        rec = torch.zeros((n, 10), dtype=torch.int16, device=device)
        rec[:, 0:2] = centre.to(torch.float32).view(torch.int16).view(n, 2)
        rec[:, 2] = lo.clamp(-32768, 32767).to(torch.int16)
        rec[:, 3] = hi.clamp(-32768, 32767).to(torch.int16)
        rec[:, 8] = 1
        self.d_gp3 = rec.view(torch.uint8).reshape(-1)
        self.gp3 = np.zeros(n, dtype=abi.UGRID_DTYPE)      # host shape only (descriptor)
        self.d_pts = torch.stack([X, Y], 1).contiguous()
        self.d_wgs = torch.stack([lon, lat], 1).contiguous()
        self.d_ncc = torch.zeros(n * abi.NCCRESULT_DTYPE.itemsize, dtype=torch.uint8,
                                 device=device)
        ims = []
        for ci in range(2):
            im = dict(rpc=sc.rpcs[ci], **rs.planes[L][ci])
            if L >= 1:
                nxt = rs.planes[L - 1][ci]
                im.update(img_n=nxt["img"], mag_n=nxt["mag"], ori_n=nxt["ori"])
            ims.append(im)
        gd = {"n": req.n_nodes, "w": req.n, "h": req.n, "res": req.spacing,
              "d_pts": self.d_pts, "d_wgs": self.d_wgs}
        self.keep = [gd, ims]
        self.desc = workloads._level_desc(ims, gd, self.gp3, pyramid_step=L,
                                          template=req.template, height_step_m=step,
                                          resolution=spec.gsd, param=sc.param, boundary=b,
                                          keep=self.keep)

    def io(self) -> tuple:
        return (self.desc, self.d_gp3.data_ptr(), self.d_ncc.data_ptr())


def request_bytes(req: TileRequest) -> int:
    """Device bytes a request holds while admitted: grid arrays (32 B), UGRID
    (20 B), NCCresult (24 B) and the pipeline's per-node scratch (~48 B) per
    node, and its per-slot float2 (8 B) plus work items for up to 2K slots."""
    return req.n_nodes * (32 + 20 + 24 + 48) + req.n_nodes * 2 * req.k * 9


class Server:
    def __init__(self, scenes: list, device: int = 0, hbm_budget: float = 120e9,
                 max_batch: int = 32, n_workers: int = 2, tuning: dict | None = None):
        self.scenes = {rs.sid: rs for rs in scenes}
        self.device = device
        self.budget = float(hbm_budget)
        self.max_batch = int(max_batch)
        self.n_workers = int(n_workers)
        self.tuning = tuning
        self.lock = threading.Condition()
        self.waiting: deque = deque()        # arrived, not admitted (arrival order)
        self.ready: deque = deque()          # admitted, not yet in a batch
        self.in_use = 0.0
        self.max_in_use = 0.0
        self.finished: list = []
        self.batches: list = []              # (size, t_start, t_end, worker)
        self.stop = False
        self.errors: list = []
        self.t0 = 0.0

    # ---- admission ------------------------------------------------------------
    def _admit_locked(self, now: float) -> None:
        while self.waiting:
            req = self.waiting[0]
            need = request_bytes(req)
            if self.in_use + need > self.budget and self.in_use > 0:
                break
            self.waiting.popleft()
            self.in_use += need
            self.max_in_use = max(self.max_in_use, self.in_use)
            req.admitted = now
            self.ready.append(req)

    def submit(self, req: TileRequest) -> None:
        with self.lock:
            self.waiting.append(req)
            self._admit_locked(time.perf_counter() - self.t0)
            self.lock.notify_all()

    # ---- workers --------------------------------------------------------------
    def _worker(self, wid: int) -> None:
        torch.cuda.set_device(self.device)
        ctx = vll.Context(self.device)
        stream = torch.cuda.Stream(device=self.device)
        ctx.set_stream(stream.cuda_stream)
        if self.tuning:
            ctx.set_tuning(**self.tuning)
        try:
            while True:
                with self.lock:
                    while not self.ready and not (self.stop and not self.waiting):
                        self.lock.wait(0.05)
                    if not self.ready and self.stop and not self.waiting:
                        return
                    batch = []
                    while self.ready and len(batch) < self.max_batch:
                        batch.append(self.ready.popleft())
                if not batch:
                    continue
                t_start = time.perf_counter() - self.t0
                with torch.cuda.stream(stream):
                    mats = [_Materialized(r, self.scenes[r.sid], torch.device("cuda", self.device))
                            for r in batch]
                    stream.synchronize()
                    acc, st = ctx.batch([m.io() for m in mats])
                    outs = [m.d_ncc.cpu().numpy().view(abi.NCCRESULT_DTYPE).copy() for m in mats]
                t_end = time.perf_counter() - self.t0
                with self.lock:
                    for r, m, o, a in zip(batch, mats, outs, acc):
                        r.nccresult = o
                        r.accessable = int(a)
                        r.done = t_end
                        r.batch_size = len(batch)
                        self.in_use -= request_bytes(r)
                        self.finished.append(r)
                    self.batches.append((len(batch), t_start, t_end, wid, int(st.evals)))
                    self._admit_locked(t_end)
                    self.lock.notify_all()
                del mats
        except Exception as e:   # surfaced by run()
            with self.lock:
                self.errors.append(repr(e))
                self.stop = True
                self.lock.notify_all()
        finally:
            ctx.close()

    def run(self, requests: list, realtime: bool = True) -> dict:
        """Feeds `requests` at their arrival times (seconds from now) and
        returns the stream's statistics once every request is answered."""
        self.t0 = time.perf_counter()
        workers = [threading.Thread(target=self._worker, args=(w,), daemon=True)
                   for w in range(self.n_workers)]
        for w in workers:
            w.start()
        for req in sorted(requests, key=lambda r: r.arrival):
            if realtime:
                dt = req.arrival - (time.perf_counter() - self.t0)
                if dt > 0:
                    time.sleep(dt)
            self.submit(req)
        with self.lock:
            self.stop = True
            self.lock.notify_all()
        for w in workers:
            w.join()
        if self.errors:
            raise RuntimeError("serving worker failed: " + "; ".join(self.errors))
        return self.report()

    def report(self) -> dict:
        lat = np.array([r.done - r.arrival for r in self.finished]) * 1e3
        makespan = max(b[2] for b in self.batches) - min(b[1] for b in self.batches)
        evals = sum(b[4] for b in self.batches)
        overlap = 0.0
        bs = sorted(self.batches, key=lambda b: b[1])
        for i in range(len(bs)):
            for j in range(i + 1, len(bs)):
                if bs[j][1] >= bs[i][2]:
                    break
                overlap += min(bs[i][2], bs[j][2]) - bs[j][1]
        arr = [r.arrival for r in self.finished]
        slots = sum(r.n * r.n * r.k for r in self.finished)
        span = max(arr) - min(arr) if len(arr) > 1 else 0.0
        return {"requests": len(self.finished), "batches": len(self.batches),
                # candidate slots (grid nodes x heights) requested per second of
                # arrivals, and served per second of the makespan
                "offered_slots_per_s": slots / span if span > 0 else 0.0,
                "served_slots_per_s": slots / makespan if makespan > 0 else 0.0,
                "mean_batch": float(np.mean([b[0] for b in self.batches])),
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "max_ms": float(lat.max()), "evals": int(evals),
                "evals_per_s": evals / makespan if makespan > 0 else 0.0,
                "makespan_s": makespan, "batch_overlap_s": overlap,
                "max_admitted_gb": self.max_in_use / 1e9, "budget_gb": self.budget / 1e9}


def poisson_requests(n: int, rate: float, scenes: list, seed: int = 7, grid_min: int = 64,
                     grid_max: int = 1024, levels=(0,), templates=(11,)) -> list:
    """n requests with Poisson arrivals at `rate` per second; grid side and
    candidate count log-uniform in [grid_min, grid_max] and [8, 512]; the
    pyramid level and the window drawn uniformly from `levels` and
    `templates` (a level's grid is at 2 m << level, clipped to its scene)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        rs = scenes[int(rng.integers(len(scenes)))]
        L = int(rng.choice(levels))
        template = int(rng.choice(templates))
        spacing = 2.0 * (1 << L)
        side_max = int(rs.scene.spec.image_size * rs.scene.spec.gsd / spacing)
        n_side = int(round(math.exp(rng.uniform(math.log(grid_min), math.log(grid_max)))))
        n_side = max(8, min(n_side, side_max - 4))
        k = int(round(math.exp(rng.uniform(math.log(8), math.log(512)))))
        out.append(TileRequest(rid=i, sid=rs.sid, level=L, template=template, n=n_side,
                               spacing=spacing, k=k, fx=float(rng.random()),
                               fy=float(rng.random()), seed=seed * 100003 + i, arrival=t))
    return out


def run_alone(ctx, req: TileRequest, rs: ResidentScene, device, kernel: str = "split"):
    """One request by itself (a batch of one, or the plain FP64 kernel)."""
    m = _Materialized(req, rs, device)
    torch.cuda.synchronize(device)
    if kernel == "split":
        acc, st = ctx.batch([m.io()])
        acc = int(acc[0])
    else:
        st = ctx.vertical_line_locus_device(m.desc, m.d_gp3.data_ptr(), m.d_ncc.data_ptr(), None,
                                            None, "plain", stats=True)
        acc = int(st.accessable_grid)
    return m.d_ncc.cpu().numpy().view(abi.NCCRESULT_DTYPE).copy(), acc, int(st.evals)
