"""Device-resident VerticalLineLocus workloads.

A workload is one synthetic stereo scene with its level-0 images, magnitude and
orientation images (built on the GPU by the library's own preprocessing
kernels), a matching grid with per-node height ranges, and the level
descriptors that point at the device copies.  Host copies in pinned memory are
kept for the end-to-end (host-buffer) path and for CPU baselines.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import abi, level, synth

# Matching configurations (level 0, memory-tight route with inline peaks).
CONFIGS = {
    # C1: 2048^2 pair, 256^2 grid, 64 heights at 1 m around truth + N(0, 20 m), 7x7
    "c1": dict(image_size=2048, nodes=256, ranges="uniform", n_heights=64, height_step=1.0,
               sigma=20.0, templates=(11,)),
    # C2: 16384^2 pair, 4096^2 grid at 2 m, TIN ranges K 8-512 at 0.5 m, 7x7 and 11x11
    "c2": dict(image_size=16384, nodes=4096, ranges="tin", k_min=8, k_max=512, height_step=0.5,
               n_seeds=20000, tin_noise=3.0, templates=(11, 15)),
    # a reduced C2-like case (same generator and distributions) for profiling captures
    "c2_small": dict(image_size=4096, nodes=1024, ranges="tin", k_min=8, k_max=512,
                     height_step=0.5, n_seeds=2000, tin_noise=3.0, templates=(11, 15)),
}

WINDOW_OF_TEMPLATE = {11: "7x7", 15: "11x11"}
# algorithmic bytes per evaluation: 8 * window samples + 2 orientation bytes + 4 B NCC out
BYTES_PER_EVAL = {11: 8 * 45 + 2 + 4, 15: 8 * 109 + 2 + 4}


@dataclass
class Workload:
    name: str
    cfg: dict
    scene: synth.Scene
    grid: synth.Grid
    gp3: np.ndarray
    d_img: list = field(default_factory=list)
    d_mag: list = field(default_factory=list)
    d_ori: list = field(default_factory=list)
    d_wgs: torch.Tensor | None = None
    d_pts: torch.Tensor | None = None
    d_gp3: torch.Tensor | None = None
    d_ncc: torch.Tensor | None = None
    host: dict = field(default_factory=dict)

    @property
    def n_nodes(self) -> int:
        return self.grid.width * self.grid.height

    def level_kwargs(self, template: int) -> dict:
        return dict(pyramid_step=0, template_size=template, iteration=1, check_matching_rate=True,
                    height_step=self.cfg["height_step"], grid_resolution=self.grid.resolution,
                    resolution=self.scene.spec.gsd, dem_resolution=2.0,
                    minmax_height=(-500.0, 3000.0), sgm_py=0, param=self.scene.param)

    def device_desc(self, template: int) -> abi.LevelDesc:
        """Level descriptor whose every pointer is a device pointer."""
        li = level.LevelInputs(
            [level.ImageLevel(image=np.zeros((2, 2), np.uint16), mag=np.zeros((2, 2), np.uint16),
                              ori=np.zeros((2, 2), np.uint8), rpc=self.scene.rpcs[ci])
             for ci in range(2)],
            np.zeros((self.n_nodes, 2)), np.zeros((self.n_nodes, 2)), self.grid.width,
            self.grid.height, self.grid.boundary, self.gp3, **self.level_kwargs(template))
        d = li.desc()
        n = self.scene.spec.image_size
        for ci in range(2):
            e = d.images[ci]
            e.image = self.d_img[ci].data_ptr()
            e.mag = self.d_mag[ci].data_ptr()
            e.ori = self.d_ori[ci].data_ptr()
            e.width = n
            e.height = n
        d.grid_pts = self.d_pts.data_ptr()
        d.grid_wgs = self.d_wgs.data_ptr()
        return d

    def host_inputs(self, template: int, rows: tuple | None = None) -> level.LevelInputs:
        """LevelInputs on the pinned host copies (optionally a band of grid rows)."""
        h = self.host
        imgs = [level.ImageLevel(image=h["img"][ci], mag=h["mag"][ci], ori=h["ori"][ci],
                                 rpc=self.scene.rpcs[ci]) for ci in range(2)]
        W = self.grid.width
        if rows is None:
            r0, r1 = 0, self.grid.height
        else:
            r0, r1 = rows
        sl = slice(r0 * W, r1 * W)
        b = self.grid.boundary.copy()
        b[1] = b[1] + r0 * self.grid.resolution
        inp = level.LevelInputs(imgs, h["pts"][sl], h["wgs"][sl], W, r1 - r0, b,
                                self.gp3[sl].copy() if rows is not None else self.gp3,
                                **self.level_kwargs(template))
        return inp


def _pinned(t: torch.Tensor) -> np.ndarray:
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    h.copy_(t)
    return h.numpy()


def build(name: str, ctx, device: str = "cuda", seed: int = 1, keep_host: bool = True) -> Workload:
    """Builds a workload on `device` with the library's preprocessing kernels."""
    cfg = CONFIGS[name]
    dev = torch.device(device)
    spec = synth.SceneSpec(seed=seed, image_size=cfg["image_size"])
    scene = synth.make_scene(spec, device=dev, rows_per_chunk=512)
    n = spec.image_size
    wl_imgs, wl_mags, wl_oris = [], [], []
    for ci in range(2):
        img = scene.images[ci].contiguous()
        mag = torch.empty_like(img)
        ori = torch.empty((n, n), dtype=torch.uint8, device=dev)
        ctx.preprocess_device(img.data_ptr(), n, n, mag.data_ptr(), ori.data_ptr())
        wl_imgs.append(img)
        wl_mags.append(mag)
        wl_oris.append(ori)
    extent = n * spec.gsd
    res = extent / cfg["nodes"]
    grid = synth.make_grid(scene, cfg["nodes"], res, device=dev)
    if cfg["ranges"] == "uniform":
        lo, hi, centre = synth.ranges_uniform(grid, cfg["n_heights"], cfg["height_step"],
                                              cfg["sigma"], seed=seed + 1)
    else:
        lo, hi, centre = synth.ranges_tin(scene, grid, cfg["n_seeds"], cfg["k_min"], cfg["k_max"],
                                          cfg["height_step"], cfg["tin_noise"], seed=seed + 1,
                                          device=dev)
    gp3 = level.make_gridpt3(lo, hi, centre)
    wl = Workload(name=name, cfg=cfg, scene=scene, grid=grid, gp3=gp3, d_img=wl_imgs,
                  d_mag=wl_mags, d_ori=wl_oris)
    wl.d_wgs = torch.from_numpy(grid.wgs).to(dev)
    wl.d_pts = torch.from_numpy(grid.pts).to(dev)
    wl.d_gp3 = torch.from_numpy(gp3.view(np.uint8)).to(dev)
    wl.d_ncc = torch.zeros(wl.n_nodes * abi.NCCRESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    if keep_host:
        wl.host = {
            "img": [_pinned(t).view(np.uint16) for t in wl_imgs],
            "mag": [_pinned(t).view(np.uint16) for t in wl_mags],
            "ori": [_pinned(t) for t in wl_oris],
            "wgs": _pinned(wl.d_wgs),
            "pts": _pinned(wl.d_pts),
        }
        gp3_pinned = _pinned(wl.d_gp3).view(abi.UGRID_DTYPE)
        wl.gp3 = gp3_pinned
    torch.cuda.synchronize(dev)
    return wl


def ncc_host(wl: Workload) -> np.ndarray:
    """Copy of the device NCCresult array as a structured numpy array."""
    return wl.d_ncc.cpu().numpy().view(abi.NCCRESULT_DTYPE)


def evals_per_sample_rows(n_rows: int, wl: Workload) -> float:
    return n_rows / wl.grid.height


def rows_for_budget(wl: Workload, evals_budget: float) -> int:
    """Number of grid rows whose expected evaluation count is ~evals_budget."""
    per_row = wl.grid.width * float(np.mean((wl.gp3["maxHeight"].astype(np.int64)
                                             - wl.gp3["minHeight"]) / wl.cfg["height_step"]))
    return max(1, min(wl.grid.height, int(math.ceil(evals_budget / max(per_row, 1.0)))))
