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
        # (a Workload whose whole planes were released after cropping bands
        # has none: DeviceBand.desc sets the crops')
        for ci in range(len(self.d_img)):
            e = d.images[ci]
            e.image = self.d_img[ci].data_ptr()
            e.mag = self.d_mag[ci].data_ptr()
            e.ori = self.d_ori[ci].data_ptr()
            e.width = n
            e.height = n
        d.grid_pts = self.d_pts.data_ptr()
        d.grid_wgs = self.d_wgs.data_ptr()
        return d

    def device_band_io(self, template: int, rows: int) -> tuple:
        """(descriptor, d_gridpt3, d_nccresult) of a band of `rows` grid rows in
        the middle of the grid, on the resident device arrays (memory-tight
        route: no orthoimage raster depends on the band's boundary)."""
        rows = max(1, min(rows, self.grid.height))
        r0 = (self.grid.height - rows) // 2
        W = self.grid.width
        d = self.device_desc(template)
        d.grid_height = rows
        d.grid_pts = self.d_pts.data_ptr() + r0 * W * 16
        d.grid_wgs = self.d_wgs.data_ptr() + r0 * W * 16
        return (d, self.d_gp3.data_ptr() + r0 * W * abi.UGRID_DTYPE.itemsize,
                self.d_ncc.data_ptr() + r0 * W * abi.NCCRESULT_DTYPE.itemsize)

    def device_band(self, r0: int, r1: int) -> "DeviceBand":
        """Grid rows [r0, r1) with each image plane cut, on the device, to the
        band's footprint (shard.footprint_of: every projection of the band's
        nodes over their height range, widened by the shard margin); the cut's
        origin becomes the image's py_Startpos, as in shard.band_inputs.  The
        whole-image planes are not referenced by the band."""
        from . import shard
        W = self.grid.width
        sl = slice(r0 * W, r1 * W)
        n = self.scene.spec.image_size
        crops = []
        for ci in range(2):
            x0, x1, y0, y1 = shard.footprint_of(self.grid.wgs[sl], self.gp3[sl],
                                                self.scene.rpcs[ci], (0.0, 0.0), 0)
            x0, y0 = max(0, x0), max(0, y0)
            x1, y1 = min(n, x1), min(n, y1)
            if x1 - x0 < 2 or y1 - y0 < 2:
                x0, y0, x1, y1 = 0, 0, 2, 2
            crops.append(((x0, y0), self.d_img[ci][y0:y1, x0:x1].contiguous(),
                          self.d_mag[ci][y0:y1, x0:x1].contiguous(),
                          self.d_ori[ci][y0:y1, x0:x1].contiguous()))
        return DeviceBand(self, r0, r1, crops)

    def host_inputs(self, template: int, rows: tuple | None = None,
                    planes: dict | None = None) -> level.LevelInputs:
        """LevelInputs on the pinned host copies (optionally a band of grid
        rows; `planes` = {"mag": [..], "ori": [..]} replaces the magnitude
        and orientation planes)."""
        h = self.host
        mags = (planes or h)["mag"]
        oris = (planes or h)["ori"]
        imgs = [level.ImageLevel(image=h["img"][ci], mag=mags[ci], ori=oris[ci],
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
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=torch.cuda.is_available())
    h.copy_(t)
    return h.numpy()


@dataclass
class DeviceBand:
    """A band of grid rows on the device with its cropped image planes
    (Workload.device_band)."""
    wl: Workload
    r0: int
    r1: int
    crops: list          # per image: ((x0, y0), image, magnitude, orientation)

    @property
    def n_nodes(self) -> int:
        return (self.r1 - self.r0) * self.wl.grid.width

    def desc(self, template: int) -> abi.LevelDesc:
        """Level descriptor of the band: the band's grid rows (pointers into
        the resident grid arrays), the cropped planes with their origins as
        py_Startpos, and the whole tile's boundary."""
        wl = self.wl
        W = wl.grid.width
        d = wl.device_desc(template)
        d.grid_height = self.r1 - self.r0
        d.grid_pts = wl.d_pts.data_ptr() + self.r0 * W * 16
        d.grid_wgs = wl.d_wgs.data_ptr() + self.r0 * W * 16
        for ci, ((x0, y0), img, mag, ori) in enumerate(self.crops):
            e = d.images[ci]
            e.image = img.data_ptr()
            e.mag = mag.data_ptr()
            e.ori = ori.data_ptr()
            e.width = img.shape[1]
            e.height = img.shape[0]
            e.startpos[0] = float(x0)
            e.startpos[1] = float(y0)
        return d

    def d_gridpt3(self) -> int:
        return self.wl.d_gp3.data_ptr() + self.r0 * self.wl.grid.width * abi.UGRID_DTYPE.itemsize

    def image_bytes(self) -> int:
        return sum(t.numel() * t.element_size() for c in self.crops for t in c[1:])


def build(name: str, ctx, device: str = "cuda", seed: int = 1, keep_host: bool = True) -> Workload:
    """Builds a workload on `device` with the library's preprocessing kernels.

    With `ctx` None the magnitude and orientation planes are not made (the
    library is not used at all): the caller supplies host planes in
    ``wl.host["mag"]`` / ``wl.host["ori"]`` before calling `host_inputs`."""
    cfg = CONFIGS[name]
    dev = torch.device(device)
    spec = synth.SceneSpec(seed=seed, image_size=cfg["image_size"])
    scene = synth.make_scene(spec, device=dev, rows_per_chunk=512)
    n = spec.image_size
    wl_imgs, wl_mags, wl_oris = [], [], []
    for ci in range(2):
        img = scene.images[ci].contiguous()
        wl_imgs.append(img)
        if ctx is None:
            continue
        mag = torch.empty_like(img)
        ori = torch.empty((n, n), dtype=torch.uint8, device=dev)
        ctx.preprocess_device(img.data_ptr(), n, n, mag.data_ptr(), ori.data_ptr())
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
            "mag": [_pinned(t).view(np.uint16) for t in wl_mags] or None,
            "ori": [_pinned(t) for t in wl_oris] or None,
            "wgs": _pinned(wl.d_wgs),
            "pts": _pinned(wl.d_pts),
        }
        gp3_pinned = _pinned(wl.d_gp3).view(abi.UGRID_DTYPE)
        wl.gp3 = gp3_pinned
    if dev.type == "cuda":
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


# ---------------------------------------------------------------------------
# Multi-level workloads: batches of levels matched in one pass
# ---------------------------------------------------------------------------
def height_step(pyramid_step: int, im_resolution: float) -> float:
    """GetHeightStep (setsm_code.cpp:5741-5757): half the level's pixel size,
    truncated to mm, capped at 3 m."""
    hs = im_resolution * (1 << pyramid_step) / 2.0
    hs = math.floor(hs * 1000.0 + 0.1) / 1000.0
    return min(hs, 3.0)


@dataclass
class LevelWork:
    """One level of a batch: its device planes, grid and UGRID / NCCresult."""
    name: str
    template: int
    pyramid_step: int
    grid_w: int
    grid_h: int
    gp3: np.ndarray                # host UGRID (pinned)
    desc: abi.LevelDesc            # every pointer on the device
    host_desc_kwargs: dict
    d_gp3: torch.Tensor
    d_ncc: torch.Tensor
    keep: list = field(default_factory=list)

    @property
    def n_nodes(self) -> int:
        return self.grid_w * self.grid_h

    def io(self) -> tuple:
        return (self.desc, self.d_gp3.data_ptr(), self.d_ncc.data_ptr())

    def slots(self, step: float) -> int:
        return int(np.sum(((self.gp3["maxHeight"].astype(np.int64) - self.gp3["minHeight"])
                           / step).astype(np.int64)))


@dataclass
class MultiWorkload:
    name: str
    levels: list
    scenes: list
    info: dict = field(default_factory=dict)

    @property
    def n_nodes(self) -> int:
        return sum(lv.n_nodes for lv in self.levels)

    def ios(self) -> list:
        return [lv.io() for lv in self.levels]


def _level_desc(images, grid, gp3, *, pyramid_step, template, height_step_m, resolution,
                param, boundary, keep) -> abi.LevelDesc:
    """Descriptor of a level whose planes (dict per camera) are device tensors."""
    li = level.LevelInputs(
        [level.ImageLevel(image=np.zeros((2, 2), np.uint16), mag=np.zeros((2, 2), np.uint16),
                          ori=np.zeros((2, 2), np.uint8), rpc=im["rpc"]) for im in images],
        np.zeros((grid["n"], 2)), np.zeros((grid["n"], 2)), grid["w"], grid["h"], boundary, gp3,
        pyramid_step=pyramid_step, template_size=template, iteration=1, check_matching_rate=True,
        height_step=height_step_m, grid_resolution=grid["res"], resolution=resolution,
        dem_resolution=2.0, minmax_height=(-500.0, 3000.0), sgm_py=0, param=param)
    d = li.desc()
    for ci, im in enumerate(images):
        e = d.images[ci]
        e.image, e.mag, e.ori = (im["img"].data_ptr(), im["mag"].data_ptr(), im["ori"].data_ptr())
        e.height, e.width = im["img"].shape
        if im.get("img_n") is not None:
            e.image_next = im["img_n"].data_ptr()
            e.mag_next = im["mag_n"].data_ptr()
            e.ori_next = im["ori_n"].data_ptr()
            e.height_next, e.width_next = im["img_n"].shape
    d.grid_pts = grid["d_pts"].data_ptr()
    d.grid_wgs = grid["d_wgs"].data_ptr()
    keep.append(li)
    return d


def _planes(ctx, img: torch.Tensor) -> dict:
    n_h, n_w = img.shape
    mag = torch.empty_like(img)
    ori = torch.empty((n_h, n_w), dtype=torch.uint8, device=img.device)
    ctx.preprocess_device(img.data_ptr(), n_w, n_h, mag.data_ptr(), ori.data_ptr())
    return {"img": img.contiguous(), "mag": mag, "ori": ori}


def _grid_dev(grid, dev) -> dict:
    return {"n": grid.width * grid.height, "w": grid.width, "h": grid.height,
            "res": grid.resolution, "d_pts": torch.from_numpy(grid.pts).to(dev),
            "d_wgs": torch.from_numpy(grid.wgs).to(dev)}


def _level_work(name, images, grid, gd, lo, hi, centre, *, pyramid_step, template, step,
                resolution, param, dev) -> LevelWork:
    gp3 = level.make_gridpt3(lo, hi, centre)
    keep = [gd, images]
    d = _level_desc(images, gd, gp3, pyramid_step=pyramid_step, template=template,
                    height_step_m=step, resolution=resolution, param=param,
                    boundary=grid.boundary, keep=keep)
    d_gp3 = torch.from_numpy(gp3.view(np.uint8).copy()).to(dev)
    d_ncc = torch.zeros(gd["n"] * abi.NCCRESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    return LevelWork(name=name, template=template, pyramid_step=pyramid_step, grid_w=grid.width,
                     grid_h=grid.height, gp3=gp3, desc=d,
                     host_desc_kwargs=dict(step=step), d_gp3=d_gp3, d_ncc=d_ncc, keep=keep)


def build_c3(ctx, device: str = "cuda", seed: int = 1, n_tiles: int = 64,
             grid_min: int = 128, grid_max: int = 2048, template: int = 11) -> MultiWorkload:
    """C3: n_tiles independent stereo tiles; grid side log-uniform in
    [grid_min, grid_max] nodes at 2 m, images sized to match (4 px per node
    at 0.5 m), convergence 20-40 degrees, each tile with its own fBm DEM and
    TIN ranges of 8-512 candidates at 0.5 m; 7x7 window."""
    dev = torch.device(device)
    rng = np.random.default_rng(seed)
    levels, scenes = [], []
    for t in range(n_tiles):
        g = int(round(math.exp(rng.uniform(math.log(grid_min), math.log(grid_max)))))
        g = max(16, g - g % 2)
        size = 8 * int(math.ceil(4 * g / 8))
        conv = float(rng.uniform(20.0, 40.0))
        cams = (synth.CameraSpec(conv / 2, float(rng.uniform(-1.5, 1.5))),
                synth.CameraSpec(-conv / 2, float(rng.uniform(-1.5, 1.5))))
        spec = synth.SceneSpec(seed=seed * 1000 + t, image_size=size, cameras=cams)
        scene = synth.make_scene(spec, device=dev, rows_per_chunk=512)
        grid = synth.make_grid(scene, g, 2.0, device=dev)
        n_seeds = max(200, int(20000 * (g / 4096.0) ** 2))
        lo, hi, centre = synth.ranges_tin(scene, grid, n_seeds, 8, 512, 0.5, 3.0,
                                          seed=seed * 1000 + t + 1, device=dev)
        ims = [dict(rpc=scene.rpcs[ci], **_planes(ctx, scene.images[ci])) for ci in range(2)]
        scene.images = []        # the planes live in `ims`
        gd = _grid_dev(grid, dev)
        levels.append(_level_work(f"tile{t}", ims, grid, gd, lo, hi, centre, pyramid_step=0,
                                  template=template, step=0.5, resolution=spec.gsd,
                                  param=scene.param, dev=dev))
        scenes.append(scene)
    torch.cuda.synchronize(dev)
    return MultiWorkload(name="c3", levels=levels, scenes=scenes)


def tin_heights(pts: np.ndarray, tris: np.ndarray, grid) -> tuple:
    """Heights at `grid`'s nodes interpolated linearly over a TIN (pts:
    POINT3 records in projected metres, tris: vertex indices); nodes outside
    every triangle take the height of the nearest point.  Returns (heights,
    covered mask)."""
    W, Hn, res = grid.width, grid.height, grid.resolution
    x0, y0 = grid.boundary[0], grid.boundary[1]
    h = np.full(W * Hn, np.nan)

    def fill(X, Y, Z, det, c, r):
        # barycentric coordinates of nodes (c, r) in their triangles' rows
        m = (c >= 0) & (c < W) & (r >= 0) & (r < Hn)
        if not m.any():
            return
        X, Y, Z, det, c, r = X[m], Y[m], Z[m], det[m], c[m], r[m]
        px, py = x0 + c * res, y0 + r * res
        l0 = ((Y[:, 1] - Y[:, 2]) * (px - X[:, 2]) + (X[:, 2] - X[:, 1]) * (py - Y[:, 2])) / det
        l1 = ((Y[:, 2] - Y[:, 0]) * (px - X[:, 2]) + (X[:, 0] - X[:, 2]) * (py - Y[:, 2])) / det
        l2 = 1.0 - l0 - l1
        inside = (l0 >= -1e-9) & (l1 >= -1e-9) & (l2 >= -1e-9)
        h[(r * W + c)[inside]] = (l0 * Z[:, 0] + l1 * Z[:, 1] + l2 * Z[:, 2])[inside]

    if len(tris):
        v = np.stack([tris["a"], tris["b"], tris["c"]], 1).astype(np.int64)
        X, Y, Z = pts["x"][v], pts["y"][v], pts["z"][v]          # [T, 3]
        det = (Y[:, 1] - Y[:, 2]) * (X[:, 0] - X[:, 2]) + (X[:, 2] - X[:, 1]) * (Y[:, 0] - Y[:, 2])
        ok = np.abs(det) > 1e-12
        X, Y, Z, det = X[ok], Y[ok], Z[ok], det[ok]
        c0 = np.ceil((X.min(1) - x0) / res).astype(np.int64)
        c1 = np.floor((X.max(1) - x0) / res).astype(np.int64)
        r0 = np.ceil((Y.min(1) - y0) / res).astype(np.int64)
        r1 = np.floor((Y.max(1) - y0) / res).astype(np.int64)
        span = np.maximum(c1 - c0, r1 - r0) + 1
        small = span <= 8
        # small triangles: every offset of an 8 x 8 box, vectorised over them
        for dr in range(8):
            for dc in range(8):
                sel = small & (c0 + dc <= c1) & (r0 + dr <= r1)
                if sel.any():
                    fill(X[sel], Y[sel], Z[sel], det[sel], c0[sel] + dc, r0[sel] + dr)
        # the few large ones (long triangles along the hull): each over its box
        for t in np.nonzero(~small)[0]:
            cc, rr = np.meshgrid(np.arange(max(c0[t], 0), min(c1[t], W - 1) + 1),
                                 np.arange(max(r0[t], 0), min(r1[t], Hn - 1) + 1))
            n = cc.size
            if n:
                rep = lambda a: np.repeat(a[t:t + 1], n, axis=0)
                fill(rep(X), rep(Y), rep(Z), np.repeat(det[t], n), cc.ravel(), rr.ravel())
    covered = np.isfinite(h)
    if (~covered).any() and len(pts):
        from scipy.spatial import cKDTree
        tree = cKDTree(np.stack([pts["x"], pts["y"]], 1))
        _, j = tree.query(grid.pts[~covered])
        h[~covered] = pts["z"][j]
    return h, covered


def _match_level_points(ctx, lw: "LevelWork", grid, dev) -> tuple:
    """The chain step of C4 on the device: VerticalLineLocus of level work
    `lw` (synchronously), SelectMPs on its records (thresholds of a first iteration), and
    TINCreate_list of the matched points.  Returns (points, triangles) on the
    host."""
    n = lw.n_nodes
    ctx.vertical_line_locus_device(lw.desc, lw.d_gp3.data_ptr(), lw.d_ncc.data_ptr(), None,
                                   None, "split")
    d_g = lw.d_gp3.clone()        # SelectMPs updates its UGRID
    torch.cuda.synchronize(dev)   # (the library runs on its own stream)
    d_pts = torch.empty(n * abi.POINT3_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    n_pts = ctx.select_mps_device(lw.desc, lw.d_ncc.data_ptr(), d_g.data_ptr(), d_pts.data_ptr(),
                                  n, 0.6, 0.2, 0.8, 0.7, 1, 1.5, 1, 10.0)
    cap = 2 * max(n_pts, 1) + 16
    d_tris = torch.empty(cap * abi.TRI_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    n_tris = ctx.tin_create_device(d_pts.data_ptr(), n_pts, grid.boundary, grid.resolution,
                                   d_tris.data_ptr(), cap) if n_pts >= 3 else 0
    pts = d_pts[:n_pts * abi.POINT3_DTYPE.itemsize].cpu().numpy().view(abi.POINT3_DTYPE)
    tris = d_tris[:n_tris * abi.TRI_DTYPE.itemsize].cpu().numpy().view(abi.TRI_DTYPE)
    return pts.copy(), tris.copy()


# C4 candidates per level (level 4 .. 0) and grid spacing (m)
C4_LEVELS = {4: (256, 32.0), 3: (128, 16.0), 2: (64, 8.0), 1: (32, 4.0), 0: (16, 2.0)}


def build_c4(ctx, device: str = "cuda", seed: int = 1, image_size: int = 16384,
             templates=(11, 15), chain: bool = True) -> MultiWorkload:
    """C4: a 5-level pyramid of one stereo pair (the reference's 9x9,
    sigma = 1.5 Gaussian 2x downsample, CreateImagePyramid), grid spacing 32 m
    at level 4 down to 2 m at level 0, K = 256 .. 16 candidates per level at
    that level's GetHeightStep, every level with the 7x7 and 11x11 windows.

    Level 4 searches +-3 sigma around truth + N(0, sigma) (6 sigma = K steps).
    With `chain`, every finer level's ranges follow the previous level's
    matches, coarse to fine as Matching_SETSM carries them: the previous
    level's 7x7 records -> SelectMPs -> TINCreate_list (all on the GPU) ->
    heights interpolated over the TIN at the level's nodes, each node
    searching +-3 sigma (K steps) around its interpolated height.  The chain
    runs once while the workload is built; the timed batch then matches every
    level and window with these ranges.  Per-level chain statistics are kept
    in the workload's `info`."""
    dev = torch.device(device)
    spec = synth.SceneSpec(seed=seed, image_size=image_size)
    scene = synth.make_scene(spec, device=dev, rows_per_chunk=512)
    pyr = [[scene.images[ci].contiguous()] for ci in range(2)]
    for ci in range(2):
        for _ in range(4):
            src = pyr[ci][-1]
            h, w = src.shape
            out = torch.empty((h // 2, w // 2), dtype=torch.int16, device=dev)
            ctx.pyramid_down_device(src.data_ptr(), w, h, out.data_ptr())
            pyr[ci].append(out)
    planes = [[_planes(ctx, pyr[ci][lv]) for lv in range(5)] for ci in range(2)]
    scene.images = []
    levels, info, prev = [], {"chain": bool(chain), "levels": []}, None
    for L in (4, 3, 2, 1, 0):
        k, spacing = C4_LEVELS[L]
        n = int(round(image_size * spec.gsd / spacing))
        grid = synth.make_grid(scene, n, spacing, device=dev)
        gd = _grid_dev(grid, dev)
        step = height_step(L, spec.gsd)
        lv_info = {"level": L, "grid": n, "k": k, "height_step": step}
        if prev is None:
            lo, hi, centre = synth.ranges_uniform(grid, k, step, k * step / 6.0,
                                                  seed=seed + 10 + L)
        else:
            centre, covered = tin_heights(prev[0], prev[1], grid)
            span = k * step
            lo = np.floor(centre - span / 2).astype(np.int64)
            hi = lo + int(round(span))
            err = np.abs(centre - grid.truth)
            lv_info.update(from_points=int(len(prev[0])), from_triangles=int(len(prev[1])),
                           tin_covered=float(covered.mean()),
                           centre_err_m_p50=float(np.median(err)),
                           centre_err_m_p90=float(np.percentile(err, 90)),
                           truth_in_range=float(((grid.truth >= lo) & (grid.truth <= hi)).mean()))
        info["levels"].append(lv_info)
        ims = []
        for ci in range(2):
            im = dict(rpc=scene.rpcs[ci], **planes[ci][L])
            if L >= 1:
                im.update(img_n=planes[ci][L - 1]["img"], mag_n=planes[ci][L - 1]["mag"],
                          ori_n=planes[ci][L - 1]["ori"])
            ims.append(im)
        for t in templates:
            levels.append(_level_work(f"L{L}_T{t}", ims, grid, gd, lo, hi, centre,
                                      pyramid_step=L, template=t, step=step,
                                      resolution=spec.gsd, param=scene.param, dev=dev))
        if chain and L > 0:
            lw = levels[-len(templates)]        # the level's first window
            prev = _match_level_points(ctx, lw, grid, dev)
            lw.d_ncc.zero_()
    torch.cuda.synchronize(dev)
    return MultiWorkload(name="c4", levels=levels, scenes=[scene], info=info)
