"""Row-band sharding of one VerticalLineLocus level across GPUs.

Grid nodes are independent given the images and RPCs: VerticalLineLocus
loops over nodes (setsm_code.cpp:6139-6145) and every read it makes for a node
-- its UGRID range, its blunder-cell test (:6162-6204), its projections and
windows -- belongs to that node alone.  A level therefore splits into bands of
grid rows with no collective on the NCC math: one process per GPU matches one
band, and the NCCresult rows are gathered afterwards (or stay where a
downstream stage on that GPU consumes them).

Each rank keeps only its band's image footprint in its own HBM.  The footprint
is the bounding box of every projection of the band's nodes over their height
range (and their UGRID height), widened by a margin larger than any window
plus the image-boundary test's band (check_image_boundary,
setsm_code.cpp:11002-11083), and clipped to the image.  The crop is expressed
through py_Startpos, which the reference subtracts from every pyramid
coordinate (OriginalToPyramid_single, CoordConversion.hpp:96-106) -- the same
mechanism SETSM's own tile subsets use (SetsubsetImage / GetsubareaImage,
SubFunctions.cpp:232-300).  Where the crop edge lies inside the image, no
band node comes within the margin of it, so every bounds test has the outcome
it has on the full image and the band's results are bit-identical.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi, level

NCC_BYTES = abi.NCCRESULT_DTYPE.itemsize   # bytes of one NCCresult record

# Margin (pyramid pixels) kept around the projected footprint: the largest
# window radius (half-size 8, rotated: 8 * sqrt(2) + 2) plus the image
# boundary test's H + 1 band, with room to spare.
MARGIN = 32


def row_bands(grid_height: int, world: int) -> list:
    """[(r0, r1)) grid-row bands, one per rank, as equal as possible."""
    if world < 1:
        raise ValueError("world must be >= 1")
    base, extra = divmod(int(grid_height), world)
    out, r = [], 0
    for k in range(world):
        n = base + (1 if k < extra else 0)
        out.append((r, r + n))
        r += n
    return out


def _rpc_eval(rpc: np.ndarray, lon, lat, h):
    """Line / sample of the 20-term cubic RPC in the reference's row layout
    (GetObjectToImageRPC_single, CoordConversion.hpp:26-86) without the clamp;
    used only to size footprints, so plain numpy arithmetic suffices."""
    L = (lon - rpc[2]) / rpc[7]
    P = (lat - rpc[3]) / rpc[8]
    H = (h - rpc[4]) / rpc[9]
    L = np.where(np.abs(L) > 10, ((np.where(lon > 0, lon - 360, lon + 360)) - rpc[2]) / rpc[7], L)
    P = np.where(np.abs(P) > 10, ((np.where(lat > 0, lat - 360, lat + 360)) - rpc[3]) / rpc[8], P)
    t = [np.ones_like(L), L, P, H, L * P, L * H, P * H, L * L, P * P, H * H, P * L * H, L * L * L,
         L * P * P, L * H * H, L * L * P, P * P * P, P * H * H, L * L * H, P * P * H, H * H * H]
    poly = [sum(rpc[10 + 20 * j + k] * t[k] for k in range(20)) for j in range(4)]
    line = poly[0] / poly[1] * rpc[5] + rpc[0]
    samp = poly[2] / poly[3] * rpc[6] + rpc[1]
    return samp, line


def footprint(inputs: level.LevelInputs, r0: int, r1: int, ti: int, pyramid_step: int,
              margin: int = MARGIN):
    """Pixel box [x0, x1) x [y0, y1) of image `ti` at `pyramid_step` (in that
    level's full-image pixel coordinates) that the band's nodes can touch."""
    W = inputs.grid_width
    sl = slice(r0 * W, r1 * W)
    im = inputs.images[ti]
    return footprint_of(inputs.grid_wgs[sl], inputs.gridpt3[sl], im.rpc, im.adjust,
                        pyramid_step, margin)


def footprint_of(wgs: np.ndarray, g: np.ndarray, rpc: np.ndarray, adjust, pyramid_step: int,
                 margin: int = MARGIN):
    """The box of `footprint` for grid nodes `wgs` (lon, lat) with UGRID rows
    `g`, in an image of RPC `rpc` and (line, sample) adjustment `adjust`."""
    lo = g["minHeight"].astype(np.float64)
    hi = g["maxHeight"].astype(np.float64)
    hs = [lo, hi, 0.5 * (lo + hi), g["Height"].astype(np.float64)]
    xs, ys = [], []
    for h in hs:
        x, y = _rpc_eval(rpc, wgs[:, 0], wgs[:, 1], h)
        xs.append(x + adjust[1])
        ys.append(y + adjust[0])
    scale = 1.0 / (1 << pyramid_step)
    x = np.concatenate(xs) * scale
    y = np.concatenate(ys) * scale
    ok = np.isfinite(x) & np.isfinite(y)
    if not ok.any():
        return 0, 0, 0, 0
    return (int(math.floor(x[ok].min())) - margin, int(math.ceil(x[ok].max())) + margin,
            int(math.floor(y[ok].min())) - margin, int(math.ceil(y[ok].max())) + margin)


def _crop(a: np.ndarray | None, sx: int, sy: int, x0: int, x1: int, y0: int, y1: int):
    """Crop of plane `a` whose pixel (0, 0) sits at full-level pixel (sx, sy)."""
    if a is None:
        return None, (x0, y0)
    h, w = a.shape
    cx0 = max(0, x0 - sx)
    cy0 = max(0, y0 - sy)
    cx1 = min(w, x1 - sx)
    cy1 = min(h, y1 - sy)
    if cx1 - cx0 < 2 or cy1 - cy0 < 2:
        cx0, cy0, cx1, cy1 = 0, 0, min(w, 2), min(h, 2)
    return np.ascontiguousarray(a[cy0:cy1, cx0:cx1]), (sx + cx0, sy + cy0)


def band_inputs(inputs: level.LevelInputs, r0: int, r1: int, crop: bool = True,
                margin: int = MARGIN) -> level.LevelInputs:
    """LevelInputs of grid rows [r0, r1): the rows' grid arrays and UGRID
    slice, and (with `crop`) each image cut to the band's footprint with
    py_Startpos moved to the cut's origin."""
    W = inputs.grid_width
    sl = slice(r0 * W, r1 * W)
    L = inputs.pyramid_step
    imgs = []
    for ti, im in enumerate(inputs.images):
        if not crop or not im.selected:
            imgs.append(im)
            continue
        sx, sy = int(round(im.startpos[0])), int(round(im.startpos[1]))
        if (sx, sy) != tuple(im.startpos):
            raise ValueError("cropping needs integer py_Startpos")
        x0, x1, y0, y1 = footprint(inputs, r0, r1, ti, L, margin)
        img, (nx, ny) = _crop(im.image, sx, sy, x0, x1, y0, y1)
        mag, _ = _crop(im.mag, sx, sy, x0, x1, y0, y1)
        ori, _ = _crop(im.ori, sx, sy, x0, x1, y0, y1)
        kw = dict(image=img, mag=mag, ori=ori, rpc=im.rpc, startpos=(float(nx), float(ny)),
                  adjust=im.adjust, selected=im.selected)
        if im.image_next is not None:
            snx, sny = int(round(im.startpos_next[0])), int(round(im.startpos_next[1]))
            x0n, x1n, y0n, y1n = footprint(inputs, r0, r1, ti, L - 1, margin)
            imn, (nxn, nyn) = _crop(im.image_next, snx, sny, x0n, x1n, y0n, y1n)
            magn, _ = _crop(im.mag_next, snx, sny, x0n, x1n, y0n, y1n)
            orin, _ = _crop(im.ori_next, snx, sny, x0n, x1n, y0n, y1n)
            kw.update(image_next=imn, mag_next=magn, ori_next=orin,
                      startpos_next=(float(nxn), float(nyn)))
        imgs.append(level.ImageLevel(**kw))
    band = level.LevelInputs(
        imgs, inputs.grid_pts[sl], inputs.grid_wgs[sl], W, r1 - r0, inputs.boundary,
        inputs.gridpt3[sl].copy(), pyramid_step=L, template_size=inputs.template_size,
        iteration=inputs.iteration, check_matching_rate=inputs.check_matching_rate,
        height_step=inputs.height_step, grid_resolution=inputs.grid_resolution,
        resolution=inputs.resolution, dem_resolution=inputs.dem_resolution,
        minmax_height=inputs.minmax_height, sgm_py=inputs.sgm_py,
        py_combined_level=inputs.py_combined_level, bin_angle=inputs.bin_angle,
        is_ra=inputs.is_ra, pre_dem_tif=inputs.pre_dem_tif, check_matchtag=inputs.check_matchtag,
        param=inputs.param, reference_id=inputs.reference_id)
    return band


def shardable(inputs: level.LevelInputs) -> bool:
    """Row bands reproduce the whole-grid call on the memory-tight route
    without orthoimage GNCC (the GNCC raster spans the tile's Boundary and is
    left whole)."""
    return bool(inputs.check_matching_rate)


def match_band(ctx, inputs: level.LevelInputs, rank: int, world: int, kernel: str = "split",
               crop: bool = True):
    """Runs this rank's band on its GPU context; returns (band nccresult,
    accessable count, (r0, r1))."""
    r0, r1 = row_bands(inputs.grid_height, world)[rank]
    band = band_inputs(inputs, r0, r1, crop=crop)
    ncc = band.new_nccresult()
    if r1 > r0:
        st = ctx.vertical_line_locus(band, ncc, None, kernel)
        acc = int(st.accessable_grid)
    else:
        acc = 0
    return ncc, acc, (r0, r1)


def gather_bands(ncc_band: np.ndarray, acc: int, grid_width: int, grid_height: int, group=None,
                 device=None):
    """All-gathers the bands' NCCresult rows over torch.distributed; returns
    the whole grid's NCCresult and the summed Accessable_grid on every rank.
    `device` is where the collective's buffers live (None: the CPU, for
    gloo; a CUDA device for NCCL)."""
    import torch
    full, total = gather_bands_tensor(torch.from_numpy(ncc_band.view(np.uint8).copy()), acc,
                                      grid_width, grid_height, group=group, device=device)
    return full.cpu().numpy().view(ncc_band.dtype), total


def gather_bands_tensor(band, acc: int, grid_width: int, grid_height: int, group=None,
                        device=None):
    """The same for a band held as a uint8 tensor (its rows' records first,
    any length up to the largest band's bytes): every rank's band is padded
    to the largest band and gathered with one all_gather_into_tensor; the
    counts are summed with all_reduce.  Returns (whole-grid uint8 tensor,
    Accessable_grid) on `device`."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    bands = row_bands(grid_height, world)
    rec = NCC_BYTES
    cap = max(r1 - r0 for r0, r1 in bands) * grid_width * rec
    dev = device if device is not None else band.device
    send = torch.zeros(cap, dtype=torch.uint8, device=dev)
    n = min(int(band.numel()), cap)
    send[:n].copy_(band.reshape(-1)[:n])
    recv = torch.empty(world * cap, dtype=torch.uint8, device=dev)
    dist.all_gather_into_tensor(recv, send, group=group)
    cnt = torch.tensor([int(acc)], dtype=torch.int64, device=dev)
    dist.all_reduce(cnt, group=group)
    full = torch.empty(grid_width * grid_height * rec, dtype=torch.uint8, device=dev)
    for k, (r0, r1) in enumerate(bands):
        nb = (r1 - r0) * grid_width * rec
        full[r0 * grid_width * rec:r0 * grid_width * rec + nb].copy_(recv[k * cap:k * cap + nb])
    return full, int(cnt.item())
