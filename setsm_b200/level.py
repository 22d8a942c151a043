"""Host-side assembly of one VerticalLineLocus call.

``LevelInputs`` gathers what the reference's caller (Matching_SETSM,
setsm_code.cpp:3560-3830) hands to VerticalLineLocus -- pyramid images,
RPCs, grid coordinates, UGRID ranges, flags -- as numpy arrays and builds the
``vll_level_desc`` that points at them.  The arrays are kept alive by the
object for as long as the descriptor is used.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import abi


@dataclass
class ImageLevel:
    image: np.ndarray            # uint16 [H, W]
    mag: np.ndarray              # uint16 [H, W]
    ori: np.ndarray              # uint8  [H, W]
    rpc: np.ndarray              # float64[90]
    startpos: tuple = (0.0, 0.0)
    adjust: tuple = (0.0, 0.0)
    image_next: np.ndarray | None = None
    mag_next: np.ndarray | None = None
    ori_next: np.ndarray | None = None
    startpos_next: tuple = (0.0, 0.0)
    selected: bool = True
    # the blunder-selected pyramid level (None: the matched level)
    image_b: np.ndarray | None = None
    mag_b: np.ndarray | None = None
    startpos_b: tuple = (0.0, 0.0)


def _c(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


class LevelInputs:
    """Inputs of one VerticalLineLocus call plus the matching descriptor."""

    def __init__(self, images: list[ImageLevel], grid_pts: np.ndarray, grid_wgs: np.ndarray,
                 grid_width: int, grid_height: int, boundary, gridpt3: np.ndarray,
                 *, pyramid_step: int = 0, template_size: int = 11, iteration: int = 1,
                 check_matching_rate: bool = True, height_step: float = 1.0,
                 grid_resolution: float = 8.0, resolution: float = 0.5,
                 dem_resolution: float = 2.0, minmax_height=(-500.0, 3000.0),
                 sgm_py: int = 0, py_combined_level: int = 0, bin_angle: float = 20.0,
                 is_ra: bool = False, pre_dem_tif: bool = False, check_matchtag: bool = False,
                 param: dict | None = None, reference_id: int = 0, blunder_level: int | None = None):
        self.images = []
        for im in images:
            self.images.append(ImageLevel(
                image=_c(im.image, np.uint16), mag=_c(im.mag, np.uint16), ori=_c(im.ori, np.uint8),
                rpc=_c(im.rpc, np.float64), startpos=im.startpos, adjust=im.adjust,
                image_next=_c(im.image_next, np.uint16), mag_next=_c(im.mag_next, np.uint16),
                ori_next=_c(im.ori_next, np.uint8), startpos_next=im.startpos_next,
                selected=im.selected, image_b=_c(im.image_b, np.uint16),
                mag_b=_c(im.mag_b, np.uint16), startpos_b=im.startpos_b))
        self.grid_pts = _c(grid_pts, np.float64)
        self.grid_wgs = _c(grid_wgs, np.float64)
        self.grid_width = int(grid_width)
        self.grid_height = int(grid_height)
        self.n = self.grid_width * self.grid_height
        assert self.grid_pts.shape == (self.n, 2) and self.grid_wgs.shape == (self.n, 2)
        assert gridpt3.dtype == abi.UGRID_DTYPE and gridpt3.shape == (self.n,)
        self.gridpt3 = gridpt3
        self.boundary = np.asarray(boundary, dtype=np.float64)
        self.pyramid_step = int(pyramid_step)
        self.template_size = int(template_size)
        self.iteration = int(iteration)
        self.check_matching_rate = bool(check_matching_rate)
        self.height_step = float(height_step)
        self.grid_resolution = float(grid_resolution)
        self.resolution = float(resolution)
        self.dem_resolution = float(dem_resolution)
        self.minmax_height = np.asarray(minmax_height, dtype=np.float64)
        self.sgm_py = int(sgm_py)
        self.py_combined_level = int(py_combined_level)
        self.bin_angle = float(bin_angle)
        self.is_ra = bool(is_ra)
        self.pre_dem_tif = bool(pre_dem_tif)
        self.check_matchtag = bool(check_matchtag)
        self.param = dict(param) if param is not None else {}
        self.reference_id = int(reference_id)
        self.blunder_level = int(pyramid_step if blunder_level is None else blunder_level)

    def desc(self) -> abi.LevelDesc:
        d = abi.LevelDesc()
        d.num_images = len(self.images)
        d.reference_id = self.reference_id
        d.pyramid_step = self.pyramid_step
        d.template_size = self.template_size
        d.py_combined_level = self.py_combined_level
        d.iteration = self.iteration
        d.check_matching_rate = int(self.check_matching_rate)
        d.is_ra = int(self.is_ra)
        d.pre_dem_tif = int(self.pre_dem_tif)
        d.check_matchtag = int(self.check_matchtag)
        d.sgm_py = self.sgm_py
        d.sensor_type = 0
        d.resolution = self.resolution
        d.dem_resolution = self.dem_resolution
        d.height_step = self.height_step
        d.grid_resolution = self.grid_resolution
        d.bin_angle = self.bin_angle
        for i in range(4):
            d.boundary[i] = self.boundary[i]
        d.minmax_height[0] = self.minmax_height[0]
        d.minmax_height[1] = self.minmax_height[1]
        d.grid_width = self.grid_width
        d.grid_height = self.grid_height
        d.grid_pts = abi.ptr(self.grid_pts)
        d.grid_wgs = abi.ptr(self.grid_wgs)
        abi.set_transparam(d.param, self.param)
        for ti, im in enumerate(self.images):
            e = d.images[ti]
            e.image = abi.ptr(im.image)
            e.mag = abi.ptr(im.mag)
            e.ori = abi.ptr(im.ori)
            e.height, e.width = im.image.shape
            e.startpos[0], e.startpos[1] = im.startpos
            if im.image_next is not None:
                e.image_next = abi.ptr(im.image_next)
                e.mag_next = abi.ptr(im.mag_next)
                e.ori_next = abi.ptr(im.ori_next)
                e.height_next, e.width_next = im.image_next.shape
            e.startpos_next[0], e.startpos_next[1] = im.startpos_next
            for k in range(90):
                e.rpc[k] = im.rpc[k]
            e.image_adjust[0], e.image_adjust[1] = im.adjust
            e.selected = int(im.selected)
            if im.image_b is not None:
                e.image_b = abi.ptr(im.image_b)
                e.mag_b = abi.ptr(im.mag_b)
                e.height_b, e.width_b = im.image_b.shape
                e.startpos_b[0], e.startpos_b[1] = im.startpos_b
        d.blunder_level = self.blunder_level
        return d

    def new_nccresult(self) -> np.ndarray:
        return np.zeros(self.n, dtype=abi.NCCRESULT_DTYPE)


def make_gridpt3(lo: np.ndarray, hi: np.ndarray, height: np.ndarray, matched_flag=1,
                 ortho_ncc=None) -> np.ndarray:
    """UGRID array with per-node [lo, hi] height ranges (int16 metres)."""
    n = lo.shape[0]
    g = np.zeros(n, dtype=abi.UGRID_DTYPE)
    g["minHeight"] = np.clip(lo, -32768, 32767)
    g["maxHeight"] = np.clip(hi, -32768, 32767)
    g["Height"] = height.astype(np.float32)
    g["Matched_flag"] = matched_flag
    if ortho_ncc is not None:
        g["ortho_ncc"][:, 1] = ortho_ncc
    return g
