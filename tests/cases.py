"""Seeded synthetic VerticalLineLocus cases shared by the tests.

Inputs only: images from setsm_b200.synth; magnitude / orientation / pyramid
images from the C oracle (so every implementation reads the same bytes).
"""
from __future__ import annotations

import functools

import numpy as np

from setsm_b200 import level, synth
from oracle import oraclepy as op


@functools.lru_cache(maxsize=8)
def scene(seed: int, size: int, n_cams: int = 2):
    if n_cams == 2:
        return synth.make_scene(synth.SceneSpec(seed=seed, image_size=size))
    return synth.make_scene(synth.SceneSpec(seed=seed, image_size=size, cameras=CAMS[:n_cams]))


# a third, near-nadir view for the multi-image cases
CAMS = (synth.CameraSpec(15.0, 0.7), synth.CameraSpec(-15.0, -0.9), synth.CameraSpec(4.0, 0.25))


@functools.lru_cache(maxsize=32)
def pyramid(seed: int, size: int, ci: int, lev: int, n_cams: int = 2):
    """(image, mag, ori) of camera ci at pyramid level lev."""
    if lev == 0:
        im = scene(seed, size, n_cams).images[ci].numpy().view(np.uint16).copy()
    else:
        im = op.pyramid_down(pyramid(seed, size, ci, lev - 1, n_cams)[0])
    mag, ori = op.preprocess(im)
    return im, mag, ori


def make_case(*, seed=3, size=768, nodes=48, res=7.5, template=11, cmr=True, L=0, it=1,
              sgm=0, n_heights=64, hs=1.0, sigma=20.0, ortho_frac=0.0, unmatched_frac=0.0,
              zero_patch=False, minmax=(-500.0, 3000.0), dem_res=2.0, combined_level=0,
              iters=None, n_images=2, unselected=()):
    sc = scene(seed, size, n_images)
    g = synth.make_grid(sc, nodes, res)
    lo, hi, _ = synth.ranges_uniform(g, n_heights, hs, sigma, seed=seed + 1)
    rng = np.random.default_rng(seed + 2)
    imgs = []
    for ci in range(n_images):
        im, mag, ori = pyramid(seed, size, ci, L, n_images)
        if zero_patch:
            im = im.copy()
            h, w = im.shape
            im[h // 3: h // 3 + h // 10, w // 4: w // 4 + w // 8] = 0
        kw = {}
        if L >= 1:
            imn, magn, orin = pyramid(seed, size, ci, L - 1, n_images)
            kw = dict(image_next=imn, mag_next=magn, ori_next=orin)
        imgs.append(level.ImageLevel(image=im, mag=mag, ori=ori, rpc=sc.rpcs[ci],
                                     selected=ci not in unselected, **kw))
    on = None
    if ortho_frac > 0:
        on = np.where(rng.random(lo.shape) < ortho_frac, 800, 100)
    matched = np.where(rng.random(lo.shape) < unmatched_frac, 0, 1)
    gp3 = level.make_gridpt3(lo, hi, g.truth, matched_flag=matched, ortho_ncc=on)
    inp = level.LevelInputs(imgs, g.pts, g.wgs, g.width, g.height, g.boundary, gp3,
                            pyramid_step=L, template_size=template, iteration=it,
                            check_matching_rate=cmr, height_step=hs, grid_resolution=g.resolution,
                            resolution=sc.spec.gsd, dem_resolution=dem_res, minmax_height=minmax,
                            sgm_py=sgm, param=sc.param, py_combined_level=combined_level)
    inp.iters = list(iters) if iters else [it]
    return inp


def make_variant_case(*, seed=5, size=512, nodes=32, res=8.0, template=11, L=0,
                      blunder_level=None, matchtag=False, off_frac=0.4, off_m=40.0,
                      void_frac=0.08, minmax=(-60.0, 420.0), n_images=2):
    """A case for the orthoimage-window variants (VerticalLineLocus_seeddem /
    _blunder): node heights at the truth, off by up to `off_m` metres on
    `off_frac` of the nodes (low ortho NCC) and -1000 (unmatched) on
    `void_frac`; the blunder level's images (images[].image_b) at
    `blunder_level` (default: the matched level)."""
    inp = make_case(seed=seed, size=size, nodes=nodes, res=res, template=template, L=L,
                    cmr=False, sgm=-1, n_heights=32, minmax=minmax, n_images=n_images)
    bl = L if blunder_level is None else int(blunder_level)
    for ci, im in enumerate(inp.images):
        im.image_b, im.mag_b, _ = pyramid(seed, size, ci, bl, n_images)
    inp.blunder_level = bl
    inp.check_matchtag = bool(matchtag)
    rng = np.random.default_rng(seed + 17)
    g = inp.gridpt3
    n = len(g)
    off = rng.random(n) < off_frac
    g["Height"][off] += rng.uniform(-off_m, off_m, int(off.sum())).astype(np.float32)
    g["Height"][rng.random(n) < void_frac] = -1000
    return inp


def make_tin_case(*, seed=9, size=512, nodes=32, res=8.0, template=11, L=0, point_frac=0.3,
                  anchor_frac=0.6, off_m=25.0, range_m=40.0, n_images=2):
    """Inputs of Ortho_blunder: matched points on a random subset of the grid
    nodes (height = truth, candidates off by up to `off_m`), anchor flags 1
    (anchored) or 2 (candidate) on their nodes, candidate nodes' height range
    truth +- `range_m`, and the Delaunay triangulation of the points (scipy).
    Returns (inputs, pts, tris)."""
    from setsm_b200 import abi
    inp = make_case(seed=seed, size=size, nodes=nodes, res=res, template=template, L=L,
                    cmr=False, sgm=-1, n_heights=32, n_images=n_images)
    rng = np.random.default_rng(seed + 31)
    g = inp.gridpt3
    n = len(g)
    sel = np.sort(rng.choice(n, size=max(4, int(point_frac * n)), replace=False))
    truth = g["Height"][sel].astype(np.float64)
    anchor = rng.random(len(sel)) < anchor_frac
    pts = np.zeros(len(sel), dtype=abi.POINT3_DTYPE)
    pts["x"] = inp.grid_pts[sel, 0]
    pts["y"] = inp.grid_pts[sel, 1]
    pts["z"] = np.where(anchor, truth, truth + rng.uniform(-off_m, off_m, len(sel)))
    pts["flag"] = 1
    g["anchor_flag"] = 0
    g["anchor_flag"][sel] = np.where(anchor, 1, 2)
    lo = np.floor(truth - range_m).astype(np.int16)
    hi = np.ceil(truth + range_m).astype(np.int16)
    g["minHeight"][sel] = lo
    g["maxHeight"][sel] = hi
    return inp, pts, delaunay(pts)


def make_range_case(*, seed=13, flag4_frac=0.2, unmatched_frac=0.2, **kw):
    """Inputs of SetHeightRange: make_tin_case's points and TIN, with the
    UGRID fields it reads varied: Matched_flag 0 / 1 / 4 and Mean_ortho_ncc
    over [-1, 1]."""
    inp, pts, tris = make_tin_case(seed=seed, **kw)
    rng = np.random.default_rng(seed + 57)
    g = inp.gridpt3
    n = len(g)
    r = rng.random(n)
    g["Matched_flag"] = np.where(r < unmatched_frac, 0, np.where(r < unmatched_frac + flag4_frac,
                                                                   4, 1))
    g["Mean_ortho_ncc"] = rng.integers(-1000, 1000, n).astype(np.int16)
    g["roh"] = rng.integers(-1000, 1000, n).astype(np.int16)
    return inp, pts, tris


@functools.lru_cache(maxsize=8)
def _matched(name: str):
    from oracle import refpy
    base = make_case(**CASES[name])
    return run_cpu(refpy, base, base.iters)


def make_select_case(name: str, seed: int = 71, flag_frac=(0.5, 0.1, 0.2)):
    """Inputs of SelectMPs: the NCCresult of the reference build's matching
    of case `name` (VerticalLineLocus [+ AWNCC]), and its UGRID with
    Matched_flag drawn from 0 / 1 / 2 / 4 (fractions of 1, 2, 4 given) and
    roh over [-0.2, 0.9].  Returns (inputs, nccresult)."""
    import copy
    r = _matched(name)
    inp = copy.copy(r["inputs"])
    inp.gridpt3 = r["gp3"].copy()
    rng = np.random.default_rng(seed)
    g = inp.gridpt3
    n = len(g)
    u = rng.random(n)
    f1, f2, f4 = flag_frac
    g["Matched_flag"] = np.where(u < f1, 1, np.where(u < f1 + f2, 2, np.where(u < f1 + f2 + f4,
                                                                               4, 0)))
    g["roh"] = rng.integers(-200, 900, n).astype(np.int16)
    inp.grid_pts = r["inputs"].grid_pts.copy()
    return inp, r["ncc"].copy()


def make_tin_blunder_case(*, seed=17, flagged_frac=0.1, low_ncc_frac=0.2, **kw):
    """Inputs of blunder_detection_TIN: make_tin_case's points (heights off
    the truth on its candidates) and TIN, point flags 0 with `flagged_frac`
    already 1, and an orthoimage NCC per grid node over [-1, 1] (low on
    `low_ncc_frac` of the nodes).  Returns (inputs, pts, tris, ortho_ncc)."""
    inp, pts, tris = make_tin_case(seed=seed, **kw)
    rng = np.random.default_rng(seed + 91)
    pts["flag"] = np.where(rng.random(len(pts)) < flagged_frac, 1, 0)
    n = inp.n
    oncc = np.where(rng.random(n) < low_ncc_frac, rng.uniform(-1.0, 0.3, n),
                    rng.uniform(0.3, 1.0, n)).astype(np.float32)
    oncc[rng.random(n) < 0.05] = -1.0
    return inp, pts, tris, oncc


def delaunay(pts):
    """Triangles (abi.TRI_DTYPE) of the Delaunay triangulation of the points'
    x, y (scipy's Qhull) -- a stand-in for the matcher's own TIN."""
    from scipy.spatial import Delaunay
    from setsm_b200 import abi
    tri = Delaunay(np.stack([pts["x"], pts["y"]], axis=1)).simplices
    tris = np.zeros(len(tri), dtype=abi.TRI_DTYPE)
    tris["a"], tris["b"], tris["c"] = tri[:, 0], tri[:, 1], tri[:, 2]
    return tris


# name -> kwargs
CASES = {
    "m7": dict(),
    "m11": dict(template=15),
    "m7_edges": dict(zero_patch=True, unmatched_frac=0.1, minmax=(0.0, 260.0), nodes=56, res=7.0),
    "v7_gncc": dict(cmr=False, sgm=-1, ortho_frac=0.5),
    "v11": dict(cmr=False, sgm=-1, template=15, ortho_frac=0.3, n_heights=40),
    "l2_combined": dict(L=2, it=2, iters=(1, 2), cmr=False, sgm=-1, ortho_frac=0.5, nodes=24,
                        res=16.0, n_heights=24, hs=2.0, template=15),
    "l2_max": dict(L=2, it=1, cmr=False, sgm=-1, ortho_frac=0.5, nodes=24, res=16.0,
                   n_heights=24, hs=2.0, template=15),
    "l3_m": dict(L=3, it=1, cmr=True, nodes=16, res=24.0, n_heights=20, hs=3.0, template=15),
    "v7_it2": dict(cmr=False, sgm=-1, it=2, iters=(1, 2), ortho_frac=0.5, n_heights=48),
    # three images (the FP64 kernel): every selected target image enters the sums
    "m7_3img": dict(n_images=3, nodes=40, n_heights=48),
    "v7_3img": dict(n_images=3, cmr=False, sgm=-1, ortho_frac=0.5, nodes=40, n_heights=40),
    "v7_3img_unsel": dict(n_images=3, unselected=(1,), cmr=False, sgm=-1, ortho_frac=0.5,
                          nodes=40, n_heights=40),
}


def field_mismatch(a: np.ndarray, b: np.ndarray) -> dict:
    """Per-field count of differing records (structured arrays)."""
    out = {}
    for f in a.dtype.names:
        x, y = a[f], b[f]
        if x.dtype.kind == "f":
            bad = ~((x == y) | (np.isnan(x) & np.isnan(y)))
        else:
            bad = x != y
        n = int(np.count_nonzero(bad))
        if n:
            out[f] = n
    return out


def run_cpu(impl, inp, iterations=None):
    """Runs a case through `impl` (oracle.refpy or oracle.oraclepy) the way
    Matching_SETSM does (setsm_code.cpp:3774-3845), once per iteration:
    [InitializeVoxel ->] VerticalLineLocus [-> AWNCC].  The returned state
    (init_* = inputs of the last VerticalLineLocus call) lets a GPU test
    replay exactly the last call."""
    import copy
    inp = copy.copy(inp)
    inp.gridpt3 = inp.gridpt3.copy()
    iters = iterations or [inp.iteration]
    ncc = inp.new_nccresult()
    vox = None
    out = {}
    for it in iters:
        inp.iteration = it
        if not inp.check_matching_rate:
            vox = impl.initialize_voxel(inp, ncc, vox)
        out["init_ncc"] = ncc.copy()
        out["init_vox"] = None if vox is None else vox.copy()
        out["init_gp3"] = inp.gridpt3.copy()
        out["acc"] = impl.vertical_line_locus(inp, ncc, vox)
        out["vll_ncc"] = ncc.copy()
        if vox is not None:
            out["vll_vox"] = vox.copy()
            impl.awncc(inp, ncc, vox)
    out["ncc"] = ncc
    out["vox"] = vox
    out["gp3"] = inp.gridpt3
    out["inputs"] = inp
    return out


def device_level(torch, inp, ncc: np.ndarray, voxels: np.ndarray | None = None):
    """Device copies of a case's inputs (planes, grid arrays, UGRID, NCCresult,
    packed voxel rows and their offsets) and a descriptor whose every pointer
    is a device pointer.  Returns (desc, io tuple, tensors to keep alive)."""
    keep = []

    def dev(a):
        a = np.ascontiguousarray(a)
        src = a.view(np.int16) if a.dtype == np.uint16 else a
        if a.dtype.names is not None:
            src = a.view(np.uint8)
        t = torch.from_numpy(src.copy()).cuda()
        keep.append(t)
        return t

    d = inp.desc()
    for ti, im in enumerate(inp.images):
        for name, arr in (("image", im.image), ("mag", im.mag), ("ori", im.ori)):
            setattr(d.images[ti], name, dev(arr).data_ptr())
        if im.image_next is not None:
            for name, arr in (("image_next", im.image_next), ("mag_next", im.mag_next),
                              ("ori_next", im.ori_next)):
                setattr(d.images[ti], name, dev(arr).data_ptr())
        if im.image_b is not None:
            for name, arr in (("image_b", im.image_b), ("mag_b", im.mag_b)):
                setattr(d.images[ti], name, dev(arr).data_ptr())
    d.grid_wgs = dev(inp.grid_wgs).data_ptr()
    d.grid_pts = dev(inp.grid_pts).data_ptr()
    gp3 = dev(inp.gridpt3)
    d_ncc = dev(ncc)
    io = [d, gp3.data_ptr(), d_ncc.data_ptr()]
    if voxels is not None:
        off = np.concatenate([[0], np.cumsum(ncc["NumOfHeight"].astype(np.int64))]).astype(np.int64)
        io += [dev(voxels).data_ptr(), dev(off).data_ptr()]
    return tuple(io), {"keep": keep, "gp3": gp3, "ncc": d_ncc,
                       "vox": keep[-2] if voxels is not None else None}


def from_device(t, dtype) -> np.ndarray:
    return t.cpu().numpy().view(dtype)
