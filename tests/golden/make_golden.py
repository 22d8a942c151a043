"""Generates the golden vectors in this folder from the reference SETSM code.

The reference ships no tests, fixtures or sample imagery, so its known answers
are produced here: seeded synthetic cases (tests/cases.py) are run through the
reference's own InitializeVoxel / VerticalLineLocus / AWNCC, compiled from its
sources into oracle/_ref/libsetsm_ref.so (``make -C oracle ref``).  Each
fixture holds a digest of the case's inputs and the reference's outputs, so
tests/test_oracle_golden.py can pin the oracle (and the CUDA kernels) on a
machine without the reference sources.

    python tests/golden/make_golden.py [name ...]
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# small versions of the parity cases: every route the matcher takes
GOLDEN = {
    "m7": dict(size=512, nodes=24, res=8.0, n_heights=32),
    "m11": dict(size=512, nodes=24, res=8.0, n_heights=32, template=15),
    "m7_edges": dict(size=512, nodes=24, res=8.0, n_heights=32, zero_patch=True,
                     unmatched_frac=0.1, minmax=(0.0, 260.0)),
    "v7_gncc": dict(size=512, nodes=20, res=9.0, n_heights=24, cmr=False, sgm=-1,
                    ortho_frac=0.5),
    "v11_it2": dict(size=512, nodes=16, res=10.0, n_heights=24, cmr=False, sgm=-1, it=2,
                    iters=(1, 2), template=15, ortho_frac=0.5),
    "l2_combined": dict(L=2, it=2, iters=(1, 2), cmr=False, sgm=-1, ortho_frac=0.5, nodes=16,
                        res=16.0, n_heights=16, hs=2.0, template=15),
    "l3_m": dict(L=3, it=1, cmr=True, nodes=12, res=24.0, n_heights=16, hs=3.0, template=15),
}


# AWNCC with semi-global aggregation (Pyramid_step <= SGM_py): the voxel route
# at level 0 (iterations 1 and 2; level 0 from iteration 2 keeps the peak's
# window NCC) and at level 1.  The C restatement of the oracle covers the
# non-SGM peak loop only; these are checked against the reference build and
# its fixtures.
GOLDEN_SGM = {
    "v7_sgm": dict(size=512, nodes=24, res=8.0, n_heights=32, cmr=False, sgm=1, ortho_frac=0.5),
    "v7_sgm_it2": dict(size=512, nodes=20, res=9.0, n_heights=24, cmr=False, sgm=1, it=2,
                       iters=(1, 2), ortho_frac=0.5),
    "v11_sgm": dict(size=512, nodes=20, res=9.0, n_heights=32, cmr=False, sgm=1, template=15),
    "l1_sgm": dict(L=1, it=1, cmr=False, sgm=1, nodes=16, res=12.0, n_heights=20, hs=1.0,
                   template=15, ortho_frac=0.5),
}


# The orthoimage-window variants (VerticalLineLocus_seeddem, setsm_code.cpp:
# 7720-7880; VerticalLineLocus_blunder, :7882-8026): kwargs of
# tests/cases.py:make_variant_case plus the call ("seeddem", or "blunder"
# with its iteration and bblunder flag).
GOLDEN_VARIANTS = {
    "sd_l0": dict(kind="seeddem", case=dict(seed=5, nodes=28, res=8.0, L=0)),
    "sd_mt_l1": dict(kind="seeddem", case=dict(seed=6, nodes=20, res=10.0, L=1, template=15,
                                               blunder_level=2, matchtag=True)),
    "bl_l0": dict(kind="blunder", iteration=1, bblunder=False,
                  case=dict(seed=7, nodes=28, res=8.0, L=0, blunder_level=1)),
    "bl_l3_bb": dict(kind="blunder", iteration=2, bblunder=True,
                     case=dict(seed=8, nodes=16, res=16.0, L=3, template=15, blunder_level=3)),
}


# Ortho_blunder (setsm_code.cpp:8028-8232) with VerticalLineLocus_Ortho:
# kwargs of tests/cases.py:make_tin_case; the fixture keeps the points,
# triangles and UGRID it starts from.
GOLDEN_TIN = {
    "tin_l0": dict(mpp=1.5, case=dict(seed=9)),
    "tin_l1_3img": dict(mpp=2.0, case=dict(seed=12, L=1, res=12.0, template=15, n_images=3)),
}


# SetHeightRange (setsm_code.cpp:9851-10255): kwargs of
# tests/cases.py:make_range_case and the call's iteration / MPP / level
# check_matching_rate / pre_DEMtif and seedDEMsigma.  It reads no image, so
# the fixture keeps every input it reads (grid geometry, points, triangles,
# UGRID).
GOLDEN_RANGE = {
    "range_l0": dict(iteration=1, mpp=1.5, lcmr=False, case=dict(seed=13)),
    "range_l3": dict(iteration=2, mpp=2.0, lcmr=True,
                     case=dict(seed=14, L=3, res=24.0, template=15, nodes=16)),
    "range_l1_seed": dict(iteration=3, mpp=1.0, lcmr=False, pre_dem=True, sigma=2.5,
                          case=dict(seed=15, L=1, res=12.0, template=15, nodes=24, n_images=3)),
}


# SelectMPs (setsm_code.cpp:8535-8895) on the reference build's matching of
# a case; the fixture keeps every input it reads (NCCresult, UGRID, grid
# points) and the call's arguments: (Th_roh, Th_roh_min, Th_roh_start,
# Th_roh_next, iteration, MPP, final_level_iteration, MPP_stereo_angle).
GOLDEN_SELECT = {
    "select_l0": dict(case="m7", level=0, args=(0.6, 0.2, 0.8, 0.7, 1, 1.5, 1, 10.0)),
    "select_l1": dict(case="v7_gncc", level=1, args=(0.5, 0.45, 0.5, 0.4, 2, 2.0, 3, 10.0)),
    "select_l3": dict(case="l3_m", level=3, args=(0.3, 0.25, 0.3, 0.2, 3, 2.0, 3, 3.0)),
}


def select_case(name):
    """(inputs, nccresult, fixture arrays) of SelectMPs fixture `name`."""
    from setsm_b200 import abi
    from tests import cases
    z = np.load(fixture_path(name))
    v = GOLDEN_SELECT[name]
    inp = cases.make_case(**cases.CASES[v["case"]])
    inp.pyramid_step = v["level"]
    inp.gridpt3 = z["init_gp3"].view(abi.UGRID_DTYPE).copy()
    inp.grid_pts = z["grid_pts"].copy()
    return inp, z["ncc"].view(abi.NCCRESULT_DTYPE).copy(), z


# blunder_detection_TIN (setsm_code.cpp:9158-9787): kwargs of
# tests/cases.py:make_tin_blunder_case and the call's (iteration,
# flag_blunder, count_bl, Hinterval); the fixture keeps every input it reads.
GOLDEN_TINB = {
    "tinb_l0": dict(call=(1, True, 1, 60.0), case=dict(seed=17)),
    "tinb_l3": dict(call=(2, True, 2, 40.0),
                    case=dict(seed=18, L=3, res=24.0, template=15, nodes=16)),
    "tinb_l1_anchor": dict(call=(1, False, 3, 80.0),
                           case=dict(seed=19, L=1, res=12.0, template=15, nodes=24)),
}


def tinb_case(name):
    """(inputs, pts, tris, ortho_ncc, fixture arrays) of fixture `name`."""
    from setsm_b200 import abi
    from tests import cases
    z = np.load(fixture_path(name))
    inp, _, _, _ = cases.make_tin_blunder_case(**GOLDEN_TINB[name]["case"])
    inp.boundary = z["boundary"].copy()
    inp.grid_resolution = float(z["grid_resolution"])
    inp.gridpt3 = z["init_gp3"].view(abi.UGRID_DTYPE).copy()
    return (inp, z["init_pts"].view(abi.POINT3_DTYPE).copy(), z["tris"].view(abi.TRI_DTYPE).copy(),
            z["oncc"].copy(), z)


def range_case(name):
    """(inputs, pts, tris, fixture arrays) of SetHeightRange fixture `name`."""
    from setsm_b200 import abi
    from tests import cases
    z = np.load(fixture_path(name))
    v = GOLDEN_RANGE[name]
    inp, _, _ = cases.make_range_case(**v["case"])
    inp.boundary = z["boundary"].copy()
    inp.grid_resolution = float(z["grid_resolution"])
    inp.pre_dem_tif = bool(v.get("pre_dem", False))
    inp.gridpt3 = z["init_gp3"].view(abi.UGRID_DTYPE).copy()
    return inp, z["pts"].view(abi.POINT3_DTYPE).copy(), z["tris"].view(abi.TRI_DTYPE).copy(), z


def tin_case(name):
    """(inputs, pts, tris, fixture arrays) of TIN fixture `name`: images from
    the seeded case, RPCs, points, triangles and UGRID from the fixture."""
    from setsm_b200 import abi
    from tests import cases
    z = np.load(fixture_path(name))
    inp, _, _ = cases.make_tin_case(**GOLDEN_TIN[name]["case"])
    for im, rpc in zip(inp.images, z["rpc"]):
        im.rpc = np.ascontiguousarray(rpc)
    inp.gridpt3 = z["init_gp3"].view(abi.UGRID_DTYPE).copy()
    pts = z["init_pts"].view(abi.POINT3_DTYPE).copy()
    tris = z["tris"].view(abi.TRI_DTYPE).copy()
    return inp, pts, tris, z


def variant_case(name):
    """The inputs of variant fixture `name` (RPCs from the fixture) and the
    fixture's arrays."""
    from tests import cases
    z = np.load(fixture_path(name))
    inp = cases.make_variant_case(**GOLDEN_VARIANTS[name]["case"])
    for im, rpc in zip(inp.images, z["rpc"]):
        im.rpc = np.ascontiguousarray(rpc)
    return inp, z


def image_digest(inp) -> str:
    h = hashlib.sha256()
    for im in inp.images:
        for a in (im.image, im.mag):
            h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def input_digest(inp) -> str:
    h = hashlib.sha256()
    for im in inp.images:
        for a in (im.image, im.mag, im.ori, np.asarray(im.rpc, dtype=np.float64)):
            h.update(np.ascontiguousarray(a).tobytes())
        for a in (im.image_next, im.mag_next, im.ori_next, im.image_b, im.mag_b):
            if a is not None:
                h.update(np.ascontiguousarray(a).tobytes())
    for a in (inp.grid_pts, inp.grid_wgs, inp.gridpt3):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def clean(rec: np.ndarray) -> np.ndarray:
    """Record array with its padding bytes zeroed (they carry whatever the
    reference's allocations held and are not part of any result)."""
    out = np.zeros(rec.shape, dtype=rec.dtype)
    for f in rec.dtype.names:
        out[f] = rec[f]
    return out


def fixture_path(name: str) -> str:
    return os.path.join(HERE, f"{name}.npz")


def main(only=None) -> None:
    """Writes every fixture, or only the names in `only`."""
    from oracle import refpy
    from tests import cases
    if not refpy.available():
        raise SystemExit("reference build missing: make -C oracle ref")
    refpy.set_threads(os.cpu_count() or 1)
    for name, kw in list(GOLDEN.items()) + list(GOLDEN_SGM.items()):
        if only and name not in only:
            continue
        inp = cases.make_case(**kw)
        r = cases.run_cpu(refpy, inp, inp.iters)
        arrays = {
            "digest": np.array(input_digest(inp)),
            "acc": np.array(r["acc"]),
            "init_ncc": clean(r["init_ncc"]).view(np.uint8),
            "init_gp3": clean(r["init_gp3"]).view(np.uint8),
            "vll_ncc": clean(r["vll_ncc"]).view(np.uint8),
            "ncc": clean(r["ncc"]).view(np.uint8),
        }
        if r["vox"] is not None:
            arrays["init_vox"] = clean(r["init_vox"]).view(np.uint8)
            arrays["vll_vox"] = clean(r["vll_vox"]).view(np.uint8)
        np.savez_compressed(fixture_path(name), **arrays)
        print(f"{name}: acc {r['acc']}, peaks {(r['ncc']['result4'] > 0).sum()}, "
              f"{os.path.getsize(fixture_path(name))} bytes")

    for name, v in GOLDEN_VARIANTS.items():
        if only and name not in only:
            continue
        inp = cases.make_variant_case(**v["case"])
        # the RPC fit of the synthetic scene rounds differently on other CPUs
        # (its least-squares solve); the fixture carries the coefficients
        arrays = {"digest": np.array(input_digest(inp)),
                  "rpc": np.stack([np.asarray(im.rpc, dtype=np.float64) for im in inp.images]),
                  "init_gp3": clean(inp.gridpt3).view(np.uint8)}
        if v["kind"] == "seeddem":
            refpy.vll_seeddem(inp)
        else:
            arrays["ncc"] = refpy.vll_blunder(inp, v["iteration"], v["bblunder"])
        arrays["gp3"] = clean(inp.gridpt3).view(np.uint8)
        np.savez_compressed(fixture_path(name), **arrays)
        print(f"{name}: {os.path.getsize(fixture_path(name))} bytes")

    for name, v in GOLDEN_TIN.items():
        if only and name not in only:
            continue
        inp, pts, tris = cases.make_tin_case(**v["case"])
        arrays = {"rpc": np.stack([np.asarray(im.rpc, dtype=np.float64) for im in inp.images]),
                  "img_digest": np.array(image_digest(inp)),
                  "init_gp3": clean(inp.gridpt3).view(np.uint8),
                  "init_pts": clean(pts).view(np.uint8), "tris": tris.view(np.uint8)}
        refpy.ortho_blunder(inp, v["mpp"], pts, tris)
        arrays["gp3"] = clean(inp.gridpt3).view(np.uint8)
        arrays["pts"] = clean(pts).view(np.uint8)
        np.savez_compressed(fixture_path(name), **arrays)
        print(f"{name}: {os.path.getsize(fixture_path(name))} bytes")

    for name, v in GOLDEN_RANGE.items():
        if only and name not in only:
            continue
        inp, pts, tris = cases.make_range_case(**v["case"])
        inp.pre_dem_tif = bool(v.get("pre_dem", False))
        out, ext = refpy.set_height_range(inp, pts, tris, v["iteration"], v["mpp"], v["lcmr"],
                                          v.get("sigma", 0.0))
        np.savez_compressed(fixture_path(name), boundary=np.asarray(inp.boundary),
                            grid_resolution=np.array(inp.grid_resolution),
                            init_gp3=clean(inp.gridpt3).view(np.uint8),
                            pts=clean(pts).view(np.uint8), tris=tris.view(np.uint8),
                            result=clean(out).view(np.uint8), extent=np.array(ext))
        print(f"{name}: extent {ext}, {os.path.getsize(fixture_path(name))} bytes")

    for name, v in GOLDEN_SELECT.items():
        if only and name not in only:
            continue
        inp, ncc = cases.make_select_case(v["case"])
        inp.pyramid_step = v["level"]
        init = clean(inp.gridpt3)
        r, pts = refpy.select_mps(inp, ncc, *v["args"])
        np.savez_compressed(fixture_path(name), ncc=clean(ncc).view(np.uint8),
                            init_gp3=init.view(np.uint8), grid_pts=inp.grid_pts,
                            gp3=clean(inp.gridpt3).view(np.uint8), pts=clean(pts).view(np.uint8),
                            ret=np.array(r))
        print(f"{name}: {r} points, {os.path.getsize(fixture_path(name))} bytes")

    for name, v in GOLDEN_TINB.items():
        if only and name not in only:
            continue
        inp, pts, tris, oncc = cases.make_tin_blunder_case(**v["case"])
        init_gp3, init_pts = clean(inp.gridpt3), clean(pts)
        det = np.zeros(len(pts), np.uint8)
        counts = np.zeros(2, np.int64)
        zext = np.array([1e5, -1e5])
        it, fb, cbl, hint = v["call"]
        refpy.blunder_detection_tin(inp, it, oncc, fb, cbl, hint, pts, det, tris, counts, zext)
        np.savez_compressed(fixture_path(name), boundary=np.asarray(inp.boundary),
                            grid_resolution=np.array(inp.grid_resolution),
                            init_gp3=init_gp3.view(np.uint8), init_pts=init_pts.view(np.uint8),
                            tris=tris.view(np.uint8), oncc=oncc, gp3=clean(inp.gridpt3).view(np.uint8),
                            pts=clean(pts).view(np.uint8), detected=det, counts=counts, zext=zext)
        print(f"{name}: {int(det.sum())} new blunders, {os.path.getsize(fixture_path(name))} bytes")


if __name__ == "__main__":
    main(set(sys.argv[1:]) or None)
