"""Seeded synthetic stereo scenes for the vertical-line-locus path.

No public imagery or RPC metadata is available offline, so every workload is
generated here, with the shapes, sizes and value distributions of the matching
configurations:

* DEM: fBm (spectral synthesis, Hurst exponent ``hurst``) scaled to
  ``[0, relief]`` metres plus Gaussian hills.
* Texture: band-limited fBm reflectance (hash-lattice value noise, octaves from
  ``tex_lambda_max`` down to ``tex_lambda_min`` metres), quantised to 11-bit
  values in uint16, plus per-image sensor noise.
* Cameras: pushbroom, ``altitude`` metres, along-track view angle per image
  (stereo convergence), small yaw; images rendered by ray/DEM intersection
  (fixed-point iteration on the DEM height).
* RPC: each camera is fitted with a 20+20+20+20-coefficient cubic rational
  polynomial in normalised (lon, lat, h), stored in the reference's row layout
  (offsets, scales, LINE_NUM, LINE_DEN, SAMP_NUM, SAMP_DEN; SubFunctions.cpp:1494-1582)
  so that GetObjectToImageRPC_single (CoordConversion.hpp:26-86) evaluates it.
* Grid: SetDEMGrid's convention (SubFunctions.cpp:3363-3381), polar-stereographic
  metres, with Grid_wgs from the inverse projection.

Everything is torch so the same code runs on the CPU for small cases and on a
GPU for the 16384^2 scenes.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

# --------------------------------------------------------------------------
# Polar stereographic (north) constants and transforms.  Same published
# formulas as wgs2ps_single / ps2wgs_single (CoordConversion.cpp:103, :396),
# restated for generating inputs on any device.
# --------------------------------------------------------------------------
_DEG = math.pi / 180.0


def transparam_north() -> dict:
    """TransParam for north polar stereographic (SubFunctions.cpp:1186-1221)."""
    a = 6378137.0
    e = 0.08181919
    phi_c = 70.0 * (3.141592653589793 / 180)
    lambda_0 = -45.0 * (3.141592653589793 / 180)
    t_c = math.tan(math.pi / 4.0 - phi_c / 2.0) / (
        ((1.0 - e * math.sin(phi_c)) / (1.0 + e * math.sin(phi_c))) ** (e / 2.0))
    m_c = math.cos(phi_c) / math.sqrt(1.0 - e ** 2 * math.sin(phi_c) ** 2)
    sa = 6378137.0
    sb = 6356752.314245
    e2 = math.sqrt(sa * sa - sb * sb) / sb
    return dict(t_c=t_c, m_c=m_c, sa=sa, sb=sb, e2=e2, e2cuadrada=e2 * e2,
                c=sa * sa / sb, a=a, e=e, phi_c=phi_c, lambda_0=lambda_0, pm=1,
                projection=1, utm_zone=0, direction=b"X\x00", bHemisphere=1)


def wgs2ps(p: dict, lon, lat):
    lam = lon * p["pm"] * _DEG
    phi = lat * p["pm"] * _DEG
    e = p["e"]
    t = torch.tan(math.pi / 4.0 - phi / 2.0) / torch.pow(
        (1.0 - e * torch.sin(phi)) / (1.0 + e * torch.sin(phi)), e / 2.0)
    rho = p["a"] * p["m_c"] * t / p["t_c"]
    x = p["pm"] * rho * torch.sin(lam - p["lambda_0"])
    y = -p["pm"] * rho * torch.cos(lam - p["lambda_0"])
    return x, y


def ps2wgs(p: dict, x, y):
    e = p["e"]
    e2 = e * e
    e4 = e2 * e2
    e6 = e2 * e4
    e8 = e4 * e4
    x = x * p["pm"]
    y = y * p["pm"]
    rho = torch.sqrt(x * x + y * y)
    t = rho * p["t_c"] / (p["a"] * p["m_c"])
    chi = math.pi / 2 - 2 * torch.atan(t)
    phi = (chi + (e2 / 2 + 5 * e4 / 24 + e6 / 12 + 13 * e8 / 360) * torch.sin(2 * chi)
           + (7 * e4 / 48 + 29 * e6 / 240 + 811 * e8 / 11520) * torch.sin(4 * chi)
           + (7 * e6 / 120 + 81 * e8 / 1120) * torch.sin(6 * chi)
           + (4279 * e8 / 161280) * torch.sin(8 * chi))
    lam = p["lambda_0"] + torch.atan2(x, -y)
    phi = p["pm"] * phi
    lam = p["pm"] * lam
    lam = torch.where(lam > math.pi, lam - 2 * math.pi, lam)
    lam = torch.where(lam < -math.pi, lam + 2 * math.pi, lam)
    return lam / _DEG, phi / _DEG


# --------------------------------------------------------------------------
# RPC (RPC00B term order of GetObjectToImageRPC_single)
# --------------------------------------------------------------------------
def rpc_terms(L, P, H):
    one = torch.ones_like(L)
    return torch.stack([one, L, P, H, L * P, L * H, P * H, L * L, P * P, H * H,
                        (P * L) * H, (L * L) * L, (L * P) * P, (L * H) * H, (L * L) * P,
                        (P * P) * P, (P * H) * H, (L * L) * H, (P * P) * H, (H * H) * H], dim=-1)


def rpc_eval(rpc: np.ndarray, lon, lat, h, adjust=(0.0, 0.0)):
    """Evaluate a 90-double RPC (no wrap / clamp); returns (sample, line)."""
    r = torch.as_tensor(rpc, dtype=torch.float64, device=lon.device)
    L = (lon - r[2]) / r[7]
    P = (lat - r[3]) / r[8]
    H = (h - r[4]) / r[9]
    t = rpc_terms(L, P, H)
    c = [t @ r[10 + 20 * j: 30 + 20 * j] for j in range(4)]
    line = (c[0] / c[1]) * r[5] + r[0] + adjust[0]
    samp = (c[2] / c[3]) * r[6] + r[1] + adjust[1]
    return samp, line


def fit_rpc(lon, lat, h, line, samp) -> np.ndarray:
    """Least-squares cubic RPC fit (denominator constant term fixed to 1)."""
    lon = lon.double().cpu(); lat = lat.double().cpu(); h = h.double().cpu()
    line = line.double().cpu(); samp = samp.double().cpu()
    off = [float(line.mean()), float(samp.mean()), float(lon.mean()), float(lat.mean()),
           float(h.mean())]
    sc = [float((line - off[0]).abs().max()), float((samp - off[1]).abs().max()),
          float((lon - off[2]).abs().max()), float((lat - off[3]).abs().max()),
          float((h - off[4]).abs().max())]
    L = (lon - off[2]) / sc[2]
    P = (lat - off[3]) / sc[3]
    H = (h - off[4]) / sc[4]
    t = rpc_terms(L, P, H)
    rpc = np.zeros(90)
    rpc[0:5] = off
    rpc[5:10] = sc
    for j, target in enumerate([(line - off[0]) / sc[0], (samp - off[1]) / sc[1]]):
        A = torch.cat([t, -target[:, None] * t[:, 1:]], dim=1)
        sol = torch.linalg.lstsq(A, target[:, None], driver="gelsd").solution[:, 0]
        num = sol[:20]
        den = torch.cat([torch.ones(1, dtype=torch.float64), sol[20:]])
        rpc[10 + 40 * j: 30 + 40 * j] = num.numpy()
        rpc[30 + 40 * j: 50 + 40 * j] = den.numpy()
    return rpc


# --------------------------------------------------------------------------
# Noise
# --------------------------------------------------------------------------
_M32 = 0xFFFFFFFF


def _hash01(ix, iy, salt: int):
    h = (ix * 0x27D4EB2D + iy * 0x165667B1 + (salt * 0x9E3779B1 & _M32)) & _M32
    h = ((h ^ (h >> 15)) * 0x2C1B3C6D) & _M32
    h = ((h ^ (h >> 12)) * 0x297A2D39) & _M32
    h = h ^ (h >> 15)
    return h.to(torch.float32) * (1.0 / 4294967296.0)


def value_noise_fbm(x, y, lam_max: float, lam_min: float, hurst: float, salt: int):
    """Band-limited fBm value noise at metric coords (x, y >= 0); ~unit std."""
    out = torch.zeros_like(x, dtype=torch.float32)
    norm = 0.0
    lam = lam_max
    k = 0
    while lam >= lam_min:
        amp = (lam / lam_max) ** hurst
        u = x / lam
        v = y / lam
        iu = torch.floor(u)
        iv = torch.floor(v)
        fu = (u - iu).float()
        fv = (v - iv).float()
        iu = iu.long()
        iv = iv.long()
        su = fu * fu * (3 - 2 * fu)
        sv = fv * fv * (3 - 2 * fv)
        s = salt * 131 + k
        n00 = _hash01(iu, iv, s)
        n10 = _hash01(iu + 1, iv, s)
        n01 = _hash01(iu, iv + 1, s)
        n11 = _hash01(iu + 1, iv + 1, s)
        val = (n00 * (1 - su) + n10 * su) * (1 - sv) + (n01 * (1 - su) + n11 * su) * sv
        out += amp * (val - 0.5)
        norm += amp * amp
        lam *= 0.5
        k += 1
    # value noise with smoothstep blending has std ~0.21 per octave
    return out / (0.21 * math.sqrt(norm))


def fbm_surface(n: int, hurst: float, gen: torch.Generator, device) -> torch.Tensor:
    """n x n fBm by spectral synthesis, normalised to [0, 1]."""
    white = torch.randn((n, n), generator=gen, dtype=torch.float64).to(device)
    f = torch.fft.fftfreq(n, device=device, dtype=torch.float64)
    k = torch.sqrt(f[:, None] ** 2 + f[None, :] ** 2)
    k[0, 0] = 1.0
    amp = k ** (-(hurst + 1.0))
    amp[0, 0] = 0.0
    s = torch.fft.ifft2(torch.fft.fft2(white) * amp).real
    s = (s - s.min()) / (s.max() - s.min())
    return s


# --------------------------------------------------------------------------
# Scene
# --------------------------------------------------------------------------
@dataclass
class CameraSpec:
    view_deg: float            # along-track off-nadir view angle (+ forward)
    yaw_deg: float             # rotation of the image axes w.r.t. grid axes
    altitude: float = 770e3


@dataclass
class SceneSpec:
    seed: int = 1
    image_size: int = 2048     # pixels (square), level 0
    gsd: float = 0.5
    dem_spacing: float = 2.0
    dem_relief: float = 300.0
    hurst: float = 0.8
    n_hills: int = 3
    hill_height: tuple = (50.0, 150.0)
    cameras: tuple = (CameraSpec(15.0, 0.7), CameraSpec(-15.0, -0.9))
    center_lon: float = -49.5
    center_lat: float = 69.0
    tex_lambda_max: float = 48.0
    tex_lambda_min: float = 1.5
    tex_hurst: float = 0.5
    tex_mean: float = 900.0
    tex_gain: float = 260.0
    noise_dn: float = 3.0
    iterations: int = 10


@dataclass
class Scene:
    spec: SceneSpec
    param: dict
    center_xy: tuple
    dem: torch.Tensor          # float64 [nd, nd], metres
    dem_origin: tuple          # (x0, y0) of dem[0, 0]
    images: list = field(default_factory=list)   # torch int16 [H, W] (uint16 bits) per camera
    rpcs: list = field(default_factory=list)     # np float64[90] per camera
    rpc_residual_px: float = 0.0

    @property
    def h0(self) -> float:
        return float(self.dem.mean())

    def dem_at(self, x, y):
        """Bilinear DEM height at metric (x, y)."""
        d = self.dem
        nd = d.shape[0]
        u = ((x - self.dem_origin[0]) / self.spec.dem_spacing).clamp(0, nd - 1.000001)
        v = ((y - self.dem_origin[1]) / self.spec.dem_spacing).clamp(0, nd - 1.000001)
        iu = torch.floor(u).long()
        iv = torch.floor(v).long()
        fu = u - iu
        fv = v - iv
        a = d[iv, iu]
        b = d[iv, iu + 1]
        c = d[iv + 1, iu]
        e = d[iv + 1, iu + 1]
        return (a * (1 - fu) + b * fu) * (1 - fv) + (c * (1 - fu) + e * fu) * fv

    # ---- physical pushbroom camera --------------------------------------
    def cam_forward(self, ci: int, x, y, h):
        """Ground (x, y, h) -> (sample, line) with the exact pushbroom model."""
        cam = self.spec.cameras[ci]
        n = self.spec.image_size
        g = self.spec.gsd
        yaw = cam.yaw_deg * _DEG
        tv = math.tan(cam.view_deg * _DEG)
        dx = x - self.center_xy[0]
        dy = y - self.center_xy[1]
        u = math.cos(yaw) * dx + math.sin(yaw) * dy
        v = -math.sin(yaw) * dx + math.cos(yaw) * dy
        z0 = cam.altitude - self.h0
        line = n / 2 + (v + (h - self.h0) * tv) / g
        samp = n / 2 + u * (z0 / (cam.altitude - h)) / g
        return samp, line

    def cam_ground(self, ci: int, samp, line, h):
        cam = self.spec.cameras[ci]
        n = self.spec.image_size
        g = self.spec.gsd
        yaw = cam.yaw_deg * _DEG
        tv = math.tan(cam.view_deg * _DEG)
        z0 = cam.altitude - self.h0
        v = (line - n / 2) * g - (h - self.h0) * tv
        u = (samp - n / 2) * g * (cam.altitude - h) / z0
        x = self.center_xy[0] + math.cos(yaw) * u - math.sin(yaw) * v
        y = self.center_xy[1] + math.sin(yaw) * u + math.cos(yaw) * v
        return x, y

    def reflectance(self, x, y):
        """Two anisotropic (4:1) fBm layers with different dominant directions,
        blended by a slowly varying mask, plus an isotropic component: gives the
        locally consistent gradient orientation that real scenes have."""
        sp = self.spec
        xo = x - (self.center_xy[0] - 1e5)
        yo = y - (self.center_xy[1] - 1e5)
        out = 0.45 * value_noise_fbm(xo, yo, sp.tex_lambda_max, sp.tex_lambda_min,
                                     sp.tex_hurst, salt=sp.seed)
        mask = value_noise_fbm(xo, yo, 400.0, 200.0, 0.0, salt=sp.seed + 7)
        mask = torch.clamp(0.5 + 1.5 * mask, 0.0, 1.0)
        for li, ang in enumerate((0.5, 2.1)):
            ca, sa = math.cos(ang), math.sin(ang)
            u = ca * xo + sa * yo
            v = (-sa * xo + ca * yo) * 4.0
            lay = value_noise_fbm(u + 1e5, v + 4e5, sp.tex_lambda_max * 2, sp.tex_lambda_min * 2,
                                  sp.tex_hurst, salt=sp.seed + 11 * (li + 1))
            out = out + (mask if li == 0 else 1.0 - mask) * lay
        return out


def _render(scene: Scene, ci: int, device, rows_per_chunk: int) -> torch.Tensor:
    spec = scene.spec
    n = spec.image_size
    out = torch.empty((n, n), dtype=torch.int32, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(spec.seed * 1000 + 17 * ci + 5)
    cols = torch.arange(n, device=device, dtype=torch.float64)
    for r0 in range(0, n, rows_per_chunk):
        r1 = min(n, r0 + rows_per_chunk)
        line = torch.arange(r0, r1, device=device, dtype=torch.float64)[:, None].expand(-1, n)
        samp = cols[None, :].expand(r1 - r0, -1)
        h = torch.full_like(line, scene.h0)
        for _ in range(spec.iterations):
            x, y = scene.cam_ground(ci, samp, line, h)
            h = scene.dem_at(x, y)
        x, y = scene.cam_ground(ci, samp, line, h)
        tex = scene.reflectance(x, y)
        noise = torch.randn(tex.shape, generator=gen, device=device, dtype=torch.float32)
        dn = spec.tex_mean + spec.tex_gain * tex + spec.noise_dn * noise
        out[r0:r1] = torch.round(dn).clamp(0, 2047).to(torch.int32)
    # values are in [0, 2047], so the int16 bits are the uint16 image
    return out.to(torch.int16)


def make_scene(spec: SceneSpec, device="cpu", rows_per_chunk: int = 512) -> Scene:
    device = torch.device(device)
    gen = torch.Generator()
    gen.manual_seed(spec.seed)
    param = transparam_north()
    cx, cy = wgs2ps(param, torch.tensor(spec.center_lon, dtype=torch.float64),
                    torch.tensor(spec.center_lat, dtype=torch.float64))
    cx = float(cx); cy = float(cy)
    extent = spec.image_size * spec.gsd
    margin = 0.25 * extent + 400.0
    nd = int(math.ceil((extent + 2 * margin) / spec.dem_spacing)) + 1
    dem = fbm_surface(nd, spec.hurst, gen, device) * spec.dem_relief
    x0 = cx - (nd - 1) * spec.dem_spacing / 2
    y0 = cy - (nd - 1) * spec.dem_spacing / 2
    gx = x0 + torch.arange(nd, device=device, dtype=torch.float64) * spec.dem_spacing
    gy = y0 + torch.arange(nd, device=device, dtype=torch.float64) * spec.dem_spacing
    for _ in range(spec.n_hills):
        r = torch.rand(4, generator=gen, dtype=torch.float64)
        hh = spec.hill_height[0] + (spec.hill_height[1] - spec.hill_height[0]) * float(r[0])
        hx = cx + (float(r[1]) - 0.5) * extent * 0.8
        hy = cy + (float(r[2]) - 0.5) * extent * 0.8
        sig = extent * (0.05 + 0.1 * float(r[3]))
        dem = dem + hh * torch.exp(-((gx[None, :] - hx) ** 2 + (gy[:, None] - hy) ** 2)
                                   / (2 * sig * sig))
    scene = Scene(spec=spec, param=param, center_xy=(cx, cy), dem=dem, dem_origin=(x0, y0))

    # RPC fit per camera on a 3-D control grid over the footprint.
    hmin = float(dem.min()) - 60.0
    hmax = float(dem.max()) + 60.0
    half = extent * 0.6
    cg = torch.linspace(-half, half, 21, dtype=torch.float64)
    hg = torch.linspace(hmin, hmax, 9, dtype=torch.float64)
    X = (cx + cg[None, :, None]).expand(9, 21, 21).reshape(-1)
    Y = (cy + cg[None, None, :]).expand(9, 21, 21).reshape(-1)
    Hh = hg[:, None, None].expand(9, 21, 21).reshape(-1)
    lon, lat = ps2wgs(param, X, Y)
    resid = 0.0
    for ci in range(len(spec.cameras)):
        samp, line = scene.cam_forward(ci, X, Y, Hh)
        rpc = fit_rpc(lon, lat, Hh, line, samp)
        s2, l2 = rpc_eval(rpc, lon, lat, Hh)
        resid = max(resid, float(torch.max(torch.abs(s2 - samp))),
                    float(torch.max(torch.abs(l2 - line))))
        scene.rpcs.append(rpc)
    scene.rpc_residual_px = resid
    for ci in range(len(spec.cameras)):
        scene.images.append(_render(scene, ci, device, rows_per_chunk))
    return scene


# --------------------------------------------------------------------------
# Grids and per-node height ranges
# --------------------------------------------------------------------------
@dataclass
class Grid:
    boundary: np.ndarray       # [minX, minY, maxX, maxY]
    resolution: float
    width: int
    height: int
    pts: np.ndarray            # float64 [N, 2] projected metres
    wgs: np.ndarray            # float64 [N, 2] lon, lat
    truth: np.ndarray          # float64 [N] DEM height at each node


def make_grid(scene: Scene, n_nodes: int, resolution: float, device="cpu") -> Grid:
    """n_nodes x n_nodes grid centred on the scene, SetDEMGrid's convention."""
    cx, cy = scene.center_xy
    ext = n_nodes * resolution
    b = np.array([cx - ext / 2, cy - ext / 2, cx + ext / 2, cy + ext / 2])
    w = int(math.ceil((b[2] - b[0]) / resolution))
    hgt = int(math.ceil((b[3] - b[1]) / resolution))
    col = torch.arange(w, dtype=torch.float64, device=device)
    row = torch.arange(hgt, dtype=torch.float64, device=device)
    X = (b[0] + col[None, :] * resolution).expand(hgt, w).reshape(-1)
    Y = (b[1] + row[:, None] * resolution).expand(hgt, w).reshape(-1)
    lon, lat = ps2wgs(scene.param, X, Y)
    truth = scene.dem_at(X.to(scene.dem.device), Y.to(scene.dem.device))
    return Grid(boundary=b, resolution=resolution, width=w, height=hgt,
                pts=torch.stack([X, Y], 1).cpu().numpy(),
                wgs=torch.stack([lon, lat], 1).cpu().numpy(),
                truth=truth.cpu().numpy())


def ranges_uniform(grid: Grid, n_heights: int, step: float, sigma: float, seed: int):
    """Each node searches n_heights at `step` around truth + N(0, sigma)."""
    rng = np.random.default_rng(seed)
    centre = grid.truth + rng.normal(0.0, sigma, size=grid.truth.shape)
    span = n_heights * step
    lo = np.floor(centre - span / 2).astype(np.int64)
    hi = lo + int(round(span))
    return lo, hi, centre


def ranges_tin(scene: Scene, grid: Grid, n_seeds: int, k_min: int, k_max: int, step: float,
               noise: float, seed: int, lattice: int = 512, device="cpu"):
    """Per-node ranges from a coarse Delaunay TIN of jittered, noisy seeds.

    The TIN (scipy Delaunay over ``n_seeds`` jittered lattice points whose
    heights are the DEM plus N(0, noise)) is evaluated on a ``lattice`` x
    ``lattice`` raster over the grid and bilinearly refined to every node,
    which gives each node a prior height.  The candidate count is log-uniform
    in [k_min, k_max] at ``step`` metres; ranges are whole metres (UGRID keeps
    heights as short).  Returns (lo, hi, prior) as numpy arrays.
    """
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    b = grid.boundary
    side = int(math.ceil(math.sqrt(n_seeds)))
    gx, gy = np.meshgrid(np.linspace(b[0], b[2], side), np.linspace(b[1], b[3], side))
    jit = (b[2] - b[0]) / side * 0.35
    sx = (gx.ravel() + rng.uniform(-jit, jit, gx.size)).clip(b[0], b[2])
    sy = (gy.ravel() + rng.uniform(-jit, jit, gy.size)).clip(b[1], b[3])
    corners = np.array([[b[0], b[1]], [b[2], b[1]], [b[0], b[3]], [b[2], b[3]]])
    sx = np.concatenate([sx, corners[:, 0]])
    sy = np.concatenate([sy, corners[:, 1]])
    sh = scene.dem_at(torch.tensor(sx, dtype=torch.float64, device=scene.dem.device),
                      torch.tensor(sy, dtype=torch.float64, device=scene.dem.device)).cpu().numpy()
    sh = sh + rng.normal(0.0, noise, sx.size)
    tri = Delaunay(np.stack([sx, sy], 1))
    lx = np.linspace(b[0], b[2], lattice)
    ly = np.linspace(b[1], b[3], lattice)
    LX, LY = np.meshgrid(lx, ly)
    q = np.stack([LX.ravel(), LY.ravel()], 1)
    simplex = tri.find_simplex(q)
    simplex = np.where(simplex < 0, 0, simplex)
    T = tri.transform[simplex]
    bary = np.einsum("nij,nj->ni", T[:, :2], q - T[:, 2])
    w3 = np.concatenate([bary, 1 - bary.sum(1, keepdims=True)], 1)
    lat_prior = (w3 * sh[tri.simplices[simplex]]).sum(1).reshape(lattice, lattice)
    # bilinear refinement to the node grid
    dev = torch.device(device)
    P = torch.tensor(lat_prior, dtype=torch.float64, device=dev)
    u = (torch.tensor(grid.pts[:, 0], device=dev) - b[0]) / (b[2] - b[0]) * (lattice - 1)
    v = (torch.tensor(grid.pts[:, 1], device=dev) - b[1]) / (b[3] - b[1]) * (lattice - 1)
    u = u.clamp(0, lattice - 1.000001)
    v = v.clamp(0, lattice - 1.000001)
    iu, iv = torch.floor(u).long(), torch.floor(v).long()
    fu, fv = u - iu, v - iv
    prior = ((P[iv, iu] * (1 - fu) + P[iv, iu + 1] * fu) * (1 - fv)
             + (P[iv + 1, iu] * (1 - fu) + P[iv + 1, iu + 1] * fu) * fv).cpu().numpy()
    k = np.exp(rng.uniform(math.log(k_min), math.log(k_max), prior.shape))
    span = np.maximum(1, np.round(k * step)).astype(np.int64)
    lo = np.floor(prior - span / 2).astype(np.int64)
    hi = lo + span
    return lo, hi, prior
