"""Seeded synthetic grids and SSH fields standing in for the reference's MPAS CSVs.

The reference reads five CSVs of a 2,313,486-cell MPAS ocean grid
(code.f90:37-49, mom6_code.f90:95-99) that are not distributed with it.  These
generators build grids with the same sizes and value ranges:

* Fibonacci-lattice cells on the unit sphere (the kernel assumes |t| = 1,
  fast_sum_module.f90:20-27), masked to an "ocean" by a random real
  spherical-harmonic field;
* 0.25 degree logically rectangular lon-lat cells with exact spherical areas;
* SSH fields as sums of real spherical harmonics with a red spectrum, scaled to
  1 m RMS, optionally with Gaussian bumps.

Spherical harmonics are evaluated with the standard fully normalised associated
Legendre recurrences (sectoral seed, then three-term recurrence in degree),
vectorised over points with torch so that degree 128 on 3.3M points runs in
about a second on a GPU.  Only numpy's default_rng drives randomness, so a seed
fully determines a grid on any machine.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

EARTH_RADIUS_M = 6371220.0


@dataclass
class Grid:
    """Ocean cells of one grid: unit-sphere coordinates and cell areas (m^2)."""
    name: str
    xs: np.ndarray
    ys: np.ndarray
    zs: np.ndarray
    areas: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return len(self.xs)


def fibonacci_points(n: int) -> np.ndarray:
    """n points of the Fibonacci lattice, (n, 3) float64 unit vectors."""
    i = np.arange(n, dtype=np.float64)
    z = 1.0 - (2.0 * i + 1.0) / n
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = i * (math.pi * (3.0 - math.sqrt(5.0)))
    p = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    return p


def lonlat_points(nlon: int = 1440, nlat: int = 720):
    """Cell centres of a regular lon-lat grid plus exact cell areas on the unit sphere."""
    dlon = 2.0 * math.pi / nlon
    dlat = math.pi / nlat
    lon = (np.arange(nlon) + 0.5) * dlon
    lat_edges = -0.5 * math.pi + np.arange(nlat + 1) * dlat
    lat = 0.5 * (lat_edges[:-1] + lat_edges[1:])
    LAT, LON = np.meshgrid(lat, lon, indexing="ij")
    p = np.stack([np.cos(LAT) * np.cos(LON), np.cos(LAT) * np.sin(LON), np.sin(LAT)], axis=-1).reshape(-1, 3)
    band = dlon * (np.sin(lat_edges[1:]) - np.sin(lat_edges[:-1]))
    area = np.repeat(band, nlon)
    return p, area


def _device(device):
    if device is None:
        return torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu")
    return torch.device(device)


def harmonic_fields(pts: np.ndarray, lmin: int, lmax: int, coeffs: list, device=None) -> np.ndarray:
    """Evaluate real SH expansions at points.

    coeffs[m] is an array (F, lmax-m+1, 2): cosine and sine coefficients of
    degrees l = m..lmax for order m (entries for l < lmin are ignored).
    Returns (F, N) float64.
    """
    dev = _device(device)
    P = torch.as_tensor(pts, dtype=torch.float64, device=dev)
    ct = P[:, 2].clamp(-1.0, 1.0)
    st = torch.sqrt(torch.clamp(1.0 - ct * ct, min=0.0))
    phi = torch.atan2(P[:, 1], P[:, 0])
    F = coeffs[0].shape[0]
    out = torch.zeros(F, P.shape[0], dtype=torch.float64, device=dev)
    pmm = torch.ones_like(ct)                       # normalised P_00 (4pi convention, up to a constant)
    for m in range(0, lmax + 1):
        if m > 0:
            pmm = pmm * st * math.sqrt((2.0 * m + 1.0) / (2.0 * m))
        nl = lmax - m + 1
        rows = torch.empty(nl, P.shape[0], dtype=torch.float64, device=dev)
        rows[0] = pmm
        if nl > 1:
            rows[1] = math.sqrt(2.0 * m + 3.0) * ct * pmm
        for k in range(2, nl):
            l = m + k
            a = math.sqrt((4.0 * l * l - 1.0) / (l * l - m * m))
            b = math.sqrt(((l - 1.0) ** 2 - m * m) / (4.0 * (l - 1.0) ** 2 - 1.0))
            rows[k] = a * (ct * rows[k - 1] - b * rows[k - 2])
        c = torch.as_tensor(np.array(coeffs[m], dtype=np.float64), device=dev)      # (F, nl, 2)
        keep = torch.as_tensor((np.arange(m, lmax + 1) >= lmin).astype(np.float64), device=dev)
        c = c * keep[None, :, None]
        A = c[:, :, 0] @ rows                                                       # (F, N)
        if m == 0:
            out += A
        else:
            B = c[:, :, 1] @ rows
            out += A * torch.cos(m * phi)[None, :] + B * torch.sin(m * phi)[None, :]
    return out.cpu().numpy()


def random_coeffs(rng: np.random.Generator, lmax: int, nfields: int, spectrum) -> list:
    """Per-order coefficient blocks with standard deviation spectrum(l)."""
    out = []
    for m in range(lmax + 1):
        ls = np.arange(m, lmax + 1, dtype=np.float64)
        sd = spectrum(ls)
        out.append(rng.standard_normal((nfields, len(ls), 2)) * sd[None, :, None])
    return out


def ssh_fields(pts, rng, nfields=1, lmin=1, lmax=32, rms=1.0, bumps=0, bump_amp=0.5,
               bump_width_m=200e3, device=None) -> np.ndarray:
    """SSH fields (F, N): SH degrees lmin..lmax with coefficients N(0, (l+1)^-2),
    each field scaled to `rms` metres RMS over the cells, plus `bumps` Gaussian
    bumps of amplitude bump_amp and standard deviation bump_width_m."""
    co = random_coeffs(rng, lmax, nfields, lambda l: 1.0 / (l + 1.0))
    h = harmonic_fields(pts, lmin, lmax, co, device=device)
    h *= rms / np.sqrt(np.mean(h * h, axis=1, keepdims=True))
    if bumps:
        sites = rng.standard_normal((nfields, bumps, 3))
        sites /= np.linalg.norm(sites, axis=2, keepdims=True)
        w = bump_width_m / EARTH_RADIUS_M
        for f in range(nfields):
            for k in range(bumps):
                cosd = np.clip(pts @ sites[f, k], -1.0, 1.0)
                d = np.arccos(cosd)
                h[f] += bump_amp * np.exp(-0.5 * (d / w) ** 2)
    return h


def ocean_mask(pts, rng, lmax, keep=None, keep_frac=0.7, device=None) -> np.ndarray:
    """Boolean mask of ocean cells: the cells where a seeded real SH field of
    degree <= lmax is largest, keeping `keep` cells or a fraction keep_frac."""
    co = random_coeffs(rng, lmax, 1, lambda l: np.ones_like(l))
    f = harmonic_fields(pts, 1, lmax, co, device=device)[0]
    n = len(f)
    k = keep if keep is not None else int(round(keep_frac * n))
    order = np.argsort(-f, kind="stable")
    mask = np.zeros(n, bool)
    mask[order[:k]] = True
    return mask


def fibonacci_grid(n_cells: int, seed: int = 0, n_lattice: int | None = None, area_jitter: float = 0.05,
                   mask_lmax: int = 8, device=None, name=None) -> Grid:
    """Fibonacci-lattice grid of n_lattice points masked to exactly n_cells ocean
    cells (n_lattice defaults to n_cells / 0.7).  Areas are the lattice's mean
    cell area times (1 + area_jitter * U(-1, 1))."""
    rng = np.random.default_rng(seed)
    nl = n_lattice or int(round(n_cells / 0.7))
    pts = fibonacci_points(nl)
    mask = ocean_mask(pts, rng, mask_lmax, keep=n_cells, device=device)
    p = pts[mask]
    base = 4.0 * math.pi * EARTH_RADIUS_M ** 2 / nl
    areas = base * (1.0 + area_jitter * rng.uniform(-1.0, 1.0, size=len(p)))
    return Grid(name or f"fib{n_cells}", np.ascontiguousarray(p[:, 0]), np.ascontiguousarray(p[:, 1]),
                np.ascontiguousarray(p[:, 2]), areas,
                {"n_lattice": nl, "seed": seed, "area_jitter": area_jitter, "mask_lmax": mask_lmax})


def lonlat_grid(nlon=1440, nlat=720, seed=1, mask_lmax=12, keep_frac=0.7, device=None) -> Grid:
    """MOM6-style logically rectangular 0.25 degree grid with a seeded land mask."""
    rng = np.random.default_rng(seed)
    pts, area = lonlat_points(nlon, nlat)
    mask = ocean_mask(pts, rng, mask_lmax, keep_frac=keep_frac, device=device)
    p = pts[mask]
    return Grid(f"lonlat{nlon}x{nlat}", np.ascontiguousarray(p[:, 0]), np.ascontiguousarray(p[:, 1]),
                np.ascontiguousarray(p[:, 2]), area[mask] * EARTH_RADIUS_M ** 2,
                {"nlon": nlon, "nlat": nlat, "seed": seed, "mask_lmax": mask_lmax})


def grid_points(g: Grid) -> np.ndarray:
    return np.stack([g.xs, g.ys, g.zs], axis=1)


# --------------------------------------------------------------------- named configs
def config_grid(name: str, device=None) -> Grid:
    """The grids of the five benchmark configurations.

    cfg0: 40,962-point Fibonacci lattice, ~70% kept (degree-8 mask).
    cfg1: 1440x720 lon-lat, degree-12 mask.
    cfg2 / cfg3: 3.3M-point lattice masked to 2,313,486 cells, areas jitter 0.1.
    serve_<n>: n-cell masked Fibonacci grid (serving mix).
    small_<n>: n-cell masked Fibonacci grid for tests.
    """
    if name == "cfg0":
        return fibonacci_grid(28673, seed=0, n_lattice=40962, area_jitter=0.05, mask_lmax=8, device=device,
                              name="cfg0")
    if name == "cfg1":
        return lonlat_grid(device=device)
    if name in ("cfg2", "cfg3"):
        return fibonacci_grid(2313486, seed=2, n_lattice=3300000, area_jitter=0.1, mask_lmax=8, device=device,
                              name="cfg2")
    if name.startswith("serve_"):
        n = int(name.split("_")[1])
        return fibonacci_grid(n, seed=4, area_jitter=0.1, mask_lmax=8, device=device, name=name)
    if name.startswith("small_"):
        n = int(name.split("_")[1])
        return fibonacci_grid(n, seed=7, area_jitter=0.05, mask_lmax=8, device=device, name=name)
    raise KeyError(name)


def config_ssh(name: str, g: Grid, nfields: int = 1, seed: int = 11, device=None) -> np.ndarray:
    """SSH fields (F, N) for a configuration: degree 1-32 for cfg0/cfg1/small,
    degree 1-128 plus 8 bumps for cfg2, degree 1-128 for cfg3/serving."""
    rng = np.random.default_rng(seed)
    pts = grid_points(g)
    if name in ("cfg0", "cfg1") or name.startswith("small_"):
        return ssh_fields(pts, rng, nfields, 1, 32, device=device)
    if name == "cfg2":
        return ssh_fields(pts, rng, nfields, 1, 128, bumps=8, device=device)
    return ssh_fields(pts, rng, nfields, 1, 128, device=device)
