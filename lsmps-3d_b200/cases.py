"""Seeded synthetic particle cases for the LSMPS step.

Portable random stream: splitmix64, mapped to doubles by (x >> 11) * 2**-53,
so that a C++, CUDA or Python generator seeded alike produces bit-identical
inputs.  Lattice and wall conventions follow the reference's hydrostatic box
generator (tool/generate_hydrostatic_box.cpp:50-99): fluid particles sit at
((i + 1/2) l0, (j + 1/2) l0, (k + 1/2) l0); wall particles sit on integer
planes with unit normals pointing into the fluid; edge and corner samples
belong to the x faces first, then the y faces, then the bottom.  Here every
face has `layers` parallel planes (0, -l0, -2 l0 on the low side and
n l0, (n+1) l0, (n+2) l0 on the high side).

The cell grid is derived from the particle bounds exactly as the reference
driver does it (src/app/simulation_driver.cu:83-108): padding = support
radius, origin = min - padding, dims = ceil((max + padding - origin) / h) + 1.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import abi

GAMMA = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """Values offset .. offset+n-1 of the splitmix64 stream started at `seed`."""
    with np.errstate(over="ignore"):
        k = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        z = np.uint64(seed) + k * GAMMA
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, n: int, offset: int = 0) -> np.ndarray:
    return (splitmix64(seed, n, offset) >> np.uint64(11)).astype(np.float64) * (2.0**-53)


def normal(seed: int, n: int) -> np.ndarray:
    """Box-Muller on pairs of the stream: u1 from even slots (mapped to (0, 1]),
    u2 from odd slots."""
    u = uniform01(seed, 2 * n)
    u1 = 1.0 - u[0::2]
    u2 = u[1::2]
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


@dataclass
class Case:
    name: str
    l0: float
    fluid: dict
    walls: dict
    params: abi.Params
    meta: dict = field(default_factory=dict)

    @property
    def n_fluid(self) -> int:
        return int(self.fluid["x"].shape[0])

    @property
    def n_wall(self) -> int:
        return int(self.walls["x"].shape[0])

    @property
    def n_cells(self) -> int:
        d = self.params.grid.dims
        return int(d[0]) * int(d[1]) * int(d[2])


def fluid_block(nx: int, ny: int, nz: int, l0: float) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """x-fastest lattice, as make_hydrostatic_box loops iz -> iy -> ix."""
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    x = (ix.ravel().astype(np.float64) + 0.5) * l0
    y = (iy.ravel().astype(np.float64) + 0.5) * l0
    z = (iz.ravel().astype(np.float64) + 0.5) * l0
    return x, y, z


def tank_walls(nx: int, ny: int, nz_top: int, l0: float, layers: int = 3):
    """Wall samples of an open-top tank whose interior is [0, nx l0] x [0, ny l0]
    with walls up to z = nz_top l0.  Returns (x, y, z, nx, ny, nz) arrays."""
    lo = -(layers - 1)
    pts = []
    for iz in range(lo, nz_top + 1):
        for iy in range(lo, ny + layers):
            for m in range(layers):
                pts.append((-m, iy, iz, 1.0, 0.0, 0.0))
                pts.append((nx + m, iy, iz, -1.0, 0.0, 0.0))
        for ix in range(1, nx):
            for m in range(layers):
                pts.append((ix, -m, iz, 0.0, 1.0, 0.0))
                pts.append((ix, ny + m, iz, 0.0, -1.0, 0.0))
    for iy in range(1, ny):
        for ix in range(1, nx):
            for m in range(layers):
                pts.append((ix, iy, -m, 0.0, 0.0, 1.0))
    a = np.asarray(pts, dtype=np.float64)
    return a[:, 0] * l0, a[:, 1] * l0, a[:, 2] * l0, a[:, 3].copy(), a[:, 4].copy(), a[:, 5].copy()


def _tank_walls_fast(nx: int, ny: int, nz_top: int, l0: float, layers: int = 3):
    """Vectorised tank_walls (identical output order) for large tanks."""
    lo = -(layers - 1)
    zs = np.arange(lo, nz_top + 1)
    ys = np.arange(lo, ny + layers)
    ms = np.arange(layers)
    inner_x = np.arange(1, nx)
    blocks = []
    for iz in zs:
        # x faces: for iy: for m: (low, high)
        iy_g, m_g = np.meshgrid(ys, ms, indexing="ij")
        n = iy_g.size
        xf = np.empty((n, 2, 6))
        xf[:, 0, 0] = -m_g.ravel()
        xf[:, 1, 0] = nx + m_g.ravel()
        xf[:, :, 1] = iy_g.ravel()[:, None]
        xf[:, :, 2] = iz
        xf[:, 0, 3:] = (1.0, 0.0, 0.0)
        xf[:, 1, 3:] = (-1.0, 0.0, 0.0)
        blocks.append(xf.reshape(-1, 6))
        ix_g, m_g = np.meshgrid(inner_x, ms, indexing="ij")
        n = ix_g.size
        yf = np.empty((n, 2, 6))
        yf[:, :, 0] = ix_g.ravel()[:, None]
        yf[:, 0, 1] = -m_g.ravel()
        yf[:, 1, 1] = ny + m_g.ravel()
        yf[:, :, 2] = iz
        yf[:, 0, 3:] = (0.0, 1.0, 0.0)
        yf[:, 1, 3:] = (0.0, -1.0, 0.0)
        blocks.append(yf.reshape(-1, 6))
    iy_g, ix_g, m_g = np.meshgrid(np.arange(1, ny), inner_x, ms, indexing="ij")
    bf = np.empty((iy_g.size, 6))
    bf[:, 0] = ix_g.ravel()
    bf[:, 1] = iy_g.ravel()
    bf[:, 2] = -m_g.ravel()
    bf[:, 3:] = (0.0, 0.0, 1.0)
    blocks.append(bf)
    a = np.concatenate(blocks, axis=0)
    return a[:, 0] * l0, a[:, 1] * l0, a[:, 2] * l0, a[:, 3].copy(), a[:, 4].copy(), a[:, 5].copy()


def derive_grid(params: abi.Params, xs: list[np.ndarray], ys: list[np.ndarray], zs: list[np.ndarray]) -> None:
    """derive_cell_grid_from_particles, src/app/simulation_driver.cu:83-108."""
    mins = [min(float(a.min()) for a in arrs if a.size) for arrs in (xs, ys, zs)]
    maxs = [max(float(a.max()) for a in arrs if a.size) for arrs in (xs, ys, zs)]
    pad = params.support_radius
    h = params.grid.cell_size
    for d in range(3):
        origin = mins[d] - pad
        params.grid.origin[d] = origin
        span = (maxs[d] + pad) - origin
        params.grid.dims[d] = int(math.ceil(span / h)) + 1


def hydrostatic_pressure(z: np.ndarray, height: float, l0: float, rho: float, g: float) -> np.ndarray:
    """make_hydrostatic_pressure, tests/reference/hydrostatic_surface_diagnostics.cu:170-183."""
    return rho * g * np.maximum(height - 0.5 * l0 - z, 0.0)


def _make_case(name, l0, fx, fy, fz, walls, fluid_height, params=None, meta=None) -> Case:
    p = params if params is not None else abi.default_params()
    p.particle_spacing = l0
    p.support_radius = 3.1 * l0
    p.grid.cell_size = p.support_radius
    p.near_surface_radius = 1.5 * l0
    p.density = 1000.0
    p.gravity[:] = (0.0, 0.0, -9.81)
    wx, wy, wz, wnx, wny, wnz = walls
    derive_grid(p, [fx, wx], [fy, wy], [fz, wz])
    n = fx.shape[0]
    nw = wx.shape[0]
    fluid = {
        "x": np.ascontiguousarray(fx),
        "y": np.ascontiguousarray(fy),
        "z": np.ascontiguousarray(fz),
        "vx": np.zeros(n),
        "vy": np.zeros(n),
        "vz": np.zeros(n),
        "pressure": hydrostatic_pressure(fz, fluid_height, l0, p.density, 9.81),
        "surface_type": np.zeros(n, dtype=np.int32),
    }
    wallsd = {
        "x": np.ascontiguousarray(wx),
        "y": np.ascontiguousarray(wy),
        "z": np.ascontiguousarray(wz),
        "vx": np.zeros(nw),
        "vy": np.zeros(nw),
        "vz": np.zeros(nw),
        "normal_x": wnx,
        "normal_y": wny,
        "normal_z": wnz,
    }
    return Case(name, l0, fluid, wallsd, p, meta or {})


def hydrostatic_box(n: int = 20, l0: float = 0.01, layers: int = 3) -> Case:
    """n^3 fluid lattice in an open-top tank of side n l0 whose walls reach
    4 l0 above the fluid; hydrostatic pressure, zero velocity."""
    fx, fy, fz = fluid_block(n, n, n, l0)
    walls = _tank_walls_fast(n, n, n + 4, l0, layers)
    return _make_case(f"hydrostatic_{n}^3", l0, fx, fy, fz, walls, n * l0)


def dam_break(nx: int = 100, ny: int = 50, nz: int = 100, l0: float = 0.005, jitter: float = 0.05,
              seed: int = 1, layers: int = 3) -> Case:
    """Fluid block nx x ny x nz in the corner of a (2 L, L/2, L) tank, L = nx l0,
    positions jittered by U(-jitter l0, +jitter l0) per coordinate."""
    fx, fy, fz = fluid_block(nx, ny, nz, l0)
    n = fx.shape[0]
    if jitter > 0.0:
        u = uniform01(seed, 3 * n).reshape(n, 3)
        d = (2.0 * u - 1.0) * (jitter * l0)
        fx = fx + d[:, 0]
        fy = fy + d[:, 1]
        fz = fz + d[:, 2]
    walls = _tank_walls_fast(2 * nx, nx // 2, nx, l0, layers)
    return _make_case(f"dam_break_{nx}x{ny}x{nz}", l0, fx, fy, fz, walls, nz * l0,
                      meta={"jitter": jitter, "seed": seed})


def splash_dam_break(nx: int = 200, ny: int = 50, nz: int = 200, l0: float = 0.0025, fraction: float = 0.05,
                     seed: int = 3, layers: int = 3) -> Case:
    """Dam break in the (1.0 x 0.25 x 0.5 m at nx = 200) tank whose fluid fills
    half the width; a seeded `fraction` of fluid particles keep x, y and are
    lifted to z = H + U(0, 10 l0) above the free surface H = nz l0."""
    fx, fy, fz = fluid_block(nx, ny, nz, l0)
    n = fx.shape[0]
    u = uniform01(seed, 2 * n).reshape(n, 2)
    sel = u[:, 0] < fraction
    height = nz * l0
    fz = fz.copy()
    fz[sel] = height + u[sel, 1] * (10.0 * l0)
    walls = _tank_walls_fast(2 * nx, ny * 2, nx, l0, layers)
    case = _make_case(f"splash_dam_break_{nx}x{ny}x{nz}", l0, fx, fy, fz, walls, height,
                      meta={"fraction": fraction, "seed": seed, "splash_count": int(sel.sum())})
    return case


def splash_scattered(nx: int = 200, ny: int = 50, nz: int = 200, l0: float = 0.0025, fraction: float = 0.05,
                     seed: int = 3, layers: int = 3) -> Case:
    """The splash dam break with the lifted particles scattered off the
    lattice: the same seeded `fraction` of the fluid is placed uniformly over
    the whole tank floor plan (x in [0, 2 nx l0], y in [0, 2 ny l0]) and
    z = H + U(0, 10 l0) above the free surface H = nz l0 (stream seed + 100).
    The lifted layer is then about a quarter of the bulk density with
    Poisson-scattered gaps, so it holds sparse neighbourhoods (Splash
    particles) and ill-conditioned moment matrices, which lifted particles
    kept on lattice columns do not."""
    fx, fy, fz = fluid_block(nx, ny, nz, l0)
    n = fx.shape[0]
    u = uniform01(seed, 2 * n).reshape(n, 2)
    sel = u[:, 0] < fraction
    m = int(sel.sum())
    v = uniform01(seed + 100, 3 * m).reshape(m, 3)
    height = nz * l0
    fx, fy, fz = fx.copy(), fy.copy(), fz.copy()
    fx[sel] = v[:, 0] * (2 * nx * l0)
    fy[sel] = v[:, 1] * (2 * ny * l0)
    fz[sel] = height + v[:, 2] * (10.0 * l0)
    walls = _tank_walls_fast(2 * nx, ny * 2, nx, l0, layers)
    return _make_case(f"splash_scattered_{nx}x{ny}x{nz}", l0, fx, fy, fz, walls, height,
                      meta={"fraction": fraction, "seed": seed, "splash_count": m})


def lattice_box(n: int = 64, l0: float = 0.01, jitter: float = 0.1, seed: int = 40, layers: int = 3) -> Case:
    """n^3 jittered lattice inside a closed-bottom tank (adjoint check case)."""
    fx, fy, fz = fluid_block(n, n, n, l0)
    m = fx.shape[0]
    u = uniform01(seed, 3 * m).reshape(m, 3)
    d = (2.0 * u - 1.0) * (jitter * l0)
    walls = _tank_walls_fast(n, n, n + 4, l0, layers)
    return _make_case(f"lattice_{n}^3", l0, fx + d[:, 0], fy + d[:, 1], fz + d[:, 2], walls, n * l0,
                      meta={"jitter": jitter, "seed": seed})


def batched_boxes(count: int = 64, seed: int = 7, n_min: int = 8_000, n_max: int = 200_000,
                  l0: float = 0.005) -> list[Case]:
    """The batched workload: `count` independent boxes whose fluid counts are
    drawn log-uniform in [n_min, n_max] (seeded); each box is a hydrostatic
    cube (side round(N^(1/3))) or a dam-break block (2:1:2, ny =
    round((N/4)^(1/3))) by a seeded coin flip, with 3 wall layers and
    r_e = 3.1 l0."""
    u = uniform01(seed, 2 * count)
    boxes = []
    for b in range(count):
        target = float(np.exp(np.log(n_min) + u[2 * b] * (np.log(n_max) - np.log(n_min))))
        if u[2 * b + 1] < 0.5:
            side = max(4, int(round(target ** (1.0 / 3.0))))
            c = hydrostatic_box(n=side, l0=l0)
        else:
            ny = max(2, int(round((target / 4.0) ** (1.0 / 3.0))))
            c = dam_break(nx=2 * ny, ny=ny, nz=2 * ny, l0=l0, seed=seed * 1000 + b)
        c.name = f"box{b}_{c.name}"
        boxes.append(c)
    return boxes


def shuffled(case: Case, seed: int = 11) -> Case:
    """The same particles with the fluid numbered in a seeded random order
    (input whose numbering does not follow space)."""
    n = case.n_fluid
    perm = np.argsort(uniform01(seed, n), kind="stable")
    fluid = {k: np.ascontiguousarray(np.asarray(v)[perm]) for k, v in case.fluid.items()}
    meta = dict(case.meta, shuffle_seed=seed)
    return Case(case.name + "_shuffled", case.l0, fluid, case.walls, case.params, meta)


def splash_shuffled(**kw) -> Case:
    """splash_dam_break with the fluid numbered in a seeded random order."""
    return shuffled(splash_dam_break(**kw))


def dam_break_shuffled(**kw) -> Case:
    """dam_break with the fluid numbered in a seeded random order."""
    return shuffled(dam_break(**kw))


CASES = {
    "hydrostatic": hydrostatic_box,
    "dam_break": dam_break,
    "splash": splash_dam_break,
    "splash_scattered": splash_scattered,
    "lattice": lattice_box,
    "splash_shuffled": splash_shuffled,
    "dam_break_shuffled": dam_break_shuffled,
}
