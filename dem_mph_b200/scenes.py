"""Seeded synthetic scenes in the reference's particle format.

The reference ships only the two quasi-2D SYSU cases.  The benchmark
workloads are 3D dam breaks with debris, generated here from a seed:

* a tank of interior L (x) x H (y, up) x W (z) with `wall_layers` lattice
  layers of wall particles (type 4) under the floor and outside the four side
  walls (no lid);
* a fluid column (type 1) against the x=0 wall;
* debris cuboids (type 2) of a x b x c particles at seeded uniform-random
  positions downstream of the column, resting on the floor, optionally with a
  seeded yaw (rotation about the vertical y axis) and per-body densities;
* a periodic domain that leaves more than the neighbour cut-off beyond the
  walls, so the periodic wrap of the reference never couples opposite walls.

Gravity is along -y as in the reference's data (results/SYSU/2mm/dem.data:21).
Particles are listed fluid, then solid, then wall, like the reference
generator's output for the SYSU cases.  Positions are cell-centred lattice
points (i + 0.5) * dx, the reference generator's Cuboid rule
(generator/generator.cpp:664-668).
"""
import math
from dataclasses import dataclass, field

import numpy as np

from .abi import Params, default_params, PRECISION_FP64


@dataclass
class Scene:
    params: Params
    type: np.ndarray          # int32[N]
    x: np.ndarray             # float64[N,3]
    v: np.ndarray             # float64[N,3]
    body: np.ndarray          # int32[N], -1 for particles that belong to no debris body
    body_density: np.ndarray  # float64[B]
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return len(self.type)

    def counts(self):
        t = self.type
        return {"fluid": int(np.sum(t < 2)), "solid": int(np.sum((t >= 2) & (t < 4))),
                "wall": int(np.sum(t >= 4)), "total": int(len(t))}


def _lattice(lo, n, dx):
    """cell-centred lattice points lo + (i + 0.5) dx, i < n, per axis"""
    axes = [lo[d] + (np.arange(n[d]) + 0.5) * dx for d in range(3)]
    g = np.meshgrid(*axes, indexing="ij")
    return np.stack([a.ravel() for a in g], axis=1)


def dam_break_params(dx, dt, rho_f=1000.0, nu=1.0e-6, H_col=0.3, g=9.81,
                     rho_debris=600.0, young=1.0e8, poisson=0.3, restitution=0.5,
                     friction=0.3, bulk_viscosity=1.0, dem_substeps=2,
                     radius_ratio=3.0):
    """dem.data of the 3D dam-break workloads: K = rho c0^2 with
    c0 = 10 sqrt(2 g H), mu = rho nu, InteractionRatio 0 (no surface tension),
    DEM restitution 0.5 and friction 0.3, E = 1e8 with DEMDt = Dt / substeps."""
    p = default_params()
    p.dim = 3
    p.precision = PRECISION_FP64
    p.dt = dt
    p.dem_dt = dt / dem_substeps
    p.output_interval = 1.0
    p.vtk_output_interval = 1.0
    p.end_time = 1.0
    p.radius_ratio_a = radius_ratio
    p.radius_ratio_p = radius_ratio
    p.radius_ratio_v = radius_ratio
    c0 = 10.0 * math.sqrt(2.0 * g * H_col)
    K = rho_f * c0 * c0
    mu = rho_f * nu
    for t in range(6):
        p.density[t] = rho_f
        p.bulk_modulus[t] = K
        p.bulk_viscosity[t] = bulk_viscosity
        p.shear_viscosity[t] = mu
        p.young_modulus[t] = young
        p.poisson_ratio[t] = poisson
        p.restitution_coefficient[t] = restitution
        p.viscous_friction_coefficient[t] = friction
    for t in (0, 1):  # fluids carry no DEM contact parameters, as in the reference data
        p.young_modulus[t] = 0.0
        p.poisson_ratio[t] = 0.0
        p.restitution_coefficient[t] = 0.0
        p.viscous_friction_coefficient[t] = 0.0
    for t in (2, 3):  # debris
        p.density[t] = rho_debris
        p.bulk_modulus[t] = 0.0
        p.bulk_viscosity[t] = 0.0
    p.gravity[0], p.gravity[1], p.gravity[2] = 0.0, -g, 0.0
    return p


def dam_break(dx=0.01, tank=(1.6, 0.6, 0.6), column=(0.4, 0.3, 0.6), n_debris=8,
              debris_sides=((4, 4), (4, 4), (4, 4)), debris_density=(600.0, 600.0),
              debris_x=(0.55, 0.85), yaw=False, wall_layers=3, seed=1234, dt=None,
              dem_substeps=2, headroom=0.3, name="dam_break"):
    """Build a seeded 3D dam-break scene.

    tank = (L, H, W) interior, column = (Lc, Hc, Wc) fluid block at x=0, y=0,
    z=0.  debris_sides[d] = (min, max) particles along x, y, z of each cuboid;
    debris_density = (min, max) per-body density; debris_x = fraction of L
    where debris centres are drawn.  Returns a Scene.
    """
    rng = np.random.default_rng(seed)
    L, H, W = tank
    nl = wall_layers
    nx, ny, nz = (int(round(L / dx)), int(round(H / dx)), int(round(W / dx)))
    cx, cy, cz = (int(round(column[0] / dx)), int(round(column[1] / dx)), int(round(column[2] / dx)))
    cz = min(cz, nz)

    fluid = _lattice((0.0, 0.0, 0.0), (cx, cy, cz), dx)

    # walls: floor slab (with the corners), x walls (full z incl. corners), z walls
    floor = _lattice((-nl * dx, -nl * dx, -nl * dx), (nx + 2 * nl, nl, nz + 2 * nl), dx)
    xw0 = _lattice((-nl * dx, 0.0, -nl * dx), (nl, ny, nz + 2 * nl), dx)
    xw1 = _lattice((nx * dx, 0.0, -nl * dx), (nl, ny, nz + 2 * nl), dx)
    zw0 = _lattice((0.0, 0.0, -nl * dx), (nx, ny, nl), dx)
    zw1 = _lattice((0.0, 0.0, nz * dx), (nx, ny, nl), dx)
    walls = np.concatenate([floor, xw0, xw1, zw0, zw1])

    # debris bodies: rejection-sample footprints that do not overlap each other
    # (one particle of clearance) nor the walls
    bodies, placed = [], []
    tries = 0
    while len(bodies) < n_debris and tries < 100000:
        tries += 1
        a = int(rng.integers(debris_sides[0][0], debris_sides[0][1] + 1))
        b = int(rng.integers(debris_sides[1][0], debris_sides[1][1] + 1))
        c = int(rng.integers(debris_sides[2][0], debris_sides[2][1] + 1))
        ang = float(rng.uniform(0.0, 2.0 * math.pi)) if yaw else 0.0
        rad = 0.5 * math.hypot(a, c) * dx if yaw else 0.0
        hx = rad if yaw else 0.5 * a * dx
        hz = rad if yaw else 0.5 * c * dx
        x0 = float(rng.uniform(debris_x[0] * L + hx, debris_x[1] * L - hx))
        z0 = float(rng.uniform(hz + dx, W - hz - dx))
        if not yaw:  # snap to the lattice so the block sits in lattice registry
            x0 = (round(x0 / dx - 0.5 * a) + 0.5 * a) * dx
            z0 = (round(z0 / dx - 0.5 * c) + 0.5 * c) * dx
        box = (x0 - hx - dx, x0 + hx + dx, z0 - hz - dx, z0 + hz + dx)
        if any(not (box[1] <= q[0] or q[1] <= box[0] or box[3] <= q[2] or q[3] <= box[2]) for q in placed):
            continue
        rho = float(rng.uniform(debris_density[0], debris_density[1]))
        local = _lattice((-0.5 * a * dx, 0.0, -0.5 * c * dx), (a, b, c), dx)
        ca, sa = math.cos(ang), math.sin(ang)
        px = x0 + ca * local[:, 0] - sa * local[:, 2]
        pz = z0 + sa * local[:, 0] + ca * local[:, 2]
        pts = np.stack([px, local[:, 1], pz], axis=1)
        placed.append(box)
        bodies.append((pts, rho))
    if len(bodies) < n_debris:
        raise ValueError("could not place %d debris bodies without overlap" % n_debris)

    solid = np.concatenate([b[0] for b in bodies]) if bodies else np.zeros((0, 3))
    body = np.concatenate([np.full(len(b[0]), k, np.int32) for k, b in enumerate(bodies)]) \
        if bodies else np.zeros(0, np.int32)
    body_density = np.array([b[1] for b in bodies], dtype=np.float64)

    x = np.concatenate([fluid, solid, walls])
    typ = np.concatenate([np.full(len(fluid), 1, np.int32), np.full(len(solid), 2, np.int32),
                          np.full(len(walls), 4, np.int32)])
    bod = np.concatenate([np.full(len(fluid), -1, np.int32), body, np.full(len(walls), -1, np.int32)])
    v = np.zeros_like(x)

    if dt is None:
        c0 = 10.0 * math.sqrt(2.0 * 9.81 * column[1])
        dt = float("%.1e" % (0.2 * dx / c0))
    rho_lo, rho_hi = debris_density
    p = dam_break_params(dx, dt, H_col=column[1], rho_debris=0.5 * (rho_lo + rho_hi),
                         dem_substeps=dem_substeps)
    rc = 3.1 * dx
    margin = nl * dx + rc + 2 * dx
    p.particle_spacing = dx
    p.domain_min[0], p.domain_max[0] = -margin, L + margin
    p.domain_min[1], p.domain_max[1] = -margin, H + headroom
    p.domain_min[2], p.domain_max[2] = -margin, W + margin
    p.time = 0.0
    return Scene(p, typ, x, v, bod, body_density, name=name,
                 meta={"dx": dx, "tank": tank, "column": column, "seed": seed,
                       "n_debris": n_debris, "dt": dt})


def config1(seed=1234, dx=0.01):
    """Config 1: 1.6 x 0.6 x 0.6 m tank, 0.4 x 0.3 (H) x 0.6 m column at
    10 mm (72,000 fluid), 3 wall layers, 8 debris 4x4x4 of density 600."""
    return dam_break(dx=dx, tank=(1.6, 0.6, 0.6), column=(0.4, 0.3, 0.6), n_debris=8,
                     debris_sides=((4, 4), (4, 4), (4, 4)), debris_density=(600.0, 600.0),
                     seed=seed, name="config1_dambreak_3d_dx10mm")


def config2(seed=1234, dx=0.005):
    """Config 2: 3.2 x 1.0 x 1.0 m tank at 5 mm, 0.5 x 0.3 (H) x 1.0 m column
    (1.2 M fluid), 200 debris cuboids with sides of 3-8 particles, densities
    400-900 kg/m^3 and seeded yaw."""
    return dam_break(dx=dx, tank=(3.2, 1.0, 1.0), column=(0.5, 0.3, 1.0), n_debris=200,
                     debris_sides=((3, 8), (3, 8), (3, 8)), debris_density=(400.0, 900.0),
                     debris_x=(0.3, 0.95), yaw=True, seed=seed, name="config2_dambreak_3d_dx5mm")


def config4(seed=1234, n_scenes=32, dx=0.0088):
    """Config 4 (the surrogate's training corpus): 32 seeded dam breaks of the
    config-1 type (1.6 x 0.6 x 0.6 m tank, 8 debris cuboids of 4 particles a
    side) at 8.8 mm, about 250k particles each, with seeded column length
    0.35-0.45 m, height 0.25-0.35 m and debris densities 400-900 kg/m^3."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        Lc = float(rng.uniform(0.35, 0.45))
        H = float(rng.uniform(0.25, 0.35))
        sub = int(rng.integers(1 << 30))
        out.append(dam_break(dx=dx, tank=(1.6, 0.6, 0.6), column=(Lc, H, 0.6), n_debris=8,
                             debris_sides=((4, 4), (4, 4), (4, 4)), debris_density=(400.0, 900.0),
                             yaw=True, seed=sub, name="config4_scene%02d" % k))
    return out


def config5(seed=1234, dx=0.0035):
    """Config 5 (the surrogate's production case): 3.2 x 1.0 x 1.0 m tank at
    3.5 mm, a 0.5 x 0.35 (H) x 1.0 m column (4.09 M fluid), 1000 debris
    cuboids with sides of 3-6 particles, densities 400-900 kg/m^3 and seeded
    yaw, drawn over 20-97% of the tank length."""
    return dam_break(dx=dx, tank=(3.2, 1.0, 1.0), column=(0.5, 0.35, 1.0), n_debris=1000,
                     debris_sides=((3, 6), (3, 6), (3, 6)), debris_density=(400.0, 900.0),
                     debris_x=(0.2, 0.97), yaw=True, seed=seed, name="config5_dambreak_3d_dx3p5mm")


def small(seed=7, dx=0.02, n_debris=3, yaw=False):
    """A small 3D dam break (about 5k particles) for parity tests."""
    return dam_break(dx=dx, tank=(0.6, 0.3, 0.3), column=(0.16, 0.12, 0.3), n_debris=n_debris,
                     debris_sides=((3, 4), (3, 4), (3, 4)), debris_density=(600.0, 600.0),
                     debris_x=(0.35, 0.95), yaw=yaw, seed=seed, name="small_dambreak_3d")


def _dam_break_particles(nh, nw, nl=3):
    """particle count of a config-3 scene before debris: column nh x nh x nw,
    tank 3 nh x 1.2 nh x nw (in particles), nl wall layers (floor with
    corners, x walls over the full z extent, z walls)"""
    nx, ny = int(round(3.0 * nh)), int(round(1.2 * nh))
    walls = (nx + 2 * nl) * nl * (nw + 2 * nl) + 2 * nl * ny * (nw + 2 * nl) + 2 * nx * ny * nl
    return nh * nh * nw + walls


def config3(seed=1234, n_scenes=64, n_range=(20000, 300000), debris_range=(5, 50)):
    """Config 3: an ensemble of independent dam breaks with seeded column
    height H in [0.2, 0.6] m and spacing dx in [5, 10] mm (0.25 mm steps);
    a particle count (walls and debris included) drawn log-uniformly between
    20k (or the smallest tank of that column) and 300k; 5 to 50 debris bodies
    (cuboids of 3 to 4 particles a side, densities 400-900 kg/m^3, seeded
    yaw), drawn uniformly in [5, 50] and clipped to what 40% of the
    downstream half of the floor holds.  The column is H x H x W with W chosen for the drawn
    particle count (widened when fewer than 5 debris would fit); tank
    3H x 1.2H x W.  A draw that leaves the particle range is drawn again."""
    rng = np.random.default_rng(seed)
    out = []
    side_hi = 4
    foot = (1.5 * side_hi + 2) ** 2  # yawed footprint with clearance, in dx^2
    while len(out) < n_scenes:
        k = len(out)
        H = float(rng.uniform(0.2, 0.6))
        dx = float(rng.uniform(0.005, 0.010))
        dx = round(dx * 4000.0) / 4000.0  # 0.25 mm steps
        u_n, u_deb = float(rng.uniform(0.0, 1.0)), float(rng.uniform(0.0, 1.0))
        sub_seed = int(rng.integers(1 << 30))
        nh = max(8, int(round(H / dx)))
        n_min = max(n_range[0], _dam_break_particles(nh, 10))
        if n_min >= n_range[1]:
            continue
        target = float(np.exp(np.log(n_min) + u_n * (np.log(n_range[1]) - np.log(n_min))))
        nw = 10
        while nw < 2000 and _dam_break_particles(nh, nw + 1) <= target:
            nw += 1

        def fit(w):
            return int(0.4 * 0.5 * 3.0 * nh * w / foot)
        while fit(nw) < debris_range[0] and nw < 2000:
            nw += 1
        # uniform in the range, clipped to what the floor holds
        n_deb = debris_range[0] + int(u_deb * (debris_range[1] - debris_range[0] + 1))
        n_deb = min(n_deb, debris_range[1], fit(nw))
        try:
            sc = dam_break(dx=dx, tank=(3.0 * nh * dx, 1.2 * nh * dx, nw * dx), column=(nh * dx, nh * dx, nw * dx),
                           n_debris=n_deb, debris_sides=((3, side_hi), (3, side_hi), (3, side_hi)),
                           debris_density=(400.0, 900.0), debris_x=(0.45, 0.95), yaw=True, seed=sub_seed,
                           name="config3_scene%02d" % k)
        except ValueError:
            continue
        if n_range[0] <= sc.n <= n_range[1]:
            out.append(sc)
    return out
