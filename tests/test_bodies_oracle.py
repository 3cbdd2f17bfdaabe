"""Rigid debris bodies in the oracle restatement (CPU): conservation laws of
the FP64 rigid-body model (no reference counterpart exists for this mode,
so these laws are its pins)."""
import numpy as np

from dem_mph_b200.abi import default_params
from oracle.oracle import Oracle


def vacuum_params(dx=0.01, dt=1e-4, substeps=2):
    p = default_params()
    p.dim = 3
    p.dt = dt
    p.dem_dt = dt / substeps
    p.radius_ratio_a = p.radius_ratio_p = p.radius_ratio_v = 3.0
    for t in range(6):
        p.density[t] = 1000.0
        p.shear_viscosity[t] = 1e-3
        p.young_modulus[t] = 1e8
        p.poisson_ratio[t] = 0.3
        p.restitution_coefficient[t] = 0.5
        p.viscous_friction_coefficient[t] = 0.3
    p.particle_spacing = dx
    for d in range(3):
        p.domain_min[d] = -0.3
        p.domain_max[d] = 0.3
    return p


def cube(n, dx, centre):
    g = (np.arange(n) - 0.5 * (n - 1)) * dx
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1) + np.asarray(centre)


def test_free_spinning_body_conserves_angular_momentum():
    dx = 0.01
    p = vacuum_params(dx)
    x = cube(4, dx, (0.0, 0.0, 0.0))
    # a slab body: 4 x 4 x 2 -> asymmetric inertia
    x = x[x[:, 2] < 0.0]
    w = np.array([3.0, 1.0, 2.0])
    v = np.cross(w, x - x.mean(0))
    typ = np.full(len(x), 2, np.int32)
    o = Oracle(p, typ, x, v)
    o.set_bodies(np.zeros(len(x), np.int32), np.array([800.0]))
    b0 = o.bodies()
    o.step(200)
    b1 = o.bodies()
    assert np.allclose(b1["L"], b0["L"], rtol=0, atol=1e-15 * np.abs(b0["L"]).max())
    assert np.allclose(b1["V"], 0.0, atol=1e-14)
    assert abs(np.linalg.norm(b1["q"][0]) - 1.0) < 1e-14
    assert not np.allclose(b1["q"], b0["q"])  # it did rotate


def test_head_on_collision_conserves_momentum():
    """One DEM substep per step: the contact forces are pair-antisymmetric and
    act at the contact midpoint, so linear and angular momentum are conserved
    to rounding.  (With several substeps the fluid forces of the step are
    reused with moved lever arms, an O(dt) effect, as in the reference.)"""
    dx = 0.01
    p = vacuum_params(dx, dt=2.5e-5, substeps=1)
    xa = cube(3, dx, (-0.021, 0.0, 0.0))
    xb = cube(3, dx, (0.021, 0.003, 0.0))
    x = np.concatenate([xa, xb])
    v = np.concatenate([np.tile([0.5, 0.0, 0.1], (len(xa), 1)), np.tile([-0.5, 0.0, 0.0], (len(xb), 1))])
    typ = np.full(len(x), 2, np.int32)
    body = np.concatenate([np.zeros(len(xa), np.int32), np.ones(len(xb), np.int32)])
    o = Oracle(p, typ, x, v)
    o.set_bodies(body, np.array([700.0, 900.0]))
    b0 = o.bodies()
    P0 = (b0["M"][:, None] * b0["V"]).sum(0)
    L0 = (b0["L"] + b0["M"][:, None] * np.cross(b0["X"], b0["V"])).sum(0)
    o.step(800)
    b1 = o.bodies()
    P1 = (b1["M"][:, None] * b1["V"]).sum(0)
    L1 = (b1["L"] + b1["M"][:, None] * np.cross(b1["X"], b1["V"])).sum(0)
    scale = np.abs(b0["M"][:, None] * b0["V"]).sum()
    assert np.max(np.abs(P1 - P0)) <= 1e-12 * scale
    Lscale = np.abs(b0["M"][:, None] * np.cross(b0["X"], b0["V"])).sum()
    assert np.max(np.abs(L1 - L0)) <= 1e-12 * Lscale
    # they did collide: body velocities changed
    assert np.abs(b1["V"] - b0["V"]).max() > 0.1
