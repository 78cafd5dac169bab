"""Seeded synthetic particle sets for the five benchmark/parity workloads.

Each generator returns plain numpy FP64 property dicts (one per particle
array) plus the scheme parameters, so the same inputs feed the CUDA path,
the oracle and the reference.  Geometries follow the reference's own problem
generators:

* elliptical drop -- ``get_circular_patch`` (S/solver/fluid_solver.py:16-53),
  here on a dx lattice inside the unit circle, u=-s*x, v=s*y;
* dam break -- ``create_2D_tank`` / ``create_2D_filled_region``
  (S/tools/geometry_utils.py:25-60) and examples/dam-break/dam_break.py,
  with summation density and three layers of fixed wall particles;
* 3D jittered lattice -- the shape of bench/cl_summation_density.py.

No public dataset is involved; every input is generated here from a seed.
"""
from __future__ import annotations

import math

import numpy as np

FLUID = 0   # ParticleType.Fluid (S/base/particle_types.py:28)
SOLID = 1   # ParticleType.Solid


def drop_lattice(dx: float):
    """Square lattice of spacing dx on [-1, 1]^2 clipped to the unit disc
    with get_circular_patch's removal rule sqrt(x^2+y^2) - 1 > 1e-10
    (S/solver/fluid_solver.py:36-38)."""
    x, y = np.mgrid[-1.0:1.0 + 1e-4:dx, -1.0:1.0 + 1e-4:dx]
    x = x.ravel()
    y = y.ravel()
    keep = ~(np.sqrt(x * x + y * y) - 1 > 1e-10)
    return x[keep].copy(), y[keep].copy()


def elliptical_drop(dx: float = 0.025, vel_scale: float = 100.0,
                    rho0: float = 1.0, c0: float = 1400.0, h_fac: float = 1.3):
    """2D elliptical drop: radius 1, u=-s*x, v=s*y, m=rho0*dx^2, h=1.3dx."""
    x, y = drop_lattice(dx)
    n = len(x)
    props = dict(
        x=x, y=y, z=np.zeros(n), u=-vel_scale * x, v=vel_scale * y,
        w=np.zeros(n), m=np.full(n, rho0 * dx * dx), h=np.full(n, h_fac * dx),
        rho=np.full(n, rho0), p=np.zeros(n), cs=np.full(n, c0))
    params = dict(dim=2, c0=c0, rho0=rho0, gamma=7.0, alpha=0.1, beta=0.0,
                  eta=0.1, gravity=(0.0, 0.0, 0.0))
    return [props], [FLUID], params


def dam_break(dx: float = 0.0025, rho0: float = 1000.0, h_fac: float = 1.3,
              width: float = 1.0, height: float = 2.0, tank_w: float = 4.0,
              tank_h: float = 3.0, layers: int = 3):
    """2D dam break: a width x height water column at the left of a
    tank_w x tank_h tank whose bottom and side walls carry `layers` rows of
    fixed particles at spacing dx outside the wall."""
    nx = int(round(width / dx))
    ny = int(round(height / dx))
    fx = (np.arange(nx) + 0.5) * dx
    fy = (np.arange(ny) + 0.5) * dx
    x, y = np.meshgrid(fx, fy, indexing="ij")
    x = x.ravel()
    y = y.ravel()
    n = len(x)
    h = h_fac * dx
    c0 = 10.0 * math.sqrt(2 * 9.81 * height)
    fluid = dict(x=x, y=y, z=np.zeros(n), u=np.zeros(n), v=np.zeros(n),
                 w=np.zeros(n), m=np.full(n, rho0 * dx * dx), h=np.full(n, h),
                 rho=np.full(n, rho0), p=np.zeros(n), cs=np.full(n, c0))
    bx, by = [], []
    nbx = int(round(tank_w / dx))
    nwy = int(round(tank_h / dx))
    for k in range(layers):
        off = (k + 0.5) * dx
        # bottom row spans the side-wall layers too
        xb = (np.arange(-layers, nbx + layers) + 0.5) * dx
        bx.append(xb)
        by.append(np.full(len(xb), -off))
        yw = (np.arange(nwy) + 0.5) * dx
        bx.append(np.full(len(yw), -off))
        by.append(yw)
        bx.append(np.full(len(yw), tank_w + off))
        by.append(yw)
    bx = np.concatenate(bx)
    by = np.concatenate(by)
    nb = len(bx)
    wall = dict(x=bx, y=by, z=np.zeros(nb), u=np.zeros(nb), v=np.zeros(nb),
                w=np.zeros(nb), m=np.full(nb, rho0 * dx * dx),
                h=np.full(nb, h), rho=np.full(nb, rho0), p=np.zeros(nb),
                cs=np.full(nb, c0))
    params = dict(dim=2, c0=c0, rho0=rho0, gamma=7.0, alpha=0.1, beta=0.0,
                  eta=0.1, gravity=(0.0, -9.81, 0.0), cfl=0.3, dt_initial=1e-4)
    return [fluid, wall], [FLUID, SOLID], params


def tait_pressure(rho, c0, rho0, gamma=7.0):
    B = c0 * c0 * rho0 / gamma
    return (np.power(rho / rho0, gamma) - 1.0) * B


def lattice3d(n: int = 128, jitter: float = 0.2, seed: int = 0,
              h_fac: float = 1.2, c0: float = 10.0, rho0: float = 1.0,
              rho_sigma: float = 0.01):
    """n^3 cell-centred lattice in the unit cube, each point jittered by
    U(+-jitter*dx); rho = rho0 + N(0, rho_sigma) drawn after the jitter;
    p from Tait (c0, rho0, gamma=7); uniform mass dx^3, h = h_fac*dx."""
    dx = 1.0 / n
    c = (np.arange(n) + 0.5) * dx
    x, y, z = np.meshgrid(c, c, c, indexing="ij")
    x = x.ravel()
    y = y.ravel()
    z = z.ravel()
    N = len(x)
    rng = np.random.default_rng(seed)
    j = rng.uniform(-jitter * dx, jitter * dx, size=(3, N))
    x = x + j[0]
    y = y + j[1]
    z = z + j[2]
    rho = rho0 + rng.normal(0.0, rho_sigma, N)
    p = tait_pressure(rho, c0, rho0)
    B = c0 * c0 * rho0 / 7.0
    cs = np.power(rho / rho0, 3.0) * c0
    props = dict(x=x, y=y, z=z, u=np.zeros(N), v=np.zeros(N), w=np.zeros(N),
                 m=np.full(N, dx ** 3), h=np.full(N, h_fac * dx), rho=rho, p=p,
                 cs=cs)
    params = dict(dim=3, c0=c0, rho0=rho0, gamma=7.0, alpha=0.0, beta=0.0,
                  eta=0.1, gravity=(0.0, 0.0, 0.0), B=B)
    return [props], [FLUID], params


def batched_drops(num_scenes: int = 256, seed: int = 0, n_lo: int = 1000,
                  n_hi: int = 20000, s_lo: float = 50.0, s_hi: float = 150.0):
    """Independent elliptical drops: N_s ~ U[n_lo, n_hi] sets dx_s =
    sqrt(pi / N_s) at radius 1; velocity scale s ~ U[s_lo, s_hi].  Each
    scene's time step keeps the single drop's acoustic CFL number, c0 dt / h
    = 1400 * 1e-5 / (1.3 * 0.025) = 0.43: dt_s = 1e-5 dx_s / 0.025 (one fixed
    dt of 1e-5 for every scene would put the 20k-particle drops at 0.86 and
    blow them up within tens of steps)."""
    rng = np.random.default_rng(seed)
    ns = rng.uniform(n_lo, n_hi, num_scenes)
    ss = rng.uniform(s_lo, s_hi, num_scenes)
    scenes = []
    for n_target, s in zip(ns, ss):
        dx = math.sqrt(math.pi / n_target)
        arrays, types, params = elliptical_drop(dx=dx, vel_scale=float(s))
        params["dt"] = 1e-5 * dx / 0.025
        scenes.append((arrays, types, params))
    return scenes


def drop_positions_target(dx: float, steps: int, dt: float, vel_scale: float):
    """Parameters of the target run of the differentiable rollout."""
    return dict(dx=dx, steps=steps, dt=dt, vel_scale=vel_scale)
