"""Benchmark scenes: the channel-with-cylinders configurations and the
reference's flat plate, as ippi_params keywords, initial fields and markers.

Inputs are synthetic and seeded: rho = 1 and u = inlet profile plus uniform
noise of +-1e-4 drawn once on the host (numpy PCG64, seed 0), so the GPU path
and the FP64 oracle start from the same arrays.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib as L


def cylinder_markers(cx, cy, d, n=None):
    """n equispaced markers on a circle of diameter d (Mesh::InitialIBParticle,
    mesh.cpp:180-181); n defaults to ceil(pi d), about one per lattice unit."""
    n = n or int(math.ceil(math.pi * d))
    i = np.arange(n, dtype=np.float64)
    x = cx + 0.5 * d * np.sin(2.0 * math.pi * i / n)
    y = cy + 0.5 * d * np.cos(2.0 * math.pi * i / n)
    return np.stack([x, y], axis=1), np.full(n, math.pi * d / n)


def cylinder_solid(nx, ny, cx, cy, d):
    """Solid mask [ny][nx] of a staircase cylinder: nodes (x, y) with
    (x - cx)^2 + (y - cy)^2 <= (d / 2)^2."""
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    return ((xx - cx) ** 2 + (yy - cy) ** 2 <= 0.25 * d * d).astype(np.uint8)


def channel_init(nx, ny, u_max, noise=1e-4, seed=0):
    y = np.arange(ny, dtype=np.float64) + 0.5
    prof = 4.0 * u_max * y * (ny - y) / ny ** 2
    rng = np.random.default_rng(seed)
    ux = np.tile(prof[:, None], (1, nx)) + rng.uniform(-noise, noise, (ny, nx))
    uy = rng.uniform(-noise, noise, (ny, nx))
    return np.ones((ny, nx)), ux, uy


def cylinder_channel(nx, ny, d, cx, cy, u_max, re, collision=L.MRT, storage=L.F32, cs=0.1,
                     les=True, seed=0):
    """One cylinder of diameter d at (cx, cy): nu = u_max d / Re, tau = 3 nu + 1/2."""
    nu = u_max * d / re
    params = dict(collision=collision, storage=storage, bc_set=L.BC_CHANNEL,
                  les_model=L.LES_SMAGORINSKY if les else L.LES_NONE, tau0=3.0 * nu + 0.5,
                  cs=cs, u_in=u_max, rho0=1.0, delta_kernel=L.DELTA_PESKIN4, mdf_iters=1,
                  avg_start=1 << 30)
    xy, ds = cylinder_markers(cx, cy, d)
    rho, ux, uy = channel_init(nx, ny, u_max, seed=seed)
    return dict(nx=nx, ny=ny, params=params, init=(rho, ux, uy), markers=xy, ds=ds, d=d,
                u_ref=u_max)


# the configurations of the benchmark suite (sizes as stated for the method)
def config1():
    """400x100 BGK FP64, D = 20 at (100, 50), Re 100, u_max 0.05."""
    return cylinder_channel(400, 100, 20, 100, 50, 0.05, 100, collision=L.BGK, storage=L.F64,
                            les=False)


def config2(collision=L.MRT, storage=L.F32, seed=0):
    """4096x1024, D = 128 at (1024, 512), Re 3900, u_max 0.04, Smagorinsky Cs 0.1
    (initial noise from `seed`)."""
    return cylinder_channel(4096, 1024, 128, 1024, 512, 0.04, 3900, collision=collision,
                            storage=storage, cs=0.1, seed=seed)


def drag_lift(force_xy, d, u_ref, rho0=1.0):
    """Cd, Cl from body forces (lattice units): F / (1/2 rho U^2 D)."""
    f = np.asarray(force_xy, dtype=np.float64).reshape(-1, 2)
    q = 0.5 * rho0 * u_ref ** 2 * d
    return f[:, 0] / q, f[:, 1] / q
