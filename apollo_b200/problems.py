"""The benchmark problems: meshes, equation and boundary plugins, initial states.

Initial conditions are nodal interpolants of closed-form fields, as Apollo's
``exprFunc`` initial condition evaluates its expressions at every node
(src/subsolvers/wxnodaldg2dmethod.cc:183-199).  The formulas are those of the
reference's example inputs (examples/unstructuredDG/euler/isentropicVortex/
isentropicVortex.pin, .../maxwell/transverseMagnetic/transverseMagnetic.pin).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .mesh import Mesh, grid_for_elements, jittered_square


@dataclass
class Problem:
    name: str
    N: int
    cfl: float
    equation: str
    eq_params: tuple
    mesh: Mesh
    bcs: tuple = ()
    steps: int = 0
    ic: object = None          # callable (x, y) -> U[K][Np][m]
    exact: object = None       # callable (x, y, t) -> U, where an exact solution exists
    meta: dict = field(default_factory=dict)


def gaussian_advection_ic(x, y, x0=0.5, y0=0.5, width=0.01):
    r2 = (x - x0) ** 2 + (y - y0) ** 2
    return np.exp(-r2 / width)[..., None]


def vortex_fields(x, y, t=0.0, x0=5.0, y0=5.0, u0=1.0, v0=0.0, beta=5.0, gamma=1.4):
    """Isentropic vortex (the isentropicVortex.pin progn, advected by (u0, v0))."""
    xm = x - u0 * t
    ym = y - v0 * t
    r2 = (xm - x0) ** 2 + (ym - y0) ** 2
    u = u0 - beta * np.exp(1.0 - r2) * (ym - y0) / (2.0 * np.pi)
    v = v0 + beta * np.exp(1.0 - r2) * (xm - x0) / (2.0 * np.pi)
    base = 1.0 - ((gamma - 1.0) * beta * beta * np.exp(2.0 * (1.0 - r2)) / (16.0 * gamma * np.pi * np.pi))
    rho = base ** (1.0 / (gamma - 1.0))
    p = rho ** gamma
    en = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    return rho, rho * u, rho * v, en


def vortex_ic(x, y, fields=4, t=0.0, **kw):
    rho, ru, rv, en = vortex_fields(x, y, t, **kw)
    if fields == 5:
        return np.stack([rho, ru, rv, np.zeros_like(rho), en], axis=-1)
    return np.stack([rho, ru, rv, en], axis=-1)


def tm_ic(x, y, fields=3, t=0.0):
    """Cavity mode Ez = sin(pi x) sin(pi y) cos(sqrt(2) pi t), B from Faraday's law."""
    w = np.sqrt(2.0) * np.pi
    ez = np.sin(np.pi * x) * np.sin(np.pi * y) * np.cos(w * t)
    # dBx/dt = -dEz/dy, dBy/dt = dEz/dx (with the reference's sign convention
    # f[By] = -Ez in x, f[Bx] = Ez in y): Bx = -pi/w sin(pi x) cos(pi y) sin(w t)
    bx = -(np.pi / w) * np.sin(np.pi * x) * np.cos(np.pi * y) * np.sin(w * t)
    by = (np.pi / w) * np.cos(np.pi * x) * np.sin(np.pi * y) * np.sin(w * t)
    if fields == 8:
        z = np.zeros_like(ez)
        return np.stack([z, z, ez, bx, by, z, z, z], axis=-1)
    return np.stack([ez, bx, by], axis=-1)


def advection(n: int = 32, N: int = 3, seed: int = 0, steps: int = 200) -> Problem:
    """Config 1: periodic unit square, n x n vertex grid (K = 2 (n-1)^2), N = 3, CFL 0.5."""
    mesh = jittered_square(n, (0.0, 0.0), (1.0, 1.0), jitter=0.2, seed=seed, periodic=True)
    return Problem("advection", N, 0.5, "advectionEqn", (1.0, 0.5, 0.0), mesh, (), steps,
                   ic=lambda x, y: gaussian_advection_ic(x, y))


def euler_vortex(n: int = 256, N: int = 4, seed: int = 0, steps: int = 500, fields: int = 4, beta: float = 5.0,
                 cfl: float = 0.5) -> Problem:
    """Config 2: periodic [0,10]^2, n x n vertex grid (n = 256: K = 130,050), N = 4, Rusanov/LF flux."""
    mesh = jittered_square(n, (0.0, 0.0), (10.0, 10.0), jitter=0.2, seed=seed, periodic=True)
    kind = "eulerEqn" if fields == 5 else "eulerEqn2d"
    return Problem("euler_vortex", N, cfl, kind, (1.4, 0.0, 0.0), mesh, (), steps,
                   ic=lambda x, y: vortex_ic(x, y, fields, beta=beta),
                   exact=lambda x, y, t: vortex_ic(x, y, fields, t=t, beta=beta),
                   meta={"beta": beta})


def maxwell_tm(n: int = 512, N: int = 5, seed: int = 0, steps: int = 1000, fields: int = 3,
               cfl: float = 0.5) -> Problem:
    """Config 3: unit square with PEC walls (TM mirror BC), n = 512: K = 522,242, N = 5."""
    mesh = jittered_square(n, (0.0, 0.0), (1.0, 1.0), jitter=0.2, seed=seed, periodic=False, wall_tag=1)
    if fields == 8:
        kind, params = "phMaxwellEqn", (1.0, 0.0, 0.0)
    else:
        kind, params = "maxwellTM", (1.0,)
    return Problem("maxwell_tm", N, cfl, kind, params, mesh, (("maxwellTransverseMagneticBC", ()),), steps,
                   ic=lambda x, y: tm_ic(x, y, fields),
                   exact=lambda x, y, t: tm_ic(x, y, fields, t=t))


def euler_ensemble(count: int = 64, k_range=(1000, 64000), orders=(2, 3, 4, 5), beta_range=(1.0, 5.0),
                   seed: int = 0, cfl: float = 0.5, fields: int = 4) -> list:
    """Ensemble of independent isentropic vortices: per instance a seed-drawn
    element count K uniform in k_range (a jittered periodic [0,10]^2 grid of
    about that many elements), an order from ``orders`` and a vortex strength
    uniform in beta_range.  Returns a list of Problems."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        K = int(rng.integers(k_range[0], k_range[1] + 1))
        N = int(rng.choice(orders))
        beta = float(rng.uniform(beta_range[0], beta_range[1]))
        n = grid_for_elements(K)
        p = euler_vortex(n=n, N=N, seed=seed * 1000 + i, fields=fields, beta=beta, cfl=cfl)
        p.name = f"ensemble_{i}"
        p.meta.update({"K_drawn": K})
        out.append(p)
    return out
