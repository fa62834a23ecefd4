"""Synthetic inputs of the benchmark workloads (seeded; no datasets exist).

Each builder returns (forest, mesh, config, soln) with the reference's
layout. The reference has no initial condition, noise generator, inflow
boundary or final-time stop for most of these workloads; the extensions
used here are implemented identically in the oracle and the GPU path (see
initialize_quadrant_host in csrc/host_physics.cpp).
"""
import math

import numpy as np

from . import Config, Forest


def riemann_64x64(seed=0, time_scheme=3, steps=200):
    """Planar Riemann problem on the unit square: 64 quads of 8x8 (level 3),
    left (1,0,0,1) / right (0.125,0,0,0.1) split at x=0.5, slip walls,
    CFL 0.5, density noise 1e-6."""
    n = 8
    cfg = Config.from_input(cfl=0.5, time_scheme=time_scheme, nelem_subgrid=n, coarse_grid_h=1.0,
                            initial_condition=2, time_steps=steps, dt=1.0, bc=[1] * 6, gamma=1.4,
                            ic_seed=seed, noise_amplitude=1e-6)
    cfg.apply()
    f = Forest(1, 1, periodic=(0, 0), lo=(0.0, 0.0, 0.0), scale=1.0, level=3)
    return f, f.mesh(n), cfg, f.initialize(n)


def vortex_1024(level=6, n=16, time_scheme=3, final_time=10.0, form=0, steps=100000, trees_x=1):
    """Isentropic vortex of strength 5 at (5,5) advected by the free stream
    (rho,u,v,p) = (1,1,1,1) on the periodic square [0,10]^2; level 6 with
    16x16 patches = 1024^2 cells. CFL 0.5; one period is t = 10.
    trees_x > 1 widens the periodic domain to [0,10*trees_x] x [0,10] with
    one level-``level`` tree per 10 x 10 square (the weak-scaling mesh: one
    tree per rank)."""
    mach = math.sqrt(2.0) / math.sqrt(1.4)
    cfg = Config.from_input(cfl=0.5, time_scheme=time_scheme, nelem_subgrid=n, coarse_grid_h=10.0,
                            initial_condition=4, time_steps=steps, dt=1.0, bc=[1] * 6, gamma=1.4,
                            density=1.0, pressure=1.0, mach=mach, alpha=45.0, beta=0.0,
                            ic_params=[5.0, 5.0, 5.0, 0.5], final_time=final_time, form=form)
    cfg.apply()
    f = Forest(int(trees_x), 1, periodic=(1, 1), lo=(0.0, 0.0, 0.0), scale=10.0, level=level)
    return f, f.mesh(n), cfg, f.initialize(n)


def four_quadrant(seed=0, min_level=4, max_level=9, n=16, form=1, jump_tol=0.05, time_scheme=3):
    """Four-quadrant Riemann problem on the unit square split at (0.5,0.5),
    each quadrant's (rho,p) ~ U[0.1,1.5] and (u,v) ~ U[-0.8,0.8] from the
    seed; slip walls; CFL 0.5; density-jump tagging (method 5, relative jump
    >= jump_tol) from min_level to max_level. Returns the forest after the
    start-up refinement, its mesh, the configuration and the state."""
    from .amr import host_tags, initial_forest
    cfg = Config.from_input(cfl=0.5, time_scheme=time_scheme, nelem_subgrid=n, coarse_grid_h=1.0,
                            initial_condition=3, time_steps=10 ** 9, dt=1.0, bc=[1] * 6, gamma=1.4,
                            ic_seed=seed, form=form, amr_ntag_methods=1, amr_tag_methods=[5, 0, 0, 0, 0],
                            amr_tag_tolerances=[jump_tol, 0, 0, 0, 0])
    cfg.apply()
    f = Forest(1, 1, periodic=(0, 0), lo=(0.0, 0.0, 0.0), scale=1.0, level=min_level)
    soln = initial_forest(f, n, max_level, host_tags(n, jump_tol, 5), cfg)
    return f, f.mesh(n), cfg, soln


def shock_bubble(seed=0, min_level=5, max_level=11, n=16, form=1, jump_tol=0.1, time_scheme=3):
    """Shock-bubble interaction on [0,2]x[0,1] (a brick of 2x1 trees):
    ambient (rho,p) = (1,1) at rest, a Mach-2 planar shock at x = 0.1
    entering from the left (post-shock state from the Rankine-Hugoniot
    relations, also the inflow state of the left boundary, bc 3), a bubble
    of density 0.1375 and radius 0.2 in pressure equilibrium, centre
    ~ U([0.6,0.9]x[0.4,0.6]) from the seed; outflow (bc 0) on the right,
    slip walls top and bottom; density-jump tagging (method 5) from
    min_level to max_level; SSP-RK3, CFL 0.5. Returns the forest after the
    start-up refinement, its mesh, the configuration and the state."""
    from .amr import host_tags, initial_forest
    cfg = Config.from_input(cfl=0.5, time_scheme=time_scheme, nelem_subgrid=n, coarse_grid_h=1.0,
                            initial_condition=5, time_steps=10 ** 9, dt=1.0, bc=[3, 0, 1, 1, 1, 1], gamma=1.4,
                            ic_seed=seed, ic_params=[2.0, 0.1, 0.1375, 0.2], form=form, amr_ntag_methods=1,
                            amr_tag_methods=[5, 0, 0, 0, 0], amr_tag_tolerances=[jump_tol, 0, 0, 0, 0])
    cfg.apply()
    f = Forest(2, 1, periodic=(0, 0), lo=(0.0, 0.0, 0.0), scale=1.0, level=min_level)
    soln = initial_forest(f, n, max_level, host_tags(n, jump_tol, 5), cfg)
    return f, f.mesh(n), cfg, soln


def vortex_exact(mesh, t, n=16, beta=5.0, a=0.5, center=(5.0, 5.0), L=10.0):
    """Exact translated vortex at time t (periodic images summed over the
    nearest copy), AoS like the solver state."""
    g = mesh.geom.reshape(-1, 12)
    nq = len(g)
    s = 2.0 / n
    out = np.zeros((nq, n, n, 4))
    gm1 = 0.4
    xi = (s * (np.arange(n) + 0.5) - 1.0)
    X = 0.5 * (1 - xi)[None, :] * g[:, 0:1] + 0.5 * (1 + xi)[None, :] * g[:, 3:4]
    Y = 0.5 * (1 - xi)[None, :] * g[:, 1:2] + 0.5 * (1 + xi)[None, :] * g[:, 7:8]
    xx = X[:, None, :]
    yy = Y[:, :, None]
    xc = (center[0] + t) % L
    yc = (center[1] + t) % L
    dx = (xx - xc + L / 2) % L - L / 2
    dy = (yy - yc + L / 2) % L - L / 2
    r2 = dx * dx + dy * dy
    dT = -(gm1 * beta * beta) / (16.0 * a * 1.4 * math.pi ** 2) * np.exp(2 * a * (1 - r2))
    rho = (1 + dT) ** (1 / gm1)
    ff = beta / (2 * math.pi) * np.exp(a * (1 - r2))
    u = 1.0 - dy * ff
    v = 1.0 + dx * ff
    p = 1.0 + rho ** 1.4 - 1.0
    out[..., 0] = rho
    out[..., 1] = rho * u
    out[..., 2] = rho * v
    out[..., 3] = p / gm1 + 0.5 * rho * (u * u + v * v)
    return out.reshape(-1)
