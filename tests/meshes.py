"""Small meshes and states for parity tests (built with the host forest)."""
import numpy as np

import amrgpu as ag


def make_config(n, time_scheme=3, cfl=0.5, bc=(1, 1, 1, 1), ic=1, dt=1.0, time_steps=10, h=4.0, **kw):
    c = ag.Config.from_input(cfl=cfl, time_scheme=time_scheme, nelem_subgrid=n, coarse_grid_h=h,
                             initial_condition=ic, time_steps=time_steps, dt=dt,
                             bc=list(bc) + [1, 1], mach=0.5, density=1.0, pressure=1.0 / 1.4, **kw)
    return c


def uniform(n, level, periodic=(0, 0), lo=(-2.0, -2.0, 0.0), scale=4.0, nx=1, ny=1):
    f = ag.Forest(nx, ny, periodic=periodic, lo=lo, scale=scale, level=level)
    return f


def hanging(n, level=2, refine=(3, 6), periodic=(0, 0), lo=(-2.0, -2.0, 0.0), scale=4.0, nx=1, ny=1):
    """A uniform forest with a few quads refined once, then 2:1 balanced."""
    f = ag.Forest(nx, ny, periodic=periodic, lo=lo, scale=scale, level=level)
    fl = np.zeros(f.num_quads, np.int32)
    for q in refine:
        fl[q % f.num_quads] = 1
    f.refine(fl)
    f.balance()
    return f


def two_level_ring(n, level=2, periodic=(1, 1)):
    """Refine twice around the centre to get hanging faces at two level jumps."""
    f = ag.Forest(1, 1, periodic=periodic, lo=(-2.0, -2.0, 0.0), scale=4.0, level=level)
    tree, lev, x, y = f.quads()
    L = 2 ** 30
    cx = (x + (L >> lev) / 2) / L
    cy = (y + (L >> lev) / 2) / L
    fl = ((np.abs(cx - 0.5) < 0.3) & (np.abs(cy - 0.5) < 0.3)).astype(np.int32)
    f.refine(fl)
    f.balance()
    tree, lev, x, y = f.quads()
    cx = (x + (L >> lev) / 2) / L
    cy = (y + (L >> lev) / 2) / L
    fl = ((np.abs(cx - 0.45) < 0.12) & (np.abs(cy - 0.55) < 0.12)).astype(np.int32)
    f.refine(fl)
    f.balance()
    return f


def perturbed(soln, seed, amp=1e-3):
    """Small seeded density/momentum perturbation so every face carries flux."""
    rng = np.random.default_rng(seed)
    s = soln.copy()
    s[0::4] *= 1.0 + amp * rng.uniform(-1, 1, s[0::4].shape)
    s[1::4] += amp * rng.uniform(-1, 1, s[1::4].shape)
    s[2::4] += amp * rng.uniform(-1, 1, s[2::4].shape)
    return s
