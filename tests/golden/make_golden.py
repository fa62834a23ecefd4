"""Generates the golden fixtures of tests/golden/ from the reference's own
C physics driver (src/physics/src/*.c compiled unmodified into
oracle/_ref/libref_physics.so, over the Fortran-kernel restatement in
oracle/solver2d.c).

Run from the repository root after `make -C oracle` in a tree where the
reference is present:

    python tests/golden/make_golden.py

Each case stores its inputs (mesh arrays, initial state, configuration) and
the reference driver's outputs, so the tests can replay them anywhere.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "amr-demo_b200"), os.path.join(ROOT, "tests")]

import amrgpu as ag  # noqa: E402
from oracle import oracle as O  # noqa: E402
import meshes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CFG_KEYS = ["time_scheme", "time_steps", "dt", "cfl", "coarse_grid_h", "initial_condition", "gamma",
            "density", "pressure", "mach", "alpha", "beta", "checkpoint_interval", "visualization_interval",
            "regrid_interval"]


def pack_cfg(cfg):
    d = {k: np.array(cfg[k]) for k in CFG_KEYS}
    d["bc"] = np.array(cfg["bc"], np.int32)
    return d


def save(name, n, mesh, soln0, cfg, **out):
    np.savez_compressed(os.path.join(OUT, name + ".npz"), n=n, cell_info=mesh.cell_info, face_info=mesh.face_info,
                        geom=mesh.geom, nface=mesh.nface, dof=mesh.dof, soln0=soln0, **pack_cfg(cfg), **out)
    print("wrote", name)


def rhs_case(name, n, forest, cfg, seed):
    cfg.apply()
    mesh = forest.mesh(n)
    soln = meshes.perturbed(forest.initialize(n), seed)
    r = O.reference_rhs(mesh, soln, n, cfg)
    save(name, n, mesh, soln, cfg, rhs=r)


def go_case(name, n, forest, cfg, seed, soln=None):
    cfg.apply()
    mesh = forest.mesh(n)
    if soln is None:
        soln = meshes.perturbed(forest.initialize(n), seed)
    s = soln.copy()
    res = O.reference_go(mesh, s, n, cfg)
    save(name, n, mesh, soln, cfg, soln1=s, istep=res["istep"], regrid=res["regrid"],
         visualize=res["visualize"], checkpoint=res["checkpoint"], evolve_solution=res["evolve_solution"])


def main():
    if not O.reference_available():
        raise SystemExit("oracle/_ref/libref_physics.so is missing: build it with `make -C oracle` "
                         "where the reference tree is present")
    # one residual evaluation
    rhs_case("rhs_uniform_n2_wall", 2, meshes.uniform(2, 1), meshes.make_config(2), 1)
    rhs_case("rhs_uniform_n8_periodic", 8, meshes.uniform(8, 2, periodic=(1, 1)), meshes.make_config(8), 2)
    rhs_case("rhs_hanging_n8_wall", 8, meshes.hanging(8), meshes.make_config(8), 3)
    rhs_case("rhs_hanging_n4_periodic", 4, meshes.hanging(4, periodic=(1, 1)), meshes.make_config(4), 4)
    rhs_case("rhs_twolevel_n4", 4, meshes.two_level_ring(4), meshes.make_config(4), 5)
    rhs_case("rhs_bc_noslip_extrap_n4", 4, meshes.hanging(4), meshes.make_config(4, bc=(2, 0, 2, 0)), 6)
    # whole evolve segments, every time scheme
    for ts in (1, 2, 3, 4, 5):
        go_case(f"go_rk{ts}_hanging_n4", 4, meshes.hanging(4, periodic=(1, 0)),
                meshes.make_config(4, time_scheme=ts, time_steps=12, dt=0.05 if ts == 2 else 1.0), 10 + ts)
    # interval flags stop a segment early
    go_case("go_rk3_intervals_n4", 4, meshes.hanging(4),
            meshes.make_config(4, time_steps=50, regrid_interval=7, visualization_interval=5), 20)
    # planar Riemann problem of the CPU-runnable workload: unit square,
    # 64 quads of 8x8, slip walls, RK3, CFL 0.5, 200 steps, density noise 1e-6
    cfg = ag.Config.from_input(cfl=0.5, time_scheme=3, nelem_subgrid=8, coarse_grid_h=1.0, initial_condition=2,
                               time_steps=200, dt=1.0, bc=[1] * 6, gamma=1.4, ic_seed=0, noise_amplitude=1e-6)
    cfg.apply()
    f = ag.Forest(1, 1, periodic=(0, 0), lo=(0.0, 0.0, 0.0), scale=1.0, level=3)
    go_case("go_riemann_64x64_rk3_200", 8, f, cfg, 0, soln=f.initialize(8))


if __name__ == "__main__":
    main()
