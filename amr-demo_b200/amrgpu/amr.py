"""AMR evolve loop on the GPU path: the reference's driver loop
(src/amr/src/amr_evolve.c:15-73) and regrid (src/amr/src/amr_regrid.c:15-125)
restated over the host forest, with the tagging, refine and coarsen data
operations done by the library's batched GPU kernels.

Per regrid (amr_regrid.c:15-81): every quad is tagged (plain indicator,
solver_tag_feature.F90:9-52, or the density-jump extension); tagged quads
below max_level are refined once (non-recursive after start-up,
amr_regrid.c:239-244); complete families with no tagged child above
min_level are coarsened (amr_tag.c:202-220); the forest is 2:1 balanced
across faces and corners; the state moves to the new mesh by injection /
same-index averaging (solver_refine_operator_2d.F90:49-52,
solver_coarsen_operator_2d.F90:49-50).
"""
import time

import numpy as np

from . import Forest, Session


def initial_forest(forest, n, max_level, tag_fn, config):
    """Start-up build (amr_regrid.c:227-237): refine level by level where
    the tagger fires on the initial condition, re-evaluating the IC on the
    new quads."""
    config.apply()
    for _ in range(64):
        soln = forest.initialize(n)
        tags = tag_fn(soln)
        _, lev, _, _ = forest.quads()
        flags = ((tags > 0) & (lev < max_level)).astype(np.int32)
        if not flags.any():
            break
        forest.refine(flags, max_level=max_level)
        forest.balance()
    return forest.initialize(n)


def host_tags(n, rho_tol, method=5):
    """Host tagger on an AoS state, used only for the start-up build."""
    def tag(soln):
        q = soln.reshape(-1, n, n, 4)[..., 0]
        if method == 1:
            return (q <= rho_tol).any(axis=(1, 2)).astype(np.int32)
        if method == 2:
            return (q >= rho_tol).any(axis=(1, 2)).astype(np.int32)
        jx = np.abs(np.diff(q, axis=2)) / np.minimum(q[:, :, 1:], q[:, :, :-1])
        jy = np.abs(np.diff(q, axis=1)) / np.minimum(q[:, 1:, :], q[:, :-1, :])
        return ((jx.max(axis=(1, 2)) >= rho_tol) | (jy.max(axis=(1, 2)) >= rho_tol)).astype(np.int32)
    return tag


def regrid(forest, session, n, min_level, max_level, config, form):
    """One regrid; returns the new session with the remapped state."""
    tags = session.tag()
    _, lev, _, _ = forest.quads()
    forest.begin_regrid()
    forest.set_tags(tags)
    forest.refine(((tags > 0) & (lev < max_level)).astype(np.int32), max_level=max_level)
    tags2 = forest.get_tags()
    _, lev2, _, _ = forest.quads()
    forest.coarsen(((tags2 == 0) & (lev2 > min_level)).astype(np.int32), min_level=min_level)
    forest.balance()
    kind, src = forest.remap()
    mesh = forest.mesh(n)
    new = Session(mesh, config, form=form)
    new.remap_from(session, kind, src)
    return new


def run(forest, soln, n, config, form, final_time, regrid_interval, min_level, max_level, max_steps=10 ** 7):
    """Evolve to final_time with a regrid every regrid_interval steps.
    Returns (session, stats)."""
    config["final_time"] = final_time
    config.apply()
    mesh = forest.mesh(n)
    s = Session(mesh, config, form=form)
    s.upload(soln)
    steps = 0
    cell_updates = 0
    t_solve = 0.0
    t_regrid = 0.0
    time_now = 0.0
    regrids = 0
    while time_now < final_time and steps < max_steps:
        t0 = time.perf_counter()
        s.step(regrid_interval)
        rep = s.sync()
        t1 = time.perf_counter()
        t_solve += t1 - t0
        done = rep["steps"]
        cell_updates += s.mesh.ncells * done
        steps += done
        time_now = rep["time"]
        if rep["error"]:
            break
        if time_now >= final_time:
            break
        s2 = regrid(forest, s, n, min_level, max_level, config, form)
        s.close()
        s = s2
        regrids += 1
        t_regrid += time.perf_counter() - t1
    return s, {"steps": steps, "time": time_now, "cell_updates": cell_updates, "solve_s": t_solve,
               "regrid_s": t_regrid, "regrids": regrids, "cells": s.mesh.ncells, "quads": s.mesh.ncell}
