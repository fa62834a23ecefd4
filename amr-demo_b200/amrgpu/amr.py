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
        tags = tag_fn(soln, forest.mesh(n))
        _, lev, _, _ = forest.quads()
        flags = ((tags > 0) & (lev < max_level)).astype(np.int32)
        if not flags.any():
            break
        forest.refine(flags, max_level=max_level)
        forest.balance()
    return forest.initialize(n)


def side_table(mesh):
    """Per-quad side neighbours decoded from face_info (the same decode as
    the device quad descriptors): kind 0 none/boundary, 1 full or fine side
    of a hanging face (one neighbour), 2 coarse side of a hanging face (two
    fine neighbours)."""
    nq = mesh.ncell
    kind = np.zeros((nq, 4), np.int32)
    nbr = np.zeros((nq, 4, 2), np.int64)
    fi = mesh.face_info.reshape(-1, 11)[: mesh.nface]

    def put(q, s, k, a, b):
        if q < nq:
            kind[q, s] = k
            nbr[q, s] = (a, b)

    for f in fi:
        ftype, side, cell = int(f[0]), int(f[1]), int(f[2])
        if ftype == 2:
            left, right = (int(f[3]), cell) if side % 2 == 0 else (cell, int(f[3]))
            hs = side + 1 if side % 2 == 0 else side
            put(left, hs, 1, right, right)
            put(right, hs - 1, 1, left, left)
        elif ftype == 3:
            fs = side + 1 if side % 2 == 0 else side - 1
            put(cell, side, 2, int(f[3]), int(f[4]))
            put(int(f[3]), fs, 1, cell, cell)
            put(int(f[4]), fs, 1, cell, cell)
    return kind, nbr


def _edge(q, s, own):
    """Edge cells of side s (own=True) or the opposite edge a neighbour
    presents to side s (own=False); q is (nq, n_j, n_i)."""
    if own:
        return (q[:, :, 0], q[:, :, -1], q[:, 0, :], q[:, -1, :])[s]
    return (q[:, :, -1], q[:, :, 0], q[:, -1, :], q[:, 0, :])[s]


def host_tags(n, rho_tol, method=5):
    """Host restatement of the library's plain indicator on an AoS state
    (methods 1 and 2 of solver_tag_feature.F90:9-52; method 5 = relative
    density jump inside the patch or across its faces, with the flux
    kernels' cell pairing). Used for the start-up build and as a checker."""
    def tag(soln, mesh=None):
        q = soln.reshape(-1, n, n, 4)[..., 0]
        if method == 1:
            return (q <= rho_tol).any(axis=(1, 2)).astype(np.int32)
        if method == 2:
            return (q >= rho_tol).any(axis=(1, 2)).astype(np.int32)
        jx = np.abs(np.diff(q, axis=2)) / np.minimum(q[:, :, 1:], q[:, :, :-1])
        jy = np.abs(np.diff(q, axis=1)) / np.minimum(q[:, 1:, :], q[:, :-1, :])
        hit = (jx.max(axis=(1, 2)) >= rho_tol) | (jy.max(axis=(1, 2)) >= rho_tol)
        if mesh is not None:
            kind, nbr = side_table(mesh)
            for s in range(4):
                own = _edge(q, s, True)
                for k in range(2):
                    sel = kind[:, s] >= k + 1
                    if not sel.any():
                        continue
                    other = _edge(q[nbr[sel, s, k]], s, False)
                    mine = own[sel]
                    jump = np.abs(mine - other) / np.minimum(mine, other)
                    hit[np.nonzero(sel)[0]] |= (jump >= rho_tol).any(axis=1)
        return hit.astype(np.int32)
    return tag


def regrid(forest, session, n, min_level, max_level, config=None, form=None, device_mesh=True, size_of_level=None):
    """One regrid of the session in place (its mesh and state follow the
    forest); returns the session. device_mesh: the 2:1 balance passes and
    the quad descriptors run on the GPU (Forest.balance(session=...),
    Session.regrid_forest); otherwise the host balances, lists the mesh
    arrays and the session decodes them. size_of_level: mixed patch sizes
    (a level -> 8 / 16 rule, Forest.patch_sizes): the host path, with the
    mesh of Forest.mesh_mixed."""
    if device_mesh:
        # tags, refine / coarsen and balance in one call (on the device too
        # when the session's last regrid came from this forest)
        if size_of_level is not None:
            session.set_patch_rule(size_of_level)
        session.adapt_regrid(forest, min_level, max_level)
        return session
    tags = session.tag()
    if size_of_level is not None:
        forest.adapt(tags, 1, 0, min_level, max_level)
        forest.balance()
        kind, src = forest.remap()
        session.regrid(forest.mesh_mixed(forest.patch_sizes(size_of_level)), kind, src)
    else:
        _, lev, _, _ = forest.quads()
        forest.begin_regrid()
        forest.set_tags(tags)
        forest.refine(((tags > 0) & (lev < max_level)).astype(np.int32), max_level=max_level)
        tags2 = forest.get_tags()
        _, lev2, _, _ = forest.quads()
        forest.coarsen(((tags2 == 0) & (lev2 > min_level)).astype(np.int32), min_level=min_level)
        forest.balance()
        kind, src = forest.remap()
        session.regrid(forest.mesh(n), kind, src)
    return session


def run(forest, soln, n, config, form, final_time, regrid_interval, min_level, max_level, max_steps=10 ** 7,
        size_of_level=None, headroom=3.0):
    """Evolve to final_time with a regrid every regrid_interval steps.
    size_of_level: mixed 8x8 / 16x16 patches by level (soln is then
    ignored: the initial state is evaluated at each quad's size).
    headroom: the session's buffers are reserved up front for meshes this
    many times the initial one (cells and quads), so that regrids within it
    allocate nothing. Returns (session, stats)."""
    config["final_time"] = final_time
    config.apply()
    if size_of_level is not None:
        sizes = forest.patch_sizes(size_of_level)
        mesh = forest.mesh_mixed(sizes)
        soln = forest.initialize(sizes)
    else:
        mesh = forest.mesh(n)
    s = Session(mesh, config, form=form)
    if headroom > 1.0:
        s.reserve(int(headroom * mesh.ncells), int(headroom * mesh.ncell))
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
        regrid(forest, s, n, min_level, max_level, size_of_level=size_of_level)
        regrids += 1
        t_regrid += time.perf_counter() - t1
    return s, {"steps": steps, "time": time_now, "cell_updates": cell_updates, "solve_s": t_solve,
               "regrid_s": t_regrid, "regrids": regrids, "cells": s.mesh.ncells, "quads": s.mesh.ncell}
