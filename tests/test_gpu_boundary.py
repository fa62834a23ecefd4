"""The reference-facing evolve entry keeps one device session across calls
(the reference rebuilds its arrays on every call, amr_external.c:69-113).
These tests pin down when that session may be reused: only for a mesh that
is byte-identical to the cached one, and simulated time (the final-time
stop, an extension) only carries over when a call continues where the last
one ended."""
import os

import numpy as np
import pytest

import meshes

pytestmark = pytest.mark.gpu

os.environ.setdefault("AMRGPU_QUIET", "1")


def _fp64(cfg):
    cfg["form"] = 0
    cfg.apply()
    return cfg


def test_same_sized_mesh_with_other_bytes_is_rebuilt(ag, oracle):
    """Two meshes with identical counts, cell_info and face_info but other
    corner coordinates: the second call must not reuse the first's
    quad descriptors."""
    n = 4
    fa = meshes.hanging(n, periodic=(1, 0))
    fb = meshes.hanging(n, periodic=(1, 0), lo=(-1.0, -3.0, 0.0), scale=3.0)
    cfg = _fp64(meshes.make_config(n, time_steps=6))
    ma, mb = fa.mesh(n), fb.mesh(n)
    assert np.array_equal(ma.cell_info, mb.cell_info) and np.array_equal(ma.face_info, mb.face_info)
    assert not np.array_equal(ma.geom, mb.geom)
    s0 = meshes.perturbed(fa.initialize(n), 1, amp=1e-2)
    a = s0.copy()
    assert ag.evolve_solver(ma, a, 0)["error"] == 0
    b = s0.copy()
    assert ag.evolve_solver(mb, b, 0)["error"] == 0
    ref = s0.copy()
    oracle.evolve(mb, ref, oracle.make_config(n, cfg))
    assert np.array_equal(b, ref), np.abs(b - ref).max()
    assert not np.array_equal(a, b)


def test_final_time_run_restarts_from_zero(ag, oracle):
    """A run that reached its final time, then a new run from istep 0 on the
    same mesh: the second starts at t = 0 again and repeats the first."""
    n = 4
    f = meshes.hanging(n, periodic=(1, 1))
    cfg = meshes.make_config(n, time_steps=10000, dt=1.0)
    cfg["final_time"] = 0.05
    cfg = _fp64(cfg)
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), 3, amp=1e-2)
    a = s0.copy()
    r1 = ag.evolve_solver(m, a, 0)
    assert r1["error"] == 0 and r1["evolve_solution"] == 0 and r1["istep"] > 1
    b = s0.copy()
    r2 = ag.evolve_solver(m, b, 0)
    assert r2["error"] == 0 and r2["istep"] == r1["istep"]
    assert np.array_equal(a, b)
    ref = s0.copy()
    out = oracle.evolve(m, ref, oracle.make_config(n, cfg))
    assert out["istep"] == r1["istep"]
    assert np.array_equal(a, ref), np.abs(a - ref).max()


def test_final_time_carries_over_a_continuing_run(ag, oracle):
    """Segments cut by the regrid interval continue in simulated time: two
    calls (istep 0 -> k -> end) give the oracle's two segments."""
    n = 4
    f = meshes.hanging(n, periodic=(1, 1))
    cfg = meshes.make_config(n, time_steps=10000, dt=1.0, regrid_interval=3)
    cfg["final_time"] = 0.2
    cfg = _fp64(cfg)
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), 4, amp=1e-2)
    got = s0.copy()
    ref = s0.copy()
    oc = oracle.make_config(n, cfg)
    istep, oistep = 0, 0
    for _ in range(100):
        r = ag.evolve_solver(m, got, istep)
        o = oracle.evolve(m, ref, oc, istep=oistep)
        assert r["error"] == 0
        assert r["istep"] == o["istep"] and r["evolve_solution"] == o["evolve_solution"]
        istep, oistep = r["istep"], o["istep"]
        if not r["evolve_solution"]:
            break
    assert r["evolve_solution"] == 0 and istep > 6
    assert np.array_equal(got, ref), np.abs(got - ref).max()


def test_pageable_and_pinned_transfers_agree(ag):
    """The 1024^2 state (33.5 MB: four 8 MB chunks of the session's pinned
    ring and a partial fifth) makes the same round trip from pageable numpy
    memory as from page-locked memory."""
    import torch
    from amrgpu import workloads as W
    f, m, cfg, s0 = W.vortex_1024(form=0)
    rng = np.random.default_rng(5)
    q = s0 * (1.0 + 1e-3 * rng.uniform(-1, 1, s0.shape))
    s = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    s.upload(q)
    assert np.array_equal(s.download(), q)
    pin = torch.empty(m.dof, dtype=torch.float64, pin_memory=True).numpy()
    pin[:] = q[::-1]
    s.upload(pin)
    back = torch.empty(m.dof, dtype=torch.float64, pin_memory=True).numpy()
    s.download(back)
    assert np.array_equal(back, q[::-1])
    s.upload(q)
    r_pageable = s.rhs()
    s.upload(pin[::-1].copy())
    assert np.array_equal(s.rhs(), r_pageable)
    s.close()
