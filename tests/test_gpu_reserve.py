"""amrgpu_session_reserve: buffers grown up front for an adaptive run.

A reservation moves the session's state, descriptors and tables into larger
buffers; it must change no result. Each test runs the same adaptive loop
(GPU tagging, host forest adapt, GPU balance / descriptors / remap) with and
without a reservation -- made before the first step, and again between
steps after a captured step graph has run -- and compares the states bit for
bit after every remap and every segment of steps.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
os.environ.setdefault("AMRGPU_QUIET", "1")


def adaptive_run(ag, form, reserve, rule=None, cycles=4):
    from amrgpu import workloads as W
    f, mesh, cfg, soln = W.four_quadrant(seed=0, min_level=4, max_level=6, n=16, form=form)
    cfg["final_time"] = 0.0
    if rule is not None:
        sizes = f.patch_sizes(rule)
        mesh = f.mesh_mixed(sizes)
        soln = f.initialize(sizes)
    s = ag.Session(mesh, cfg, form=form)
    if rule is not None:
        s.set_patch_rule(rule)
    if reserve:
        s.reserve(4 * mesh.ncells, 4 * mesh.ncell)
    s.upload(soln)
    states = []
    for c in range(cycles):
        if c == 2:
            s.step(6, graph_steps=6)  # a captured graph, released by the reservation below
            if reserve:
                s.reserve(8 * mesh.ncells, 8 * mesh.ncell)
        s.step(3)
        rep = s.sync()
        assert rep["error"] == 0
        states.append(s.download())
        tags = s.tag()
        f.adapt(tags, 1, 0, 4, 6)
        s.balance_regrid(f)
        states.append(s.download())
    s.step(6, graph_steps=6)
    assert s.sync()["error"] == 0
    states.append(s.download())
    s.close()
    assert all(np.isfinite(x).all() for x in states)
    return states


@pytest.mark.parametrize("form", [0, 1])
def test_reserved_run_is_bit_identical(ag, form):
    a = adaptive_run(ag, form, reserve=False)
    b = adaptive_run(ag, form, reserve=True)
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert x.shape == y.shape and np.array_equal(x, y)


def test_reserved_mixed_run_is_bit_identical(ag):
    rule = lambda lv: 8 if lv <= 5 else 16  # noqa: E731
    a = adaptive_run(ag, 1, reserve=False, rule=rule)
    b = adaptive_run(ag, 1, reserve=True, rule=rule)
    for x, y in zip(a, b):
        assert x.shape == y.shape and np.array_equal(x, y)


def test_reserve_rejects_negative_sizes(ag):
    from amrgpu import workloads as W
    f, mesh, cfg, soln = W.four_quadrant(seed=0, min_level=2, max_level=3, n=8, form=1)
    s = ag.Session(mesh, cfg, form=1)
    s.upload(soln)
    with pytest.raises(RuntimeError):
        s.reserve(-1, 10)
    with pytest.raises(RuntimeError):
        s.reserve(10, -1)
    s.reserve(0, 0)  # no-op
    s.step(1)
    assert s.sync()["steps"] == 1
    s.close()
