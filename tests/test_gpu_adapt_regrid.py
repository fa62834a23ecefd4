"""amrgpu_session_adapt_regrid: tags, refine / coarsen, 2:1 balance, quad
descriptors and remap in one call, with the refine / coarsen on the device
(at the head of the balance's single launch, from the leaves the session
still holds) when the session's last regrid came from the same unchanged
forest, and the host forest adapted from the copied-back tags meanwhile.

Every test runs the same adaptive loop twice -- once step by step
(Session.tag, Forest.adapt, Session.balance_regrid, each checked on its
own elsewhere) and once through adapt_regrid -- and compares, after every
regrid, the tags, the forest's leaves and remap table, the quad
descriptors and the state, bit for bit."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
os.environ.setdefault("AMRGPU_QUIET", "1")


def pair(ag, form, which="four_quadrant"):
    from amrgpu import workloads as W
    out = []
    for _ in range(2):
        if which == "four_quadrant":
            f, mesh, cfg, soln = W.four_quadrant(seed=0, min_level=4, max_level=6, n=16, form=form)
            lo, hi = 4, 6
        else:
            f, mesh, cfg, soln = W.shock_bubble(seed=0, min_level=3, max_level=7, n=16, form=form)
            lo, hi = 3, 7
        cfg["final_time"] = 0.0
        s = ag.Session(mesh, cfg, form=form)
        s.upload(soln)
        out.append((f, s))
    return out, lo, hi


def same(a, b):
    (fa, sa), (fb, sb) = a, b
    for x, y in zip(fa.quads(), fb.quads()):
        assert np.array_equal(x, y)
    for x, y in zip(fa.remap(), fb.remap()):
        assert np.array_equal(x, y)
    assert np.array_equal(sa.quad_descriptors(), sb.quad_descriptors())
    qa, qb = sa.download(), sb.download()
    assert qa.shape == qb.shape and np.array_equal(qa, qb)


def stepwise(f, s, lo, hi, tags=None):
    t = s.tag() if tags is None else np.asarray(tags, np.int32)
    f.adapt(t, 1, 0, lo, hi)
    s.balance_regrid(f)
    return t


@pytest.mark.parametrize("form,which", [(1, "four_quadrant"), (0, "four_quadrant"), (1, "shock_bubble")])
def test_adapt_regrid_matches_the_stepwise_regrid(ag, form, which):
    (a, b), lo, hi = pair(ag, form, which)
    for c in range(6):
        for f, s in (a, b):
            s.step(3)
            assert s.sync()["error"] == 0
        ta = stepwise(*a, lo, hi)
        assert b[1].holds_forest(b[0]) == (c > 0)  # the first regrid stages the host forest
        tb = b[1].adapt_regrid(b[0], lo, hi, return_tags=True)
        assert np.array_equal(ta, tb)
        assert b[1].holds_forest(b[0])
        same(a, b)
    for f, s in (a, b):
        s.step(3)
        assert s.sync()["error"] == 0
    same(a, b)
    for f, s in (a, b):
        s.close()


def test_adapt_regrid_with_caller_tags_and_growth_mid_adapt(ag):
    """Caller tags that refine every quad: the adapt needs 4x the leaves,
    more than the balance buffers hold, so the device grows them and runs
    the adapt again from the kept leaves; then tags that coarsen
    everything."""
    (a, b), lo, hi = pair(ag, 1)
    for f, s in (a, b):
        s.step(2)
        s.sync()
    stepwise(*a, lo, hi)
    b[1].adapt_regrid(b[0], lo, hi)
    same(a, b)
    assert b[1].holds_forest(b[0])
    n = a[0].num_quads
    up = np.ones(n, np.int32)
    stepwise(*a, lo, hi + 1, tags=up)
    b[1].adapt_regrid(b[0], lo, hi + 1, tags=up)
    assert b[0].num_quads > 3 * n
    same(a, b)
    n = a[0].num_quads
    down = np.zeros(n, np.int32)
    stepwise(*a, lo, hi + 1, tags=down)
    b[1].adapt_regrid(b[0], lo, hi + 1, tags=down)
    assert b[0].num_quads < n
    same(a, b)
    for f, s in (a, b):
        s.step(3)
        assert s.sync()["error"] == 0
    same(a, b)
    for f, s in (a, b):
        s.close()


def test_adapt_regrid_after_host_changes_and_a_reservation(ag):
    """A change of the forest on the host, or a reservation that moves the
    balance buffers, sends the next regrid back through the staged path;
    the results stay the same."""
    (a, b), lo, hi = pair(ag, 1)
    for c in range(5):
        for f, s in (a, b):
            s.step(2)
            s.sync()
        if c == 2:
            for f, s in (a, b):
                f.begin_regrid()  # a host call that may change the leaves
            assert not b[1].holds_forest(b[0])
        if c == 3:
            for f, s in (a, b):
                s.reserve(4 * s.mesh.ncells, 4 * s.mesh.ncell)
            assert not b[1].holds_forest(b[0])
        stepwise(*a, lo, hi)
        b[1].adapt_regrid(b[0], lo, hi)
        same(a, b)
    for f, s in (a, b):
        s.close()


def test_adapt_regrid_with_a_patch_rule(ag):
    """With mixed patch sizes the host adapt and the rule's build run (no
    device adapt); same results as the stepwise regrid."""
    (a, b), lo, hi = pair(ag, 1)
    rule = lambda lv: 8 if lv <= 4 else 16  # noqa: E731
    for f, s in (a, b):
        s.set_patch_rule(rule)
    for c in range(3):
        for f, s in (a, b):
            s.step(2)
            s.sync()
        stepwise(*a, lo, hi)
        b[1].adapt_regrid(b[0], lo, hi)
        assert not b[1].holds_forest(b[0])
        same(a, b)
    for f, s in (a, b):
        s.close()


@pytest.mark.parametrize("seed", range(3))
def test_adapt_regrid_equals_the_host_path_on_bricks(ag, seed):
    """Against code that shares nothing with the device path: the host
    forest's adapt and balance, its mesh arrays, decoded by the session
    (Session.regrid). Random refine / coarsen tags on bricks of up to 3x2
    periodic trees, eight regrids (the device adapt from the second on);
    leaves, descriptors and states bit for bit."""
    import meshes
    n = 8
    rng = np.random.default_rng(700 + seed)
    nx, ny = int(rng.integers(1, 4)), int(rng.integers(1, 3))
    per = (int(rng.integers(2)), int(rng.integers(2)))
    fa = ag.Forest(nx, ny, periodic=per, level=2)
    fb = ag.Forest(nx, ny, periodic=per, level=2)
    cfg = meshes.make_config(n, time_scheme=3, time_steps=10 ** 6, dt=0.005, h=1.0)
    cfg.apply()
    s0 = meshes.perturbed(fa.initialize(n), seed, amp=1e-2)
    a = ag.Session(fa.mesh(n), cfg, form=1)
    b = ag.Session(fb.mesh(n), cfg, form=1)
    for s in (a, b):
        s.upload(s0)
    for rnd in range(8):
        for s in (a, b):
            s.step(2)
        u = rng.random(fa.num_quads)
        tags = np.where(u < 0.2, 1, np.where(u < 0.8, 0, 2)).astype(np.int32)
        fa.adapt(tags, 1, 0, 1, 6)
        fa.balance()
        kind, src = fa.remap()
        a.regrid(fa.mesh(n), kind, src)
        assert b.holds_forest(fb) == (rnd > 0)
        b.adapt_regrid(fb, 1, 6, tags=tags)
        for x, y in zip(fa.quads(), fb.quads()):
            assert np.array_equal(x, y), rnd
        assert a.quad_descriptors().tobytes() == b.quad_descriptors().tobytes(), rnd
        qa = a.download()
        assert np.isfinite(qa).all() and np.array_equal(qa, b.download()), rnd
    for s in (a, b):
        s.step(3)
    assert np.array_equal(a.download(), b.download())
    a.close()
    b.close()
