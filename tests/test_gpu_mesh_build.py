"""Quad descriptors built on the GPU from the forest
(amrgpu_session_regrid_forest) against the host path (amrgpu_forest_external
+ decode): byte-identical descriptors (face types, neighbours, face order,
levels, boundary conditions, corners), the same face count, and the same
states after the remap and after stepping, on bricks of several trees,
periodic or not, with hanging faces at every level jump."""
import os

import numpy as np
import pytest

import meshes

pytestmark = pytest.mark.gpu
os.environ.setdefault("AMRGPU_QUIET", "1")


def forest_case(ag, seed):
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(1, 4)), int(rng.integers(1, 3))
    per = (int(rng.integers(2)), int(rng.integers(2)))
    level = int(rng.integers(1, 3))
    f = ag.Forest(nx, ny, periodic=per, lo=(-1.0, 0.5, 0.0), scale=1.5, level=level)
    return f, rng


def regrid_pair(ag, f, rng, n, form, cfg):
    """Two sessions on the forest's current mesh; one random regrid of the
    forest; one session follows through the host path, the other through
    the device build."""
    m0 = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), int(rng.integers(1 << 30)), amp=1e-2)
    a = ag.Session(m0, cfg, form=form)
    b = ag.Session(m0, cfg, form=form)
    for s in (a, b):
        s.upload(s0)
        s.step(2)
    _, lev, _, _ = f.quads()
    f.begin_regrid()
    f.refine((rng.random(f.num_quads) < 0.3).astype(np.int32), max_level=lev.max() + 2)
    _, lev2, _, _ = f.quads()
    f.coarsen((rng.random(f.num_quads) < 0.5).astype(np.int32), min_level=1)
    f.balance()
    kind, src = f.remap()
    m1 = f.mesh(n)
    a.regrid(m1, kind, src)
    b.regrid_forest(f)
    return a, b, m1


@pytest.mark.parametrize("seed", range(10))
def test_device_descriptors_equal_host_decode(ag, seed):
    f, rng = forest_case(ag, 100 + seed)
    n = 4
    cfg = meshes.make_config(n, time_scheme=3, time_steps=10 ** 6, dt=0.01,
                             bc=tuple(int(x) for x in rng.integers(0, 3, 4)))
    cfg.apply()
    for rnd in range(3):
        a, b, m1 = regrid_pair(ag, f, rng, n, ag.FORM_FP64_EXACT, cfg)
        da, db = a.quad_descriptors(), b.quad_descriptors()
        assert da.tobytes() == db.tobytes(), rnd
        assert b.mesh.nface == m1.nface and b.mesh.ncell == m1.ncell
        assert np.array_equal(a.download(), b.download())
        a.step(4)
        b.step(4)
        assert np.array_equal(a.download(), b.download())
        assert a.sync()["time"] == b.sync()["time"]
        # the lazily built host mesh of the device path is the forest's
        assert np.array_equal(b.mesh.face_info, m1.face_info)
        a.close()
        b.close()


def test_fp32_form_and_hanging_ring(ag):
    n = 16
    f = meshes.two_level_ring(n, periodic=(1, 1))
    cfg = meshes.make_config(n, time_scheme=3, time_steps=10 ** 6, dt=0.01)
    cfg.apply()
    rng = np.random.default_rng(5)
    a, b, m1 = regrid_pair(ag, f, rng, n, ag.FORM_FP32_FLUX, cfg)
    assert a.quad_descriptors().tobytes() == b.quad_descriptors().tobytes()
    a.step(5)
    b.step(5)
    assert np.array_equal(a.download(), b.download())


def test_single_periodic_tree_is_its_own_neighbour(ag):
    n = 4
    f = ag.Forest(1, 1, periodic=(1, 1), level=0)
    cfg = meshes.make_config(n)
    cfg.apply()
    m0 = f.mesh(n)
    a = ag.Session(m0, cfg, form=0)
    a.upload(f.initialize(n))
    f.begin_regrid()
    f.balance()
    a.regrid_forest(f)
    b = ag.Session(f.mesh(n), cfg, form=0)
    assert a.quad_descriptors().tobytes() == b.quad_descriptors().tobytes()
    assert a.mesh.nface == m0.nface == 2


def test_unbalanced_forest_is_rejected_and_session_kept(ag):
    n = 4
    f = meshes.uniform(n, 2, periodic=(0, 0))
    cfg = meshes.make_config(n)
    cfg.apply()
    s = ag.Session(f.mesh(n), cfg, form=0)
    s.upload(f.initialize(n))
    before = s.quad_descriptors()
    f.begin_regrid()
    fl = np.zeros(f.num_quads, np.int32)
    fl[5] = 1
    f.refine(fl)
    fl = np.zeros(f.num_quads, np.int32)
    fl[5] = 1
    f.refine(fl)  # two levels finer next to level-2 quads, no balance
    with pytest.raises(RuntimeError):
        s.regrid_forest(f)
    ag.clear_error()
    assert s.quad_descriptors().tobytes() == before.tobytes()
    s.step(1)
    assert s.sync()["steps"] == 1


def leaves_of(f):
    tree, lev, x, y = f.quads()
    kind, src = f.remap()
    return tree, lev, x, y, f.get_tags(), kind, src


@pytest.mark.parametrize("seed", range(8))
def test_device_balance_equals_host_balance(ag, seed):
    """Two identical forests through the same random refine / coarsen, one
    balanced on the host, one with every pass on the GPU: the same leaves,
    tags and remap tables; then a few more regrid rounds."""
    n = 4
    rng = np.random.default_rng(700 + seed)
    nx, ny = int(rng.integers(1, 4)), int(rng.integers(1, 3))
    per = (int(rng.integers(2)), int(rng.integers(2)))
    fa = ag.Forest(nx, ny, periodic=per, level=2)
    fb = ag.Forest(nx, ny, periodic=per, level=2)
    cfg = meshes.make_config(n)
    cfg.apply()
    s = ag.Session(fa.mesh(n), cfg, form=0)
    for rnd in range(4):
        _, lev, _, _ = fa.quads()
        rf = (rng.random(fa.num_quads) < 0.15).astype(np.int32)
        for f in (fa, fb):
            f.begin_regrid()
            f.set_tags(rf)
            f.refine(rf, max_level=7)
        cf = (rng.random(fa.num_quads) < 0.6).astype(np.int32)
        for f in (fa, fb):
            f.coarsen(cf, min_level=1)
        fa.balance()
        nb = fb.balance(session=s)
        assert nb == fa.num_quads == fb.num_quads
        assert fb.is_balanced()
        for u, v in zip(leaves_of(fa), leaves_of(fb)):
            assert np.array_equal(u, v), rnd


@pytest.mark.parametrize("seed", range(4))
def test_fused_balance_regrid_equals_host_path(ag, seed):
    """balance_regrid (balance passes and descriptors from the balanced
    leaves on the device) against the host balance + host mesh + decode."""
    n = 8
    rng = np.random.default_rng(900 + seed)
    nx, ny = int(rng.integers(1, 3)), int(rng.integers(1, 3))
    per = (int(rng.integers(2)), int(rng.integers(2)))
    fa = ag.Forest(nx, ny, periodic=per, level=2)
    fb = ag.Forest(nx, ny, periodic=per, level=2)
    cfg = meshes.make_config(n, time_scheme=3, time_steps=10 ** 6, dt=0.005, h=1.0)  # trees of side 1
    cfg.apply()
    s0 = meshes.perturbed(fa.initialize(n), seed, amp=1e-2)
    a = ag.Session(fa.mesh(n), cfg, form=1)
    b = ag.Session(fb.mesh(n), cfg, form=1)
    for s in (a, b):
        s.upload(s0)
    for rnd in range(4):
        for s in (a, b):
            s.step(3)
        rf = (rng.random(fa.num_quads) < 0.2).astype(np.int32)
        cf = None
        for f in (fa, fb):
            f.begin_regrid()
            f.set_tags(rf)
            f.refine(rf, max_level=6)
        cf = (rng.random(fa.num_quads) < 0.5).astype(np.int32)
        for f in (fa, fb):
            f.coarsen(cf, min_level=1)
        fa.balance()
        kind, src = fa.remap()
        a.regrid(fa.mesh(n), kind, src)
        b.balance_regrid(fb)
        for u, v in zip(leaves_of(fa), leaves_of(fb)):
            assert np.array_equal(u, v), rnd
        assert a.quad_descriptors().tobytes() == b.quad_descriptors().tobytes(), rnd
        qa = a.download()
        assert np.isfinite(qa).all() and np.array_equal(qa, b.download()), rnd
    a.step(4)
    b.step(4)
    qa = a.download()
    assert np.isfinite(qa).all() and np.array_equal(qa, b.download())


def test_fused_balance_grows_its_buffers_mid_balance(ag):
    """A deep refinement chain at the centre of a small forest: its 2:1
    ripple needs more leaves than the balance buffers hold when the leaves
    are staged (1.5 times as many, at least 64), so the one-launch balance
    loop stops, the buffers grow keeping the leaves and their marks, and the
    loop goes on; the leaves, the descriptors and the remapped state equal
    the host path's."""
    n = 4
    fa = ag.Forest(1, 1, periodic=(0, 0), level=2)
    fb = ag.Forest(1, 1, periodic=(0, 0), level=2)
    cfg = meshes.make_config(n, time_scheme=3, time_steps=10 ** 6, dt=0.002)
    cfg.apply()
    s0 = meshes.perturbed(fa.initialize(n), 5, amp=1e-2)
    a = ag.Session(fa.mesh(n), cfg, form=0)
    b = ag.Session(fb.mesh(n), cfg, form=0)
    for s in (a, b):
        s.upload(s0)
        s.step(2)
    p = (1 << 29) - 1  # just below and left of the centre, in root units
    for f in (fa, fb):
        f.begin_regrid()
        for _ in range(8):
            _, lev, x, y = f.quads()
            size = np.left_shift(np.int64(1), 30 - lev.astype(np.int64))
            hit = (x <= p) & (p < x + size) & (y <= p) & (p < y + size)
            fl = hit.astype(np.int32)
            f.refine(fl, max_level=12)
    staged = fb.num_quads
    fa.balance()
    assert fa.num_quads > max(64, staged + staged // 2)  # the ripple outgrows the staged capacity
    kind, src = fa.remap()
    a.regrid(fa.mesh(n), kind, src)
    b.balance_regrid(fb)
    for u, v in zip(leaves_of(fa), leaves_of(fb)):
        assert np.array_equal(u, v)
    assert a.quad_descriptors().tobytes() == b.quad_descriptors().tobytes()
    assert np.array_equal(a.download(), b.download())
    for s in (a, b):
        s.step(3)
    qa = a.download()
    assert np.isfinite(qa).all() and np.array_equal(qa, b.download())


def test_balance_barrier_wait_runs_out_and_the_session_stays_usable(ag):
    """The one-launch balance's device-wide barrier with its arrival count
    started out of reach: every block's wait runs out after its poll limit,
    the kernel ends with the abort flag set and the call reports an error,
    within a few seconds; the session keeps its mesh, the forest its leaves,
    and the same regrid then runs normally and equals the host path."""
    import time
    n = 4
    fa = ag.Forest(2, 1, periodic=(1, 0), level=2)
    fb = ag.Forest(2, 1, periodic=(1, 0), level=2)
    cfg = meshes.make_config(n, time_scheme=3, time_steps=10 ** 6, dt=0.002)
    cfg.apply()
    s0 = meshes.perturbed(fa.initialize(n), 9, amp=1e-2)
    a = ag.Session(fa.mesh(n), cfg, form=0)
    b = ag.Session(fb.mesh(n), cfg, form=0)
    for s in (a, b):
        s.upload(s0)
        s.step(2)
    rng = np.random.default_rng(5)
    rf = (rng.random(fa.num_quads) < 0.3).astype(np.int32)
    for f in (fa, fb):
        f.begin_regrid()
        f.refine(rf, max_level=4)
    before = leaves_of(fb)
    desc = b.quad_descriptors().tobytes()
    t0 = time.perf_counter()
    rc = ag.lib().amrgpu_session_balance_stall_test(b._s, fb._f)
    assert time.perf_counter() - t0 < 30.0
    assert rc != 0
    ag.clear_error()
    for u, v in zip(before, leaves_of(fb)):
        assert np.array_equal(u, v)
    assert b.quad_descriptors().tobytes() == desc
    fa.balance()
    kind, src = fa.remap()
    a.regrid(fa.mesh(n), kind, src)
    b.balance_regrid(fb)
    assert a.quad_descriptors().tobytes() == b.quad_descriptors().tobytes()
    assert np.array_equal(a.download(), b.download())
