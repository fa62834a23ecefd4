"""Batched regrid on the GPU: the plain indicator, refine/coarsen remap, and a
whole AMR loop (evolve segments + regrids) against the oracle doing the same
sequence on the CPU with the reference's per-quad callbacks."""
import ctypes as C
import os

import numpy as np
import pytest

import meshes

pytestmark = pytest.mark.gpu

os.environ.setdefault("AMRGPU_QUIET", "1")


def host_tag_feature(ag, soln, n):
    """hpc_amr_tag_feature quad by quad on the AoS state."""
    L = ag.lib()
    q = soln.reshape(-1, 4 * n * n)
    out = np.zeros(len(q), np.int32)
    for k in range(len(q)):
        patch = np.ascontiguousarray(q[k])
        t = C.c_int(-1)
        L.hpc_amr_tag_feature(C.byref(C.c_int(2)), C.byref(C.c_int(0)), C.byref(C.c_int(4)), C.byref(C.c_int(n)),
                              C.byref(C.c_int(0)), C.byref(C.c_double(0.1)), ag.dp(np.zeros(12)), ag.dp(patch),
                              C.byref(t))
        out[k] = t.value
    return out


def jump_tags(soln, n, tol, mesh):
    from amrgpu.amr import host_tags
    return host_tags(n, tol, 5)(soln, mesh)


def numpy_remap(old, kind, src, n):
    o = old.reshape(-1, 4 * n * n)
    new = np.empty((len(kind), 4 * n * n))
    for q, (k, s) in enumerate(zip(kind, src)):
        if k == 0:
            new[q] = o[s]
        else:
            acc = ((o[s] + o[s + 1]) + o[s + 2]) + o[s + 3]
            new[q] = 0.25 * acc
    return new.reshape(-1)


@pytest.mark.parametrize("n", [4, 8, 16])
def test_gpu_plain_indicator_matches_host_callback(ag, n):
    f = meshes.hanging(n, periodic=(1, 1))
    cfg = meshes.make_config(n)
    cfg["amr_ntag_methods"] = 2
    cfg["amr_tag_methods"] = [1, 2, 0, 0, 0]
    cfg["amr_tag_tolerances"] = [0.93, 1.02, 0, 0, 0]
    cfg.apply()
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), 1, amp=2e-2)
    s = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    s.upload(s0)
    got = s.tag()
    ref = host_tag_feature(ag, s0, n)
    assert ref.sum() > 0 and ref.sum() < len(ref)
    assert np.array_equal(got, ref)


def test_gpu_density_jump_indicator(ag):
    n = 8
    f = meshes.uniform(n, 2)
    cfg = meshes.make_config(n, ic=3)
    cfg["amr_ntag_methods"] = 1
    cfg["amr_tag_methods"] = [5, 0, 0, 0, 0]
    cfg["amr_tag_tolerances"] = [0.05, 0, 0, 0, 0]
    cfg["ic_seed"] = 4
    cfg["ic_params"] = [0.3, 0.6, 0, 0, 0, 0, 0, 0]
    cfg.apply()
    m = f.mesh(n)
    s0 = f.initialize(n)
    s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
    s.upload(s0)
    got = s.tag()
    ref = jump_tags(s0, n, 0.05, m)
    assert 0 < ref.sum() < len(ref)
    assert np.array_equal(got, ref)


def test_gpu_remap_matches_reference_operators(ag):
    n = 8
    f = meshes.uniform(n, 2, periodic=(1, 1))
    cfg = meshes.make_config(n)
    cfg.apply()
    m0 = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), 2, amp=5e-2)
    a = ag.Session(m0, cfg, form=ag.FORM_FP64_EXACT)
    a.upload(s0)
    f.begin_regrid()
    fl = np.zeros(f.num_quads, np.int32)
    fl[[2, 9]] = 1
    f.refine(fl)
    cf = np.zeros(f.num_quads, np.int32)
    _, lev, _, _ = f.quads()
    cf[(lev == 2)] = 1
    f.coarsen(cf, min_level=0)
    f.balance()
    kind, src = f.remap()
    assert (kind == 1).any() and (kind == 0).any()
    m1 = f.mesh(n)
    b = ag.Session(m1, cfg, form=ag.FORM_FP64_EXACT)
    b.remap_from(a, kind, src)
    got = b.download()
    assert np.array_equal(got, numpy_remap(s0, kind, src, n))
    # injection and same-index averaging conserve mass and energy
    ta, tb = a.totals(), b.totals()
    assert np.all(np.abs(tb - ta) <= 1e-13 * np.abs(ta) + 1e-14)


def test_amr_loop_fp64_bitwise_against_oracle(ag, oracle):
    """Segments of 3 RK3 steps with a regrid after each (tag, refine once,
    coarsen untagged families, balance, remap): GPU path and oracle path
    follow the same forest and end bit-identical."""
    n, lo, hi, tol = 4, 2, 5, 0.05
    from amrgpu import workloads as W
    fg, mg, cfg, s0 = W.four_quadrant(seed=3, min_level=lo, max_level=hi, n=n, form=ag.FORM_FP64_EXACT,
                                      jump_tol=tol)
    fo, _, _, _ = W.four_quadrant(seed=3, min_level=lo, max_level=hi, n=n, form=ag.FORM_FP64_EXACT, jump_tol=tol)
    cfg["time_steps"] = 10 ** 6
    cfg.apply()
    s = ag.Session(mg, cfg, form=ag.FORM_FP64_EXACT)
    s.upload(s0)
    ref = s0.copy()
    oc = oracle.make_config(n, cfg)
    oc.time_steps = 3  # each oracle segment starts at istep 0 and stops after 3 steps
    from amrgpu.amr import regrid
    for seg in range(4):
        s.step(3)
        out = oracle.evolve(fo.mesh(n), ref, oc, 0)
        assert out["steps"] == 3
        got = s.download()
        assert np.array_equal(got, ref), (seg, np.abs(got - ref).max())
        # same regrid on the oracle side with host tags and numpy remap
        tags = jump_tags(ref, n, tol, fo.mesh(n))
        _, lev, _, _ = fo.quads()
        fo.begin_regrid()
        fo.set_tags(tags)
        fo.refine(((tags > 0) & (lev < hi)).astype(np.int32), max_level=hi)
        t2 = fo.get_tags()
        _, lev2, _, _ = fo.quads()
        fo.coarsen(((t2 == 0) & (lev2 > lo)).astype(np.int32), min_level=lo)
        fo.balance()
        kind, src = fo.remap()
        ref = numpy_remap(ref, kind, src, n)
        regrid(fg, s, n, lo, hi)
        assert s.mesh.ncell == len(kind)
        assert np.array_equal(s.download(), ref)


@pytest.mark.parametrize("form", [0, 1])
def test_in_place_regrid_matches_new_session(ag, form):
    """amrgpu_session_regrid (capacity reuse, spare-buffer remap, device-side
    re-arm) against a fresh session filled by amrgpu_session_remap: same
    state, same time, and bit-identical steps afterwards. The first regrid
    grows past the capacity, the second shrinks into the spare buffer."""
    n = 8
    f = meshes.uniform(n, 2, periodic=(1, 1))
    cfg = meshes.make_config(n)
    cfg["time_steps"] = 10 ** 6
    cfg.apply()
    s0 = meshes.perturbed(f.initialize(n), 5, amp=5e-2)
    a = ag.Session(f.mesh(n), cfg, form=form)
    a.upload(s0)
    a.step(2)
    for flags_fn in (lambda lev: np.isin(np.arange(len(lev)), [0, 3, 5, 6, 9, 12]),
                     lambda lev: lev > 2):
        t_before = a.sync()["time"]
        _, lev, _, _ = f.quads()
        f.begin_regrid()
        fl = flags_fn(lev).astype(np.int32)
        if (lev > 2).any():
            f.coarsen(fl, min_level=2)
        else:
            f.refine(fl, max_level=4)
        f.balance()
        kind, src = f.remap()
        m1 = f.mesh(n)
        b = ag.Session(m1, cfg, form=form)
        b.remap_from(a, kind, src)
        a.regrid(m1, kind, src)
        assert np.array_equal(a.download(), b.download())
        ra, rb = a.sync(), b.sync()
        assert ra["time"] == rb["time"] == t_before
        a.step(3)
        b.step(3)
        ra, rb = a.sync(), b.sync()
        assert ra["steps"] == rb["steps"] == 3 and ra["time"] == rb["time"]
        assert np.array_equal(a.download(), b.download())
        b.close()
    a.close()


def test_in_place_regrid_rejects_bad_tables(ag):
    n = 4
    f = meshes.uniform(n, 1, periodic=(1, 1))
    cfg = meshes.make_config(n)
    cfg.apply()
    a = ag.Session(f.mesh(n), cfg, form=0)
    a.upload(f.initialize(n))
    nq = f.num_quads
    with pytest.raises(RuntimeError):
        a.regrid(f.mesh(n), np.zeros(nq, np.int32), np.full(nq, nq, np.int32))
    with pytest.raises(RuntimeError):
        a.regrid(f.mesh(n), np.ones(nq, np.int32), np.full(nq, nq - 2, np.int32))
    # the session is unchanged and still steps
    a.step(1)
    assert a.sync()["steps"] == 1
    a.close()
