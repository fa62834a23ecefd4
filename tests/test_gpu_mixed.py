"""Meshes that mix 8x8 and 16x16 patches, one stage work list (the
FP32-flux form's mixed-size row sweep, extension: the reference fixes one
patch size per build).

Checks:
* with one size everywhere the mixed path gives the uniform sweep's bits;
* the residual on a periodic mesh with random sizes (every pairing of sizes
  at full and hanging edges) is within the FP32 form's 2e-5 of max|R| of the
  FP64 restatement of the mixed rule (oracle/mixed_oracle.py);
* the conserved totals stay within 1e-12 (every edge piece is evaluated from
  the same two records by both quads);
* a mesh whose two fine quads on a hanging edge differ in size is refused
  (siblings share a patch size);
* a uniform state stays uniform bit for bit (the pieces of a coarse cell's
  edge add up to its face exactly);
* a regrid between mixed meshes moves the state as the reference's refine /
  coarsen operators do, resampled by position where the size changes;
* the isentropic vortex on a mesh with 8x8 patches away from the vortex stays
  within 2e-3 (L1 of rho, relative) of the all-16x16 run.
"""
import os

import numpy as np
import pytest

import meshes

pytestmark = pytest.mark.gpu
os.environ.setdefault("AMRGPU_QUIET", "1")


def ring(n=16):
    return meshes.two_level_ring(n, periodic=(1, 1))


def config(n, scheme=3, dt=0.01):
    cfg = meshes.make_config(n, time_scheme=scheme, time_steps=10 ** 6, dt=dt)
    cfg.apply()
    return cfg


def run(ag, mesh, cfg, s0, steps, variant=None):
    s = ag.Session(mesh, cfg, form=ag.FORM_FP32_FLUX)
    if variant is not None:
        s.set_launch_variant(variant)
    s.upload(s0)
    s.step(steps)
    rep = s.sync()
    q = s.download()
    s.close()
    return q, rep


@pytest.mark.parametrize("n,other", [(16, 8), (8, 16)])
def test_one_size_through_the_mixed_path_is_the_uniform_sweep(ag, n, other):
    f = ring(n)
    s0 = meshes.perturbed(f.initialize(n), 21, amp=2e-2)
    ref, r0 = run(ag, f.mesh(n), config(n), s0, 6, variant=0)
    # the configured size differs from the mesh's: the session reads the
    # sizes from cell_info and takes the mixed-size sweep
    got, r1 = run(ag, f.mesh_mixed(np.full(f.num_quads, n, np.int32)), config(other), s0, 6)
    assert r0["error"] == 0 and r1["error"] == 0 and r1["steps"] == 6
    assert r1["time"] == r0["time"]
    assert np.array_equal(got, ref)


def family_sizes(f, rng):
    """A random patch size per family of siblings (the children of one
    parent), so that the two fine quads on any hanging edge share a size:
    every pairing of sizes at full and hanging edges still occurs."""
    tree, lev, x, y = f.quads()
    L = 2 ** 30
    pick = {}
    sizes = np.zeros(len(lev), np.int32)
    for q in range(len(lev)):
        span = L >> max(int(lev[q]) - 1, 0)
        key = (int(tree[q]), int(lev[q]), int(x[q]) // span, int(y[q]) // span)
        if key not in pick:
            pick[key] = int(rng.choice([8, 16]))
        sizes[q] = pick[key]
    return sizes


def mixed_mesh(seed):
    f = ring(16)
    sizes = family_sizes(f, np.random.default_rng(seed))
    return f, sizes, f.mesh_mixed(sizes)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_mixed_rhs_within_fp32_tolerance_of_the_restatement(ag, seed):
    from oracle import mixed_oracle as MO
    f, sizes, m = mixed_mesh(seed)
    cfg = config(16)
    s0 = meshes.perturbed(f.initialize(sizes), 40 + seed, amp=2e-2)
    ref = MO.rhs(m, s0, cfg["coarse_grid_h"]).reshape(-1, 4)
    s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
    s.upload(s0)
    got = s.rhs().reshape(-1, 4)
    s.close()
    for k in range(4):
        scale = np.abs(ref[:, k]).max() + 1e-300
        assert np.abs(got[:, k] - ref[:, k]).max() <= 2e-5 * scale, k


def test_mixed_mesh_conserves(ag):
    f, sizes, m = mixed_mesh(7)
    cfg = config(16)
    s0 = meshes.perturbed(f.initialize(sizes), 5, amp=1e-2)
    s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
    s.upload(s0)
    t0 = s.totals()
    s.step(40)
    rep = s.sync()
    t1 = s.totals()
    s.close()
    assert rep["error"] == 0 and rep["steps"] == 40
    assert np.all(np.abs(t1 - t0) <= 1e-12 * np.abs(t0) + 1e-13), t1 - t0


def test_siblings_of_different_sizes_are_refused(ag):
    f = ring(16)
    sizes = family_sizes(f, np.random.default_rng(1))
    m = f.mesh_mixed(sizes)
    # flip one fine quad of a hanging edge so that it differs from its sibling
    fi = m.face_info.reshape(-1, 11)[: m.nface]
    f0 = int(fi[fi[:, 0] == 3][0, 3])
    sizes[f0] = 24 - sizes[f0]
    with pytest.raises(ag.AmrGpuError) as e:
        ag.Session(f.mesh_mixed(sizes), config(16), form=ag.FORM_FP32_FLUX)
    assert e.value.code == 3  # AMRGPU_ERR_MESH


def test_uniform_state_stays_uniform_on_a_mixed_mesh(ag):
    """Forward Euler, so that a zero residual leaves the state bit for bit
    (a Runge-Kutta combination such as 0.75 q + 0.25 q may round)."""
    f, sizes, m = mixed_mesh(3)
    cfg = config(16, scheme=1)
    s0 = np.tile(np.array([1.2, 0.3, -0.2, 2.5]), m.ncells)
    q, rep = run(ag, m, cfg, s0, 10)
    assert rep["error"] == 0
    assert np.array_equal(q, s0)


def host_remap(old, osz, new_sizes, kind, src):
    """The remap's restatement: kind 0 takes the source patch (a refined
    child the parent's), kind 1 the mean of four children cell by cell;
    a size change is resampled by position (the covering cell, or the mean
    of the four covered cells)."""
    ooff = np.concatenate([[0], np.cumsum(osz.astype(np.int64) ** 2)])
    O = old.reshape(-1, 4)
    out = []

    def patch(q):
        n = int(osz[q])
        return O[ooff[q]:ooff[q] + n * n].reshape(n, n, 4)

    def resample(p, n):
        ns = p.shape[0]
        if ns == n:
            return p
        if 2 * ns == n:
            return p.repeat(2, axis=0).repeat(2, axis=1)
        return 0.25 * (((p[0::2, 0::2] + p[0::2, 1::2]) + p[1::2, 0::2]) + p[1::2, 1::2])

    for q, n in enumerate(new_sizes):
        s = int(src[q])
        if kind[q] == 0:
            p = patch(s)
        else:
            p = 0.25 * (((patch(s) + patch(s + 1)) + patch(s + 2)) + patch(s + 3))
        out.append(resample(p, int(n)).reshape(-1))
    return np.concatenate(out)


def test_regrid_between_mixed_meshes(ag):
    """Refine and coarsen with sizes by level (8x8 at the coarsest level,
    16x16 above): the remapped state equals the host restatement bit for bit
    (size changes included) and the run continues."""
    f = meshes.two_level_ring(16, periodic=(1, 1))
    rule = lambda lv: 8 if lv <= 2 else 16  # noqa: E731
    sizes = f.patch_sizes(rule)
    assert set(np.unique(sizes)) == {8, 16}
    cfg = config(16)
    s0 = meshes.perturbed(f.initialize(sizes), 9, amp=1e-2)
    s = ag.Session(f.mesh_mixed(sizes), cfg, form=ag.FORM_FP32_FLUX)
    s.upload(s0)
    s.step(3)
    s.sync()
    q_old = s.download()
    # refine a few coarse quads, coarsen one complete family of fine ones
    f.begin_regrid()
    tree, lev, x, y = f.quads()
    fl = np.zeros(f.num_quads, np.int32)
    fl[np.flatnonzero(lev == 2)[:3]] = 1
    f.refine(fl)
    tree, lev, x, y = f.quads()
    cf = np.zeros(f.num_quads, np.int32)
    cf[np.flatnonzero(lev == 4)[:4]] = 1
    f.coarsen(cf, min_level=0)
    f.balance()
    kind, src = f.remap()
    new_sizes = f.patch_sizes(rule)
    s.regrid(f.mesh_mixed(new_sizes), kind, src)
    got = s.download()
    want = host_remap(q_old, sizes, new_sizes, kind, src)
    assert np.array_equal(got, want)
    s.step(5)
    rep = s.sync()
    s.close()
    assert rep["error"] == 0 and rep["steps"] == 5  # counted from the regrid


def test_vortex_on_mixed_patches_stays_close_to_all_16(ag):
    """The isentropic vortex (periodic [0,10]^2, level 3 = 64 quads) with
    8x8 patches on the quads away from the vortex (distance > 3.5 from its
    centre) against all 16x16: L1(rho) of the difference after t = 0.5 is
    within 2e-3 of L1(rho), and the mixed run has fewer cells."""
    from amrgpu import workloads as W
    f, m16, cfg, s16 = W.vortex_1024(level=3, n=16, form=1, final_time=0.5)
    tree, lev, x, y = f.quads()
    L = 2 ** 30
    cx = (x + (L >> lev) / 2) / L * 10.0
    cy = (y + (L >> lev) / 2) / L * 10.0
    sizes = np.where(np.hypot(cx - 5.0, cy - 5.0) > 3.5, 8, 16).astype(np.int32)
    assert 0 < (sizes == 8).sum() < len(sizes)
    mm = f.mesh_mixed(sizes)
    smx = f.initialize(sizes)

    def to_end(mesh, s0):
        s = ag.Session(mesh, cfg, form=ag.FORM_FP32_FLUX)
        s.upload(s0)
        for _ in range(200):
            s.step(20)
            rep = s.sync()
            if rep["time"] >= 0.5 - 1e-12:
                break
        q = s.download()
        s.close()
        return q, rep

    q16, r16 = to_end(m16, s16)
    qmx, rmx = to_end(mm, smx)
    assert r16["error"] == 0 and rmx["error"] == 0
    assert abs(rmx["time"] - 0.5) < 1e-9 and abs(r16["time"] - 0.5) < 1e-9
    # compare on the 16x16 cells: 8x8 patches injected onto 16x16
    ones = np.full(len(sizes), 16, np.int32)
    kind = np.zeros(len(sizes), np.int32)
    src = np.arange(len(sizes), dtype=np.int32)
    qmx16 = host_remap(qmx, sizes, ones, kind, src).reshape(-1, 4)
    q16 = q16.reshape(-1, 4)
    l1 = np.abs(qmx16[:, 0] - q16[:, 0]).sum() / np.abs(q16[:, 0]).sum()
    assert l1 <= 2e-3, l1
    assert mm.ncells < m16.ncells


def on_fine_grid(forest, sizes, q, level_max, nmax=16):
    """rho of every quad's cells injected onto the uniform grid of the
    finest cells (one tree, unit square), so that two adaptive runs compare
    cell by cell."""
    tree, lev, x, y = forest.quads()
    res = (2 ** level_max) * nmax
    grid = np.zeros((res, res))
    rho = q.reshape(-1, 4)[:, 0]
    off = 0
    L = 2 ** 30
    for k in range(len(lev)):
        n = int(sizes[k])
        patch = rho[off:off + n * n].reshape(n, n)
        off += n * n
        cells = res >> int(lev[k])          # fine cells across this quad
        rep = cells // n
        i0 = int(x[k]) * res // L
        j0 = int(y[k]) * res // L
        grid[j0:j0 + cells, i0:i0 + cells] = patch.repeat(rep, axis=0).repeat(rep, axis=1)
    return grid


def test_adaptive_four_quadrant_with_mixed_patches(ag):
    """Config 3's workload at levels 4-6: the AMR loop (GPU tagging, host
    forest, in-place GPU remap) with 8x8 patches on levels 4-5 and 16x16 on
    level 6 against all 16x16, both to t = 0.05; on the finest uniform grid
    L1(rho) of the difference is within 2% of L1(rho), with fewer cells."""
    from amrgpu import amr, workloads as W
    out = {}
    for mixed in (False, True):
        f, mesh, cfg, soln = W.four_quadrant(seed=0, min_level=4, max_level=6, n=16, form=1)
        rule = (lambda lv: 8 if lv <= 5 else 16) if mixed else None
        s, st = amr.run(f, soln, 16, cfg, 1, 0.05, 5, 4, 6, size_of_level=rule)
        q = s.download()
        sizes = f.patch_sizes(rule) if mixed else np.full(f.num_quads, 16, np.int32)
        assert s.sync()["error"] == 0 and st["time"] >= 0.05 - 1e-12, st
        out[mixed] = (on_fine_grid(f, sizes, q, 6), st["cell_updates"] / max(st["steps"], 1))
        s.close()
    a, b = out[False][0], out[True][0]
    l1 = np.abs(b - a).sum() / np.abs(a).sum()
    assert l1 <= 2e-2, l1
    assert out[True][1] < out[False][1]  # fewer cells per step


def test_device_built_mixed_regrid_equals_the_host_built_one(ag):
    """A regrid with a patch-size rule built on the device (GPU 2:1 balance,
    descriptors, sizes / offsets / work list by scans) gives the state the
    host-built mixed mesh gives, bit for bit, after the remap and after
    further steps -- from a uniform 16x16 session that turns mixed, and
    again from the mixed one."""
    rule = lambda lv: 8 if lv <= 2 else 16  # noqa: E731
    runs = []
    for device in (False, True):
        f = meshes.two_level_ring(16, periodic=(1, 1))
        cfg = config(16)
        s0 = meshes.perturbed(f.initialize(16), 13, amp=1e-2)
        s = ag.Session(f.mesh(16), cfg, form=ag.FORM_FP32_FLUX)
        s.upload(s0)
        s.step(2)
        s.sync()
        states = []
        for cycle in range(2):
            tags = s.tag()
            tags[: max(1, len(tags) // 5)] = 1  # refine some, coarsen the rest where possible
            if device:
                s.set_patch_rule(rule)
                f.adapt(tags, 1, 0, 1, 4)
                s.balance_regrid(f)
            else:
                f.adapt(tags, 1, 0, 1, 4)
                f.balance()
                kind, src = f.remap()
                s.regrid(f.mesh_mixed(f.patch_sizes(rule)), kind, src)
            states.append(s.download())
            s.step(3)
            rep = s.sync()
            assert rep["error"] == 0
            states.append(s.download())
        s.close()
        runs.append(states)
    for a, b in zip(*runs):
        assert a.shape == b.shape and np.array_equal(a, b)


def test_refused_regrid_leaves_the_session_on_its_mesh(ag):
    """A mixed regrid the library refuses (two fine siblings of different
    sizes) raises and changes nothing: the session's state and its next
    steps equal those of a session that never saw the regrid."""
    f = ring(16)
    sizes = family_sizes(f, np.random.default_rng(2))
    m = f.mesh_mixed(sizes)
    cfg = config(16)
    s0 = meshes.perturbed(f.initialize(sizes), 6, amp=1e-2)
    runs = []
    for attempt in (False, True):
        s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
        s.upload(s0)
        s.step(2)
        s.sync()
        if attempt:
            bad = sizes.copy()
            fi = m.face_info.reshape(-1, 11)[: m.nface]
            f0 = int(fi[fi[:, 0] == 3][0, 3])
            bad[f0] = 24 - bad[f0]
            kind = np.zeros(len(sizes), np.int32)
            src = np.arange(len(sizes), dtype=np.int32)
            with pytest.raises(ag.AmrGpuError):
                s.regrid(f.mesh_mixed(bad), kind, src)
            s.mesh = m
        s.step(3)
        rep = s.sync()
        assert rep["error"] == 0
        runs.append(s.download())
        s.close()
    assert np.array_equal(runs[0], runs[1])
