"""Host-side logic on CPU: the host forest (p4est stand-in), the reference
ABI's configuration parsing and per-quad callbacks, and the library's
exported symbols. No GPU needed."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import meshes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    # the MPI adapter physics_go_gpu.h compiles into the caller (static
    # functions over the caller's MPI) declares nothing this library exports
    txt = re.sub(r"#ifndef AMRGPU_NO_MPI_ADAPTER.*?#endif", "", txt, flags=re.S)
    # function-pointer members, e.g. "int (*rank)(...)", name no function
    txt = re.sub(r"\b[a-z_][a-z0-9_]*\s*\(\s*\*\s*[a-z_][a-z0-9_]*\s*\)", "", txt)
    return sorted(set(re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", txt)) - {"defined"})


def test_library_exports_every_declared_symbol(ag):
    L = ag.lib()
    names = declared_functions("amrgpu.h")
    assert "hpc_amr_evolve_solver" in names and "physics_go_gpu" in names
    for name in names:
        assert hasattr(L, name), name
    for name in declared_functions("physics_go_gpu.h"):
        assert hasattr(L, name), name
    # the Python mirror binds every exported entry point with a prototype
    assert set(names) <= set(ag.PROTOTYPES)


def test_session_without_gpu_reports_no_device(ag):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    f = meshes.uniform(4, 1)
    meshes.make_config(4).apply()
    m = f.mesh(4)
    with pytest.raises(ag.AmrGpuError) as e:
        ag.Session(m)
    assert e.value.code == 6


def test_uniform_brick_counts():
    import amrgpu as ag
    for per in ((0, 0), (1, 0), (1, 1)):
        f = ag.Forest(2, 1, periodic=per, lo=(0, 0, 0), scale=1.0, level=2)
        assert f.num_quads == 2 * 16
        m = f.mesh(4)
        types = np.bincount(m.face_info[0::11], minlength=4)
        nx, ny = 8, 4
        full = (nx - (0 if per[0] else 1)) * ny + nx * (ny - (0 if per[1] else 1))
        bnd = (0 if per[0] else 2 * ny) + (0 if per[1] else 2 * nx)
        assert types[2] == full and types[1] == bnd and types[3] == 0


def side_coverage(m):
    cover = np.zeros((m.ncell, 4), int)
    for row in m.face_info.reshape(-1, 11):
        t, s, c = row[:3]
        cover[c, s] += 1
        if t == 2:
            cover[row[3], row[7]] += 1
        elif t == 3:
            cover[row[3], row[7]] += 1
            cover[row[4], row[8]] += 1
    return cover


@pytest.mark.parametrize("seed", range(6))
def test_random_refinement_is_balanced_and_every_side_has_one_face(seed):
    import amrgpu as ag
    rng = np.random.default_rng(seed)
    f = ag.Forest(int(rng.integers(1, 3)), int(rng.integers(1, 3)), periodic=(int(rng.integers(2)), int(rng.integers(2))),
                  lo=(0, 0, 0), scale=1.0, level=2)
    for _ in range(3):
        fl = (rng.random(f.num_quads) < 0.2).astype(np.int32)
        f.refine(fl, max_level=7)
        f.balance()
        assert f.is_balanced()
    m = f.mesh(4)
    assert np.all(side_coverage(m) == 1)
    # cell_info offsets follow amr_external.c: 4 n^2 * local id
    assert np.array_equal(m.cell_info[2::3], 64 * np.arange(m.ncell))


def test_geometry_matches_quadrant_coordinates():
    """geom corners (amr_p4est_utilities.c:15-81) against the quad's integer
    position: x = lo + scale*(tree_x + qx/2^30)."""
    import amrgpu as ag
    f = ag.Forest(2, 2, periodic=(0, 0), lo=(-1.0, 2.0, 0.0), scale=0.5, level=3)
    fl = np.zeros(f.num_quads, np.int32)
    fl[::7] = 1
    f.refine(fl)
    f.balance()
    m = f.mesh(2)
    tree, lev, x, y = f.quads()
    g = m.geom.reshape(-1, 4, 3)
    L = 2.0 ** 30
    # trees follow the Morton order of the 2x2 brick
    tx = np.array([0, 1, 0, 1])[tree]
    ty = np.array([0, 0, 1, 1])[tree]
    x0 = -1.0 + 0.5 * (tx + x / L)
    y0 = 2.0 + 0.5 * (ty + y / L)
    h = 0.5 / 2.0 ** lev
    assert np.allclose(g[:, 0, 0], x0) and np.allclose(g[:, 0, 1], y0)
    assert np.allclose(g[:, 3, 0], x0 + h) and np.allclose(g[:, 3, 1], y0 + h)


def test_hanging_faces_pair_the_coarse_quad_with_two_fine_quads():
    f = meshes.hanging(4)
    m = f.mesh(4)
    lev = m.cell_info[1::3]
    for row in m.face_info.reshape(-1, 11):
        if row[0] != 3:
            continue
        coarse, f0, f1 = row[2], row[3], row[4]
        assert lev[f0] == lev[f1] == lev[coarse] + 1
        assert row[7] == row[8] == (row[1] ^ 1)


def test_refine_then_coarsen_remap_and_operators(ag):
    """Remap kinds from the forest and the reference's refine (injection)
    and coarsen (same-index average) callbacks on host."""
    f = ag.Forest(1, 1, periodic=(1, 1), lo=(0, 0, 0), scale=1.0, level=2)
    f.begin_regrid()
    fl = np.zeros(16, np.int32)
    fl[5] = 1
    f.refine(fl)
    kind, src = f.remap()
    assert f.num_quads == 19
    assert list(src[5:9]) == [5] * 4 and np.all(kind == 0)
    f.begin_regrid()
    cf = np.zeros(f.num_quads, np.int32)
    cf[5:9] = 1
    f.coarsen(cf, min_level=0)
    kind, src = f.remap()
    assert f.num_quads == 16 and kind[5] == 1 and src[5] == 5
    L = ag.lib()
    n, nf = 2, 4
    rng = np.random.default_rng(0)
    parent = rng.random(nf * n * n)
    kids = [np.zeros(nf * n * n) for _ in range(4)]
    args = [C.byref(C.c_int(v)) for v in (0, nf, n, 0)] + [C.byref(C.c_double(0.1)), ag.dp(np.zeros(12))]
    L.hpc_amr_refine_operator_2d(*args, ag.dp(parent), *[ag.dp(k) for k in kids])
    assert all(np.array_equal(k, parent) for k in kids)
    out = np.zeros(nf * n * n)
    L.hpc_amr_coarsen_operator_2d(*args, *[ag.dp(k + i) for i, k in enumerate(kids)], ag.dp(out))
    assert np.array_equal(out, 0.25 * (parent + (parent + 1) + (parent + 2) + (parent + 3)))


def test_input_physics_keyword_rules(ag, tmp_path):
    """physics_initialize.c:61-197: defaults, cfl <- 0.25*cfl*time_scheme,
    intervals <= 0 become INT_MAX, extension keywords."""
    p = tmp_path / "input.physics"
    p.write_text("<SIMULATION PROPERTIES>\ncheckpoint_interval: 0\nvisualization_interval: 1000\n"
                 "regrid_interval: 10\namr_ntag_methods: 2\namr_tag_methods: 1 2\n"
                 "amr_tag_tolerances: 0.996, 1.5\ntime_scheme: 3\ntime_steps: 10000\ndt: 0.01000\n"
                 "</SIMULATION PROPERTIES>\n<FLUID PROPERTIES>\ninitial_condition: 1\nbc_xlo: 2\ncfl: 0.5\n"
                 "gamma: 1.4\npressure: 0.714286\nmach: 0.5\ngpu_form: 1\nfinal_time: 2.5\n</FLUID PROPERTIES>\n")
    c = ag.Config.read(str(p))
    assert c["time_scheme"] == 3 and c["time_steps"] == 10000 and c["dt"] == 0.01
    assert c["cfl"] == 0.25 * 0.5 * 3
    assert c["checkpoint_interval"] == 2147483647 and c["regrid_interval"] == 10
    assert c["amr_ntag_methods"] == 2 and c["amr_tag_methods"][:2] == [1, 2]
    assert c["amr_tag_tolerances"][:2] == [0.996, 1.5]
    assert c["bc"][:4] == [2, 1, 1, 1] and c["mach"] == 0.5 and c["alpha"] == 0.0
    assert c["form"] == 1 and c["final_time"] == 2.5


def test_initialize_solver_reads_input_from_cwd(ag, tmp_path, monkeypatch):
    (tmp_path / "input.physics").write_text("time_scheme: 2\ntime_steps: 7\ncfl: 1.0\n")
    monkeypatch.chdir(tmp_path)
    os.environ["AMRGPU_QUIET"] = "1"
    ag.clear_error()
    assert ag.initialize_solver(2.0, 8, nlevels=3) == 0
    c = ag.Config.current()
    assert c["time_scheme"] == 2 and c["time_steps"] == 7 and c["cfl"] == 0.5
    assert c["coarse_grid_h"] == 2.0 and c["nelem_subgrid"] == 8
    (tmp_path / "input.physics").unlink()
    assert ag.initialize_solver(2.0, 8) == 7  # missing file: defaults kept, error reported
    ag.clear_error()


def test_host_tag_feature_matches_restated_fortran(ag, oracle):
    L = ag.lib()
    n, nf = 4, 4
    rng = np.random.default_rng(3)
    for meth, tol in ((1, 0.5), (2, 1.2)):
        c = ag.Config.current()
        c["amr_ntag_methods"] = 1
        c["amr_tag_methods"] = [meth, 0, 0, 0, 0]
        c["amr_tag_tolerances"] = [tol, 0, 0, 0, 0]
        c.apply()
        for _ in range(20):
            soln = rng.uniform(0.4, 1.3, nf * n * n)
            tag = C.c_int(-1)
            L.hpc_amr_tag_feature(C.byref(C.c_int(2)), C.byref(C.c_int(0)), C.byref(C.c_int(nf)), C.byref(C.c_int(n)),
                                  C.byref(C.c_int(0)), C.byref(C.c_double(0.1)), ag.dp(np.zeros(12)), ag.dp(soln),
                                  C.byref(tag))
            rho = soln[0::4]
            expect = int((rho <= tol).any()) if meth == 1 else int((rho >= tol).any())
            assert tag.value == expect


@pytest.mark.parametrize("seed,rv,cv,level,lo,hi,rounds", [(3, 1, 0, 3, 1, 6, 8), (4, 2, 1, 3, 1, 6, 8),
                                                             (5, 1, 2, 3, 1, 6, 8), (6, 0, 1, 3, 1, 6, 8),
                                                             (7, 1, 0, 7, 5, 9, 3)])
def test_adapt_equals_the_step_by_step_regrid(ag, seed, rv, cv, level, lo, hi, rounds):
    """Forest.adapt (begin_regrid, tags, refine, coarsen in one pass) gives
    the same leaves, tags and remap table as the separate calls, also when
    the coarsen tag is the one refined children carry (1); also on a forest
    of 32k+ leaves."""
    import numpy as np
    rng = np.random.default_rng(seed)
    fa = ag.Forest(2, 1, periodic=(1, 0), level=level)
    fb = ag.Forest(2, 1, periodic=(1, 0), level=level)
    for rnd in range(rounds):
        tags = rng.integers(0, 3, fa.num_quads).astype(np.int32)
        _, lev, _, _ = fa.quads()
        fa.begin_regrid()
        fa.set_tags(tags)
        fa.refine(((tags == rv) & (lev < hi)).astype(np.int32), max_level=hi)
        t2 = fa.get_tags()
        _, lev2, _, _ = fa.quads()
        fa.coarsen(((t2 == cv) & (lev2 > lo)).astype(np.int32), min_level=lo)
        nb = fb.adapt(tags, rv, cv, lo, hi)
        assert nb == fa.num_quads == fb.num_quads
        for u, v in zip(fa.quads() + fa.remap() + (fa.get_tags(),), fb.quads() + fb.remap() + (fb.get_tags(),)):
            assert np.array_equal(u, v), rnd
        fa.balance()
        fb.balance()


def _py_refine(leaves, flags, max_level):
    """Refinement as the reference's regrid does it (amr_regrid.c:239-244):
    a flagged leaf below max_level becomes its four z-ordered children,
    which carry the refine tag; other leaves are kept. Leaves are tuples
    (tree, level, x, y, tag, kind, src)."""
    out = []
    for leaf, f in zip(leaves, flags):
        tree, lev, x, y, tag, kind, src = leaf
        if f and lev < max_level:
            h = 1 << (30 - (lev + 1))
            out += [(tree, lev + 1, x + (c & 1) * h, y + ((c >> 1) & 1) * h, 1, kind, src) for c in range(4)]
        else:
            out.append(leaf)
    return out


def _py_coarsen(leaves, flags, min_level):
    """Coarsening of complete families (amr_tag.c:202-220): four flagged
    siblings above min_level, untouched since the regrid began (copies of
    consecutive old leaves), become their parent (tag 0, averaged from the
    first sibling's source)."""
    out, i, n = [], 0, len(leaves)
    while i < n:
        tree, lev, x, y, tag, kind, src = leaves[i]
        fam = False
        if lev > 0 and lev > min_level and i + 3 < n:
            P, h = 1 << (30 - (lev - 1)), 1 << (30 - lev)
            px, py = (x // P) * P, (y // P) * P
            if (x, y) == (px, py):
                fam = all(leaves[i + c][:4] == (tree, lev, px + (c & 1) * h, py + ((c >> 1) & 1) * h)
                          and flags[i + c] and leaves[i + c][5] == 0 and leaves[i + c][6] == src + c
                          for c in range(4))
        if fam:
            out.append((tree, lev - 1, px, py, 0, 1, src))
            i += 4
        else:
            out.append(leaves[i])
            i += 1
    return out


def _lib_leaves(f):
    tree, lev, x, y = f.quads()
    kind, src = f.remap()
    tags = f.get_tags()
    return [tuple(int(v) for v in t) for t in zip(tree, lev, x, y, tags, kind, src)]


@pytest.mark.parametrize("seed", range(4))
def test_forest_edits_match_a_list_restatement(ag, seed):
    """The forest's refine and coarsen (rewritten in place in the leaf
    array) give the same leaves, tags and remap table as a plain list
    restatement, over random rounds of refine, coarsen and 2:1 balance on a
    periodic 2x1 brick."""
    rng = np.random.default_rng(seed)
    f = ag.Forest(2, 1, periodic=(1, 1), level=2)
    for rnd in range(8):
        f.begin_regrid()
        tags = rng.integers(0, 3, f.num_quads).astype(np.int32)
        f.set_tags(tags)
        ref = _lib_leaves(f)
        flags = (rng.random(f.num_quads) < 0.3).astype(np.int32)
        f.refine(flags, max_level=7)
        ref = _py_refine(ref, flags, 7)
        assert _lib_leaves(f) == ref, rnd
        flags = (rng.random(f.num_quads) < 0.7).astype(np.int32)
        f.coarsen(flags, min_level=1)
        ref = _py_coarsen(ref, flags, 1)
        assert _lib_leaves(f) == ref, rnd
        f.balance()
        assert f.is_balanced()
