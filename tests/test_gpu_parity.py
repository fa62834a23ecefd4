"""GPU parity: the CUDA path against the oracle and the reference's golden
fixtures. The plain FP64 form must be bit-identical (same operations, same
order, no contracted multiply-adds); the FP32-flux form is held to the
tolerances written in each test."""
import os

import numpy as np
import pytest

import meshes
from test_oracle import GMesh, golden_cases

pytestmark = pytest.mark.gpu

os.environ.setdefault("AMRGPU_QUIET", "1")


def to_mesh(ag, gm):
    return ag.Mesh(gm.n, gm.cell_info, gm.face_info, gm.geom, gm.nface, gm.dof)


def config_from_golden(ag, z):
    c = ag.Config(nelem_subgrid=int(z["n"]))
    for k in ("time_scheme", "time_steps", "dt", "cfl", "coarse_grid_h", "initial_condition", "gamma", "density",
              "pressure", "mach", "alpha", "beta", "checkpoint_interval", "visualization_interval",
              "regrid_interval"):
        c[k] = z[k].item()
    c["bc"] = [int(b) for b in z["bc"]][:6]
    return c


@pytest.mark.parametrize("path", golden_cases("rhs_"), ids=os.path.basename)
def test_fp64_rhs_bitwise_equals_reference_golden(ag, path):
    z = np.load(path)
    gm = GMesh(z)
    s = ag.Session(to_mesh(ag, gm), config_from_golden(ag, z), form=ag.FORM_FP64_EXACT)
    s.upload(z["soln0"])
    r = s.rhs()
    assert np.array_equal(r, z["rhs"]), np.abs(r - z["rhs"]).max()


@pytest.mark.parametrize("entry", ["hpc_amr_evolve_solver", "physics_go_gpu"])
@pytest.mark.parametrize("path", golden_cases("go_"), ids=os.path.basename)
def test_fp64_evolve_through_c_abi_bitwise(ag, path, entry):
    """The reference-facing entry point on host arrays reproduces the
    reference driver's segment: state bits and the interval flags."""
    z = np.load(path)
    gm = GMesh(z)
    cfg = config_from_golden(ag, z)
    cfg["form"] = ag.FORM_FP64_EXACT
    cfg.apply()
    s = z["soln0"].copy()
    res = ag.evolve_solver(to_mesh(ag, gm), s, 0, entry=entry)
    assert res["error"] == 0, ag.last_error()
    assert np.array_equal(s, z["soln1"]), np.abs(s - z["soln1"]).max()
    for k in ("istep", "regrid", "visualize", "checkpoint", "evolve_solution"):
        assert res[k] == int(z[k]), k


def random_case(ag, seed, n=None, scheme=None):
    rng = np.random.default_rng(seed)
    n = n or int(rng.choice([2, 4, 8, 16]))
    per = (int(rng.integers(2)), int(rng.integers(2)))
    f = meshes.uniform(n, 2, periodic=per)
    fl = (rng.random(f.num_quads) < 0.35).astype(np.int32)
    f.refine(fl)
    f.balance()
    cfg = meshes.make_config(n, time_scheme=scheme or int(rng.integers(1, 6)), time_steps=9, dt=0.01,
                             bc=tuple(int(b) for b in rng.integers(0, 3, 4)))
    cfg.apply()
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), seed, amp=1e-2)
    return f, m, cfg, s0


@pytest.mark.parametrize("seed", range(8))
def test_fp64_random_meshes_bitwise(ag, oracle, seed):
    f, m, cfg, s0 = random_case(ag, seed)
    n = m.n
    oc = oracle.make_config(n, cfg)
    ref = s0.copy()
    out = oracle.evolve(m, ref, oc)
    s = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    s.upload(s0)
    assert s.cfl_dt() == oracle.time_step(m, s0, oracle.make_config(n, cfg)) or cfg["time_scheme"] == 2
    s.step(out["steps"])
    rep = s.sync()
    got = s.download()
    assert np.array_equal(got, ref), np.abs(got - ref).max()
    assert rep["steps"] == out["steps"]
    assert rep["time"] == out["time"]
    assert abs(rep["residual_norm"] - out["residual_norm"]) <= 1e-12 * out["residual_norm"]


@pytest.mark.parametrize("n", [2, 4, 8, 16])
def test_every_launch_variant_gives_identical_bits(ag, oracle, n):
    from amrgpu._lib import lib
    f, m, cfg, s0 = random_case(ag, 100 + n, n=n, scheme=3)
    ref = s0.copy()
    oracle.evolve(m, ref, oracle.make_config(n, cfg))
    import ctypes as C
    tried = 0
    for qpb in (1, 2, 4, 8, 16, 32):
        for thr in (64, 96, 128, 160, 192, 256, 288, 320, 384, 544, 576):
            s = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
            if lib().amrgpu_session_set_launch(s._s, qpb, thr) != 0:
                ag.clear_error()
                continue
            s.upload(s0)
            s.step(cfg["time_steps"])
            got = s.download()
            assert np.array_equal(got, ref), (qpb, thr)
            tried += 1
    assert tried >= 1


@pytest.mark.parametrize("n", [8, 16])
@pytest.mark.parametrize("scheme", [1, 2, 3, 4, 5])
def test_every_fp64_variant_every_scheme_bitwise(ag, oracle, n, scheme):
    """Every compiled FP64 stage kernel for the patch size (block kernels and
    row sweeps) reproduces the oracle's segment bit for bit, for every RK
    scheme, on a mesh with hanging faces and mixed boundaries."""
    f, m, cfg, s0 = random_case(ag, 200 + 7 * n + scheme, n=n, scheme=scheme)
    ref = s0.copy()
    out = oracle.evolve(m, ref, oracle.make_config(n, cfg))
    s = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    nv = len(s.launch_variants())
    assert nv >= 3
    for k in range(nv):
        s.set_launch_variant(k)
        s.upload(s0)
        s.step(out["steps"])
        rep = s.sync()
        got = s.download()
        assert np.array_equal(got, ref), (k, np.abs(got - ref).max())
        assert rep["time"] == out["time"], k
        assert abs(rep["residual_norm"] - out["residual_norm"]) <= 1e-12 * out["residual_norm"], k
    s.close()


def test_graph_replay_equals_eager_launches(ag):
    f, m, cfg, s0 = random_case(ag, 7, n=8, scheme=3)
    a = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    a.upload(s0)
    a.step(50)
    b = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    b.upload(s0)
    b.step(50, graph_steps=12)
    assert np.array_equal(a.download(), b.download())
    assert a.sync()["time"] == b.sync()["time"]


def test_two_runs_are_bitwise_identical(ag):
    f, m, cfg, s0 = random_case(ag, 9, n=16, scheme=3)
    outs = []
    for form in (ag.FORM_FP64_EXACT, ag.FORM_FP32_FLUX):
        for _ in range(2):
            s = ag.Session(m, cfg, form=form)
            s.upload(s0)
            s.step(20)
            outs.append((form, s.download(), s.sync()["residual_norm"]))
    assert np.array_equal(outs[0][1], outs[1][1]) and outs[0][2] == outs[1][2]
    assert np.array_equal(outs[2][1], outs[3][1]) and outs[2][2] == outs[3][2]


@pytest.mark.parametrize("seed", range(3))
def test_fp32_flux_rhs_within_tolerance(ag, oracle, seed):
    """FP32 flux arithmetic: per-field max error of one residual evaluation
    <= 2e-5 of that field's max |R| (FP32 eps 6e-8 times ~300 operations)."""
    f, m, cfg, s0 = random_case(ag, 200 + seed)
    ref = oracle.rhs(m, s0, oracle.make_config(m.n, cfg)).reshape(-1, 4)
    s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
    s.upload(s0)
    got = s.rhs().reshape(-1, 4)
    for k in range(4):
        scale = np.abs(ref[:, k]).max() + 1e-300
        assert np.abs(got[:, k] - ref[:, k]).max() <= 2e-5 * scale, k


def test_fp32_form_riemann_200_steps_l1_rho(ag, oracle):
    """The CPU-runnable workload (64x64 planar Riemann, RK3, 200 steps): the
    FP32-flux form's density stays within 1e-3 relative L1 of the FP64 run
    (the accuracy bound of the FP32 form)."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "go_riemann_64x64_rk3_200.npz"))
    gm = GMesh(z)
    cfg = config_from_golden(ag, z)
    s = ag.Session(to_mesh(ag, gm), cfg, form=ag.FORM_FP32_FLUX)
    s.upload(z["soln0"])
    s.step(200)
    got = s.download().reshape(-1, 4)
    ref = z["soln1"].reshape(-1, 4)
    l1 = np.abs(got[:, 0] - ref[:, 0]).sum() / np.abs(ref[:, 0]).sum()
    assert l1 < 1e-3, l1


def test_periodic_conservation_on_gpu(ag):
    f, m, cfg, s0 = random_case(ag, 11, n=8, scheme=3)
    cfg2 = meshes.make_config(8, time_scheme=3, time_steps=40, dt=0.01)
    f2 = meshes.two_level_ring(8, periodic=(1, 1))
    cfg2.apply()
    m2 = f2.mesh(8)
    s2 = meshes.perturbed(f2.initialize(8), 3, amp=1e-2)
    for form in (ag.FORM_FP64_EXACT, ag.FORM_FP32_FLUX):
        s = ag.Session(m2, cfg2, form=form)
        s.upload(s2)
        t0 = s.totals()
        s.step(40)
        t1 = s.totals()
        assert np.all(np.abs(t1 - t0) <= 1e-12 * np.abs(t0) + 1e-13), (form, t1 - t0)


def test_nonfinite_state_is_reported_not_trapped(ag):
    """A NaN planted in the host input comes back as AMRGPU_ERR_NONFINITE
    through the C ABI, with evolve_solution cleared (the reference aborts)."""
    f, m, cfg, s0 = random_case(ag, 12, n=4, scheme=3)
    cfg.apply()
    bad = s0.copy()
    bad[4 * 17] = np.nan
    ag.clear_error()
    res = ag.evolve_solver(m, bad, 0)
    assert res["error"] == 4
    assert res["evolve_solution"] == 0
    ag.clear_error()
    good = s0.copy()
    res = ag.evolve_solver(m, good, 0)
    assert res["error"] == 0 and np.isfinite(good).all()


def test_segment_stops_at_interval_flags(ag, oracle):
    f, m, cfg, s0 = random_case(ag, 13, n=4, scheme=3)
    cfg["time_steps"] = 30
    cfg["regrid_interval"] = 4
    cfg["visualization_interval"] = 6
    cfg.apply()
    a = s0.copy()
    b = s0.copy()
    ist_g = ist_o = 0
    oc = oracle.make_config(4, cfg)
    for _ in range(4):
        rg = ag.evolve_solver(m, a, ist_g)
        ro = oracle.evolve(m, b, oc, ist_o)
        assert (rg["istep"], rg["regrid"], rg["visualize"]) == (ro["istep"], ro["regrid"], ro["visualize"])
        ist_g, ist_o = rg["istep"], ro["istep"]
        assert np.array_equal(a, b)
    assert ist_g == 12
