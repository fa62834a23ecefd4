"""The oracle itself: pinned against the reference's own C driver (golden
fixtures made by tests/golden/make_golden.py, and live when oracle/_ref is
built) and against analytic facts of the reference scheme. CPU only."""
import glob
import os

import numpy as np
import pytest

import meshes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


class GMesh:
    def __init__(self, z):
        self.n = int(z["n"])
        self.cell_info = z["cell_info"].astype(np.int32)
        self.face_info = z["face_info"].astype(np.int32)
        self.geom = z["geom"].astype(np.float64)
        self.nface = int(z["nface"])
        self.dof = int(z["dof"])
        self.ncell = len(self.cell_info) // 3
        self.nghost = 0


def golden_cfg(z):
    keys = ["time_scheme", "time_steps", "dt", "cfl", "coarse_grid_h", "initial_condition", "gamma", "density",
            "pressure", "mach", "alpha", "beta", "checkpoint_interval", "visualization_interval", "regrid_interval"]
    d = {k: z[k].item() for k in keys}
    d["bc"] = [int(b) for b in z["bc"]][:6]
    d["final_time"] = 0.0
    return d


def golden_cases(prefix):
    return sorted(glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))


@pytest.mark.parametrize("path", golden_cases("rhs_"), ids=os.path.basename)
def test_restatement_rhs_matches_reference_golden(oracle, path):
    z = np.load(path)
    m = GMesh(z)
    cfg = golden_cfg(z)
    r = oracle.rhs(m, z["soln0"], oracle.make_config(m.n, cfg))
    assert np.array_equal(r, z["rhs"]), np.abs(r - z["rhs"]).max()


@pytest.mark.parametrize("path", golden_cases("go_"), ids=os.path.basename)
def test_restatement_evolve_matches_reference_golden(oracle, path):
    z = np.load(path)
    m = GMesh(z)
    cfg = golden_cfg(z)
    s = z["soln0"].copy()
    res = oracle.evolve(m, s, oracle.make_config(m.n, cfg))
    assert np.array_equal(s, z["soln1"]), np.abs(s - z["soln1"]).max()
    for k in ("istep", "regrid", "visualize", "checkpoint", "evolve_solution"):
        assert res[k] == int(z[k]), k


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                    "libref_physics.so")), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", range(4))
def test_restatement_matches_reference_live(ag, oracle, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.choice([2, 4, 8]))
    per = (int(rng.integers(2)), int(rng.integers(2)))
    f = meshes.uniform(n, 2, periodic=per)
    fl = (rng.random(f.num_quads) < 0.3).astype(np.int32)
    f.refine(fl)
    f.balance()
    cfg = meshes.make_config(n, time_scheme=int(rng.integers(1, 6)), time_steps=6, dt=0.01,
                             bc=tuple(int(b) for b in rng.integers(0, 3, 4)))
    cfg.apply()
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), seed)
    r1 = oracle.rhs(m, s0, oracle.make_config(n, cfg))
    r2 = oracle.reference_rhs(m, s0, n, cfg)
    assert np.array_equal(r1, r2)
    a, b = s0.copy(), s0.copy()
    oracle.evolve(m, a, oracle.make_config(n, cfg))
    oracle.reference_go(m, b, n, cfg)
    assert np.array_equal(a, b)


def test_free_stream_is_preserved(ag, oracle):
    """Uniform flow on a periodic mesh with hanging faces: R(Q) = 0 to round-off."""
    n = 4
    f = meshes.hanging(n, periodic=(1, 1))
    cfg = meshes.make_config(n, ic=0)
    cfg.apply()
    m = f.mesh(n)
    s = f.initialize(n)
    r = oracle.rhs(m, s, oracle.make_config(n, cfg))
    assert np.abs(r).max() < 1e-12


def cell_volumes(m):
    n = m.n
    g = m.geom.reshape(-1, 12)
    dx = (g[:, 3] - g[:, 0]) / n
    dy = (g[:, 7] - g[:, 1]) / n
    return np.repeat(dx * dy, n * n)


def test_periodic_conservation_with_hanging_faces(ag, oracle):
    """sum(vol * rhs) = 0: every face flux enters two cells with opposite sign."""
    n = 4
    f = meshes.two_level_ring(n, periodic=(1, 1))
    cfg = meshes.make_config(n)
    cfg.apply()
    m = f.mesh(n)
    s = meshes.perturbed(f.initialize(n), 7, amp=1e-2)
    r = oracle.rhs(m, s, oracle.make_config(n, cfg)).reshape(-1, 4)
    vol = cell_volumes(m)
    tot = (vol[:, None] * r).sum(axis=0)
    scale = (vol[:, None] * np.abs(r)).sum(axis=0)
    assert np.all(np.abs(tot) <= 1e-12 * scale + 1e-14)


def test_slip_walls_conserve_mass_and_energy(ag, oracle):
    n = 8
    f = meshes.hanging(n)
    cfg = meshes.make_config(n, bc=(1, 1, 1, 1))
    cfg.apply()
    m = f.mesh(n)
    s = meshes.perturbed(f.initialize(n), 8)
    r = oracle.rhs(m, s, oracle.make_config(n, cfg)).reshape(-1, 4)
    vol = cell_volumes(m)
    for k in (0, 3):
        tot = (vol * r[:, k]).sum()
        assert abs(tot) <= 1e-12 * (vol * np.abs(r[:, k])).sum() + 1e-14


def test_planar_riemann_stays_y_invariant(ag, oracle):
    """No noise: a y-uniform state keeps rho*v = 0 and every row identical, to
    the round-off of the bilinear sub-cell geometry (tiny normal components)."""
    n = 8
    cfg = ag.Config.from_input(cfl=0.5, time_scheme=3, nelem_subgrid=n, coarse_grid_h=1.0, initial_condition=2,
                               time_steps=20, dt=1.0, bc=[1] * 6)
    cfg.apply()
    f = ag.Forest(1, 1, periodic=(0, 0), lo=(0.0, 0.0, 0.0), scale=1.0, level=2)
    m = f.mesh(n)
    s = f.initialize(n)
    oracle.evolve(m, s, oracle.make_config(n, cfg))
    q = s.reshape(-1, n, n, 4)
    assert np.abs(q[..., 2]).max() < 1e-13
    tree, lev, x, y = f.quads()
    # gather the global grid and compare rows
    N = n * 4
    grid = np.zeros((N, N, 4))
    L = 2 ** 30
    for k in range(len(x)):
        i0 = int(x[k] * 4 // L) * n
        j0 = int(y[k] * 4 // L) * n
        grid[j0:j0 + n, i0:i0 + n] = q[k]
    for k in (0, 1, 3):
        assert np.abs(grid[..., k] - grid[0:1, :, k]).max() < 1e-12


def test_flux_consistency(oracle):
    """F(q, q, n) is the physical flux F(q).n (HLL with equal states)."""
    rng = np.random.default_rng(0)
    for _ in range(50):
        rho, u, v, p = rng.uniform(0.2, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.2, 2)
        q = np.array([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)])
        nv = rng.uniform(-1, 1, 2)
        F = oracle.flux(q, q, nv)
        pp = 0.3999999999999999 * (q[3] - 0.5 * rho * (u * u + v * v))
        phys = np.array([rho * u, rho * u * u + pp, rho * u * v, u * (q[3] + pp)]) * nv[0] + \
            np.array([rho * v, rho * u * v, rho * v * v + pp, v * (q[3] + pp)]) * nv[1]
        assert np.allclose(F, phys, rtol=1e-12, atol=1e-12)


def test_flux_is_antisymmetric_in_the_normal(oracle):
    """F(qL, qR, n) = -F(qR, qL, -n): the scheme's conservation across a face."""
    rng = np.random.default_rng(1)
    for _ in range(50):
        def st():
            rho, u, v, p = rng.uniform(0.2, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.2, 2)
            return np.array([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)])
        a, b = st(), st()
        nv = rng.uniform(-1, 1, 2)
        assert np.allclose(oracle.flux(a, b, nv), -oracle.flux(b, a, -nv), rtol=1e-12, atol=1e-13)


def test_product_ic_matches_oracle_ic(ag, oracle):
    """Host IC 0/1 of libamrgpu equal the restated Fortran IC bit for bit."""
    import ctypes as C
    L = C.CDLL(oracle.RESTATEMENT)
    f = meshes.hanging(8)
    for ic in (0, 1):
        cfg = meshes.make_config(8, ic=ic)
        cfg["alpha"] = 30.0
        cfg.apply()
        s = f.initialize(8)
        m = f.mesh(8)
        ref = np.zeros_like(s)
        for q in range(m.ncell):
            g = np.ascontiguousarray(m.geom[12 * q:12 * q + 12])
            out = np.zeros(4 * 64)
            args = [C.c_int(ic), C.c_int(2), C.c_int(0), C.c_int(4), C.c_int(8), C.c_int(0), C.c_double(0.0)]
            dv = [C.c_double(cfg[k]) for k in ("mach", "alpha", "beta", "gamma", "density", "pressure")]
            L.solver_initialize_quadrant(*[C.byref(a) for a in args[:6]], C.byref(args[6]), oracle.dp(g),
                                         oracle.dp(out), *[C.byref(d) for d in dv])
            ref[256 * q:256 * q + 256] = out
        assert np.array_equal(s, ref)


def test_oracle_inflow_state_matches_the_library_ic(ag, oracle):
    """bc 3 (extension): the oracle's inflow state is the post-shock state
    the library's shock-bubble IC puts left of the shock, bit for bit."""
    cfg = ag.Config.from_input(cfl=0.5, time_scheme=3, nelem_subgrid=4, coarse_grid_h=1.0, initial_condition=5,
                               time_steps=1, dt=1.0, bc=[3, 0, 1, 1, 1, 1], gamma=1.4,
                               ic_params=[2.0, 0.1, 0.1375, 0.2])
    cfg.apply()
    f = ag.Forest(2, 1, periodic=(0, 0), lo=(0.0, 0.0, 0.0), scale=1.0, level=5)
    s = f.initialize(4).reshape(-1, 4, 4, 4)
    m = f.mesh(4)
    g = m.geom.reshape(-1, 12)
    left = int(np.argmin(g[:, 0] + g[:, 1]))  # the quad at the lower-left corner, behind the shock
    q = oracle.set_inflow(cfg)
    assert np.array_equal(s[left, 0, 0], q)
