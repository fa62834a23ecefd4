"""The CPU baseline's NumPy workload builder (oracle/workload.py) against
the library's own forest: identical external_t arrays (cell_info, face_info,
geom) for the uniform periodic vortex mesh, and the same initial state to
the rounding of exp / pow."""
import numpy as np
import pytest


@pytest.mark.parametrize("level,n", [(1, 4), (2, 8), (3, 16), (5, 16), (6, 16)])
def test_mesh_arrays_equal_the_library_forest(ag, level, n):
    from oracle import workload as WL
    from amrgpu import workloads as W
    f, m, cfg, s0 = W.vortex_1024(level=level, n=n, form=0)
    w = WL.uniform_periodic_mesh(level, n)
    assert (w.ncell, w.nface, w.dof) == (m.ncell, m.nface, m.dof)
    assert np.array_equal(w.cell_info, m.cell_info[: 3 * m.ncell])
    assert np.array_equal(w.face_info, m.face_info[: 11 * m.nface])
    assert np.array_equal(w.geom, m.geom[: 12 * m.ncell])


@pytest.mark.parametrize("level,n", [(3, 16), (6, 16)])
def test_vortex_state_matches_the_library_ic(ag, level, n):
    from oracle import workload as WL
    from amrgpu import workloads as W
    f, m, cfg, s0 = W.vortex_1024(level=level, n=n, form=0)
    q = WL.vortex_state(WL.uniform_periodic_mesh(level, n))
    assert q.shape == s0.shape
    np.testing.assert_allclose(q, s0, rtol=1e-14, atol=1e-15)
    c = WL.vortex_config()
    for k in ("time_scheme", "dt", "cfl", "coarse_grid_h", "initial_condition", "gamma", "density", "pressure",
              "mach", "alpha", "beta"):
        assert c[k] == cfg[k], k
