"""Edge cases of the device path: a rank with no quads, a single periodic
quad that is its own neighbour on every side, a patch size without a
compiled kernel, and a single quad with walls on all four sides."""
import os

import numpy as np
import pytest

import meshes

pytestmark = pytest.mark.gpu
os.environ.setdefault("AMRGPU_QUIET", "1")


def test_empty_mesh_steps_nothing(ag):
    """A session of zero quads (an MPI rank whose partition is empty) is
    created, uploaded, stepped and downloaded without launching work."""
    n = 4
    cfg = meshes.make_config(n)
    cfg.apply()
    m = ag.Mesh(n, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0), 0, 0)
    for form in (ag.FORM_FP64_EXACT, ag.FORM_FP32_FLUX):
        s = ag.Session(m, cfg, form=form)
        s.upload(np.zeros(0))
        s.step(3)
        rep = s.sync()
        assert rep["steps"] == 0 and rep["error"] == 0
        assert s.download().size == 0
        assert np.array_equal(s.totals(), np.zeros(4))
        s.close()


@pytest.mark.parametrize("n", [2, 8])
@pytest.mark.parametrize("scheme", [1, 3, 5])
def test_single_periodic_quad_is_bitwise(ag, oracle, n, scheme):
    """One quad whose four sides are faces with itself (level 0, periodic in
    x and y): the FP64 form against the oracle, bit for bit."""
    f = ag.Forest(1, 1, periodic=(1, 1), lo=(-2.0, -2.0, 0.0), scale=4.0, level=0)
    cfg = meshes.make_config(n, time_scheme=scheme, time_steps=10, dt=0.01)
    cfg.apply()
    m = f.mesh(n)
    assert m.ncell == 1
    s0 = meshes.perturbed(f.initialize(n), 7, amp=2e-2)
    ref = s0.copy()
    out = oracle.evolve(m, ref, oracle.make_config(n, cfg))
    s = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    s.upload(s0)
    s.step(out["steps"])
    got = s.download()
    s.close()
    assert np.array_equal(got, ref), np.abs(got - ref).max()


def test_single_walled_quad_conserves_mass(ag):
    """One quad with slip walls on all four sides: the plain form keeps the
    total mass and energy to round-off (a wall face's normal is exactly
    +-1 there, so its mass flux is exactly zero)."""
    n = 16
    f = ag.Forest(1, 1, periodic=(0, 0), lo=(-2.0, -2.0, 0.0), scale=4.0, level=0)
    cfg = meshes.make_config(n, time_scheme=3, time_steps=10 ** 6, dt=0.01, bc=(1, 1, 1, 1))
    cfg.apply()
    m = f.mesh(n)
    s = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    s.upload(meshes.perturbed(f.initialize(n), 8, amp=2e-2))
    t0 = s.totals()
    s.step(30)
    t1 = s.totals()
    s.close()
    for k in (0, 3):
        assert abs(t1[k] - t0[k]) <= 1e-12 * abs(t0[k]), (k, t1[k] - t0[k])


@pytest.mark.parametrize("form", [0, 1])
def test_patch_size_without_a_kernel_is_an_error(ag, form):
    """32x32 patches have no compiled stage kernel: session creation fails
    with AMRGPU_ERR_UNSUPPORTED instead of launching anything."""
    n = 32
    f = ag.Forest(1, 1, periodic=(1, 1), level=1)
    cfg = meshes.make_config(n)
    cfg.apply()
    with pytest.raises(RuntimeError):
        ag.Session(f.mesh(n), cfg, form=form)
    code, _ = ag.last_error()
    assert code == 5
    ag.clear_error()
