"""The FP64 restatement of the mixed-patch-size residual
(oracle/mixed_oracle.py) on meshes whose quads all have one size must give
the reference's residual (the C restatement of the reference's 2D kernels,
oracle.rhs, itself pinned to the reference's own driver): the mixed rule
reduces to the reference's face pairing when sizes agree. Periodic meshes
with hanging faces; only summation order differs (1e-12 of max|R|)."""
import numpy as np
import pytest

import meshes


@pytest.mark.parametrize("n", [8, 16])
def test_mixed_restatement_equals_reference_at_one_size(ag, oracle, n):
    from oracle import mixed_oracle as MO
    f = meshes.two_level_ring(n, periodic=(1, 1))
    cfg = meshes.make_config(n, time_scheme=3, dt=0.01, time_steps=10)
    cfg.apply()
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), 3, amp=2e-2)
    ref = oracle.rhs(m, s0, oracle.make_config(n, cfg)).reshape(-1, 4)
    mm = f.mesh_mixed(np.full(f.num_quads, n, np.int32))
    assert np.array_equal(mm.cell_info, m.cell_info) and mm.dof == m.dof
    got = MO.rhs(mm, s0, cfg["coarse_grid_h"]).reshape(-1, 4)
    for k in range(4):
        scale = np.abs(ref[:, k]).max()
        assert np.abs(got[:, k] - ref[:, k]).max() <= 1e-12 * scale, k


def test_mixed_mesh_layout(ag):
    """cell_info[2] is the running sum of 4 n^2, dof the total, faces and
    corners are the forest's; initial patches come at each quad's size."""
    f = meshes.two_level_ring(16, periodic=(1, 1))
    cfg = meshes.make_config(16, time_scheme=3, dt=0.01, time_steps=10)
    cfg.apply()
    rng = np.random.default_rng(0)
    sizes = rng.choice([8, 16], f.num_quads).astype(np.int32)
    m = f.mesh_mixed(sizes)
    m16 = f.mesh(16)
    off = m.cell_info[2::3]
    assert off[0] == 0
    assert np.array_equal(np.diff(off), 4 * sizes[:-1] ** 2)
    assert m.dof == 4 * int((sizes.astype(np.int64) ** 2).sum()) and m.ncells == m.dof // 4
    assert np.array_equal(m.face_info, m16.face_info) and np.array_equal(m.geom, m16.geom)
    s = f.initialize(sizes)
    assert s.size == m.dof
    a8, a16 = f.initialize(8).reshape(f.num_quads, -1), f.initialize(16).reshape(f.num_quads, -1)
    for q in (0, f.num_quads // 2, f.num_quads - 1):
        want = (a8 if sizes[q] == 8 else a16)[q]
        assert np.array_equal(s[4 * (off[q] // 4):4 * (off[q] // 4) + want.size], want)
