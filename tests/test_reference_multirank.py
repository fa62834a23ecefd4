"""The reference's own multi-rank path (its physics_go with the ghost
exchange of physics_mpi_real_to_ghost, physics_mpi.c:47-122) on P ranks as
P threads over the MPI stand-in (oracle/mpi_shim/mpi_threads.c,
oracle/mt_driver.c), fed with Morton-range shards: every rank's quads end
bit-identical to the one-rank reference run of the whole mesh. This pins
the multi-rank CPU baseline (and the stand-in's exchange and reductions) to
the reference's one-rank result."""
import os

import numpy as np
import pytest

import meshes

pytestmark = pytest.mark.skipif(
    not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "oracle", "_ref", "libref_physics_mt.so")),
    reason="oracle/_ref/libref_physics_mt.so not built (reference tree absent)")


def _run(ag, oracle, mesh, cfg, s0, n, nranks):
    from amrgpu import shard as S
    offs = S.partition(mesh.ncell, nranks)
    shards = [S.make_shard(mesh, offs, r) for r in range(nranks)]
    states = [sh.local_state(s0) for sh in shards]
    out = oracle.reference_mt_go(shards, states, n, cfg)
    rec = 4 * n * n
    got = np.concatenate([st[: sh.nlocal * rec] for sh, st in zip(shards, states)])
    return got, out


@pytest.mark.parametrize("nranks", [1, 2, 3, 5])
def test_multirank_reference_equals_one_rank(ag, oracle, nranks):
    n = 4
    f = meshes.hanging(n, periodic=(1, 0), refine=(3, 6, 9))
    cfg = meshes.make_config(n, time_scheme=3, time_steps=7, dt=1.0, bc=(2, 0, 1, 1))
    cfg.apply()
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), 7, amp=1e-2)
    one = s0.copy()
    oracle.reference_go(m, one, n, cfg)
    got, out = _run(ag, oracle, m, cfg, s0, n, nranks)
    assert out["istep"] == [7] * nranks and out["abort"] == 0
    assert np.array_equal(got, one), np.abs(got - one).max()


def test_multirank_reference_on_the_vortex_workload(ag, oracle):
    """The benchmark's mesh family (uniform periodic vortex, here level 3),
    built without the product library, on 4 ranks."""
    from oracle import workload as WL
    n = 16
    mesh = WL.uniform_periodic_mesh(3, n)
    cfg = WL.vortex_config(n, steps=3)
    s0 = WL.vortex_state(mesh)
    one = s0.copy()
    oracle.reference_go(mesh, one, n, cfg)
    got, out = _run(ag, oracle, mesh, cfg, s0, n, 4)
    assert np.array_equal(got, one), np.abs(got - one).max()
