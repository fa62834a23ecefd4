"""Sharded meshes on the CPU: the partition, the ghost and send lists, and
the two drivers of amrgpu.shard with the oracle computing each rank's
stages -- in one process (LocalCluster) and as two gloo processes
(Distributed over torch.distributed). A sharded run must reproduce the
unsharded oracle_evolve bit for bit (state, time, steps); the residual
norm is a sum over ranks in another order, within 1e-12."""
import os
import socket

import numpy as np
import pytest

import meshes
from shard_oracle import OracleRank


def build(seed, n=4, scheme=3):
    rng = np.random.default_rng(seed)
    per = (int(rng.integers(2)), int(rng.integers(2)))
    f = meshes.uniform(n, 2, periodic=per)
    fl = (rng.random(f.num_quads) < 0.4).astype(np.int32)
    f.refine(fl)
    f.balance()
    cfg = meshes.make_config(n, time_scheme=scheme, time_steps=6, dt=0.01,
                             bc=tuple(int(b) for b in rng.integers(0, 3, 4)))
    cfg.apply()
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), seed, amp=2e-2)
    return m, cfg, s0


def faces_of(mesh):
    fi = mesh.face_info.reshape(-1, 11)[: mesh.nface]
    return fi


@pytest.mark.parametrize("nranks", [1, 2, 3, 5])
def test_shards_cover_every_face_and_agree_on_lists(ag, nranks):
    from amrgpu import shard as S
    m, cfg, s0 = build(1)
    off = S.partition(m.ncell, nranks)
    assert off[0] == 0 and off[-1] == m.ncell and np.all(np.diff(off) >= m.ncell // nranks)
    shards = [S.make_shard(m, off, r) for r in range(nranks)]
    rec = 4 * m.n * m.n
    gfi = faces_of(m)
    for sh in shards:
        lm = sh.mesh
        assert lm.ncell == sh.nlocal and lm.nghost == len(sh.ghosts) and lm.dof == rec * sh.nlocal
        assert np.all(np.diff(sh.ghosts) > 0)
        assert np.all((sh.ghosts < sh.lo) | (sh.ghosts >= sh.lo + sh.nlocal))
        # faces: exactly those touching a local quad, in global order, remapped
        glob = np.concatenate([np.arange(sh.lo, sh.lo + sh.nlocal), sh.ghosts])
        lfi = faces_of(lm)
        back = lfi.copy()
        for k in range(2, 7):
            sel = back[:, k] >= 0
            back[sel, k] = glob[back[sel, k]]
        hit = np.zeros(len(gfi), bool)
        for k in (2, 3, 4):
            ok = (gfi[:, k] >= sh.lo) & (gfi[:, k] < sh.lo + sh.nlocal)
            ok &= (k == 2) | ((k == 3) & (gfi[:, 0] >= 2)) | ((k == 4) & (gfi[:, 0] == 3))
            hit |= ok
        assert np.array_equal(back, gfi[hit])
        # each local quad has 4 sides covered: the local mesh decodes
        ag.Mesh(lm.n, lm.cell_info, lm.face_info, lm.geom, lm.nface, lm.dof, nghost=lm.nghost)
        # ghost run of each peer equals that peer's send list to this rank
        for peer, gfirst, gcount in sh.recv:
            src = shards[peer]
            sf, sc = next((f, c) for p, f, c in src.send if p == sh.rank)
            assert sc == gcount
            sent = src.send_quads[sf:sf + sc] + src.lo
            assert np.array_equal(sent, sh.ghosts[gfirst:gfirst + gcount])
        snd, rcv = sh.reference_lists()
        assert len(snd) == 2 * len(sh.send_quads) and len(rcv) == 2 * len(sh.ghosts)
    # every ghost is received once, every send is somebody's ghost
    assert sum(len(s.ghosts) for s in shards) == sum(len(s.send_quads) for s in shards)


@pytest.mark.parametrize("scheme", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("nranks", [2, 3])
def test_local_cluster_of_oracle_ranks_equals_unsharded(ag, oracle, scheme, nranks):
    from amrgpu import shard as S
    m, cfg, s0 = build(10 + scheme, scheme=scheme)
    oc = oracle.make_config(m.n, cfg)
    ref = s0.copy()
    out = oracle.evolve(m, ref, oc)
    off = S.partition(m.ncell, nranks)
    ranks = [OracleRank(S.make_shard(m, off, r), cfg) for r in range(nranks)]
    cl = S.LocalCluster(ranks)
    cl.start(s0)
    cl.step(out["steps"])
    got = cl.download()
    rep = cl.report()
    assert np.array_equal(got, ref)
    assert rep["steps"] == out["steps"] and rep["time"] == out["time"]
    assert abs(rep["residual_norm"] - out["residual_norm"]) <= 1e-12 * out["residual_norm"]


def test_uneven_partition_with_hanging_faces_across_ranks(ag, oracle):
    from amrgpu import shard as S
    f = meshes.two_level_ring(4, periodic=(1, 1))
    cfg = meshes.make_config(4, time_scheme=3, time_steps=5, dt=0.01)
    cfg.apply()
    m = f.mesh(4)
    s0 = meshes.perturbed(f.initialize(4), 3, amp=1e-2)
    ref = s0.copy()
    out = oracle.evolve(m, ref, oracle.make_config(4, cfg))
    off = np.array([0, 7, m.ncell // 3, m.ncell // 2 + 3, m.ncell], np.int64)
    assert np.all(np.diff(off) > 0)
    ranks = [OracleRank(S.make_shard(m, off, r), cfg) for r in range(4)]
    assert sum(len(r.shard.ghosts) for r in ranks) > 0
    cl = S.LocalCluster(ranks)
    cl.start(s0)
    cl.step(out["steps"])
    assert np.array_equal(cl.download(), ref)


def test_ghost_interiors_are_never_read(ag, oracle):
    """Ghosts travel as their one-cell edge strips: with every ghost quad's
    interior cells set to NaN after the start, a sharded run still equals
    the unsharded one bit for bit (nothing reads a ghost off its strips)."""
    from amrgpu import shard as S
    n = 4
    f = meshes.two_level_ring(n, periodic=(1, 1))
    cfg = meshes.make_config(n, time_scheme=3, time_steps=5, dt=0.01)
    cfg.apply()
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), 4, amp=1e-2)
    ref = s0.copy()
    out = oracle.evolve(m, ref, oracle.make_config(n, cfg))
    off = S.partition(m.ncell, 3)
    ranks = [OracleRank(S.make_shard(m, off, r), cfg) for r in range(3)]
    cl = S.LocalCluster(ranks)
    cl.start(s0)
    interior = np.array([j * n + i for j in range(1, n - 1) for i in range(1, n - 1)], np.int64)
    poisoned = 0
    for r in ranks:
        nl, ng, rec = r.shard.nlocal, len(r.shard.ghosts), r.shard.record
        if ng:
            g = r.Q[nl * rec:(nl + ng) * rec].reshape(ng, n * n, 4)
            g[:, interior, :] = np.nan
            poisoned += ng
    assert poisoned > 0
    cl.step(out["steps"])
    assert np.array_equal(cl.download(), ref)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, seed, steps, outdir, scheme=3, fail_rank=-1, timeout_s=60):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    for p in (os.path.dirname(here), os.path.join(os.path.dirname(here), "amr-demo_b200"), here):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime
    import torch.distributed as dist
    from amrgpu import shard as S
    from shard_oracle import OracleRank as OR
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s))
    try:
        if rank == fail_rank:
            raise RuntimeError("rank failed before its first exchange")
        m, cfg, s0 = build(seed, scheme=scheme)
        off = S.partition(m.ncell, world)
        drv = S.Distributed(OR(S.make_shard(m, off, rank), cfg))
        drv.start(drv.r.shard.local_state(s0))
        drv.step(steps)
        rep = drv.report()
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), q=drv.download(), time=rep["time"],
                 steps=rep["steps"], norm=rep["residual_norm"])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,scheme", [(2, 3), (3, 4)])
def test_gloo_ranks_equal_unsharded(ag, oracle, tmp_path, world, scheme):
    import torch.multiprocessing as mp
    seed, steps = 21, 5
    m, cfg, s0 = build(seed, scheme=scheme)
    ref = s0.copy()
    oc = oracle.make_config(m.n, cfg)
    oc.time_steps = steps
    out = oracle.evolve(m, ref, oc)
    assert out["steps"] == steps
    port = _free_port()
    mp.start_processes(_gloo_rank, args=(world, port, seed, steps, str(tmp_path), scheme), nprocs=world,
                       start_method="spawn", join=True)
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    got = np.concatenate([p["q"] for p in parts])
    assert np.array_equal(got, ref)
    for p in parts:
        assert int(p["steps"]) == steps and float(p["time"]) == out["time"]
        assert abs(float(p["norm"]) - out["residual_norm"]) <= 1e-12 * out["residual_norm"]


def test_a_failed_rank_ends_the_others_with_an_error(ag, tmp_path):
    """Failure detection without a GPU: one of two gloo ranks raises before
    its first exchange. The launcher reports the failure and ends the run
    (the other rank, stuck in its first collective, has a 5 s process-group
    timeout as the last bound); nothing waits for good and no result is
    written."""
    import time
    import torch.multiprocessing as mp
    port = _free_port()
    t0 = time.perf_counter()
    with pytest.raises(Exception):
        mp.start_processes(_gloo_rank, args=(2, port, 21, 3, str(tmp_path), 3, 1, 5), nprocs=2,
                           start_method="spawn", join=True)
    assert time.perf_counter() - t0 < 120
    assert not (tmp_path / "rank0.npz").exists()
