"""Sharded meshes on the GPU: device sessions of the ranks' ghosted meshes,
stepped stage by stage with the halo pack / unpack kernels, against one
unsharded session of the whole mesh. All ranks share the one GPU and run
one after another at every stage (LocalCluster): no kernel waits on another
rank's. The sharded state, time and step count are bit-identical to the
unsharded run in both forms; the residual norm (a sum over ranks in another
order) agrees to 1e-12."""
import datetime
import os
import socket

import numpy as np
import pytest

import meshes

pytestmark = pytest.mark.gpu
os.environ.setdefault("AMRGPU_QUIET", "1")


def build(ag, seed, n, scheme, steps=8):
    rng = np.random.default_rng(seed)
    per = (int(rng.integers(2)), int(rng.integers(2)))
    f = meshes.uniform(n, 3, periodic=per)
    fl = (rng.random(f.num_quads) < 0.3).astype(np.int32)
    f.refine(fl)
    f.balance()
    # scheme 2 runs at the fixed dt (no CFL): small enough for the finest cells
    cfg = meshes.make_config(n, time_scheme=scheme, time_steps=10 ** 6, dt=0.002 if scheme == 2 else 0.01,
                             bc=tuple(int(b) for b in rng.integers(0, 3, 4)))
    cfg.apply()
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), seed, amp=2e-2)
    return m, cfg, s0


def unsharded(ag, m, cfg, s0, form, steps):
    s = ag.Session(m, cfg, form=form)
    s.upload(s0)
    s.step(steps)
    rep = s.sync()
    q = s.download()
    s.close()
    return q, rep


def cluster(ag, m, cfg, s0, form, steps, offsets):
    from amrgpu import shard as S
    cfg["form"] = form
    ranks = [S.GpuRank(S.make_shard(m, offsets, r), cfg) for r in range(len(offsets) - 1)]
    cl = S.LocalCluster(ranks)
    cl.start(s0)
    cl.step(steps)
    rep = cl.report()
    q = cl.download()
    for r in ranks:
        r.close()
    return q, rep


CASES = [(0, 16, 3, 0), (1, 16, 3, 1), (2, 8, 1, 0), (3, 8, 2, 0), (4, 4, 4, 0), (5, 16, 5, 0),
         (6, 16, 5, 1), (7, 2, 3, 0), (8, 16, 2, 1)]


@pytest.mark.parametrize("seed,n,scheme,form", CASES)
@pytest.mark.parametrize("nranks", [2, 3])
def test_local_cluster_bitwise_equals_unsharded(ag, seed, n, scheme, form, nranks):
    from amrgpu import shard as S
    m, cfg, s0 = build(ag, 500 + seed, n, scheme)
    ref, rep0 = unsharded(ag, m, cfg, s0, form, 8)
    got, rep = cluster(ag, m, cfg, s0, form, 8, S.partition(m.ncell, nranks))
    assert rep0["error"] == 0 and rep["error"] == 0 and rep["steps"] == rep0["steps"] == 8
    assert rep["time"] == rep0["time"]
    assert np.array_equal(got, ref), np.abs(got - ref).max()
    assert abs(rep["residual_norm"] - rep0["residual_norm"]) <= 1e-12 * rep0["residual_norm"]


def test_uneven_partition_on_hanging_ring(ag):
    f = meshes.two_level_ring(16, periodic=(1, 1))
    cfg = meshes.make_config(16, time_scheme=3, time_steps=10 ** 6, dt=0.01)
    cfg.apply()
    m = f.mesh(16)
    s0 = meshes.perturbed(f.initialize(16), 4, amp=1e-2)
    off = np.array([0, 5, m.ncell // 3, m.ncell // 2 + 7, m.ncell], np.int64)
    for form in (ag.FORM_FP64_EXACT, ag.FORM_FP32_FLUX):
        ref, _ = unsharded(ag, m, cfg, s0, form, 12)
        got, rep = cluster(ag, m, cfg, s0, form, 12, off)
        assert np.array_equal(got, ref), form


def _stage_input(r):
    import ctypes as C
    import torch
    from amrgpu import shard as S
    from amrgpu._lib import lib
    stride = C.c_longlong(0)
    ptr = lib().amrgpu_session_stage_input(r.session._s, C.byref(stride))
    return torch.as_tensor(S._DeviceView(ptr, (4, stride.value), "<f8"), device=r.device)


def test_halo_moves_edge_strips(ag):
    """GpuRank packs the send quads' four one-cell edge strips (16 n doubles
    per quad: per field sides 0..3 -- column 0, column n-1, row 0, row n-1);
    unpack writes them into the ghosts' edge cells and leaves the interior."""
    from amrgpu import shard as S
    import torch
    m, cfg, s0 = build(ag, 40, 8, 3)
    off = S.partition(m.ncell, 2)
    sh = S.make_shard(m, off, 1)
    r = S.GpuRank(sh, cfg)
    loc = sh.local_state(s0)
    r.upload(loc)
    with torch.cuda.stream(r.stream):
        r.pack()
    r.stream.synchronize()
    n = m.n
    strip = np.array([p * n if s == 0 else p * n + n - 1 if s == 1 else p if s == 2 else (n - 1) * n + p
                      for s in range(4) for p in range(n)])
    aos = loc.reshape(-1, n * n, 4)
    want = aos[sh.send_quads][:, strip, :].transpose(0, 2, 1).reshape(-1)
    assert sh.halo_record == 16 * n
    assert np.array_equal(r.sendbuf[: len(want)].cpu().numpy(), want)
    ng = len(sh.ghosts)
    before = _stage_input(r)[:, sh.nlocal * n * n:(sh.nlocal + ng) * n * n].cpu().numpy().reshape(4, ng, n * n)
    planted = np.arange(ng * sh.halo_record, dtype=np.float64) + 0.5
    r.recvbuf[: len(planted)].copy_(torch.from_numpy(planted))
    torch.cuda.synchronize()
    r.unpack()
    r.stream.synchronize()
    g = _stage_input(r)[:, sh.nlocal * n * n:(sh.nlocal + ng) * n * n].cpu().numpy().reshape(4, ng, n * n)
    expect = before.copy()
    expect[:, :, strip] = planted.reshape(ng, 4, 4 * n).transpose(1, 0, 2)
    assert np.array_equal(g, expect)
    r.close()


def test_whole_record_halo_calls(ag):
    """amrgpu_session_halo_pack / _unpack keep the whole-patch format
    (4 fields x n*n per quad)."""
    from amrgpu import shard as S
    from amrgpu._lib import lib
    import torch
    m, cfg, s0 = build(ag, 41, 8, 3)
    sh = S.make_shard(m, S.partition(m.ncell, 2), 1)
    r = S.GpuRank(sh, cfg)
    loc = sh.local_state(s0)
    r.upload(loc)
    n = m.n
    rec = 4 * n * n
    ns, ng = len(sh.send_quads), len(sh.ghosts)
    buf = torch.zeros(max(ns, ng) * rec, dtype=torch.float64, device=r.device)
    assert lib().amrgpu_session_halo_pack(r.session._s, 0, ns, buf.data_ptr()) == 0
    r.stream.synchronize()
    want = loc.reshape(-1, n * n, 4)[sh.send_quads].transpose(0, 2, 1).reshape(-1)
    assert np.array_equal(buf[: len(want)].cpu().numpy(), want)
    planted = torch.arange(ng * rec, dtype=torch.float64, device=r.device)
    assert lib().amrgpu_session_halo_unpack(r.session._s, 0, ng, planted.data_ptr()) == 0
    r.stream.synchronize()
    g = _stage_input(r)[:, sh.nlocal * n * n:(sh.nlocal + ng) * n * n].cpu().numpy()
    got = g.reshape(4, ng, n * n).transpose(1, 0, 2).reshape(-1)
    assert np.array_equal(got, planted.cpu().numpy())
    r.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_distributed_driver_over_nccl_single_rank(ag):
    """The per-process driver on a one-rank NCCL group: the CFL-step MIN
    runs in place on the session's device scalars through torch.distributed
    on the session stream; the result equals the plain session's."""
    import torch
    import torch.distributed as dist
    from amrgpu import shard as S
    m, cfg, s0 = build(ag, 60, 16, 3)
    ref, rep0 = unsharded(ag, m, cfg, s0, ag.FORM_FP32_FLUX, 10)
    cfg["form"] = ag.FORM_FP32_FLUX
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        r = S.GpuRank(S.make_shard(m, S.partition(m.ncell, 1), 0), cfg)
        drv = S.Distributed(r)
        drv.start(r.shard.local_state(s0))
        drv.step(10)
        rep = drv.report()
        got = drv.download()
        r.close()
    finally:
        dist.destroy_process_group()
    assert np.array_equal(got, ref)
    assert rep["time"] == rep0["time"] and rep["steps"] == 10


def test_distributed_step_graphs_single_rank(ag):
    """The per-process driver's steps captured as CUDA graphs (one per step
    phase, the CFL-step MIN all-reduce inside) on a one-rank NCCL group:
    after two eager steps, eight graph replays give the plain session's
    state and time bit for bit, and the session's counters follow."""
    import torch
    import torch.distributed as dist
    from amrgpu import shard as S
    m, cfg, s0 = build(ag, 61, 16, 3)
    ref, rep0 = unsharded(ag, m, cfg, s0, ag.FORM_FP32_FLUX, 10)
    cfg["form"] = ag.FORM_FP32_FLUX
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        r = S.GpuRank(S.make_shard(m, S.partition(m.ncell, 1), 0), cfg)
        drv = S.Distributed(r)
        drv.start(r.shard.local_state(s0))
        drv.step(2)
        assert drv.capture()
        drv.step_graphs(8)
        rep = drv.report()
        got = drv.download()
        step_index = ag.lib().amrgpu_session_step_index(r.session._s)
        drv.release_graphs()
        r.close()
    finally:
        dist.destroy_process_group()
    assert step_index == 10
    assert np.array_equal(got, ref)
    assert rep["time"] == rep0["time"] and rep["steps"] == 10
