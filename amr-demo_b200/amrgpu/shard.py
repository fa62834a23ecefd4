"""Sharded meshes: one device session per rank, ghost quads refreshed before
every RK stage, the CFL step reduced across ranks before every step.

The reference runs one MPI rank per p4est partition. Its per-rank mesh
arrays hold the rank's local quads followed by its ghost quads, "stacked in
order of processor" (src/physics/src/physics_mpi.c:54); before every call of
physics_rhs the ghosts are refreshed from their owners
(physics_mpi_real_to_ghost, rk_time_integrators.c:227,243,259 for RK3), the
time step is the MPI_MIN of the ranks' CFL steps
(physics_runge_kutta_interface.c:96,149,205,262,316) and the residual norm is
the MPI_SUM of the ranks' sums of squares (rk_time_integrators.c:74,162,274).

Here:

* :func:`partition` splits the forest's quads (Morton order) into contiguous
  ranges, as p4est_partition does with uniform weights.
* :func:`make_shard` builds one rank's mesh: local quads, then ghost quads in
  ascending global order (which groups them by owner), the faces that touch
  a local quad in their global order (the order the stage kernels accumulate
  a quad's faces in), and the send and receive lists.
* :class:`GpuRank` runs one rank's stages on the device through the C ABI
  (amrgpu_session_step_stage, _halo_pack, _halo_unpack, _dt_slot).
* :class:`Distributed` drives one rank per process over torch.distributed
  (NCCL on GPUs; any backend whose tensors match the rank's buffers).
  :class:`LocalCluster` drives several ranks in one process and moves the
  ghost records with device copies; it is the single-GPU check of the
  sharded arithmetic.

The sharded run is bit-identical to the unsharded one: every quad's
residual reads the same neighbour values in the same face order, and the
step size is the exact minimum over all cells either way.
"""
import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import Mesh, NFIELDS, Session
from ._lib import check, lib

RECORD_FIELDS = NFIELDS


# --------------------------------------------------------------------- partition
def partition(nquad, nranks):
    """offsets[r] .. offsets[r+1]-1 are rank r's quads (equal counts +-1)."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    r = np.arange(nranks + 1, dtype=np.int64)
    return (r * int(nquad)) // nranks


def owners(offsets, quads):
    return np.searchsorted(offsets, quads, side="right") - 1


def _participants(mesh):
    """(nface, 3) quads of each face (-1 where none): the full or only quad,
    then its one (full face) or two (hanging face) neighbours."""
    fi = mesh.face_info.reshape(-1, 11)[: mesh.nface]
    t = fi[:, 0]
    if np.any((t < 1) | (t > 3)):
        raise ValueError("sharding supports boundary, full and hanging 2D faces (types 1-3)")
    P = np.full((len(fi), 3), -1, np.int64)
    P[:, 0] = fi[:, 2]
    P[t >= 2, 1] = fi[t >= 2, 3]
    P[t == 3, 2] = fi[t == 3, 4]
    return fi, P


@dataclass
class Shard:
    rank: int
    nranks: int
    offsets: np.ndarray          # quad ranges of all ranks
    mesh: Mesh                   # local quads, then ghost quads
    ghosts: np.ndarray           # global ids of the ghost quads, ascending
    recv: list = field(default_factory=list)   # (peer, first ghost, count), ascending peer
    send: list = field(default_factory=list)   # (peer, first entry, count), ascending peer
    send_quads: np.ndarray = None              # local ids of the send entries

    @property
    def lo(self):
        return int(self.offsets[self.rank])

    @property
    def nlocal(self):
        return int(self.offsets[self.rank + 1] - self.offsets[self.rank])

    @property
    def record(self):
        """Doubles of one quad's whole patch (4 fields x n*n)."""
        return RECORD_FIELDS * self.mesh.n * self.mesh.n

    @property
    def halo_record(self):
        """Doubles of one ghost quad on the wire: its four one-cell edge
        strips per field (16*n), the only cells the stage kernels read of a
        ghost (amrgpu_session_halo_pack_edges)."""
        return RECORD_FIELDS * 4 * self.mesh.n

    def local_state(self, global_aos):
        """This rank's AoS input: its quads, then its ghosts."""
        rec = self.record
        g = np.asarray(global_aos, np.float64).reshape(-1, rec)
        ids = np.concatenate([np.arange(self.lo, self.lo + self.nlocal), self.ghosts])
        return np.ascontiguousarray(g[ids].reshape(-1))

    def reference_lists(self):
        """send / recv as the reference's flat (cell, rank) pairs
        (physics_mpi.c:61-63,82-83): send cells are local ids, recv cells
        are ghost ids counted from ncell."""
        send = []
        for peer, first, count in self.send:
            for q in self.send_quads[first:first + count]:
                send += [int(q), peer]
        recv = []
        for peer, first, count in self.recv:
            for g in range(first, first + count):
                recv += [self.nlocal + g, peer]
        return np.asarray(send, np.int32), np.asarray(recv, np.int32)


def make_shard(mesh, offsets, rank):
    """Rank ``rank``'s piece of the global mesh ``mesh`` under ``offsets``."""
    offsets = np.asarray(offsets, np.int64)
    nranks = len(offsets) - 1
    if offsets[0] != 0 or offsets[-1] != mesh.ncell or np.any(np.diff(offsets) < 0):
        raise ValueError("offsets must rise from 0 to the mesh's quad count")
    lo, hi = int(offsets[rank]), int(offsets[rank + 1])
    n = mesh.n
    fi, P = _participants(mesh)
    valid = P >= 0
    mine = valid & (P >= lo) & (P < hi)
    keep = mine.any(axis=1)
    ghosts = np.unique(P[keep][valid[keep] & ~mine[keep]])

    # send lists: my quads that share a face with quads of other ranks
    own = np.where(valid, owners(offsets, np.where(valid, P, 0)), -1)
    pairs = []
    for a in range(3):
        for b in range(3):
            if a == b:
                continue
            m = valid[:, a] & valid[:, b] & (own[:, a] == rank) & (own[:, b] != rank)
            if np.any(m):
                pairs.append(np.stack([own[m, b], P[m, a]], axis=1))
    if pairs:
        sp = np.unique(np.concatenate(pairs), axis=0)  # sorted by peer, then quad
    else:
        sp = np.zeros((0, 2), np.int64)
    send, start = [], 0
    for peer in np.unique(sp[:, 0]):
        cnt = int(np.count_nonzero(sp[:, 0] == peer))
        send.append((int(peer), start, cnt))
        start += cnt
    send_quads = (sp[:, 1] - lo).astype(np.int32)

    recv = []
    if len(ghosts):
        gown = owners(offsets, ghosts)
        for peer in np.unique(gown):
            idx = np.nonzero(gown == peer)[0]
            recv.append((int(peer), int(idx[0]), int(len(idx))))

    # local numbering: locals 0..nlocal-1, ghosts after them
    nloc = hi - lo
    lut = np.full(mesh.ncell, -1, np.int64)
    lut[lo:hi] = np.arange(nloc)
    lut[ghosts] = nloc + np.arange(len(ghosts))
    lf = fi[keep].copy()
    for k in range(2, 7):
        col = lf[:, k]
        sel = col >= 0
        col[sel] = lut[col[sel]]
    glob = np.concatenate([np.arange(lo, hi), ghosts]).astype(np.int64)
    ci = mesh.cell_info.reshape(-1, 3)[glob].copy()
    ci[:, 2] = RECORD_FIELDS * n * n * np.arange(len(glob))
    geom = mesh.geom.reshape(-1, 12)[glob].copy()
    lm = Mesh(n, ci.reshape(-1), lf.reshape(-1), geom.reshape(-1), int(keep.sum()),
              RECORD_FIELDS * n * n * nloc, nghost=len(ghosts))
    return Shard(rank, nranks, offsets, lm, ghosts.astype(np.int64), recv, send, send_quads)


# --------------------------------------------------------------------- one rank on the device
class _DeviceView:
    """__cuda_array_interface__ of a library-owned device buffer, so that
    torch (and NCCL through it) can read and write it in place."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 2}


class GpuRank:
    """One rank: a device session of the shard's mesh plus its halo buffers.

    Stage protocol (all work on the session's stream): ``pack`` the send
    records of the next stage's input, move them (the driver), ``unpack``
    them into the ghost quads, ``stage`` runs the stage kernel; after a
    step's last stage the driver reduces ``dt_view`` (MIN) across ranks.
    """

    def __init__(self, shard, config=None, form=None):
        import torch
        self.torch = torch
        self.shard = shard
        self.session = Session(shard.mesh, config, form)
        sq = np.ascontiguousarray(shard.send_quads, np.int32)
        check(lib().amrgpu_session_set_halo(self.session._s, sq.ctypes.data_as(C.POINTER(C.c_int)), len(sq)),
              "set_halo")
        self.device = torch.device("cuda", torch.cuda.current_device())
        rec = shard.halo_record
        self.sendbuf = torch.empty(max(len(sq), 1) * rec, dtype=torch.float64, device=self.device)
        self.recvbuf = torch.empty(max(len(shard.ghosts), 1) * rec, dtype=torch.float64, device=self.device)
        self.stream = torch.cuda.ExternalStream(self.session.stream(), device=self.device)
        self.stages_per_step = None
        self._dt_views = {}

    # -- data
    def upload(self, local_aos):
        self.session.upload(local_aos)

    def download(self, out=None):
        return self.session.download(out)

    # -- stage protocol
    def pack(self):
        nsend = len(self.shard.send_quads)
        if nsend:
            check(lib().amrgpu_session_halo_pack_edges(self.session._s, 0, nsend, self.sendbuf.data_ptr()),
                  "halo_pack")

    def unpack(self):
        ng = len(self.shard.ghosts)
        if ng:
            check(lib().amrgpu_session_halo_unpack_edges(self.session._s, 0, ng, self.recvbuf.data_ptr()),
                  "halo_unpack")

    def stage(self):
        """Runs the next stage; True when it was the step's last."""
        st, per = C.c_int(0), C.c_int(0)
        check(lib().amrgpu_session_step_stage(self.session._s, C.byref(st), C.byref(per)), "step_stage")
        self.stages_per_step = per.value
        return st.value == per.value

    def dt_view(self):
        """int64 tensor (1,) aliasing the next step's CFL step image."""
        ptr = lib().amrgpu_session_dt_slot(self.session._s)
        v = self._dt_views.get(ptr)
        if v is None:
            v = self.torch.as_tensor(_DeviceView(ptr, (1,), "<i8"), device=self.device)
            self._dt_views[ptr] = v
        return v

    def report(self):
        r = self.session.sync()
        ns, fl = C.c_double(0.0), C.c_int(0)
        check(lib().amrgpu_session_local_scalars(self.session._s, C.byref(ns), C.byref(fl)), "local_scalars")
        r["norm_sq"] = ns.value
        r["flags"] = fl.value
        return r

    def close(self):
        self.session.close()


def _combine_reports(reps, norm_sq, flags):
    r = dict(reps[0]) if isinstance(reps, list) else dict(reps)
    r["residual_norm"] = float(np.sqrt(norm_sq))
    r["norm_sq"] = float(norm_sq)
    r["flags"] = int(flags)
    r["nan"] = 1 if flags & 1 else 0
    r["error"] = 4 if flags & 1 else (5 if flags & 2 else 0)
    return r


# --------------------------------------------------------------------- drivers
class Distributed:
    """One rank of a multi-process run over torch.distributed.

    ``rank_obj`` is a :class:`GpuRank` (or any object with its stage
    protocol and tensors on the process group's device). Every rank issues
    the same collectives in the same order: per stage one all-to-all of
    ghost records (non-zero only between face neighbours), per step one MIN
    all-reduce of the CFL step image, per report two all-reduces."""

    def __init__(self, rank_obj, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.r = rank_obj
        self.group = group
        self.nranks = dist.get_world_size(group)
        if self.nranks != rank_obj.shard.nranks:
            raise ValueError("the shard's partition and the process group differ in size")

    def _plan(self):
        """The per-stage exchange as one all-to-all, built once: send records
        are grouped by destination rank and ghosts by owner, both ascending,
        so the buffers are already in rank order; ranks that share no face
        get zero-length slices."""
        plan = getattr(self, "_a2a", None)
        if plan is None:
            r = self.r
            rec = r.shard.halo_record
            out_split = [0] * self.nranks
            in_split = [0] * self.nranks
            for peer, _, count in r.shard.send:
                in_split[peer] = count * rec
            for peer, _, count in r.shard.recv:
                out_split[peer] = count * rec
            nin, nout = sum(in_split), sum(out_split)
            plan = (r.sendbuf[:nin], r.recvbuf[:nout], in_split, out_split)
            self._a2a = plan
        return plan

    def _exchange(self):
        # a collective: every rank calls it, also one with nothing to send
        if self.nranks < 2:
            return
        send, recv, in_split, out_split = self._plan()
        self.dist.all_to_all_single(recv, send, output_split_sizes=out_split, input_split_sizes=in_split,
                                    group=self.group)

    def _in_stream(self, fn):
        s = getattr(self.r, "stream", None)
        if s is None:
            return fn()
        import torch
        with torch.cuda.stream(s):
            return fn()

    def start(self, local_aos):
        self.r.upload(local_aos)
        self._in_stream(self._reduce_dt)

    def _reduce_dt(self):
        self.dist.all_reduce(self.r.dt_view(), op=self.dist.ReduceOp.MIN, group=self.group)

    def _step(self):
        while True:
            self.r.pack()
            self._exchange()
            self.r.unpack()
            if self.r.stage():
                break
        self._reduce_dt()

    def step(self, nsteps):
        def run():
            for _ in range(int(nsteps)):
                self._step()
        self._in_stream(run)

    # -- steps as CUDA graphs ---------------------------------------------
    # A step's host work -- per stage a pack, the NCCL all-to-all, an unpack
    # and the stage launch, then the MIN all-reduce of the CFL step -- costs
    # more host time than the step's kernels on a 1024^2 shard. Captured
    # once as a CUDA graph per step phase (the device addresses a step uses
    # repeat every 6 steps: three CFL slots, two buffer-role parities), a
    # step is one graph launch. The session's counters are saved before the
    # captures and restored after them (the captured work has not run), and
    # advanced by one step per replay.
    def capture(self):
        """Captures the six step graphs; needs a GPU rank whose first steps
        ran eagerly (communicators set up, launch tuned). Returns False,
        leaving the driver eager, when the capture is refused."""
        import torch
        r = self.r
        sess = getattr(r, "session", None)
        if sess is None or getattr(r, "stream", None) is None:
            return False
        L = lib()
        check(L.amrgpu_session_capture_mark(sess._s), "capture_mark")
        graphs = {}
        try:
            base = int(L.amrgpu_session_step_index(sess._s))
            for k in range(6):
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=r.stream):
                    self._step()
                graphs[(base + k) % 6] = g
        except Exception:
            graphs = None
        check(L.amrgpu_session_capture_rewind(sess._s), "capture_rewind")
        self._graphs = graphs
        return graphs is not None

    def release_graphs(self):
        """Drops the step graphs (they hold the NCCL collectives: release
        them before the process group is destroyed)."""
        self._graphs = None

    def step_graphs(self, nsteps):
        """nsteps steps, each as one replay of its phase's graph on the
        session's stream (a replay runs on the current stream)."""
        r = self.r
        L = lib()

        def run():
            for _ in range(int(nsteps)):
                k = int(L.amrgpu_session_step_index(r.session._s)) % 6
                self._graphs[k].replay()
                check(L.amrgpu_session_advance(r.session._s, 1), "advance")
        self._in_stream(run)

    def report(self):
        import torch
        rep = self.r.report()
        dev = getattr(self.r, "device", torch.device("cpu"))
        t = torch.tensor([rep["norm_sq"]], dtype=torch.float64, device=dev)
        f = torch.tensor([rep["flags"] & 1, (rep["flags"] >> 1) & 1, (rep["flags"] >> 2) & 1],
                         dtype=torch.int32, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        self.dist.all_reduce(f, op=self.dist.ReduceOp.MAX, group=self.group)
        fl = [int(v) for v in f.cpu().tolist()]
        return _combine_reports(rep, float(t.cpu().item()), fl[0] | (fl[1] << 1) | (fl[2] << 2))

    def download(self, out=None):
        return self.r.download(out)


class LocalCluster:
    """Several ranks in one process on one device: the ghost records move
    by device copies between the ranks' buffers, in the same stage order as
    :class:`Distributed`. No rank's kernels wait on another's."""

    def __init__(self, ranks):
        self.ranks = list(ranks)
        by = {r.shard.rank: r for r in self.ranks}
        self.by_rank = by
        # for each receiving (rank, peer): the sender's entry range
        self.routes = []
        for r in self.ranks:
            for peer, gfirst, gcount in r.shard.recv:
                src = by[peer]
                sfirst, scount = next((f, c) for p, f, c in src.shard.send if p == r.shard.rank)
                if scount != gcount:
                    raise RuntimeError("send and receive lists disagree")
                self.routes.append((r, gfirst, src, sfirst, gcount))

    def _sync_streams(self):
        for r in self.ranks:
            if getattr(r, "stream", None) is not None:
                r.stream.synchronize()

    def start(self, global_aos):
        for r in self.ranks:
            r.upload(r.shard.local_state(global_aos))
        self._reduce_dt()

    def _reduce_dt(self):
        if len(self.ranks) < 2:
            return
        self._sync_streams()
        views = [r.dt_view() for r in self.ranks]
        m = views[0].clone()
        for v in views[1:]:
            m = self._min(m, v.to(m.device))
        for v in views:
            v.copy_(m)
        self._sync_device()

    @staticmethod
    def _min(a, b):
        import torch
        return torch.minimum(a, b)

    def step(self, nsteps):
        for _ in range(int(nsteps)):
            done = False
            while not done:
                for r in self.ranks:
                    r.pack()
                self._sync_streams()
                for dst, gfirst, src, sfirst, cnt in self.routes:
                    rec = dst.shard.halo_record
                    dst.recvbuf[gfirst * rec:(gfirst + cnt) * rec].copy_(src.sendbuf[sfirst * rec:(sfirst + cnt) * rec])
                self._sync_device()
                ends = []
                for r in self.ranks:
                    r.unpack()
                    ends.append(r.stage())
                if len(set(ends)) != 1:
                    raise RuntimeError("ranks disagree on the stage count")
                done = ends[0]
            self._reduce_dt()

    def _sync_device(self):
        import torch
        if any(getattr(r, "stream", None) is not None for r in self.ranks):
            torch.cuda.current_stream().synchronize()

    def report(self):
        reps = [r.report() for r in self.ranks]
        ns = sum(rp["norm_sq"] for rp in reps)
        fl = 0
        for rp in reps:
            fl |= rp["flags"]
        return _combine_reports(reps, ns, fl)

    def download(self):
        """Global AoS state: the ranks' local quads in rank order."""
        return np.concatenate([r.download() for r in sorted(self.ranks, key=lambda x: x.shard.rank)])
