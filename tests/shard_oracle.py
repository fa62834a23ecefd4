"""One rank of a sharded run computed by the CPU oracle -- TEST
INFRASTRUCTURE for the sharded drivers of amrgpu.shard.

It follows amrgpu.shard.GpuRank's stage protocol (pack, unpack, stage,
dt_view, report) with the oracle's arithmetic: each stage is one oracle_rhs
of the current stage input on the rank's ghosted mesh (ghosts at indices
>= dof, read but never written, physics_rhs_structured.c:158-221) followed
by the stage update of physics2d.c's oracle_evolve in the same expression
order, so that a sharded oracle run must reproduce the unsharded
oracle_evolve bit for bit."""

import numpy as np
import torch

from oracle import oracle as O

# LSERK(4,5) coefficients of rk_time_integrators.c (lserk_45), as oracle_evolve
_RA = [0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
       -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0]
_RB = [1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
       1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
       2277821191437.0 / 14882151754819.0]
_STAGES = {1: 1, 2: 2, 3: 3, 4: 4, 5: 5}


def _bits(x):
    return int(np.float64(x).view(np.int64))


def _double(b):
    return float(np.int64(b).view(np.float64))


class OracleRank:
    device = torch.device("cpu")

    def __init__(self, shard, cfg):
        self.shard = shard
        self.mesh = shard.mesh
        self.n = shard.mesh.n
        self.oc = O.make_config(self.n, cfg)
        self.scheme = int(cfg["time_scheme"])
        self.stages_per_step = _STAGES[self.scheme]
        rec = shard.halo_record
        self.sendbuf = torch.zeros(max(len(shard.send_quads), 1) * rec, dtype=torch.float64)
        self.recvbuf = torch.zeros(max(len(shard.ghosts), 1) * rec, dtype=torch.float64)
        n = self.n
        # cells of the edge-strip format: sides 0..3 (column 0, column n-1,
        # row 0, row n-1), n cells each, as amrgpu_session_halo_pack_edges
        self.strip = np.array([p * n if s == 0 else p * n + n - 1 if s == 1 else p if s == 2 else (n - 1) * n + p
                               for s in range(4) for p in range(n)], np.int64)
        self.dt = torch.zeros(1, dtype=torch.int64)
        self.time = 0.0
        self.steps = 0
        self.norm_sq = 0.0
        self.dt_last = 0.0
        self.st = 0

    # -- data
    def _cfl(self):
        if self.scheme == 2:
            return self.oc.dt
        return O.time_step(self.mesh, self.Q, self.oc)

    def upload(self, local_aos):
        self.Q = np.array(local_aos, np.float64)
        self.dt[0] = _bits(self._cfl())
        self.st = 0

    def download(self, out=None):
        if out is None:
            return self.Q[: self.mesh.dof].copy()
        out[: self.mesh.dof] = self.Q[: self.mesh.dof]
        return out

    # -- stage protocol
    def pack(self):
        rec = self.shard.record
        if len(self.shard.send_quads):
            # per quad and field the strip cells (AoS: cell c field f at 4c + f)
            blocks = self.Q.reshape(-1, rec)[self.shard.send_quads].reshape(len(self.shard.send_quads), -1, 4)
            strips = blocks[:, self.strip, :].transpose(0, 2, 1)
            self.sendbuf[: strips.size] = torch.from_numpy(np.ascontiguousarray(strips).reshape(-1))

    def unpack(self):
        rec = self.shard.record
        ng = len(self.shard.ghosts)
        if ng:
            nl = self.shard.nlocal
            ghosts = self.Q[nl * rec:(nl + ng) * rec].reshape(ng, -1, 4)
            strips = self.recvbuf[: ng * self.shard.halo_record].numpy().reshape(ng, 4, -1)
            ghosts[:, self.strip, :] = strips.transpose(0, 2, 1)

    def _rhs(self):
        return O.rhs(self.mesh, self.Q, self.oc)

    def _norm(self, k):
        L = O.restatement()
        return L.oracle_norm(self.n, self.mesh.ncell, O.ip(self.mesh.cell_info), O.dp(np.ascontiguousarray(k)))

    def stage(self):
        dof = self.mesh.dof
        Q = self.Q
        if self.st == 0:
            dt = _double(int(self.dt[0]))
            if self.oc.final_time > 0.0:
                rem = self.oc.final_time - self.time
                if rem < dt:
                    dt = rem
                if dt < 0.0:
                    dt = 0.0
            self._dt = dt
            self.Qs = Q[:dof].copy()
            self.k = []
        dt, sc, st = self._dt, self.scheme, self.st
        k = self._rhs()
        self.k.append(k)
        Qs, K = self.Qs, self.k
        last = st + 1 == self.stages_per_step
        if sc == 1:
            Q[:dof] = Q[:dof] + (1.0 * dt) * k
        elif sc == 2:
            if st == 0:
                Q[:dof] = Qs + (1.0 * dt) * k
            else:
                Q[:dof] = Qs + (0.5 * dt) * K[0] + (0.5 * dt) * K[1]
        elif sc == 3:
            if st == 0:
                Q[:dof] = Qs + (1.00 * dt) * k
            elif st == 1:
                Q[:dof] = Qs + (0.25 * dt) * K[0] + (0.25 * dt) * K[1]
            else:
                Q[:dof] = Qs + (1.0 / 6.0 * dt) * K[0] + (1.0 / 6.0 * dt) * K[1] + (2.0 / 3.0 * dt) * K[2]
        elif sc == 4:
            if st < 3:
                a = [0.5 * dt, 0.5 * dt, 1.0 * dt][st]
                Q[:dof] = Qs + a * k
            else:
                Q[:dof] = Qs + (1.0 / 6.0 * dt) * (K[0] + 2.0 * K[1] + 2.0 * K[2] + K[3])
        elif sc == 5:
            if st == 0:
                self.S = dt * k
            else:
                self.S = self.S * _RA[st] + dt * k
            Q[:dof] = Q[:dof] + _RB[st] * self.S
        if last:
            self.norm_sq = self._norm(k)
            self.time = self.time + dt
            self.dt_last = dt
            if dt > 0.0:
                self.steps += 1
            self.dt[0] = _bits(self._cfl())
            self.st = 0
        else:
            self.st += 1
        return last

    def dt_view(self):
        return self.dt

    def report(self):
        return {"steps": self.steps, "time": self.time, "dt_last": self.dt_last,
                "residual_norm": float(np.sqrt(self.norm_sq)), "error": 0, "nan": 0,
                "norm_sq": self.norm_sq, "flags": 0 if np.isfinite(self.Q).all() else 1}

    def close(self):
        pass
