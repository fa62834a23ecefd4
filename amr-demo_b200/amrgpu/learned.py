"""Learned refinement indicator (no reference counterpart).

A 400-128-64-3 MLP (GELU) maps a quad's normalised patch (8x8 cells plus a
one-cell neighbour ring, 4 conserved fields) to coarsen / refine / keep, in
place of the plain tagger (solver_tag_feature.F90:9-52 behind
hpc_amr_tag_feature, amr_external.h:92). Training, inference and the
features all run on the GPU (csrc/mlp.cu: BF16 tcgen05 GEMMs with FP32
accumulation, AdamW on FP32 master weights); this module drives them:

  * dataset: (features, plain label) pairs collected from seeded AMR runs
    of the isentropic-vortex family, labelled by the plain three-class
    indicator (J = largest relative density jump; refine J >= tol, coarsen
    J < lo_frac*tol, keep otherwise), optionally looking ahead to the state
    at the next regrid;
  * training: AdamW, cross-entropy, shuffled batches;
  * AMR loop: the learned classes drive refine / coarsen; every regrid the
    plain indicator re-scores a sampled fraction of the quads (the judge)
    and the run falls back to the plain indicator for good once the
    disagreement exceeds the bound.
"""
import ctypes as C
import math
import time

import numpy as np

from . import Config, Forest, Session
from ._lib import JudgeStruct, check, lib

COARSEN, REFINE, KEEP = 0, 1, 2
NPARAMS = 59779
NIN = 400


def _u16(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint16))


def _f32(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _i32(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _f64(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Mlp:
    """amrgpu_mlp_t: parameters, optimiser state and device dataset."""

    def __init__(self, seed=0):
        h = C.c_void_p()
        check(lib().amrgpu_mlp_create(C.byref(h), C.c_ulonglong(seed)), "mlp_create")
        self._m = h

    def close(self):
        if getattr(self, "_m", None):
            try:
                lib().amrgpu_mlp_destroy(self._m)
            except Exception:
                pass
            self._m = None

    def __del__(self):
        self.close()

    # parameters ---------------------------------------------------------
    def get_params(self):
        p = np.zeros(NPARAMS, np.float32)
        check(lib().amrgpu_mlp_get_params(self._m, _f32(p)), "mlp_get_params")
        return p

    def set_params(self, p):
        a = np.ascontiguousarray(p, np.float32)
        assert a.size == NPARAMS
        check(lib().amrgpu_mlp_set_params(self._m, _f32(a)), "mlp_set_params")

    # dataset ------------------------------------------------------------
    def append(self, session, tol, lo_frac=0.25):
        n = lib().amrgpu_mlp_dataset_append(self._m, session._s, float(tol), float(lo_frac))
        if n < 0:
            check(int(n), "mlp_dataset_append")
        return int(n)

    def relabel(self, session, first, tol, lo_frac=0.25):
        check(lib().amrgpu_mlp_dataset_relabel(self._m, session._s, int(first), float(tol), float(lo_frac)),
              "mlp_dataset_relabel")

    def cover(self, session, first, tol, lo_frac=0.25):
        """Merges the plain classes of the session's current state into the
        labels of rows [first, first + nquad), keeping the finer demand."""
        check(lib().amrgpu_mlp_dataset_cover(self._m, session._s, int(first), float(tol), float(lo_frac)),
              "mlp_dataset_cover")

    def size(self):
        return int(lib().amrgpu_mlp_dataset_size(self._m))

    def clear(self):
        check(lib().amrgpu_mlp_dataset_clear(self._m), "mlp_dataset_clear")

    def labels(self, n=None):
        n = self.size() if n is None else n
        y = np.zeros(n, np.int32)
        check(lib().amrgpu_mlp_dataset_labels(self._m, _i32(y), n), "mlp_dataset_labels")
        return y

    # training / inference ----------------------------------------------
    def train_epoch(self, perm, batch=8192, lr=1e-3, weight_decay=1e-2):
        p = np.ascontiguousarray(perm, np.int32)
        loss, acc = C.c_double(0.0), C.c_double(0.0)
        check(lib().amrgpu_mlp_train_epoch(self._m, _i32(p), p.size, int(batch), float(lr), float(weight_decay),
                                           C.byref(loss), C.byref(acc)), "mlp_train_epoch")
        return loss.value, acc.value

    def grad(self, x_bits, y):
        x = np.ascontiguousarray(x_bits, np.uint16)
        yy = np.ascontiguousarray(y, np.int32)
        B = yy.size
        logits = np.zeros((B, 3), np.float32)
        g = np.zeros(NPARAMS, np.float32)
        loss = C.c_double(0.0)
        check(lib().amrgpu_mlp_grad(self._m, _u16(x), _i32(yy), B, _f32(logits), _f32(g), C.byref(loss)), "mlp_grad")
        return logits, g, loss.value

    def predict(self, x_bits):
        x = np.ascontiguousarray(x_bits, np.uint16)
        B = x.size // NIN
        logits = np.zeros((B, 3), np.float32)
        check(lib().amrgpu_mlp_predict(self._m, _u16(x), B, _f32(logits)), "mlp_predict")
        return logits

    def tags(self, session, tol, lo_frac=0.25, judge_fraction=0.05, seed=0):
        t = np.zeros(session.mesh.ncell, np.int32)
        j = JudgeStruct()
        check(lib().amrgpu_session_learned_tags(session._s, self._m, float(judge_fraction), C.c_ulonglong(seed),
                                                float(tol), float(lo_frac), _i32(t), C.byref(j)),
              "session_learned_tags")
        return t, {"judged": j.judged, "disagree": j.disagree, "rate": j.rate, "coarser": j.coarser}


def session_features(session):
    """Features of every quad of a session: (nquad, 400) BF16 bit patterns."""
    x = np.zeros((session.mesh.ncell, NIN), np.uint16)
    check(lib().amrgpu_session_features(session._s, _u16(x)), "session_features")
    return x


def session_jumps(session):
    j = np.zeros(session.mesh.ncell, np.float64)
    check(lib().amrgpu_session_jumps(session._s, _f64(j)), "session_jumps")
    return j


def plain_classes(jumps, tol, lo_frac=0.25):
    """The plain three-class indicator from the jumps (as label_kernel)."""
    j = np.asarray(jumps)
    return np.where(j >= tol, REFINE, np.where(j < lo_frac * tol, COARSEN, KEEP)).astype(np.int32)


def bf16_to_f32(bits):
    return (np.asarray(bits, np.uint32) << 16).view(np.float32)


# ------------------------------------------------------------------ AMR loop
def regrid_by_classes(forest, session, n, classes, min_level, max_level):
    """Regrid with indicator classes: refine class-1 quads below max_level,
    coarsen complete families whose children are all class 0 above
    min_level (a refined child inherits its parent's refine tag), 2:1
    balance, remap in place (one Session.adapt_regrid call: on the device
    too when the session's last regrid came from this forest)."""
    session.adapt_regrid(forest, min_level, max_level, tags=classes, refine_value=REFINE, coarsen_value=COARSEN)


def vortex_amr(seed=0, n=8, min_level=3, max_level=6, tol=0.02, lo_frac=0.25, form=1, beta=None, center=None):
    """Isentropic vortex on the periodic square [0,10]^2 under AMR: free
    stream (rho,u,v,p) = (1,1,1,1), vortex centre and strength from the seed
    (centre ~ U[3.5,6.5]^2, beta ~ U[3,6]) unless given, SSP-RK3, CFL 0.5;
    start-up refinement by the plain indicator. Returns (forest, config,
    state, (centre x, centre y, beta))."""
    rng = np.random.default_rng(10007 + seed)
    cx, cy = center if center is not None else rng.uniform(3.5, 6.5, 2)
    b = beta if beta is not None else rng.uniform(3.0, 6.0)
    mach = math.sqrt(2.0) / math.sqrt(1.4)
    cfg = Config.from_input(cfl=0.5, time_scheme=3, nelem_subgrid=n, coarse_grid_h=10.0, initial_condition=4,
                            time_steps=10 ** 9, dt=1.0, bc=[1] * 6, gamma=1.4, density=1.0, pressure=1.0,
                            mach=mach, alpha=45.0, beta=0.0, ic_params=[cx, cy, b, 0.5], form=form)
    cfg.apply()
    f = Forest(1, 1, periodic=(1, 1), lo=(0.0, 0.0, 0.0), scale=10.0, level=min_level)
    for _ in range(max_level - min_level + 1):
        soln = f.initialize(n)
        s = Session(f.mesh(n), cfg, form=form)
        s.upload(soln)
        cls = plain_classes(session_jumps(s), tol, lo_frac)
        s.close()
        _, lev, _, _ = f.quads()
        flags = ((cls == REFINE) & (lev < max_level)).astype(np.int32)
        if not flags.any():
            break
        f.refine(flags, max_level=max_level)
        f.balance()
    return f, cfg, f.initialize(n), (float(cx), float(cy), float(b))


def collect(mlp, seeds, n=8, min_level=3, max_level=6, tol=0.02, lo_frac=0.25, regrid_interval=5, regrids=20,
            lookahead=True, cover_every=0):
    """Runs the seeded vortex family under the plain indicator and appends
    every quad of every regrid to the model's dataset; with `lookahead` a
    row's label is the plain class of the same quad at the next regrid
    (what the indicator will ask for by then), else at the same time. With
    cover_every = k > 0 a row's label covers the whole interval instead:
    the finest of the plain classes now and every k steps until the next
    regrid (refine if any asks for it, coarsen only if all do) -- what a
    plain indicator regridding every k steps would ask of the quad over the
    interval."""
    for seed in seeds:
        f, cfg, soln, _ = vortex_amr(seed, n, min_level, max_level, tol, lo_frac)
        s = Session(f.mesh(n), cfg, form=1)
        s.upload(soln)
        for _ in range(regrids):
            start = mlp.size()
            mlp.append(s, tol, lo_frac)
            if cover_every > 0:
                done = 0
                while done < regrid_interval:
                    k = min(cover_every, regrid_interval - done)
                    s.step(k)
                    s.sync()
                    mlp.cover(s, start, tol, lo_frac)
                    done += k
            else:
                s.step(regrid_interval)
                s.sync()
                if lookahead:
                    mlp.relabel(s, start, tol, lo_frac)
            cls = plain_classes(session_jumps(s), tol, lo_frac)
            regrid_by_classes(f, s, n, cls, min_level, max_level)
        s.close()
    return mlp.size()


def train(mlp, epochs=3, batch=8192, lr=1e-3, weight_decay=1e-2, seed=0, holdout=0.1):
    """AdamW over the device dataset; returns per-epoch (loss, accuracy) on
    the training rows and the held-out accuracy (by the prediction of the
    trained model on the last `holdout` fraction, kept out of training)."""
    n = mlp.size()
    rng = np.random.default_rng(seed)
    order = rng.permutation(n).astype(np.int32)
    n_hold = int(n * holdout)
    tr, ho = order[n_hold:], order[:n_hold]
    hist = []
    for _ in range(epochs):
        perm = rng.permutation(tr).astype(np.int32)
        hist.append(mlp.train_epoch(perm, batch, lr, weight_decay))
    return hist, ho


def l1_rho_vs_exact(mesh, soln, n, t, params):
    """Volume-weighted relative L1 error of the density against the exact
    translated vortex (centre, strength) = params at time t."""
    from .workloads import vortex_exact
    cx, cy, beta = params
    ex = vortex_exact(mesh, t, n=n, beta=beta, a=0.5, center=(cx, cy)).reshape(-1, n * n, 4)[..., 0]
    rho = np.asarray(soln).reshape(-1, n * n, 4)[..., 0]
    g = mesh.geom.reshape(-1, 12)
    area = ((g[:, 3] - g[:, 0]) * (g[:, 7] - g[:, 1]))[:, None] / (n * n)
    return float((area * np.abs(rho - ex)).sum() / (area * np.abs(ex)).sum())


def to_uniform(forest, soln, n, level):
    """Density of an AMR state on the uniform grid of `level` (single tree):
    every cell's value injected into the fine cells it covers."""
    _, lev, x, y = forest.quads()
    side = n << level
    out = np.zeros((side, side))
    rho = np.asarray(soln).reshape(-1, n, n, 4)[..., 0]
    for q in range(len(lev)):
        r = 1 << (level - int(lev[q]))
        i0 = int(x[q] >> (30 - level)) * n
        j0 = int(y[q] >> (30 - level)) * n
        out[j0:j0 + n * r, i0:i0 + n * r] = np.kron(rho[q], np.ones((r, r)))
    return out


def run(forest, soln, n, config, final_time, regrid_interval, min_level, max_level, tol, lo_frac=0.25, mlp=None,
        judge_fraction=0.05, judge_bound=0.35, judge_min=200, judge_hard=0.5, form=1, seed=0, max_steps=10 ** 7,
        headroom=3.0, judge_coarser=False):
    """Evolve to final_time with a regrid every regrid_interval steps, tagged
    by the learned indicator (mlp) or the plain one (mlp None).

    The judge: every regrid the plain indicator re-scores the quads a hash
    of (seed, regrid, quad) puts below judge_fraction. The run falls back
    to the plain indicator for the rest of the run once the cumulative
    disagreement exceeds judge_bound over at least judge_min judged quads,
    or one regrid with 20 or more judged quads disagrees beyond judge_hard
    (a broken model). A look-ahead model disagrees with the plain classes
    of the current state by design (it predicts the next regrid's; about
    20% of the quads on the vortex family), which is what judge_bound
    leaves room for; an untrained model disagrees on 60% or more.
    judge_coarser: the judge counts only the judged quads that the model
    leaves coarser than the plain indicator would (plain refine and learned
    not, or learned coarsen and plain not) -- for a model trained on
    covering labels (collect(cover_every=...)), which asks for more
    refinement than the plain classes of the moment by design."""
    config["final_time"] = final_time
    s = Session(forest.mesh(n), config, form=form)
    if headroom > 1.0:
        # buffers for meshes up to headroom x the initial one: no regrid
        # within it allocates
        s.reserve(int(headroom * s.mesh.ncells), int(headroom * s.mesh.ncell))
    s.upload(soln)
    steps = cells = regrids = 0
    t_solve = t_regrid = 0.0
    judged = disagree = coarser = 0
    fallback_at = None
    time_now = 0.0
    while steps < max_steps:
        t0 = time.perf_counter()
        s.step(regrid_interval)
        r = s.sync()
        t1 = time.perf_counter()
        t_solve += t1 - t0
        steps += r["steps"]
        cells += r["steps"] * s.mesh.ncells
        time_now = r["time"]
        if r["error"] or time_now >= final_time:
            break
        if mlp is not None and fallback_at is None:
            cls, j = mlp.tags(s, tol, lo_frac, judge_fraction, seed=seed * 1000003 + regrids)
            judged += j["judged"]
            disagree += j["disagree"]
            coarser += j["coarser"]
            bad_now, bad_all = (j["coarser"], coarser) if judge_coarser else (j["disagree"], disagree)
            broken = j["judged"] >= 20 and bad_now > judge_hard * j["judged"]
            drift = judged >= judge_min and bad_all > judge_bound * judged
            if broken or drift:
                fallback_at = regrids
                cls = plain_classes(session_jumps(s), tol, lo_frac)
        else:
            cls = plain_classes(session_jumps(s), tol, lo_frac)
        regrid_by_classes(forest, s, n, cls, min_level, max_level)
        regrids += 1
        t_regrid += time.perf_counter() - t1
    return s, {"steps": steps, "time": time_now, "cell_updates": cells, "solve_s": t_solve, "regrid_s": t_regrid,
               "regrids": regrids, "quads": s.mesh.ncell, "judged": judged, "disagree": disagree,
               "disagree_rate": disagree / judged if judged else 0.0,
               "coarser_rate": coarser / judged if judged else 0.0, "fallback_at": fallback_at,
               "mean_cells": cells / max(steps, 1),
               "rate": cells / max(t_solve + t_regrid, 1e-30)}


def run_checked(make, n, final_time, min_level, max_level, tol, mlp, regrid_interval=10, plain_interval=5,
                l1_bound=1e-3, **kw):
    """The learned run validated against a plain-indicator run of the same
    problem: both final densities go to the uniform grid of max_level and
    when their relative L1 difference exceeds l1_bound the plain run's
    result is the one returned (the fallback). `make()` returns (forest,
    config, state) of the problem, fresh each call."""
    f1, c1, s1 = make()
    sl, rl = run(f1, s1, n, c1, final_time, regrid_interval, min_level, max_level, tol, mlp=mlp, **kw)
    ul = to_uniform(f1, sl.download(), n, max_level)
    f2, c2, s2 = make()
    sp, rp = run(f2, s2, n, c2, final_time, plain_interval, min_level, max_level, tol, mlp=None, **kw)
    up = to_uniform(f2, sp.download(), n, max_level)
    l1 = float(np.abs(ul - up).sum() / np.abs(up).sum())
    keep = l1 <= l1_bound
    (sp if keep else sl).close()
    return {"learned": rl, "plain": rp, "l1_rho_vs_plain": l1, "fallback": not keep,
            "session": sl if keep else sp, "forest": f1 if keep else f2}
