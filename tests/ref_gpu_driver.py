"""Drives the reference's own physics layer built with -D_GPU_
(oracle/_ref/libref_physics_gpu.so: src/physics/src/*.c, linked against
libamrgpu.so) in a fresh process, as a reference application would:

    hpc_amr_initialize_solver  (the reference's: physics_initialize reads
                                input.physics into d_physics_*)
    hpc_amr_evolve_solver      (the reference's) -> physics_evolve_interface
                               -> physics_go_gpu (libamrgpu)

A fresh process is needed because libamrgpu binds the reference's
configuration globals when it is loaded; the library must therefore be
loaded as a dependency of the reference's physics layer, not before it.

    python tests/ref_gpu_driver.py config <workdir>
    python tests/ref_gpu_driver.py evolve <workdir> <golden.npz>
    python tests/ref_gpu_driver.py unconfigured <workdir> <golden.npz>
    python tests/ref_gpu_driver.py multirank <workdir> <case.npz>

multirank: the same layer built over the multi-rank MPI stand-in
(oracle/_ref/libref_physics_gpu_mt.so): P ranks as P threads, each entering
physics_evolve_interface -> physics_go_gpu with its shard (local quads, ghost
quads, send / recv lists); the ghost exchange and the reductions go through
the MPI operations physics_go_gpu.h installs. <case.npz> holds the shards and
every rank's expected local state.

<workdir> must hold input.physics. Prints one JSON line.
"""
import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "libref_physics_gpu.so")
REF_GPU_MT = os.path.join(ROOT, "oracle", "_ref", "libref_physics_gpu_mt.so")
LIBAMRGPU = os.path.join(ROOT, "amr-demo_b200", "lib", "libamrgpu.so")
sys.path.insert(0, os.path.join(ROOT, "amr-demo_b200"))
sys.path.insert(0, ROOT)

from amrgpu._lib import ConfigStruct  # noqa: E402  (no library is loaded by this import)
from oracle.oracle import MtRank  # noqa: E402  (ctypes layout only; loads no library)

i32p = C.POINTER(C.c_int)
f64p = C.POINTER(C.c_double)


def ip(a):
    return a.ctypes.data_as(i32p)


def dp(a):
    return a.ctypes.data_as(f64p)


def iref(v):
    return C.byref(C.c_int(int(v)))


def write_input(workdir, z):
    """input.physics with the values of a golden case (raw cfl 0.5: the
    reference scales it by 0.25*time_scheme, which gives the golden's)."""
    ts = int(z["time_scheme"])
    iv = lambda k: int(z[k]) if int(z[k]) < 2147483647 else 0  # noqa: E731
    bc = [int(b) for b in z["bc"]]
    lines = [
        f"initial_condition: {int(z['initial_condition'])}",
        f"time_scheme: {ts}",
        f"time_steps: {int(z['time_steps'])}",
        f"dt: {float(z['dt'])!r}",
        f"cfl: {float(z['cfl']) / (0.25 * ts)!r}",
        f"mach: {float(z['mach'])!r}",
        f"alpha: {float(z['alpha'])!r}",
        f"beta: {float(z['beta'])!r}",
        f"gamma: {float(z['gamma'])!r}",
        f"density: {float(z['density'])!r}",
        f"pressure: {float(z['pressure'])!r}",
        f"bc_xlo: {bc[0]}", f"bc_xhi: {bc[1]}", f"bc_ylo: {bc[2]}", f"bc_yhi: {bc[3]}",
        f"bc_zlo: {bc[4]}", f"bc_zhi: {bc[5]}",
        f"checkpoint_interval: {iv('checkpoint_interval')}",
        f"visualization_interval: {iv('visualization_interval')}",
        f"regrid_interval: {iv('regrid_interval')}",
        "amr_ntag_methods: 0",
    ]
    with open(os.path.join(workdir, "input.physics"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    # the reference's physics_initialize_save_inputs writes WRK/saved.input.physics
    # (physics_initialize.c) and does not check fopen: its run directory has WRK/
    os.makedirs(os.path.join(workdir, "WRK"), exist_ok=True)


def initialize(L, n, h):
    L.hpc_amr_initialize_solver(iref(0), iref(2), C.byref(C.c_double(h)), iref(0), iref(4), iref(2), iref(n),
                                iref(3), iref(11), iref(0), iref(0), iref(2))


def evolve(L, z):
    n = int(z["n"])
    ci = np.ascontiguousarray(z["cell_info"], np.int32)
    fi = np.ascontiguousarray(z["face_info"], np.int32)
    geom = np.ascontiguousarray(z["geom"], np.float64)
    soln = np.ascontiguousarray(z["soln0"], np.float64).copy()
    ncell = len(ci) // 3
    send = np.zeros(2, np.int32)
    recv = np.zeros(2, np.int32)
    sizes = np.full(max(ncell, 1), 4 * n * n, np.int32)
    ist, rg, vis, chk, evo = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(1)
    tt, ct, rt = C.c_double(0), C.c_double(0), C.c_double(0)
    L.hpc_amr_evolve_solver.argtypes = [i32p] * 15 + [f64p] * 2 + [i32p] * 5 + [C.c_int] + [f64p] * 3
    L.hpc_amr_evolve_solver(iref(2), iref(0), iref(4), iref(n), iref(ncell), iref(0), iref(int(z["nface"])),
                            iref(int(z["dof"])), ip(ci), ip(fi), iref(0), iref(0), ip(send), ip(recv), ip(sizes),
                            dp(geom), dp(soln), C.byref(ist), C.byref(rg), C.byref(vis), C.byref(chk),
                            C.byref(evo), 0, C.byref(tt), C.byref(ct), C.byref(rt))
    return soln, {"istep": ist.value, "regrid": rg.value, "visualize": vis.value, "checkpoint": chk.value,
                  "evolve_solution": evo.value}


def multirank(z):
    """oracle_mt_evolve over the shards in z; per-rank comparison of the
    local quads with the expected state."""
    L = C.CDLL(REF_GPU_MT)  # loads libamrgpu.so as its dependency
    n, P = int(z["n"]), int(z["nranks"])
    initialize(L, n, float(z["coarse_grid_h"]))
    L.oracle_mt_evolve.restype = C.c_int
    L.oracle_mt_evolve.argtypes = [C.c_int, C.c_int, C.POINTER(MtRank)]
    ranks = (MtRank * P)()
    keep = []
    for r in range(P):
        g = lambda k: z[f"r{r}_{k}"]  # noqa: E731
        # the reference reads cell_info[3*(-1)] for absent neighbours
        # (physics_rhs_structured.c:97-128): 16 ints of -1 in front
        cbuf = np.full(len(g("cell_info")) + 16, -1, np.int32)
        cbuf[16:] = g("cell_info")
        ci = cbuf[16:]
        fi = np.ascontiguousarray(g("face_info"), np.int32)
        geom = np.ascontiguousarray(g("geom"), np.float64)
        send = np.ascontiguousarray(g("send"), np.int32)
        recv = np.ascontiguousarray(g("recv"), np.int32)
        sizes = np.ascontiguousarray(g("sizes"), np.int32)
        st = np.ascontiguousarray(g("state0"), np.float64).copy()
        R = ranks[r]
        R.ncell, R.nghost, R.nface, R.dof = int(g("ncell")), int(g("nghost")), int(g("nface")), int(g("dof"))
        R.nsend, R.nrecv = len(send) // 2, len(recv) // 2
        if R.nsend == 0:
            send = np.zeros(2, np.int32)
        if R.nrecv == 0:
            recv = np.zeros(2, np.int32)
        R.cell_info, R.face_info, R.send, R.recv, R.sizes = ip(ci), ip(fi), ip(send), ip(recv), ip(sizes)
        R.geom, R.soln = dp(geom), dp(st)
        R.istep, R.evolve_solution = 0, 1
        keep.append((cbuf, fi, geom, send, recv, sizes, st))
    rc = L.oracle_mt_evolve(P, n, ranks)
    out = {"rc": rc, "error": L.amrgpu_last_error(), "istep": [], "evolve_solution": [], "bitwise": [],
           "maxdiff": []}
    for r in range(P):
        got = keep[r][6][: int(z[f"r{r}_dof"])]
        want = z[f"r{r}_expected"]
        out["istep"].append(ranks[r].istep)
        out["evolve_solution"].append(ranks[r].evolve_solution)
        out["bitwise"].append(bool(np.array_equal(got, want)))
        out["maxdiff"].append(float(np.abs(got - want).max()) if len(want) else 0.0)
    return out


def main():
    mode, workdir = sys.argv[1], sys.argv[2]
    os.environ.setdefault("AMRGPU_QUIET", "1")
    os.chdir(workdir)
    if mode == "unconfigured":
        # libamrgpu alone, nothing configured: the evolve entry must refuse
        L = C.CDLL(LIBAMRGPU)
        z = np.load(sys.argv[3])
        soln, flags = evolve(L, z)
        out = {"error": L.amrgpu_last_error(), "evolve_solution": flags["evolve_solution"],
               "unchanged": bool(np.array_equal(soln, z["soln0"]))}
        cfg = ConfigStruct()
        out["evolve_config_rc"] = L.amrgpu_evolve_config(0, C.byref(cfg))
        print(json.dumps(out))
        return
    if mode == "multirank":
        print(json.dumps(multirank(np.load(sys.argv[3]))))
        return
    L = C.CDLL(REF_GPU)  # loads libamrgpu.so as its dependency
    L.amrgpu_evolve_config.argtypes = [C.c_int, C.POINTER(ConfigStruct)]
    L.amrgpu_evolve_config.restype = C.c_int
    if mode == "config":
        initialize(L, 8, 4.0)
        res = {}
        for layer in (1, 0):
            cfg = ConfigStruct()
            rc = L.amrgpu_evolve_config(layer, C.byref(cfg))
            res[str(layer)] = {"rc": rc, "cfl": cfg.cfl, "time_scheme": cfg.time_scheme,
                               "time_steps": cfg.time_steps, "dt": cfg.dt, "bc": list(cfg.bc),
                               "coarse_grid_h": cfg.coarse_grid_h, "nelem_subgrid": cfg.nelem_subgrid,
                               "regrid_interval": cfg.regrid_interval,
                               "visualization_interval": cfg.visualization_interval,
                               "checkpoint_interval": cfg.checkpoint_interval,
                               "initial_condition": cfg.initial_condition, "mach": cfg.mach}
        print(json.dumps(res))
        return
    z = np.load(sys.argv[3])
    initialize(L, int(z["n"]), float(z["coarse_grid_h"]))
    soln, flags = evolve(L, z)
    flags["error"] = L.amrgpu_last_error()
    flags["bitwise"] = bool(np.array_equal(soln, z["soln1"]))
    flags["maxdiff"] = float(np.abs(soln - z["soln1"]).max())
    print(json.dumps(flags))


if __name__ == "__main__":
    main()
