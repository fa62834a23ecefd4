"""ctypes access to the CPU oracle -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module, and only to verify GPU results / as the timed CPU baseline; the product
path (libamrgpu) never calls it.

Two libraries, both built by oracle/Makefile:
  * ``_build/liboracle.so``  -- restatement of the reference's 2D Fortran
    kernels (solver2d.c) and of its one-rank C driver (physics2d.c);
  * ``_ref/libref_physics.so`` -- the reference's own src/physics/src/*.c,
    compiled unmodified, linked against solver2d.c and a one-rank MPI
    stand-in. Present when the reference tree was available at build time.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT = os.path.join(HERE, "_build", "liboracle.so")
REFERENCE = os.path.join(HERE, "_ref", "libref_physics.so")
REFERENCE_MT = os.path.join(HERE, "_ref", "libref_physics_mt.so")


def _host_has_avx512():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("flags"):
                    return " avx512f " in line + " "
    except OSError:
        pass
    return False


def timing_build(base):
    """The -O3 timing build of a reference library (x86-64-v4 on AVX-512
    hosts, else x86-64-v3); the parity build when neither was built."""
    for arch in (("v4", "v3") if _host_has_avx512() else ("v3",)):
        p = os.path.join(HERE, "_ref", f"{base}_fast_{arch}.so")
        if os.path.exists(p):
            return p, f"-O3 -march=x86-64-{arch}"
    return os.path.join(HERE, "_ref", f"{base}.so"), "-O2 -ffp-contract=off (parity build)"

i32p = C.POINTER(C.c_int)
f64p = C.POINTER(C.c_double)


def ip(a):
    return a.ctypes.data_as(i32p)


def dp(a):
    return a.ctypes.data_as(f64p)


class OracleConfig(C.Structure):
    """oracle_config_t of physics2d.c."""

    _fields_ = [("nelem_subgrid", C.c_int), ("time_scheme", C.c_int), ("time_steps", C.c_int),
                ("regrid_interval", C.c_int), ("checkpoint_interval", C.c_int),
                ("visualization_interval", C.c_int), ("bc", C.c_int * 4), ("dt", C.c_double),
                ("cfl", C.c_double), ("h_base", C.c_double), ("final_time", C.c_double),
                ("time", C.c_double)]


_cache = {}


def restatement():
    if "r" not in _cache:
        if not os.path.exists(RESTATEMENT):
            raise RuntimeError(f"{RESTATEMENT} missing: run `make -C oracle`")
        L = C.CDLL(RESTATEMENT)
        L.oracle_rhs.argtypes = [C.POINTER(OracleConfig), C.c_int, i32p, C.c_int, i32p, f64p, C.c_int, f64p, f64p]
        L.oracle_rhs.restype = None
        L.oracle_time_step.argtypes = [C.POINTER(OracleConfig), C.c_int, i32p, f64p, f64p, f64p]
        L.oracle_time_step.restype = None
        L.oracle_norm.argtypes = [C.c_int, C.c_int, i32p, f64p]
        L.oracle_norm.restype = C.c_double
        L.oracle_evolve.argtypes = [C.POINTER(OracleConfig), C.c_int, i32p, C.c_int, i32p, f64p, C.c_int, f64p,
                                    i32p, i32p, i32p, i32p, i32p, f64p, f64p]
        L.oracle_evolve.restype = C.c_int
        L.oracle_flux_roe_2d.argtypes = [f64p, f64p, f64p, f64p]
        L.oracle_flux_roe_2d.restype = None
        L.oracle_set_inflow.argtypes = [f64p]
        L.oracle_set_inflow.restype = None
        L.oracle_shock_state.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, f64p]
        L.oracle_shock_state.restype = None
        _cache["r"] = L
    return _cache["r"]


def reference_available():
    return os.path.exists(REFERENCE)


def set_inflow(cfg):
    """bc 3 (extension): the shock-bubble workload's inflow state, the
    post-shock state of its Mach ic_params[0] (default 2) shock into (1, 1)."""
    L = restatement()
    out = np.zeros(4, np.float64)
    if cfg["initial_condition"] == 5:
        ms = cfg["ic_params"][0] or 2.0
        L.oracle_shock_state(cfg["gamma"], ms, 1.0, 1.0, dp(out))
    L.oracle_set_inflow(dp(out))
    if reference_available():
        reference().oracle_set_inflow(dp(out))
    return out


def make_config(n, cfg):
    """OracleConfig from an amrgpu.Config-like mapping (also sets the
    inflow state of bc 3)."""
    set_inflow(cfg)
    c = OracleConfig()
    c.nelem_subgrid = n
    c.time_scheme = cfg["time_scheme"]
    c.time_steps = cfg["time_steps"]
    big = 2147483647

    def iv(k):
        v = cfg[k]
        return 0 if v >= big or v <= 0 else v

    c.regrid_interval = iv("regrid_interval")
    c.checkpoint_interval = iv("checkpoint_interval")
    c.visualization_interval = iv("visualization_interval")
    for k in range(4):
        c.bc[k] = cfg["bc"][k]
    c.dt = cfg["dt"]
    c.cfl = cfg["cfl"]
    c.h_base = cfg["coarse_grid_h"]
    c.final_time = cfg["final_time"]
    c.time = 0.0
    return c


def rhs(mesh, soln, ocfg):
    L = restatement()
    out = np.zeros(mesh.dof, np.float64)
    s = np.ascontiguousarray(soln, np.float64).copy()
    L.oracle_rhs(C.byref(ocfg), mesh.ncell, ip(mesh.cell_info), mesh.nface, ip(mesh.face_info),
                 dp(mesh.geom), mesh.dof, dp(s), dp(out))
    return out


def time_step(mesh, soln, ocfg):
    L = restatement()
    dt = C.c_double(ocfg.dt)
    s = np.ascontiguousarray(soln, np.float64).copy()
    L.oracle_time_step(C.byref(ocfg), mesh.ncell, ip(mesh.cell_info), dp(mesh.geom), dp(s), C.byref(dt))
    return dt.value


def evolve(mesh, soln, ocfg, istep=0):
    """Runs one evolve segment on ``soln`` in place; returns the flags."""
    L = restatement()
    ist, rg, vis, chk, evo = C.c_int(istep), C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(1)
    rn, dtl = C.c_double(0), C.c_double(0)
    steps = L.oracle_evolve(C.byref(ocfg), mesh.ncell, ip(mesh.cell_info), mesh.nface, ip(mesh.face_info),
                            dp(mesh.geom), mesh.dof, dp(soln), C.byref(ist), C.byref(rg), C.byref(vis),
                            C.byref(chk), C.byref(evo), C.byref(rn), C.byref(dtl))
    return {"steps": steps, "istep": ist.value, "regrid": rg.value, "visualize": vis.value,
            "checkpoint": chk.value, "evolve_solution": evo.value, "residual_norm": rn.value,
            "dt_last": dtl.value, "time": ocfg.time}


def flux(ql, qr, normal):
    L = restatement()
    a = np.ascontiguousarray(ql, np.float64)
    b = np.ascontiguousarray(qr, np.float64)
    nv = np.ascontiguousarray(normal, np.float64)
    out = np.zeros(4, np.float64)
    L.oracle_flux_roe_2d(dp(a), dp(b), dp(nv), dp(out))
    return out


# ------------------------------------------------------------------ reference
class _Interface(C.Structure):  # physics_var_interface.h:20-36
    _fields_ = [("dim", C.c_int), ("nfringe", C.c_int), ("nfields", C.c_int), ("nelem_subgrid", C.c_int),
                ("extern_cell_size", C.c_int), ("extern_face_size", C.c_int), ("extern_edge_size", C.c_int),
                ("extern_node_size", C.c_int), ("extern_mpi_comm_size", C.c_int), ("nlevels", C.c_int),
                ("coarse_grid_h", C.c_double)]


class _Fluid(C.Structure):  # physics_var_physics.h:21-46
    _fields_ = [("initial_condition", C.c_int), ("bc", C.c_int * 6), ("amr_ntag_methods", C.c_int),
                ("amr_tag_methods", C.POINTER(C.c_int)), ("amr_tag_tolerances", C.POINTER(C.c_double)),
                ("cfl", C.c_double), ("mach", C.c_double), ("alpha", C.c_double), ("beta", C.c_double),
                ("gamma", C.c_double), ("density", C.c_double), ("pressure", C.c_double)]


class _Simulation(C.Structure):  # physics_var_simulation.h:20-30
    _fields_ = [("checkpoint_interval", C.c_int), ("visualization_interval", C.c_int),
                ("regrid_interval", C.c_int), ("time_scheme", C.c_int), ("time_steps", C.c_int),
                ("dt", C.c_double)]


def reference(path=None):
    """The reference's own C driver (oracle/_ref), with its globals; path
    selects another build of it (a timing build, the multi-rank build)."""
    path = path or REFERENCE
    key = ("ref", path)
    if key not in _cache:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
        L = C.CDLL(path)
        L.physics_rhs_structured.restype = None
        L.physics_rhs_structured.argtypes = [i32p, i32p, i32p, i32p, i32p, f64p, i32p, i32p, i32p, f64p, f64p]
        L.physics_go.restype = None
        L.physics_go.argtypes = [i32p] * 15 + [f64p] * 2 + [i32p] * 5 + [C.c_int] + [f64p] * 3
        L.oracle_mpi_take_abort_code.restype = C.c_int
        L.oracle_mpi_take_abort_code.argtypes = []
        L.oracle_set_inflow.argtypes = [f64p]
        L.oracle_set_inflow.restype = None
        if hasattr(L, "oracle_mt_go"):
            L.oracle_mt_go.restype = C.c_int
            L.oracle_mt_go.argtypes = [C.c_int, C.c_int, C.POINTER(MtRank)]
        _cache[key] = L
    return _cache[key]


class MtRank(C.Structure):
    """oracle_mt_rank_t of mt_driver.c: one rank's arrays and results."""

    _fields_ = [("ncell", C.c_int), ("nghost", C.c_int), ("nface", C.c_int), ("dof", C.c_int), ("nsend", C.c_int),
                ("nrecv", C.c_int), ("cell_info", i32p), ("face_info", i32p), ("send", i32p), ("recv", i32p),
                ("sizes", i32p), ("geom", f64p), ("soln", f64p), ("istep", C.c_int), ("regrid", C.c_int),
                ("visualize", C.c_int), ("checkpoint", C.c_int), ("evolve_solution", C.c_int),
                ("total_time", C.c_double), ("compute_time", C.c_double), ("residual_time", C.c_double),
                ("wall", C.c_double)]


def _pad_int(a, pad=16):
    """Copy with `pad` entries of -1 in front: the reference reads
    cell_info[3*(-1)] for absent neighbours (physics_rhs_structured.c:97-128)."""
    buf = np.full(len(a) + pad, -1, np.int32)
    buf[pad:] = a
    return buf, buf[pad:]


def reference_set_globals(n, cfg, L=None):
    L = L or reference()
    itf = _Interface.in_dll(L, "d_physics_interface")
    itf.dim, itf.nfringe, itf.nfields, itf.nelem_subgrid = 2, 2, 4, n
    itf.extern_cell_size, itf.extern_face_size = 3, 11
    itf.extern_edge_size, itf.extern_node_size, itf.extern_mpi_comm_size = 0, 0, 2
    itf.nlevels = 0
    itf.coarse_grid_h = cfg["coarse_grid_h"]
    fl = _Fluid.in_dll(L, "d_physics_fluid")
    for k in range(6):
        fl.bc[k] = cfg["bc"][k]
    fl.cfl = cfg["cfl"]
    fl.gamma, fl.density, fl.pressure, fl.mach = cfg["gamma"], cfg["density"], cfg["pressure"], cfg["mach"]
    fl.alpha, fl.beta = cfg["alpha"], cfg["beta"]
    fl.initial_condition = cfg["initial_condition"]
    sim = _Simulation.in_dll(L, "d_physics_simulation")
    sim.time_scheme, sim.time_steps, sim.dt = cfg["time_scheme"], cfg["time_steps"], cfg["dt"]
    big = 2147483647
    sim.checkpoint_interval = cfg["checkpoint_interval"] if cfg["checkpoint_interval"] > 0 else big
    sim.visualization_interval = cfg["visualization_interval"] if cfg["visualization_interval"] > 0 else big
    sim.regrid_interval = cfg["regrid_interval"] if cfg["regrid_interval"] > 0 else big


def reference_rhs(mesh, soln, n, cfg):
    L = reference()
    reference_set_globals(n, cfg)
    _, ci = _pad_int(mesh.cell_info)
    out = np.zeros(mesh.dof, np.float64)
    s = np.ascontiguousarray(soln, np.float64).copy()
    dim, nf, nn, nc, nface, dof = (C.c_int(2), C.c_int(4), C.c_int(n), C.c_int(mesh.ncell),
                                    C.c_int(mesh.nface), C.c_int(mesh.dof))
    L.physics_rhs_structured(C.byref(dim), C.byref(nf), C.byref(nn), C.byref(nc), ip(ci), dp(mesh.geom),
                             C.byref(nface), ip(mesh.face_info), C.byref(dof), dp(s), dp(out))
    return out


def reference_go(mesh, soln, n, cfg, istep=0, path=None):
    """physics_go (the reference's CPU evolve) on ``soln`` in place; path
    selects a build of the reference library (default: the parity build)."""
    L = reference(path)
    reference_set_globals(n, cfg, L)
    buf, ci = _pad_int(mesh.cell_info)
    dim, uns, nf, nn = C.c_int(2), C.c_int(0), C.c_int(4), C.c_int(n)
    nc, ng, nface, dof = C.c_int(mesh.ncell), C.c_int(0), C.c_int(mesh.nface), C.c_int(mesh.dof)
    nsend, nrecv = C.c_int(0), C.c_int(0)
    send = np.zeros(2, np.int32)
    recv = np.zeros(2, np.int32)
    sizes = np.full(max(mesh.ncell, 1), 4 * n * n, np.int32)
    ist = C.c_int(istep)
    rg, vis, chk, evo = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(1)
    tt, ct, rt = C.c_double(0), C.c_double(0), C.c_double(0)
    L.physics_go(C.byref(dim), C.byref(uns), C.byref(nf), C.byref(nn), C.byref(nc), C.byref(ng), C.byref(nface),
                 C.byref(dof), ip(ci), ip(mesh.face_info), C.byref(nsend), C.byref(nrecv), ip(send), ip(recv),
                 ip(sizes), dp(mesh.geom), dp(soln), C.byref(ist), C.byref(rg), C.byref(vis), C.byref(chk),
                 C.byref(evo), 0, C.byref(tt), C.byref(ct), C.byref(rt))
    return {"istep": ist.value, "regrid": rg.value, "visualize": vis.value, "checkpoint": chk.value,
            "evolve_solution": evo.value, "total_time": tt.value, "abort": L.oracle_mpi_take_abort_code()}


def reference_mt_go(shards, states, n, cfg, path=None):
    """The reference's physics_go on len(shards) ranks at once, one thread
    each, over the multi-rank MPI stand-in (mt_driver.c): every rank evolves
    its own state in ``states`` (local quads then ghost quads, AoS) with the
    ghost exchange of physics_mpi_real_to_ghost every stage. ``shards`` are
    objects with ``mesh`` (external_t arrays of the rank) and
    ``reference_lists()`` (send / recv (cell, rank) pairs). Returns the
    per-rank flags and the slowest rank's seconds in physics_go."""
    L = reference(path or REFERENCE_MT)
    reference_set_globals(n, cfg, L)
    P = len(shards)
    ranks = (MtRank * P)()
    keep = []
    for r, (sh, st) in enumerate(zip(shards, states)):
        m = sh.mesh
        buf, ci = _pad_int(m.cell_info)
        send, recv = sh.reference_lists()
        send = np.ascontiguousarray(send if len(send) else np.zeros(2, np.int32), np.int32)
        recv = np.ascontiguousarray(recv if len(recv) else np.zeros(2, np.int32), np.int32)
        nall = len(m.cell_info) // 3
        sizes = np.full(max(nall, 1), 4 * n * n, np.int32)
        fi = np.ascontiguousarray(m.face_info, np.int32)
        geom = np.ascontiguousarray(m.geom, np.float64)
        R = ranks[r]
        R.ncell, R.nghost, R.nface, R.dof = m.ncell, nall - m.ncell, m.nface, m.dof
        R.nsend, R.nrecv = len(sh.reference_lists()[0]) // 2, len(sh.reference_lists()[1]) // 2
        R.cell_info, R.face_info, R.send, R.recv, R.sizes = ip(ci), ip(fi), ip(send), ip(recv), ip(sizes)
        R.geom, R.soln = dp(geom), dp(st)
        R.istep, R.evolve_solution = 0, 1
        keep += [buf, ci, fi, geom, send, recv, sizes, st]
    rc = L.oracle_mt_go(P, n, ranks)
    if rc != 0:
        raise RuntimeError("oracle_mt_go: the rank threads could not be started")
    return {"istep": [ranks[r].istep for r in range(P)], "evolve_solution": [ranks[r].evolve_solution for r in range(P)],
            "wall": max(ranks[r].wall for r in range(P)), "abort": L.oracle_mpi_take_abort_code()}
