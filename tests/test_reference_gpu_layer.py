"""The drop-in route that keeps the reference's physics layer: its
src/physics/src/*.c built with -D_GPU_ (oracle/_ref/libref_physics_gpu.so),
so that physics_evolve_interface calls physics_go_gpu from libamrgpu
(physics_evolve_interface.c:42-46). The reference's hpc_amr_initialize_solver
configures its own globals (d_physics_*, physics_var_*.h); physics_go_gpu must
run with them, not with libamrgpu's defaults. Each case runs in a fresh
process (tests/ref_gpu_driver.py)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from test_oracle import golden_cases

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "libref_physics_gpu.so")
DRIVER = os.path.join(HERE, "ref_gpu_driver.py")

needs_ref_gpu = pytest.mark.skipif(not os.path.exists(REF_GPU),
                                   reason="oracle/_ref/libref_physics_gpu.so not built (reference tree absent)")


def run_driver(args, cwd):
    env = dict(os.environ, AMRGPU_QUIET="1")
    p = subprocess.run([sys.executable, DRIVER] + args, cwd=cwd, env=env, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


@needs_ref_gpu
def test_physics_go_gpu_takes_the_reference_configuration(tmp_path):
    """After the reference's own initialisation, the configuration libamrgpu
    resolves for physics_go_gpu is the reference's d_physics_* (scaled cfl,
    scheme, steps, dt, bc, intervals, mesh constants) -- no GPU involved."""
    sys.path.insert(0, HERE)
    import ref_gpu_driver as D
    z = dict(np.load(os.path.join(HERE, "golden", "go_rk3_intervals_n4.npz")))
    z["time_steps"] = np.array(37)
    z["bc"] = np.array([2, 0, 1, 1, 1, 1], np.int32)
    D.write_input(str(tmp_path), z)
    res = run_driver(["config", str(tmp_path)], str(tmp_path))
    for layer in ("1", "0"):  # libamrgpu unconfigured: both entries take the reference's
        c = res[layer]
        assert c["rc"] == 0
        assert c["cfl"] == 0.25 * 0.5 * 3
        assert c["time_scheme"] == 3 and c["time_steps"] == 37 and c["dt"] == 1.0
        assert c["bc"] == [2, 0, 1, 1, 1, 1]
        assert c["regrid_interval"] == 7 and c["visualization_interval"] == 5
        assert c["checkpoint_interval"] == 2147483647
        assert c["coarse_grid_h"] == 4.0 and c["nelem_subgrid"] == 8
        assert c["initial_condition"] == 1 and c["mach"] == 0.5


def test_unconfigured_evolve_is_refused(tmp_path):
    """libamrgpu with no configuration at all (no initialise call, no
    reference layer): hpc_amr_evolve_solver refuses before touching the GPU
    instead of running on defaults."""
    res = run_driver(["unconfigured", str(tmp_path), os.path.join(HERE, "golden", "go_rk3_hanging_n4.npz")],
                     str(tmp_path))
    assert res["error"] == 7  # AMRGPU_ERR_CONFIG
    assert res["evolve_solution"] == 0
    assert res["unchanged"]
    assert res["evolve_config_rc"] == 7


@needs_ref_gpu
@pytest.mark.gpu
@pytest.mark.parametrize("path", golden_cases("go_"), ids=os.path.basename)
def test_reference_layer_with_gpu_plug_point_bitwise(tmp_path, path):
    """The reference's initialise + evolve with -D_GPU_ reproduce the
    reference CPU driver's goldens bit for bit, with its interval flags."""
    sys.path.insert(0, HERE)
    import ref_gpu_driver as D
    z = np.load(path)
    D.write_input(str(tmp_path), z)
    res = run_driver(["evolve", str(tmp_path), path], str(tmp_path))
    assert res["error"] == 0
    assert res["bitwise"], res["maxdiff"]
    for k in ("istep", "regrid", "visualize", "checkpoint", "evolve_solution"):
        assert res[k] == int(z[k]), k


# ---------------------------------------------------------------- multi-rank
REF_GPU_MT = os.path.join(ROOT, "oracle", "_ref", "libref_physics_gpu_mt.so")
needs_ref_gpu_mt = pytest.mark.skipif(not os.path.exists(REF_GPU_MT),
                                      reason="oracle/_ref/libref_physics_gpu_mt.so not built (reference tree absent)")


def _write_case(path, tmp_path, ag, oracle, nranks, scheme, steps):
    """Shards of a hanging-face mesh, every rank's input and the one-rank
    reference result split by rank, plus input.physics for the reference's
    own initialisation."""
    import meshes
    from amrgpu import shard as S
    sys.path.insert(0, HERE)
    import ref_gpu_driver as D
    n = 4
    f = meshes.hanging(n, periodic=(1, 0), refine=(3, 6, 9))
    cfg = meshes.make_config(n, time_scheme=scheme, time_steps=steps, dt=1.0, bc=(2, 0, 1, 1))
    cfg.apply()
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), 11, amp=1e-2)
    one = s0.copy()
    oracle.reference_go(m, one, n, cfg)
    rec = 4 * n * n
    offs = S.partition(m.ncell, nranks)
    z = {"n": n, "nranks": nranks, "coarse_grid_h": 4.0}
    for r in range(nranks):
        sh = S.make_shard(m, offs, r)
        send, recv = sh.reference_lists()
        nall = len(sh.mesh.cell_info) // 3
        z[f"r{r}_cell_info"] = sh.mesh.cell_info
        z[f"r{r}_face_info"] = sh.mesh.face_info
        z[f"r{r}_geom"] = sh.mesh.geom
        z[f"r{r}_send"] = send
        z[f"r{r}_recv"] = recv
        z[f"r{r}_sizes"] = np.full(nall, rec, np.int32)
        z[f"r{r}_state0"] = sh.local_state(s0)
        z[f"r{r}_ncell"] = sh.nlocal
        z[f"r{r}_nghost"] = nall - sh.nlocal
        z[f"r{r}_nface"] = sh.mesh.nface
        z[f"r{r}_dof"] = sh.mesh.dof
        z[f"r{r}_expected"] = one[sh.lo * rec:(sh.lo + sh.nlocal) * rec]
    np.savez(path, **z)
    keys = {k: cfg[k] for k in ("time_scheme", "time_steps", "dt", "cfl", "mach", "alpha", "beta", "gamma",
                                "density", "pressure", "bc", "checkpoint_interval", "visualization_interval",
                                "regrid_interval", "initial_condition")}
    D.write_input(str(tmp_path), {k: np.asarray(v) for k, v in keys.items()})


@needs_ref_gpu_mt
def test_mpi_adapter_is_installed_by_the_reference_layer(tmp_path):
    """Loading the reference's -D_GPU_ physics layer installs the MPI
    operations from physics_go_gpu.h (its load-time constructor); libamrgpu
    alone has none. No GPU involved."""
    code = ("import ctypes as C, sys; L = C.CDLL(sys.argv[1]); a = L.amrgpu_has_comm_ops(); "
            "M = C.CDLL(sys.argv[2]); print(a, M.amrgpu_has_comm_ops())")
    p = subprocess.run([sys.executable, "-c", code, os.path.join(ROOT, "amr-demo_b200", "lib", "libamrgpu.so"),
                        REF_GPU_MT], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.split() == ["0", "1"]


def test_multirank_evolve_without_mpi_operations_is_refused(ag):
    """Ghost quads without the caller's MPI operations: the entry refuses
    before any device work (AMRGPU_ERR_UNSUPPORTED, evolve_solution = 0)."""
    import ctypes as C
    import meshes
    from amrgpu import shard as S
    L = ag.lib()
    assert L.amrgpu_has_comm_ops() == 0
    n = 4
    f = meshes.hanging(n, periodic=(1, 0), refine=(3, 6))
    meshes.make_config(n, time_steps=3).apply()
    m = f.mesh(n)
    sh = S.make_shard(m, S.partition(m.ncell, 2), 0)
    send, recv = sh.reference_lists()
    nall = len(sh.mesh.cell_info) // 3
    i32 = lambda a: np.ascontiguousarray(a, np.int32)  # noqa: E731
    ci, fi, send, recv = i32(sh.mesh.cell_info), i32(sh.mesh.face_info), i32(send), i32(recv)
    sizes = np.full(nall, 4 * n * n, np.int32)
    geom = np.ascontiguousarray(sh.mesh.geom, np.float64)
    st = sh.local_state(f.initialize(n))
    before = st.copy()
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))  # noqa: E731
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    ci_ = lambda v: C.byref(C.c_int(int(v)))  # noqa: E731
    ist, rg, vis, chk, evo = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(1)
    tt, ct, rt = C.c_double(0), C.c_double(0), C.c_double(0)
    L.hpc_amr_evolve_solver(ci_(2), ci_(0), ci_(4), ci_(n), ci_(sh.nlocal), ci_(nall - sh.nlocal),
                            ci_(sh.mesh.nface), ci_(sh.mesh.dof), ip(ci), ip(fi), ci_(len(send) // 2),
                            ci_(len(recv) // 2), ip(send), ip(recv), ip(sizes), dp(geom), dp(st), C.byref(ist),
                            C.byref(rg), C.byref(vis), C.byref(chk), C.byref(evo), 0, C.byref(tt),
                            C.byref(ct), C.byref(rt))
    err = L.amrgpu_last_error()
    L.amrgpu_clear_error()
    assert err == 5
    assert evo.value == 0 and ist.value == 0
    assert np.array_equal(st, before)


@needs_ref_gpu_mt
@pytest.mark.gpu
@pytest.mark.parametrize("nranks,scheme", [(2, 3), (3, 5), (4, 4)])
def test_reference_layer_multirank_on_gpu_bitwise(tmp_path, ag, oracle, nranks, scheme):
    """An unmodified multi-rank reference application on the GPU plug-point:
    the reference's physics layer built with -D_GPU_ over the multi-rank MPI
    stand-in, P ranks (threads) each calling physics_evolve_interface ->
    physics_go_gpu with its shard. Ghost records move through the MPI
    operations of physics_go_gpu.h before every stage and the CFL step is
    the MIN over ranks: every rank's quads end bit-identical to the
    reference's one-rank CPU run of the whole mesh."""
    case = str(tmp_path / "case.npz")
    _write_case(case, tmp_path, ag, oracle, nranks, scheme, steps=7)
    res = run_driver(["multirank", str(tmp_path), case], str(tmp_path))
    assert res["rc"] == 0 and res["error"] == 0, res
    assert res["istep"] == [7] * nranks
    assert all(res["bitwise"]), res["maxdiff"]
