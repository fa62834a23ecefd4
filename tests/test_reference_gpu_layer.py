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
