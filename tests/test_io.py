"""Visualisation and checkpoint output (csrc/io.cpp): the VTK file carries
what the reference's vtk_write_solution writes (amr_vtk.c:23-217: one quad
per quadrant with corners shrunk by 0.99999, tree / level / rank cell
data, patch averages as point data), the subgrid variant one quad per
cell; a checkpoint restores the forest, the state, the step and the time
exactly, and malformed files are rejected. No GPU needed."""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import meshes


def _arrays(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    out = {}
    for da in root.iter("DataArray"):
        vals = np.array(da.text.split(), dtype=np.float64)
        out[da.get("Name") or "points"] = vals
    return int(piece.get("NumberOfPoints")), int(piece.get("NumberOfCells")), out


def test_vtk_patch_averages_like_the_reference(ag, tmp_path):
    n = 4
    f = meshes.hanging(n, level=2, refine=(3, 6))
    rng = np.random.default_rng(0)
    soln = rng.random(4 * n * n * f.num_quads)
    p = tmp_path / "soln.vtu"
    f.write_vtk(p, n, soln)
    npts, ncell, a = _arrays(p)
    nq = f.num_quads
    assert (npts, ncell) == (4 * nq, nq)
    q = soln.reshape(nq, n * n, 4)
    avg = q.sum(axis=1) * (1.0 / (n * n))
    for k, name in enumerate(("rho", "rhou", "rhov", "rhoe")):
        assert np.allclose(a[name].reshape(nq, 4), avg[:, k:k + 1], rtol=0, atol=1e-15)
    tree, level, _, _ = f.quads()
    assert np.array_equal(a["level"], level) and np.array_equal(a["treeid"], tree)
    assert np.all(a["mpirank"] == 0)
    assert np.array_equal(a["types"], np.full(nq, 9))
    # each quad's points lie strictly inside its own geometry (shrunk corners)
    g = f.mesh(n).geom.reshape(nq, 4, 3)
    pts = a["points"].reshape(nq, 4, 3)
    lo, hi = g[:, :, :2].min(axis=1), g[:, :, :2].max(axis=1)
    assert np.all(pts[:, :, :2] > lo[:, None, :]) and np.all(pts[:, :, :2] < hi[:, None, :])


def test_vtk_subgrid_cells_carry_the_state(ag, tmp_path):
    n = 4
    f = meshes.uniform(n, 1)
    soln = np.arange(4 * n * n * f.num_quads, dtype=np.float64)
    p = tmp_path / "sub.vtu"
    f.write_vtk(p, n, soln, subgrid=True)
    npts, ncell, a = _arrays(p)
    assert ncell == f.num_quads * n * n and npts == 4 * ncell
    assert np.array_equal(a["rho"], soln[0::4]) and np.array_equal(a["rhoe"], soln[3::4])


def test_checkpoint_round_trip_restores_forest_state_step_and_time(ag, tmp_path):
    n = 4
    f = meshes.hanging(n, level=2, refine=(3, 6, 9), periodic=(1, 0))
    tags = np.arange(f.num_quads, dtype=np.int32) % 3
    f.set_tags(tags)
    soln = np.random.default_rng(1).random(4 * n * n * f.num_quads)
    p = tmp_path / "amr_soln_0000042.bin"
    f.save_checkpoint(p, n, soln, istep=42, time=1.25)
    g, n2, s2, ist, t = ag.Forest.load_checkpoint(p)
    assert (n2, ist, t) == (n, 42, 1.25)
    assert np.array_equal(s2, soln)
    for a, b in zip(f.quads(), g.quads()):
        assert np.array_equal(a, b)
    assert np.array_equal(g.get_tags(), tags)
    m1, m2 = f.mesh(n), g.mesh(n)
    assert np.array_equal(m1.face_info, m2.face_info) and np.array_equal(m1.geom, m2.geom)
    # the restored forest keeps adapting
    g.begin_regrid()
    g.refine(np.ones(g.num_quads, np.int32), max_level=5)
    g.balance()
    assert g.num_quads == 4 * f.num_quads


def test_malformed_checkpoints_are_rejected(ag, tmp_path):
    n = 2
    f = meshes.uniform(n, 1)
    soln = np.zeros(4 * n * n * f.num_quads)
    p = tmp_path / "c.bin"
    f.save_checkpoint(p, n, soln)
    data = p.read_bytes()
    (tmp_path / "short.bin").write_bytes(data[:-9])
    (tmp_path / "magic.bin").write_bytes(b"X" + data[1:])
    bad = bytearray(data)
    bad[48 + 8 + 16 + 32 + 8 + 8 + 4] = 7  # the first leaf's x now lies beyond its tree
    (tmp_path / "coord.bin").write_bytes(bytes(bad))
    # one leaf fewer in the count: the leaves no longer tile the trees
    few = bytearray(data)
    few[104:112] = (f.num_quads - 1).to_bytes(8, "little")
    (tmp_path / "tiles.bin").write_bytes(bytes(few))
    for name in ("short.bin", "magic.bin", "coord.bin", "tiles.bin"):
        with pytest.raises(RuntimeError):
            ag.Forest.load_checkpoint(tmp_path / name)
    with pytest.raises(RuntimeError):
        ag.Forest.load_checkpoint(tmp_path / "missing.bin")
