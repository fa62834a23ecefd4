"""The FP32-flux form's row-sweep stage kernels for 16x16 and 8x8 patches
(csrc/stage_sweep.cuh) against the block-phase FP32 kernel it replaces as
the default and against the FP64 oracle.

Both kernels evaluate every face with the same FP32 flux routine on the same
records and sum a cell's faces in the same FP64 order; they differ only at a
coarse hanging edge (the sweep adds the edge's two fluxes first) and in the
compiler's instruction selection around the inlined flux. Tolerances: the
states after 6 steps agree to 1e-6 of each field's largest magnitude, sweep
launch shapes agree bit for bit, one residual is within the FP32 form's
2e-5 of max|R| of the oracle, and periodic totals are conserved to 1e-12."""
import os

import numpy as np
import pytest

import meshes

pytestmark = pytest.mark.gpu
os.environ.setdefault("AMRGPU_QUIET", "1")

# the first block-phase FP32 variant per patch size
BLOCK = {16: (1, 288), 8: (4, 288)}
# variant indices of the row sweep, the first three of each list:
# 16x16 (4,128), (2,64), (8,256); 8x8 (8,128), (4,64), (16,256)
SWEEPS = [0, 1, 2]


def case(ag, seed, scheme, n=16):
    rng = np.random.default_rng(seed)
    per = (int(rng.integers(2)), int(rng.integers(2)))
    f = meshes.uniform(n, 2, periodic=per)
    fl = (rng.random(f.num_quads) < 0.4).astype(np.int32)
    f.refine(fl)
    f.balance()
    cfg = meshes.make_config(n, time_scheme=scheme, time_steps=10 ** 6, dt=0.01,
                             bc=tuple(int(b) for b in rng.integers(0, 3, 4)))
    cfg.apply()
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), seed, amp=2e-2)
    return f, m, cfg, s0


def run(ag, m, cfg, s0, shape, steps):
    s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
    if isinstance(shape, int):
        s.set_launch_variant(shape)
        assert s.launch_variant() == shape
    else:
        s.set_launch(*shape)
    s.upload(s0)
    s.step(steps)
    rep = s.sync()
    q = s.download()
    s.close()
    return q, rep


@pytest.mark.parametrize("n", [16, 8])
@pytest.mark.parametrize("seed,scheme", [(0, 3), (1, 1), (2, 2), (3, 4), (4, 5), (5, 3), (6, 3)])
def test_sweep_matches_block_kernel(ag, seed, scheme, n):
    f, m, cfg, s0 = case(ag, 300 + seed, scheme, n)
    ref, rep0 = run(ag, m, cfg, s0, BLOCK[n], 6)
    ref = ref.reshape(-1, 4)
    first = None
    for shape in SWEEPS:
        q, rep = run(ag, m, cfg, s0, shape, 6)
        assert rep["error"] == 0 and rep["steps"] == rep0["steps"] == 6
        assert abs(rep["time"] - rep0["time"]) <= 1e-6 * rep0["time"]
        if first is None:
            first = q
        else:
            assert np.array_equal(q, first), shape
        q = q.reshape(-1, 4)
        for k in range(4):
            scale = np.abs(ref[:, k]).max()
            assert np.abs(q[:, k] - ref[:, k]).max() <= 1e-6 * scale, (shape, k)


@pytest.mark.parametrize("seed", range(3))
@pytest.mark.parametrize("n", [16, 8])
def test_sweep_rhs_within_fp32_tolerance_of_oracle(ag, oracle, seed, n):
    f, m, cfg, s0 = case(ag, 400 + seed, 3, n)
    ref = oracle.rhs(m, s0, oracle.make_config(n, cfg)).reshape(-1, 4)
    s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
    s.set_launch_variant(SWEEPS[0])
    s.upload(s0)
    got = s.rhs().reshape(-1, 4)
    s.close()
    for k in range(4):
        scale = np.abs(ref[:, k]).max() + 1e-300
        assert np.abs(got[:, k] - ref[:, k]).max() <= 2e-5 * scale, k


@pytest.mark.parametrize("n", [16, 8])
def test_sweep_conserves_on_periodic_hanging_mesh(ag, n):
    f = meshes.two_level_ring(n, periodic=(1, 1))
    cfg = meshes.make_config(n, time_scheme=3, time_steps=10 ** 6, dt=0.01)
    cfg.apply()
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), 5, amp=1e-2)
    s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
    s.set_launch_variant(SWEEPS[0])
    s.upload(s0)
    t0 = s.totals()
    s.step(40)
    t1 = s.totals()
    s.close()
    assert np.all(np.abs(t1 - t0) <= 1e-12 * np.abs(t0) + 1e-13), t1 - t0


@pytest.mark.parametrize("n,shapes", [(16, [(4, 128), (2, 64), (8, 256)]), (8, [(8, 128), (4, 64), (16, 256)])])
def test_sweep_variants_are_the_row_sweep_kernels(ag, n, shapes):
    f, m, cfg, s0 = case(ag, 8, 3, n)
    s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
    assert s.launch_variants()[:3] == shapes
    s.close()


def test_sweep8_with_an_odd_quad_count(ag):
    """Two 8x8 quads per warp: with an odd count the last warp's second
    quad is absent; the result still matches the block kernel and nothing
    is written past the last quad (the state of every quad is finite)."""
    n = 8
    f = meshes.uniform(n, 2, periodic=(1, 1))
    fl = np.zeros(f.num_quads, np.int32)
    fl[5] = 1
    f.refine(fl)
    f.balance()
    assert f.num_quads % 2 == 1
    cfg = meshes.make_config(n, time_scheme=3, time_steps=10 ** 6, dt=0.01)
    cfg.apply()
    m = f.mesh(n)
    s0 = meshes.perturbed(f.initialize(n), 17, amp=2e-2)
    ref, _ = run(ag, m, cfg, s0, BLOCK[n], 5)
    for v in SWEEPS:
        got, rep = run(ag, m, cfg, s0, v, 5)
        assert rep["error"] == 0 and np.isfinite(got).all()
        for k in range(4):
            scale = np.abs(ref[k::4]).max()
            assert np.abs(got[k::4] - ref[k::4]).max() <= 1e-6 * scale, (v, k)


@pytest.mark.parametrize("n,level,default", [(16, 5, 0), (16, 3, 3), (8, 6, 0), (8, 5, 3)])
def test_default_launch_follows_the_mesh_size(ag, n, level, default):
    """The row sweep is the default from 1024 sweep warps on (1024 quads of
    16x16, 2048 of 8x8); smaller meshes take the first block kernel. A
    regrid re-chooses unless the caller set a launch."""
    f = meshes.uniform(n, level, periodic=(1, 1))
    cfg = meshes.make_config(n, time_scheme=3, time_steps=10 ** 6, dt=0.01)
    cfg.apply()
    s = ag.Session(f.mesh(n), cfg, form=ag.FORM_FP32_FLUX)
    assert s.launch_variant() == default
    s.upload(f.initialize(n))
    # coarsen everything once: far fewer quads -> the block kernel
    f.begin_regrid()
    f.coarsen(np.ones(f.num_quads, np.int32), min_level=0)
    f.balance()
    kind, src = f.remap()
    s.regrid(f.mesh(n), kind, src)
    assert s.launch_variant() == 3
    s.set_launch_variant(1)
    s.step(1)
    assert s.launch_variant() == 1
    s.close()
