"""The FP32-flux form's row-sweep stage kernel for 16x16 patches
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

BLOCK = (1, 288)
# variant indices of the row sweep for 16x16 patches: (4,128), (2,64), (8,256)
SWEEPS = [0, 1, 2]


def case(ag, seed, scheme):
    rng = np.random.default_rng(seed)
    n = 16
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


@pytest.mark.parametrize("seed,scheme", [(0, 3), (1, 1), (2, 2), (3, 4), (4, 5), (5, 3), (6, 3)])
def test_sweep_matches_block_kernel(ag, seed, scheme):
    f, m, cfg, s0 = case(ag, 300 + seed, scheme)
    ref, rep0 = run(ag, m, cfg, s0, BLOCK, 6)
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
def test_sweep_rhs_within_fp32_tolerance_of_oracle(ag, oracle, seed):
    f, m, cfg, s0 = case(ag, 400 + seed, 3)
    ref = oracle.rhs(m, s0, oracle.make_config(16, cfg)).reshape(-1, 4)
    s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
    s.set_launch_variant(SWEEPS[0])
    s.upload(s0)
    got = s.rhs().reshape(-1, 4)
    s.close()
    for k in range(4):
        scale = np.abs(ref[:, k]).max() + 1e-300
        assert np.abs(got[:, k] - ref[:, k]).max() <= 2e-5 * scale, k


def test_sweep_conserves_on_periodic_hanging_mesh(ag):
    n = 16
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


def test_sweep_variants_are_the_row_sweep_kernels(ag):
    f, m, cfg, s0 = case(ag, 8, 3)
    s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
    v = s.launch_variants()
    assert v[:3] == [(4, 128), (2, 64), (8, 256)]
    assert s.launch_variant() == 0
    s.close()


def test_sweep_is_the_default_for_16x16_patches(ag):
    f, m, cfg, s0 = case(ag, 7, 3)
    a, _ = run(ag, m, cfg, s0, SWEEPS[0], 3)
    s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
    s.upload(s0)
    s.step(3)
    b = s.download()
    s.close()
    assert np.array_equal(a, b)
