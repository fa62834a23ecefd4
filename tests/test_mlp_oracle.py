"""CPU checks of the learned indicator's oracle (oracle/mlp_oracle.py) and
of its host-side pieces: the oracle's own backward pass against finite
differences in FP64, BF16 rounding, the feature normalisation on states
with a known answer, the plain three-class labels, and the library's
deterministic initialisation restated. No GPU needed."""
import numpy as np
import pytest

import meshes
from oracle import mlp_oracle as M


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = M.init_params(3).astype(np.float64)
    x = rng.normal(size=(24, M.NIN))
    y = rng.integers(0, 3, 24)
    _, _, g = M.forward_backward(p, x, y, bf16_mode=False)
    for k in rng.choice(M.NPARAMS, 40, replace=False):
        e = np.zeros_like(p)
        e[k] = 1e-6
        fd = (M.loss_only(p + e, x, y) - M.loss_only(p - e, x, y)) / 2e-6
        assert abs(g[k] - fd) <= 1e-5 * abs(fd) + 1e-9, (k, g[k], fd)


def test_bf16_rounding_is_round_to_nearest_even():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 1e-3, 3.1415927], np.float32)
    got = M.bf16_bits_to_f64(M.f32_to_bf16_bits(vals))
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa (1.0) wins
    assert got[0] == 1.0 and got[1] == 1.0
    assert got[2] == 1.0 + 2 ** -7
    assert got[3] == -2.5
    assert abs(got[4] - 1e-3) <= 2 ** -9 * 1e-3
    assert abs(got[5] - np.pi) <= 2 ** -8 * np.pi


def test_features_of_a_uniform_state_are_zero_and_of_a_jump_are_scaled():
    n = 8
    f = meshes.uniform(n, 1, periodic=(1, 1))
    m = f.mesh(n)
    q = np.zeros((m.ncell, n, n, 4))
    q[..., 0] = 1.3
    q[..., 1] = 0.2
    q[..., 2] = -0.1
    q[..., 3] = 2.9
    x = M.bf16_bits_to_f64(M.features(q.ravel(), m, n))
    assert np.abs(x).max() <= 1e-12  # the patch mean is a rounded sum
    # density step inside quad 0: x0 = S (rho - mean) / mean
    q[0, :, 4:, 0] = 1.3 * 1.1
    x = M.bf16_bits_to_f64(M.features(q.ravel(), m, n)).reshape(-1, 4, 10, 10)
    mean = 1.3 * 1.05
    assert abs(x[0, 0, 5, 1] - M.bf16(M.FEAT_SCALE * (1.3 - mean) / mean)) == 0.0
    assert abs(x[0, 0, 5, 8] - M.bf16(M.FEAT_SCALE * (1.43 - mean) / mean)) == 0.0


def test_features_ring_comes_from_the_flux_paired_neighbour():
    n = 8
    f = meshes.uniform(n, 1, periodic=(1, 1))
    m = f.mesh(n)
    rng = np.random.default_rng(1)
    q = np.ones((m.ncell, n, n, 4)) + 0.01 * rng.random((m.ncell, n, n, 4))
    kind, nbr = M.sides(m)
    assert np.all(kind == 1)
    x = M.bf16_bits_to_f64(M.features(q.ravel(), m, n)).reshape(-1, 4, 10, 10)
    # the right ring of quad 0 holds the left column of its x+ neighbour
    r = nbr[0, 1, 0]
    mean = q[0, :, :, 0].mean()
    want = M.bf16(M.FEAT_SCALE * (q[r, :, 0, 0] - mean) / mean)
    assert np.max(np.abs(x[0, 0, 1:9, 9] - want)) <= 2 ** -7 * np.abs(want).max()


def test_plain_labels_and_jumps():
    assert list(M.labels([0.0, 0.004, 0.005, 0.019, 0.02, 0.5], 0.02)) == [0, 0, 2, 2, 1, 1]
    n = 4
    f = meshes.uniform(n, 1, periodic=(1, 1))
    m = f.mesh(n)
    q = np.ones((m.ncell, n, n, 4))
    q[0, 2, 1, 0] = 1.5  # a cell of quad 0: jump 0.5 inside it
    J = M.jumps(q.ravel(), m, n)
    assert J[0] == 0.5 and np.all(J[1:] == 0.0)


def test_init_params_is_deterministic_and_bounded():
    a = M.init_params(7)
    b = M.init_params(7)
    c = M.init_params(8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    W1 = a[: M.NH1 * M.NIN]
    assert np.abs(W1).max() <= 1.0 / np.sqrt(M.NIN) + 1e-7
    assert a.size == M.NPARAMS == 59779
