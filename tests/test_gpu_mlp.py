"""The learned refinement indicator on the GPU against the CPU oracle
(oracle/mlp_oracle.py): tensor-core forward pass and gradient of the
cross-entropy, patch features, density jumps and plain labels; then
training on seeded vortex runs, inference on unseen seeds, the judge and
the fallback of the AMR loop.

Tolerances: the GPU rounds to BF16 at the same points as the oracle, and
differs from it by FP32 accumulation order and FP32 GELU, which moves a
value across a BF16 rounding boundary now and then: logits within 2e-2
absolute, every gradient tensor within 1e-2 relative (L2) with cosine
>= 0.9999; features bit-equal except for at most 0.5% of entries one BF16
ulp apart; jumps bit-equal (same FP64 operations, max is order-free).
"""
import os

import numpy as np
import pytest

import meshes

pytestmark = pytest.mark.gpu
os.environ.setdefault("AMRGPU_QUIET", "1")


@pytest.fixture(scope="module")
def L(ag):
    from amrgpu import learned
    return learned


@pytest.fixture(scope="module")
def M():
    from oracle import mlp_oracle
    return mlp_oracle


def _features(rng, B, M):
    x = rng.normal(scale=1.5, size=(B, M.NIN)).astype(np.float32)
    return M.f32_to_bf16_bits(x)


@pytest.mark.parametrize("B", [128, 293, 1024])
def test_forward_logits_match_oracle(L, M, B):
    rng = np.random.default_rng(B)
    m = L.Mlp(seed=5)
    p = M.init_params(5)
    assert np.array_equal(m.get_params(), p)
    xb = _features(rng, B, M)
    got = m.predict(xb)
    want, _, _ = M.forward_backward(p, M.bf16_bits_to_f64(xb), np.zeros(B, np.int64))
    assert np.abs(got - want).max() <= 2e-2, np.abs(got - want).max()
    m.close()


@pytest.mark.parametrize("B", [256, 600, 1000])
def test_gradient_matches_oracle(L, M, B):
    rng = np.random.default_rng(100 + B)
    m = L.Mlp(seed=11)
    p = M.init_params(11).astype(np.float64)
    # larger weights than the initialisation so every layer carries signal
    p = (p * 3.0).astype(np.float32)
    m.set_params(p)
    xb = _features(rng, B, M)
    y = rng.integers(0, 3, B).astype(np.int32)
    logits, g, loss = m.grad(xb, y)
    L_ref, loss_ref, g_ref = M.forward_backward(p.astype(np.float64), M.bf16_bits_to_f64(xb), y)
    assert np.abs(logits - L_ref).max() <= 2e-2
    assert abs(loss - loss_ref) <= 1e-3 * abs(loss_ref)
    o = 0
    for name, k in (("W1", 128 * 400), ("b1", 128), ("W2", 64 * 128), ("b2", 64), ("W3", 3 * 64), ("b3", 3)):
        a, b = g[o:o + k].astype(np.float64), g_ref[o:o + k]
        o += k
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
        assert rel <= 1e-2 and cos >= 0.9999, (name, rel, cos)
    m.close()


@pytest.mark.parametrize("n,which", [(8, "hanging"), (16, "hanging"), (8, "uniform")])
def test_features_and_jumps_match_oracle(ag, L, M, n, which):
    if which == "hanging":
        f = meshes.hanging(n, level=2, refine=(3, 6, 9), periodic=(1, 0))
    else:
        f = meshes.uniform(n, 2, periodic=(1, 1))
    cfg = meshes.make_config(n, ic=1, h=4.0)
    cfg.apply()
    soln = meshes.perturbed(f.initialize(n), 3, amp=3e-2)
    m = f.mesh(n)
    s = ag.Session(m, cfg, form=1)
    s.upload(soln)
    x = L.session_features(s)
    xr = M.features(soln, m, n)
    diff = x != xr
    assert diff.mean() <= 5e-3, diff.mean()
    if diff.any():
        ulp = np.abs(x[diff].astype(np.int64) - xr[diff].astype(np.int64))
        assert ulp.max() <= 1
    J = L.session_jumps(s)
    assert np.array_equal(J, M.jumps(soln, m, n))
    s.close()


def test_dataset_append_and_relabel(ag, L, M):
    n = 8
    f = meshes.hanging(n, level=2, refine=(3, 6), periodic=(1, 1))
    cfg = meshes.make_config(n, ic=1, h=4.0)
    cfg.apply()
    soln = meshes.perturbed(f.initialize(n), 4, amp=2e-2)
    m = f.mesh(n)
    s = ag.Session(m, cfg, form=1)
    s.upload(soln)
    mlp = L.Mlp(seed=0)
    tol = 0.01
    assert mlp.append(s, tol) == m.ncell
    y0 = mlp.labels()
    assert np.array_equal(y0, M.labels(M.jumps(soln, m, n), tol))
    s.step(3)
    s.sync()
    mlp.relabel(s, 0, tol)
    assert np.array_equal(mlp.labels(), M.labels(M.jumps(s.download(), m, n), tol))
    assert mlp.append(s, tol) == 2 * m.ncell
    mlp.clear()
    assert mlp.size() == 0
    mlp.close()
    s.close()


def test_dataset_cover_keeps_the_finer_demand(ag, L, M):
    """Covering labels: a row's label merged with the plain class of a later
    state of the same mesh is refine where either asks for it, coarsen where
    both do, keep otherwise."""
    tol = 0.02
    f, cfg, soln, _ = L.vortex_amr(904, 8, 3, 5, tol)
    m = f.mesh(8)
    s = ag.Session(m, cfg, form=1)
    s.upload(soln)
    mlp = L.Mlp(seed=0)
    assert mlp.append(s, tol) == m.ncell
    ya = M.labels(M.jumps(s.download(), m, 8), tol)
    s.step(60)
    s.sync()
    mlp.cover(s, 0, tol)
    yb = M.labels(M.jumps(s.download(), m, 8), tol)
    assert not np.array_equal(ya, yb)
    assert (ya == L.REFINE).any() and (ya == L.COARSEN).any()
    want = np.where((ya == L.REFINE) | (yb == L.REFINE), L.REFINE,
                    np.where((ya == L.COARSEN) & (yb == L.COARSEN), L.COARSEN, L.KEEP))
    assert np.array_equal(mlp.labels(), want)
    mlp.close()
    s.close()


def test_train_epoch_matches_oracle_adamw_step(ag, L, M):
    """One AdamW step on one batch: the GPU update equals the oracle's
    gradient fed through AdamW (bias-corrected, decay on weights only)."""
    n = 8
    f = meshes.uniform(n, 4, periodic=(1, 1))
    cfg = meshes.make_config(n, ic=1, h=4.0)
    cfg.apply()
    soln = meshes.perturbed(f.initialize(n), 9, amp=5e-2)
    m = f.mesh(n)
    s = ag.Session(m, cfg, form=1)
    s.upload(soln)
    mlp = L.Mlp(seed=2)
    mlp.append(s, 0.02)
    p0 = mlp.get_params().astype(np.float64)
    B = 128
    perm = np.arange(B, dtype=np.int32)
    x = M.bf16_bits_to_f64(M.features(soln, m, n)[:B])
    y = mlp.labels()[:B]
    lr, wd = 1e-3, 1e-2
    loss, acc = mlp.train_epoch(perm, B, lr, wd)
    _, loss_ref, g = M.forward_backward(p0, x, y)
    assert abs(loss - loss_ref) <= 1e-3 * abs(loss_ref)
    # first Adam step: m_hat = g, v_hat = g^2 -> w -= lr (g/(|g|+eps) + wd w)
    decay = np.ones(M.NPARAMS)
    o = 0
    for k, is_w in ((128 * 400, 1), (128, 0), (64 * 128, 1), (64, 0), (3 * 64, 1), (3, 0)):
        decay[o:o + k] = is_w
        o += k
    want = p0 - lr * (g / (np.abs(g) + 1e-8) + wd * decay * p0)
    got = mlp.get_params().astype(np.float64)
    step = np.abs(want - p0)
    big = np.abs(g) > 1e-4  # sign(g) is well defined there
    assert np.abs(got - want)[big].max() <= 1e-6 + 1e-3 * step[big].max()
    mlp.close()
    s.close()


# ------------------------------------------------------------------ training and use
N8, LO, HI, TOL = 8, 3, 5, 0.02


@pytest.fixture(scope="module")
def trained(L):
    """A model trained on 8 seeded vortex runs (levels 3-5, 8x8 patches)
    with look-ahead labels (the plain class 5 steps later, at the next
    regrid), 12 epochs of AdamW."""
    m = L.Mlp(seed=1)
    L.collect(m, range(8), N8, LO, HI, TOL, regrid_interval=5, regrids=15, lookahead=True)
    hist, _ = L.train(m, epochs=12, batch=1024, lr=2e-3, seed=0)
    yield m, hist
    m.close()


def test_training_reduces_loss_and_generalises_to_unseen_seeds(ag, L, trained):
    m, hist = trained
    assert hist[-1][0] < 0.6 * hist[0][0], hist
    assert hist[-1][1] >= 0.85, hist
    agree = []
    for seed in (900, 901):
        f, cfg, soln, _ = L.vortex_amr(seed, N8, LO, HI, TOL)
        s = ag.Session(f.mesh(N8), cfg, form=1)
        s.upload(soln)
        for _ in range(6):
            pred = m.predict(L.session_features(s)).argmax(1)
            s.step(5)
            s.sync()
            later = L.plain_classes(L.session_jumps(s), TOL)
            agree.append((pred == later).mean())
            L.regrid_by_classes(f, s, N8, later, LO, HI)
        s.close()
    assert np.mean(agree) >= 0.80, agree


def test_learned_tags_equal_argmax_of_predict_and_judge_counts(ag, L, trained):
    m, _ = trained
    f, cfg, soln, _ = L.vortex_amr(902, N8, LO, HI, TOL)
    s = ag.Session(f.mesh(N8), cfg, form=1)
    s.upload(soln)
    tags, j = m.tags(s, TOL, judge_fraction=0.5, seed=3)
    assert np.array_equal(tags, m.predict(L.session_features(s)).argmax(1))
    plain = L.plain_classes(L.session_jumps(s), TOL)
    assert 0 < j["judged"] < s.mesh.ncell
    assert j["disagree"] <= j["judged"]
    # the judged quads are a subset: the disagreement cannot exceed the total one
    assert j["disagree"] <= int((tags != plain).sum())
    assert j["coarser"] <= j["disagree"]
    # every quad judged: both counts over the whole mesh
    tags, j = m.tags(s, TOL, judge_fraction=1.0, seed=3)
    assert j["judged"] == s.mesh.ncell
    assert j["disagree"] == int((tags != plain).sum())
    assert j["coarser"] == int((((plain == L.REFINE) & (tags != L.REFINE)) |
                                ((tags == L.COARSEN) & (plain != L.COARSEN))).sum())
    s.close()


def test_amr_loop_with_learned_indicator_and_fallback(ag, L, trained):
    """What the trained network gains: on an unseen seed the learned run
    keeps the density error against the exact vortex within 10% of the
    plain-indicator run's (it is lower on most seeds) with fewer cells; the
    judge keeps it; an untrained model is caught at its first regrid."""
    m, _ = trained
    f, cfg, soln, par = L.vortex_amr(903, N8, LO, HI, TOL)
    s, r = L.run(f, soln, N8, cfg, final_time=1.0, regrid_interval=5, min_level=LO, max_level=HI, tol=TOL, mlp=m,
                 judge_fraction=0.2)
    err_l = L.l1_rho_vs_exact(s.mesh, s.download(), N8, r["time"], par)
    s.close()
    assert r["fallback_at"] is None and r["judged"] > 0 and r["disagree_rate"] <= 0.35, r
    f, cfg, soln, par = L.vortex_amr(903, N8, LO, HI, TOL)
    s, rp = L.run(f, soln, N8, cfg, final_time=1.0, regrid_interval=5, min_level=LO, max_level=HI, tol=TOL)
    err_p = L.l1_rho_vs_exact(s.mesh, s.download(), N8, rp["time"], par)
    s.close()
    assert err_l <= 1.10 * err_p, (err_l, err_p)
    assert r["mean_cells"] < rp["mean_cells"], (r["mean_cells"], rp["mean_cells"])
    # an untrained model is caught by the judge at its first regrid
    bad = L.Mlp(seed=77)
    f, cfg, soln, _ = L.vortex_amr(903, N8, LO, HI, TOL)
    s, rb = L.run(f, soln, N8, cfg, final_time=0.5, regrid_interval=5, min_level=LO, max_level=HI, tol=TOL, mlp=bad,
                  judge_fraction=0.2)
    s.close()
    bad.close()
    assert rb["fallback_at"] == 0, rb


def test_checked_run_falls_back_beyond_the_l1_bound(ag, L, trained):
    m, _ = trained

    def make():
        f, cfg, soln, _ = L.vortex_amr(904, N8, LO, HI, TOL)
        return f, cfg, soln

    keep = L.run_checked(make, N8, 0.5, LO, HI, TOL, m, l1_bound=1.0)
    assert not keep["fallback"] and keep["l1_rho_vs_plain"] < 1e-2
    keep["session"].close()
    strict = L.run_checked(make, N8, 0.5, LO, HI, TOL, m, l1_bound=0.0)
    assert strict["fallback"] == (strict["l1_rho_vs_plain"] > 0.0)
    strict["session"].close()
