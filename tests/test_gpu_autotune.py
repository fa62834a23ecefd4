"""The library's stage-launch autotuner on the GPU: a session tunes on its
first step, stores the choice, a later session with the same key uses the
stored choice without timing, the FP32-flux form only ever switches within
the default's bit-identical family, and the tuned run is bit-identical to
the default launch."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

os.environ.setdefault("AMRGPU_QUIET", "1")


@pytest.fixture
def cache_env(ag, tmp_path):
    old = {k: os.environ.get(k) for k in ("AMRGPU_TUNE_CACHE", "AMRGPU_AUTOTUNE")}
    os.environ["AMRGPU_TUNE_CACHE"] = str(tmp_path / "tune.json")
    os.environ.pop("AMRGPU_AUTOTUNE", None)
    ag.lib().amrgpu_tune_cache_reload()
    yield tmp_path / "tune.json"
    for k, v in old.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v
    ag.lib().amrgpu_tune_cache_reload()


def _vortex(ag, level, form):
    from amrgpu import workloads as W
    return W.vortex_1024(level=level, form=form, final_time=0.0)


def test_tunes_once_then_reuses_the_stored_choice(ag, oracle, cache_env):
    f, m, cfg, s0 = _vortex(ag, 5, 0)  # 1024 quads of 16x16
    a = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    a.upload(s0)
    l0 = a.launch_count()
    a.step(2)
    a.sync()
    tuned_launches = a.launch_count() - l0
    nvar = len(a.launch_variants())
    assert tuned_launches >= 2 * 3 + 4 * nvar  # 2 RK3 steps + 4 timing launches per variant
    assert cache_env.exists()
    chosen = a.launch_variant()
    got = a.download()
    a.close()
    # a second session with the same key: no timing, same choice
    b = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    b.upload(s0)
    l0 = b.launch_count()
    b.step(2)
    b.sync()
    assert b.launch_count() - l0 == 2 * 3
    assert b.launch_variant() == chosen
    # the tuned run equals the oracle bit for bit
    ref = s0.copy()
    oc = oracle.make_config(16, cfg)
    oc.time_steps = 2
    oracle.evolve(m, ref, oc)
    assert np.array_equal(got, ref)
    assert np.array_equal(b.download(), ref)
    b.close()


def test_a_stored_choice_drives_the_session(ag, cache_env):
    """A choice stored for the session's key (here the last FP64 variant,
    not the default) is what a fresh session runs with after its first step."""
    import json
    from amrgpu._lib import lib
    f, m, cfg, s0 = _vortex(ag, 5, 0)
    s = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    s.upload(s0)
    s.autotune()  # stores an entry: the file then names this GPU and its SM count
    e = json.loads(cache_env.read_text())["entries"][0]
    k = len(s.launch_variants()) - 1
    qpb, thr, mb, _ = s.launch_variant_info(k)
    s.close()
    assert lib().amrgpu_tune_cache_put(e["gpu"].encode(), e["sms"], 0, 16, m.ncell, qpb, thr, mb, 0.001) == 0
    t = ag.Session(m, cfg, form=ag.FORM_FP64_EXACT)
    t.upload(s0)
    t.step(1)
    t.sync()
    assert t.launch_variant() == k
    t.close()


def test_fp32_form_stays_in_its_bit_identical_family(ag, cache_env):
    f, m, cfg, s0 = _vortex(ag, 6, 1)  # 4096 quads: the default is the row sweep
    s = ag.Session(m, cfg, form=ag.FORM_FP32_FLUX)
    s.upload(s0)
    default = s.launch_variant()
    r0 = s.rhs()
    s.autotune(retime=True)
    assert s.launch_variant_info(default)[3] == 1  # a row sweep
    assert s.launch_variant_info(s.launch_variant())[3] == 1
    s.upload(s0)
    assert np.array_equal(s.rhs(), r0)
    s.close()


def test_evolve_entry_point_tunes_its_session(ag, oracle, cache_env):
    f, m, cfg, s0 = _vortex(ag, 5, 0)
    cfg["time_steps"] = 4
    cfg.apply()
    got = s0.copy()
    res = ag.evolve_solver(m, got, 0)
    assert res["error"] == 0 and res["istep"] == 4
    assert cache_env.exists()
    ref = s0.copy()
    oracle.evolve(m, ref, oracle.make_config(16, cfg))
    assert np.array_equal(got, ref)
