"""The stage-launch autotuner's JSON cache (host side, no GPU): entries
round-trip through the file, a key's new choice replaces the old one,
malformed lines are skipped, and an empty AMRGPU_TUNE_CACHE keeps choices
in memory only."""
import json
import os

import pytest


@pytest.fixture
def cache_env(ag, tmp_path):
    old = os.environ.get("AMRGPU_TUNE_CACHE")
    path = tmp_path / "sub" / "tune.json"
    os.environ["AMRGPU_TUNE_CACHE"] = str(path)
    ag.lib().amrgpu_tune_cache_reload()
    yield path
    if old is None:
        os.environ.pop("AMRGPU_TUNE_CACHE", None)
    else:
        os.environ["AMRGPU_TUNE_CACHE"] = old
    ag.lib().amrgpu_tune_cache_reload()


def _get(ag, gpu, form, n, nquad):
    import ctypes as C
    q, t, m, ms = C.c_int(), C.c_int(), C.c_int(), C.c_double()
    found = ag.lib().amrgpu_tune_cache_get(gpu.encode(), 148, form, n, nquad, C.byref(q), C.byref(t), C.byref(m),
                                           C.byref(ms))
    return (q.value, t.value, m.value, ms.value) if found else None


def test_cache_round_trip_through_the_file(ag, cache_env):
    L = ag.lib()
    assert L.amrgpu_tune_cache_put(b"NVIDIA B200", 148, 0, 16, 4096, 4, 128, 4, 0.1189) == 0
    assert L.amrgpu_tune_cache_put(b"NVIDIA B200", 148, 1, 8, 3000, 8, 128, 4, 0.05) == 0
    doc = json.loads(cache_env.read_text())
    assert doc["amrgpu_tune"] == 1 and len(doc["entries"]) == 2
    assert doc["entries"][0] == {"gpu": "NVIDIA B200", "sms": 148, "form": 0, "n": 16, "bucket": 12, "qpb": 4,
                                 "threads": 128, "min_blocks": 4, "ms": 0.1189}
    L.amrgpu_tune_cache_reload()  # read back from the file
    assert _get(ag, "NVIDIA B200", 0, 16, 4096) == (4, 128, 4, 0.1189)
    assert _get(ag, "NVIDIA B200", 0, 16, 5000) == (4, 128, 4, 0.1189)  # same bucket: 4096..8191
    assert _get(ag, "NVIDIA B200", 0, 16, 2000) is None                 # other bucket
    assert _get(ag, "NVIDIA B200", 1, 8, 2048) == (8, 128, 4, 0.05)
    assert _get(ag, "NVIDIA H100", 0, 16, 4096) is None


def test_new_choice_replaces_old_and_bad_lines_are_skipped(ag, cache_env):
    L = ag.lib()
    L.amrgpu_tune_cache_put(b"G", 148, 0, 16, 1024, 1, 288, 2, 0.5)
    L.amrgpu_tune_cache_put(b"G", 148, 0, 16, 1500, 4, 128, 4, 0.3)  # same bucket
    text = cache_env.read_text().splitlines()
    assert sum('"gpu": "G"' in ln for ln in text) == 1
    text.insert(1, '{"gpu": "G", "sms": 148, "form": 0, "n": 8, "bucket": garbage}')
    cache_env.write_text("\n".join(text) + "\n")
    L.amrgpu_tune_cache_reload()
    assert _get(ag, "G", 0, 16, 1024) == (4, 128, 4, 0.3)
    assert _get(ag, "G", 0, 8, 1024) is None


def test_empty_path_keeps_choices_in_memory(ag, cache_env, tmp_path):
    os.environ["AMRGPU_TUNE_CACHE"] = ""
    ag.lib().amrgpu_tune_cache_reload()
    ag.lib().amrgpu_tune_cache_put(b"M", 148, 0, 16, 1024, 4, 128, 4, 0.1)
    assert _get(ag, "M", 0, 16, 1024) == (4, 128, 4, 0.1)
    assert not any(tmp_path.rglob("*.json"))
