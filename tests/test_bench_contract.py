"""bench.py's reference arm on CPU: one JSON line with the metric, unit and
direction of the GPU arm, a cpu_baseline describing the sample (the
reference's C driver over the restated kernels on all host cores, or the
restatement alone when the reference tree was not built), and an e2e entry
with no host-device traffic; under torchrun only rank 0 prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(args, env_extra=None):
    env = dict(os.environ)
    env.pop("RANK", None)
    env.update(env_extra or {})
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return [line for line in out.stdout.splitlines() if line.strip()]


def test_reference_arm_prints_one_contract_line():
    lines = run_bench(["--impl", "reference", "--steps", "10", "--warmup", "3"])
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"].startswith("RK cell-updates/s")
    assert d["unit"] == "cell-updates/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 10 and d["warmup"] == 3
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in d["config"] and d["ms_per_step"] > 0
    assert cb["same_config"] is True and cb["one_rank"]["value"] > 0


def test_reference_arm_loads_no_product_library():
    """The CPU baseline builds its mesh in NumPy and runs only the
    reference's own C code (oracle/_ref): libamrgpu.so is never mapped."""
    code = ("import sys, json; sys.argv=['bench.py']; sys.path.insert(0, %r); import bench; "
            "cb = bench.cpu_baseline(steps=1, one_rank_steps=1); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'amrgpu': 'libamrgpu' in maps, 'ref': 'libref_physics' in maps}))" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads(out.stdout.strip().splitlines()[-1])
    assert d == {"amrgpu": False, "ref": True}


def test_reference_arm_prints_nothing_on_other_ranks():
    assert run_bench(["--impl", "reference", "--steps", "10", "--warmup", "3"], {"RANK": "1"}) == []
