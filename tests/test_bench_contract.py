"""The benchmark's reference arm runs on the host alone (the oracle port on all cores), so its
JSON line can be checked without a GPU: one line with the keys the benchmark contract names,
the same `config` object as the GPU arm's, and the product library never mapped."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# Runs the reference arm in-process, then reports which shared objects the process mapped.
_DRIVER = r"""
import contextlib, io, json, sys
sys.path.insert(0, {root!r})
sys.argv = ["bench.py", "--impl", "reference", "--workload", "c2", "--steps", "2", "--warmup", "0"]
import bench
out = io.StringIO()
with contextlib.redirect_stdout(out):
    rc = bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({{"rc": rc, "stdout": out.getvalue(), "product_mapped": "libpivb200.so" in maps,
                  "oracle_mapped": "libpivoracle.so" in maps}}))
"""


def test_reference_arm_prints_one_contract_line_without_the_product():
    r = subprocess.run([sys.executable, "-c", _DRIVER.format(root=ROOT)], cwd=ROOT, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["rc"] == 0
    assert res["oracle_mapped"] and not res["product_mapped"], "the reference arm must not load libpivb200.so"
    lines = [l for l in res["stdout"].splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "vectors/s"
    assert d["warmup"] >= 3 and d["steps"] == 2 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    # whole 1024x1024 pairs: 16,129 final-pass vectors each, timed step by step
    assert d["config"]["final_pass_vectors"] == 16129
    assert "2 whole 1024x1024 pairs" in d["cpu_baseline"]["sample"]
    assert abs(d["ms_per_step"] * d["value"] * d["steps"] / 1e3 - 2 * 16129) < 1e-6 * 2 * 16129
    for k in ("workload", "image", "windows", "overlap", "final_pass_vectors", "parallelism", "inputs", "l2"):
        assert k in d["config"], k


def test_both_arms_build_the_same_config():
    """The GPU arm's `config` comes from the same function over the same inputs."""
    sys.path.insert(0, ROOT)
    import numpy as np

    import bench
    wl = dict(bench.WORKLOADS["c2"])
    a = np.zeros((wl["h"], wl["w"]), np.uint16)
    ring = bench.input_ring(a, a)
    assert bench.workload_config(wl, ring, 16129, 1) == bench.workload_config(wl, bench.input_ring(a, a), 16129, 1)
    assert len(ring) * 2 * a.nbytes >= 256 << 20
