"""bench.py's reference arm on CPU: one JSON line with the contract's keys
(the GPU arm prints the same keys plus the device measurements)."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl",
                        "reference", "--steps", "1", "--warmup", "3",
                        "--workload", "dc2d_small"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup",
                "ms_per_step", "higher_is_better", "scaling", "vs_baseline",
                "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["higher_is_better"] is False
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["config"]["workload"] == "dc2d_small"


def test_library_path_override():
    """DCT_LIB_PATH selects another build of the same sources (A/B timing);
    unset, the in-tree library is the one loaded."""
    code = "from simpeg_dc_torch_b200 import _native as n; print(n.LIB_PATH)"
    env = dict(os.environ)
    env.pop("DCT_LIB_PATH", None)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=300, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == os.path.join(ROOT, "simpeg_dc_torch_b200", "lib", "libdct.so")
    env["DCT_LIB_PATH"] = "/tmp/other/libdct.so"
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=300, cwd=ROOT, env=env)
    assert r.returncode == 0 and r.stdout.strip() == "/tmp/other/libdct.so"
