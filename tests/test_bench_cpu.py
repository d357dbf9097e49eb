"""bench.py's reference arm on CPU: the line it prints for a uniform workload.

The reference arm times the oracle (the reference algorithm's CPU
restatement) on the whole grid of the same workload, and reports exactly the
``config`` the GPU arm reports, so that the two lines describe one workload.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_reference_arm_line_has_the_same_config():
    sys.path.insert(0, ROOT)
    import bench
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "kh256",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["config"] == json.loads(json.dumps(bench._config("kh256")))
    assert line["config"]["cells"] == 256 * 256
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert "whole 256^2 grid" in line["cpu_baseline"]["sample"]


def test_configs_are_static_per_workload():
    sys.path.insert(0, ROOT)
    import bench
    c = bench._config("ot128")
    assert c["cells"] == 128 ** 3 and c["blocks"] == 512 and c["nw"] == 9
    assert "no flush" in c["l2"]
    assert "flushed" in bench._config("kh256")["l2"]
    assert set(bench._config("ens512")) == {"workload"}
