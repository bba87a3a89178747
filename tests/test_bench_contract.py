"""bench.py's reference arm runs on the host cores only (the reference built from its sources in
oracle/_ref), so its JSON contract is checked here without a GPU."""
import json
import os
import subprocess
import sys

import pytest

from helpers import require_reference_binary

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    require_reference_binary()
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3", "--workload", "poisson2d_l7_fp64"], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "ms" and d["higher_is_better"] is False
    assert d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1 and d["value"] > 0
    assert d["config"]["iterations"] == 5   # the reference's own iteration count at L7
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
