"""bench.py's reference arm (oracle/refbench.py) runs the reference's own
host build, camera, eye rays and CPU ray query, and loads nothing of the
product: no liblrt_b200.so mapping, no import of the package.  Small sizes,
a fresh process, no GPU."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import refbench  # noqa: E402

SCRIPT = r"""
import json, sys
sys.path.insert(0, "oracle")
import refbench
m = refbench.run(64, 48, 64, 8, 1, 16, 1, 1e-4, 1e9, steps=2, warmup=3, seconds=1.0, threads=2)
maps = open("/proc/self/maps").read()
print(json.dumps({"value": m["value"], "product_mapped": "liblrt_b200" in maps,
                  "package_imported": any(k.startswith("graphic_lab_task_b200") for k in sys.modules),
                  "libs": sorted({l.split()[-1].rsplit("/", 1)[-1] for l in maps.splitlines() if "oracle/" in l})}))
"""


@pytest.mark.skipif(refbench.available() is not None, reason="reference build absent (make -C oracle ref wl)")
def test_reference_arm_loads_no_product_code():
    r = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["value"] > 0
    assert not out["product_mapped"] and not out["package_imported"]
    assert out["libs"] == ["liblrt_ref_fast.so", "liblrt_workloads.so"]
