"""bench.py's reference arm (the CPU port of the reference's algorithm timed on
the host) builds its inputs with the oracle's restatement of the generator and
maps no product library: run in a fresh process, its JSON line is complete and
libds_b200.so is absent from the process's mappings."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SNIPPET = r"""
import contextlib, io, json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--workload", "plain_small", "--steps", "2", "--warmup", "0",
            "--concurrency", "2"]
buf = io.StringIO()
with contextlib.redirect_stdout(buf):
    runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print(json.dumps({"line": buf.getvalue().strip(), "product": "libds_b200" in maps, "oracle": "libds_oracle" in maps}))
"""


def test_reference_arm_loads_only_the_oracle():
    out = subprocess.run([sys.executable, "-c", SNIPPET], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    r = json.loads(out.stdout.strip().splitlines()[-1])
    line = json.loads(r["line"])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "LPs/s"
    assert line["statuses"] == ["optimal"]
    assert r["oracle"] and not r["product"]
