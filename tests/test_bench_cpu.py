"""bench.py's reference arm on the host: the JSON line of the reference's CPU
path (oracle/_ref, the reference's MeshDist and octree compiled from source)
on a reduced workload (10 vessels x 40 nuclei, where the join refines some
2e5 triangle pairs) carries every key of the line the GPU arm prints, the
same workload keys in `config`, and its process never maps this
repository's library (the tiles are generated in a child process)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_line(pkg):
    if not (ROOT / "oracle" / "_ref" / "libtdp_ref.so").exists():
        pytest.skip("the reference library is built from the reference sources")
    argv = ["bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1", "--vessels", "10",
            "--nuclei-per-vessel", "40"]
    # run bench.py in a process that reports, at exit, whether libtdp.so was mapped
    code = ("import atexit, runpy, sys; "
            "atexit.register(lambda: sys.stderr.write('LIBTDP_MAPPED=%d\\n' % ('libtdp.so' in open('/proc/self/maps').read()))); "
            f"sys.argv = {argv!r}; runpy.run_path('bench.py', run_name='__main__')")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0 and d["higher_is_better"] is True
    assert d["unit"] == "tri-pairs/s" and d["e2e"]["unit"] == d["unit"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "10 vessels x 40 nuclei" in d["config"]["workload"]
    c = d["config"]
    assert c["n_nuclei"] == 400 and c["n_vessels"] == 10 and c["tau"] == 400.0 and c["seed"] == 20260002
    assert "LIBTDP_MAPPED=0" in out.stderr, out.stderr[-2000:]
