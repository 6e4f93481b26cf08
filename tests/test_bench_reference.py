"""bench.py's reference arm on CPU: it times the reference's own executable on
the workload's pair without loading the engine's library, and describes the
workload exactly as the engine's arm does."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import os, runpy, sys, io, contextlib
sys.argv = ["bench.py", "--impl", "reference", "--workload", "sisi_plain", "--steps", "3", "--warmup", "3"]
buf = io.StringIO()
with contextlib.redirect_stdout(buf):
    try:
        runpy.run_path(os.path.join(sys.argv0_root, "bench.py"), run_name="__main__")
    except SystemExit:
        pass
maps = open("/proc/self/maps").read()
print(buf.getvalue().strip().splitlines()[-1])
print("ENGINE_LOADED" if "libsi_b200" in maps else "ENGINE_NOT_LOADED")
"""


def test_reference_arm_runs_without_the_engine(tmp_path):
    env = dict(os.environ, SI_BENCH_CACHE=str(tmp_path))
    code = "import sys; sys.argv0_root = %r\n" % ROOT + PROBE
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line, loaded = r.stdout.strip().splitlines()[-2:]
    assert loaded == "ENGINE_NOT_LOADED"
    d = json.loads(line)
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "Gelem/s"
    assert d["config"]["workload"] == "sisi_plain" and d["config"]["n_a"] == 1 << 20
    assert set(d["config"]) == {"workload", "desc", "materialize", "n_a", "n_b", "l2", "parallelism"}
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("reference", "port")


def test_reference_pair_equals_engine_pair(tmp_path, monkeypatch):
    """The reference arm's pair is the engine arm's pair, set for set."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setattr(bench, "CACHE_DIR", str(tmp_path / "ref"))
    a, b = bench.ref_pair("sisi_plain")
    monkeypatch.setattr(bench, "CACHE_DIR", str(tmp_path / "eng"))
    a2, b2 = bench.make_pair("sisi_plain")
    assert (a == a2).all() and (b == b2).all()


def test_extras_and_flags_are_well_formed():
    """Every short run a default bench adds names a known workload with a
    positive step count, and the SISI flags parse."""
    sys.path.insert(0, ROOT)
    import bench
    for wl, extra, steps in bench.EXTRAS:
        assert wl in bench.WORKLOADS
        assert isinstance(steps, int) and steps >= 1
        assert "--technique" in extra
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True, text=True,
                       timeout=120, cwd=ROOT)
    assert r.returncode == 0
    for flag in ("--no-techniques", "--no-extras", "--bucket-times", "--count-only"):
        assert flag in r.stdout
