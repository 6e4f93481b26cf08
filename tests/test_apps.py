"""The per-technique executables: the reference's flags, exit codes and result
file.  Flag handling runs on the CPU; the result files are checked on the GPU
against the reference's own result files (single run) and against the
reference writer's run order (several runs, --partition)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_path
from set_intersection_b200 import dataset as fmt

BIN = os.path.join(ROOT, "set_intersection_b200", "bin")
APPS = ["ip", "obs", "hi", "bitmap_dynamic", "bitmap_naive", "matrix_multiplication"]


@pytest.fixture(scope="module")
def apps():
    if not all(os.access(os.path.join(BIN, a), os.X_OK) for a in APPS):
        subprocess.run(["make", "-C", os.path.join(ROOT, "set_intersection_b200"), "apps"], check=True,
                       capture_output=True)
    return BIN


def run(app, *args, **kw):
    return subprocess.run([os.path.join(BIN, app), *args], capture_output=True, text=True, timeout=300, **kw)


@pytest.mark.parametrize("app", APPS)
def test_flags_and_exit_codes(apps, app):
    r = run(app, "--help")
    assert r.returncode == 0 and "--input" in r.stdout
    r = run(app)
    assert r.returncode == 1 and "No input dataset given! Exiting..." in r.stdout
    r = run(app, "--input", golden_path("misi_mixed.bin"), "--no-such-flag", "1")
    assert r.returncode == 1
    r = run(app, "--input", "/nonexistent/dataset.bin")
    assert r.returncode == 1


def test_corrupt_dataset_is_rejected(apps, tmp_path):
    raw = open(golden_path("misi_mixed.bin"), "rb").read()
    bad = tmp_path / "bad.bin"
    bad.write_bytes(raw[:-4])
    r = run("ip", "--input", str(bad))
    assert r.returncode == 1 and "corrupt" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("app", APPS)
@pytest.mark.parametrize("name", ["misi_mixed", "misi_onebased", "sisi_uniform", "sisi_skewed", "sisi_extremes"])
def test_result_file_equals_reference(cuda, apps, tmp_path, app, name):
    out = tmp_path / "result.txt"
    r = run(app, "--input", golden_path(f"{name}.bin"), "--output", str(out))
    assert r.returncode == 0, r.stdout + r.stderr
    assert out.read_text() == open(golden_path(f"{name}.std.txt")).read()


@pytest.mark.gpu
@pytest.mark.parametrize("app", APPS)
@pytest.mark.parametrize("partition", [1, 5, 11, 33])
def test_partitioned_runs_follow_reference_order(cuda, apps, tmp_path, app, partition):
    ds = fmt.read_dataset(golden_path("misi_mixed.bin"))
    counts = fmt.parse_result(golden_path("misi_mixed.std.txt"), ds.cardinality)
    out = tmp_path / "result.txt"
    r = run(app, "--input", golden_path("misi_mixed.bin"), "--output", str(out), "--partition", str(partition))
    if app == "bitmap_naive":  # the reference's bitmap_naive has no --partition (src/bitmap_naive.cu:36-41)
        assert r.returncode == 1 and "partition" in r.stdout
        return
    assert r.returncode == 0, r.stdout + r.stderr
    assert out.read_text() == "".join(fmt.format_result_lines(ds.cardinality, counts, partition))


@pytest.mark.gpu
def test_launch_geometry_flags_are_accepted(cuda, apps, tmp_path):
    out = tmp_path / "r.txt"
    r = run("hi", "--input", golden_path("misi_mixed.bin"), "--output", str(out), "--blocks", "64", "--threads",
            "128", "--buckets", "7", "--bucket-size", "9", "--warp", "--path")
    assert r.returncode == 0, r.stdout
    assert out.read_text() == open(golden_path("misi_mixed.std.txt")).read()
