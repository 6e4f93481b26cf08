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
TOOLS = ["txt2bin", "bin2txt"]


@pytest.fixture(scope="module")
def apps():
    if not all(os.access(os.path.join(BIN, a), os.X_OK) for a in APPS + TOOLS):
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


def test_txt2bin_and_bin2txt_match_the_reference_tools(apps, tmp_path):
    """Byte-identical to the reference's own txt2bin / bin2txt outputs
    (tests/golden/text_sets_*.bin were made by them)."""
    r = run("txt2bin", golden_path("text_sets.txt"), str(tmp_path / "x"))
    assert r.returncode == 0, r.stdout
    assert (tmp_path / "x_asc.bin").read_bytes() == open(golden_path("text_sets_asc.bin"), "rb").read()
    assert (tmp_path / "x_desc.bin").read_bytes() == open(golden_path("text_sets_desc.bin"), "rb").read()
    r = run("bin2txt", golden_path("text_sets_asc.bin"), str(tmp_path / "y"))
    assert r.returncode == 0, r.stdout
    ds = fmt.read_dataset(golden_path("text_sets_asc.bin"))
    want = "".join("".join(f"{v} " for v in s) + "\n" for s in ds.sets())
    assert (tmp_path / "y.txt").read_text() == want


@pytest.mark.parametrize("text,msg", [("1 2 3\n5 4\n", "not strictly increasing"), ("1 2 2\n", "not strictly"),
                                      ("1 x 3\n", "not a 32-bit"), ("4294967296\n", "not a 32-bit"),
                                      ("-1 2\n", "not a 32-bit")])
def test_txt2bin_rejects_bad_sets(apps, tmp_path, text, msg):
    src = tmp_path / "bad.txt"
    src.write_text(text)
    r = run("txt2bin", str(src), str(tmp_path / "o"))
    assert r.returncode == 1 and msg in r.stdout


def test_bin2txt_rejects_truncated_file(apps, tmp_path):
    raw = open(golden_path("text_sets_asc.bin"), "rb").read()
    (tmp_path / "t.bin").write_bytes(raw[:-1])
    r = run("bin2txt", str(tmp_path / "t.bin"), str(tmp_path / "o"))
    assert r.returncode == 1
