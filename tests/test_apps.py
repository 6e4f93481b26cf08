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
TOOLS = ["txt2bin", "bin2txt", "degree_cdf", "generate_dataset"]


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


# ---------------------------------------------------------------- dataset tools --
DEGREE_FILES = ("degree_set", "degree_element", "set_cdf", "element_cdf")


def _degree_cdf_matches(tmp_path, name, *flags):
    prefix = str(tmp_path / name)
    r = run("degree_cdf", golden_path(f"{name}.bin"), prefix, *flags)
    assert r.returncode == 0 and "Finished" in r.stdout, r.stdout
    for t in ("degree_set", "degree_element", "set_cdf"):
        assert open(f"{prefix}_{t}.txt").read() == open(golden_path(f"{name}_{t}.txt")).read(), t
    ref_el = open(golden_path(f"{name}_element_cdf.txt")).read()
    assert ref_el == open(golden_path(f"{name}_set_cdf.txt")).read()  # the reference's slip
    ds = fmt.read_dataset(golden_path(f"{name}.bin"))
    inv = np.bincount(np.asarray(ds.elements, dtype=np.int64), minlength=ds.universe)[:ds.universe]
    lens = np.sort(inv)
    want = "".join(f"{a} {b}\n" for a, b in zip(lens, np.cumsum(lens.astype(np.int64) ** 2)))
    assert open(f"{prefix}_element_cdf.txt").read() == want


@pytest.mark.parametrize("name", ["degree_ties", "degree_zipf"])
def test_degree_cdf_matches_the_reference_tool(apps, tmp_path, name):
    """degree_set, degree_element and set_cdf byte-identical to the reference's
    degree_cdf outputs (tests/golden/<name>_*.txt were made by it); element_cdf
    holds the element CDF, where the reference writes its set CDF a second time."""
    _degree_cdf_matches(tmp_path, name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["degree_ties", "degree_zipf"])
def test_degree_cdf_on_the_device_matches_the_reference_tool(apps, cuda, tmp_path, name):
    """The same files with the inverted-list lengths and per-set sums computed
    by si_degree_stats on the GPU."""
    _degree_cdf_matches(tmp_path, name, "--device")


def test_degree_cdf_usage_and_bad_input(apps, tmp_path):
    assert run("degree_cdf").returncode == 1
    assert run("degree_cdf", golden_path("degree_ties.bin"), str(tmp_path / "y"), "--gpu").returncode == 1
    bad = tmp_path / "bad.bin"
    bad.write_bytes(open(golden_path("degree_ties.bin"), "rb").read()[:-4])
    assert run("degree_cdf", str(bad), str(tmp_path / "x")).returncode == 1


def _gen(tmp_path, *args):
    r = run("generate_dataset", "--output", str(tmp_path / "g"), *args)
    assert r.returncode == 0, r.stdout
    return r


@pytest.mark.parametrize("args,name", [
    (["--universe", "100000", "--k", "10", "--iterations", "5000"], "uniform_10_100000_5000"),
    (["--universe", "1000", "--k", "4", "--distribution", "normal", "--iterations", "200", "--stdev", "2"],
     "normal_4_1000_200_2.000000"),
    (["--universe", "1000", "--k", "5", "--distribution", "bernoulli", "--prob", "0.1"], "bernoulli_5_1000_0.100000"),
    (["--universe", "5000", "--k", "6", "--distribution", "zipf", "--iterations", "300"], "zipf_6_5000_300_0.900000"),
])
def test_generate_dataset_files(apps, tmp_path, args, name):
    """Output names as the reference builds them; valid datasets of sorted
    distinct values in [1, universe]; the two files hold the same sets, by
    size ascending and descending."""
    _gen(tmp_path, *args)
    asc = fmt.read_dataset(str(tmp_path / f"g_asc_{name}.bin"))
    desc = fmt.read_dataset(str(tmp_path / f"g_desc_{name}.bin"))
    k = int(args[args.index("--k") + 1])
    U = int(args[args.index("--universe") + 1])
    assert asc.cardinality == desc.cardinality == k and asc.universe == desc.universe == U
    sa, sd = [np.asarray(s) for s in asc.sets()], [np.asarray(s) for s in desc.sets()]
    for s in sa:
        assert s.size == 0 or (np.all(np.diff(s.astype(np.int64)) > 0) and s[0] >= 1 and s[-1] <= U)
    assert [s.size for s in sa] == sorted(s.size for s in sa)
    assert [s.size for s in sd] == sorted((s.size for s in sd), reverse=True)
    assert sorted(map(bytes, sa)) == sorted(map(bytes, sd))


def test_generate_dataset_is_seeded_and_thread_independent(apps, tmp_path):
    base = ["--universe", "50000", "--k", "12", "--iterations", "3000", "--distribution", "zipf"]
    name = "g_asc_zipf_12_50000_3000_0.900000.bin"
    a, b, c = tmp_path / "a", tmp_path / "b", tmp_path / "c"
    for d in (a, b, c):
        d.mkdir()
    _gen(a, *base, "--seed", "7", "--threads", "1")
    _gen(b, *base, "--seed", "7", "--threads", "5")
    _gen(c, *base, "--seed", "8")
    assert (a / name).read_bytes() == (b / name).read_bytes()
    assert (a / name).read_bytes() != (c / name).read_bytes()


def test_generate_dataset_distributions(apps, tmp_path):
    """Bernoulli sizes near p U; Zipf puts the most draws on the smallest values."""
    _gen(tmp_path, "--universe", "20000", "--k", "40", "--distribution", "bernoulli", "--prob", "0.05")
    ds = fmt.read_dataset(str(tmp_path / "g_asc_bernoulli_40_20000_0.050000.bin"))
    sizes = np.asarray(ds.sizes, dtype=np.float64)
    assert abs(sizes.mean() - 1000) < 4 * np.sqrt(1000 * 0.95 / 40)
    _gen(tmp_path, "--universe", "1000", "--k", "50", "--distribution", "zipf", "--iterations", "200",
         "--skew", "1.2")
    ds = fmt.read_dataset(str(tmp_path / "g_asc_zipf_50_1000_200_1.200000.bin"))
    counts = np.bincount(np.asarray(ds.elements, dtype=np.int64), minlength=1001)
    assert counts[1] == 50 and counts[1] >= counts[2] >= counts[500]


@pytest.mark.parametrize("args,msg", [([], "No universe given! Exiting..."),
                                      (["--universe", "10", "--distribution", "poisson"], "unknown distribution"),
                                      (["--universe", "10", "--prob", "x"], "failed to parse"),
                                      (["--universe", "10", "--nope", "1"], "does not exist")])
def test_generate_dataset_flag_errors(apps, tmp_path, args, msg):
    r = run("generate_dataset", "--output", str(tmp_path / "g"), *args)
    assert r.returncode == 1 and msg in r.stdout
    assert run("generate_dataset", "--help").returncode == 0


@pytest.mark.gpu
@pytest.mark.parametrize("app", ["ip", "bitmap_dynamic", "matrix_multiplication"])
@pytest.mark.parametrize("partition", [7, 10000])
def test_binary_counts_dump(cuda, apps, tmp_path, app, partition):
    """--output-binary: u32 k, u32 0, u64 C(k,2), u32 counts in triangular order,
    equal to the reference's result file (streamed runs and whole-triangle paths)."""
    ds = fmt.read_dataset(golden_path("misi_mixed.bin"))
    want = fmt.parse_result(golden_path("misi_mixed.std.txt"), ds.cardinality)
    dump = tmp_path / "counts.bin"
    r = run(app, "--input", golden_path("misi_mixed.bin"), "--output-binary", str(dump), "--partition", str(partition))
    assert r.returncode == 0, r.stdout + r.stderr
    raw = dump.read_bytes()
    k, zero = np.frombuffer(raw[:8], dtype=np.uint32)
    pairs = np.frombuffer(raw[8:16], dtype=np.uint64)[0]
    assert (k, zero, pairs) == (ds.cardinality, 0, want.size)
    assert np.array_equal(np.frombuffer(raw[16:], dtype=np.uint32).astype(np.uint64), want)
