"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Inputs are small seeded datasets written in the reference's binary format
(numpy's PCG64, independent of the engine's own generator).  Outputs come from
the reference's own CPU executables, compiled from the reference sources by
`make -C oracle ref` into oracle/_ref/:

  <name>.std.txt      stdintersection  --input <name>.bin --output ...  (src/std_set_intersection.cpp)
  <name>.serial.txt   serial_intersect --input <name>.bin --output ...  (src/serial_intersect.cpp)
  <name>.bitset.txt   boost_bitset     --input <name>.bin --output ...  (src/boost_bitset.cpp; only when
                                                                          universe + 1 fits its bitset)
  <name>.elements.bin ref_elements <name>.bin ...   (std::set_intersection of sets 0 and 1 through the
                                                     reference's readDataset): u64 n + u32[n]
  text_sets_asc.bin / text_sets_desc.bin            txt2bin text_sets.txt text_sets (src/txt2bin.cpp)
  degree_<name>.bin, degree_<name>_{degree_set,degree_element,set_cdf,element_cdf}.txt
                                                    degree_cdf <bin> <prefix> (src/degree_cdf.cpp) on
                                                    datasets whose values stay below the universe
  text_roundtrip.txt                                bin2txt text_sets_asc.bin text_roundtrip (src/bin2txt.cpp)

Run from the repository root in a container that has the reference checkout:
    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from set_intersection_b200 import dataset as fmt  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")


def uniq_sorted(rng, n, lo, hi):
    return np.sort(rng.choice(np.arange(lo, hi, dtype=np.int64), size=n, replace=False)).astype(np.uint32)


def datasets():
    rng = np.random.default_rng(20240601)
    out = {}
    # single pair, plain: equal sizes, dense overlap
    out["sisi_uniform"] = fmt.from_sets([uniq_sorted(rng, 20000, 0, 1 << 17),
                                         uniq_sorted(rng, 20000, 0, 1 << 17)], universe=(1 << 17) - 1)
    # single pair, skewed sizes with planted overlap
    big = uniq_sorted(rng, 30000, 0, 1 << 20)
    small = np.union1d(uniq_sorted(rng, 300, 0, 1 << 20), rng.choice(big, 100, replace=False)).astype(np.uint32)
    out["sisi_skewed"] = fmt.from_sets([small, big], universe=(1 << 20) - 1)
    # single pair at the value extremes: 0 and 0xffffffff in both sets
    ext_a = np.array([0, 1, 7, 1 << 31, 0xfffffffe, 0xffffffff], dtype=np.uint32)
    ext_b = np.array([0, 2, 7, (1 << 31) + 1, 0xffffffff], dtype=np.uint32)
    out["sisi_extremes"] = fmt.from_sets([ext_a, ext_b], universe=0xffffffff)
    # many sets: empty, singleton, identical, disjoint, subset, ragged sizes
    U = 5000
    sets = [np.zeros(0, np.uint32), np.array([17], np.uint32), np.array([U - 1], np.uint32)]
    base = uniq_sorted(rng, 700, 0, U)
    sets += [base, base.copy(), base[::3].copy(), base[1::2].copy()]
    sets += [np.arange(0, U, 2, dtype=np.uint32), np.arange(1, U, 2, dtype=np.uint32)]
    for n in (1, 2, 3, 5, 31, 32, 33, 127, 128, 129, 1000, 2047, 4096):
        sets.append(uniq_sorted(rng, n, 0, U))
    for _ in range(12):
        sets.append(uniq_sorted(rng, int(rng.integers(0, 1500)), 0, U))
    out["misi_mixed"] = fmt.from_sets(sets, universe=U - 1)
    # many sets, 1-based elements in [1, universe] as the reference generator writes them
    U2 = 3000
    sets2 = [np.sort(rng.choice(np.arange(1, U2 + 1), size=int(n), replace=False)).astype(np.uint32)
             for n in rng.integers(1, 400, size=25)]
    out["misi_onebased"] = fmt.from_sets(sets2, universe=U2)
    return out


def degree_datasets():
    """Inputs of degree_cdf: values below the universe (the reference's inverted
    index has `universe` slots), many equal set sizes and equal inverted-list
    lengths (ties keep std::sort's order), empty sets."""
    rng = np.random.default_rng(314159)
    out = {}
    U = 2048
    sets = [np.zeros(0, np.uint32)]
    for n in rng.integers(0, 6, size=30) * 25:  # sizes 0, 25, ..., 125: many ties
        sets.append(uniq_sorted(rng, int(n), 0, U - 1))
    out["degree_ties"] = fmt.from_sets(sets, universe=U)
    # popular low values: skewed inverted-list lengths
    V = 5000
    p = 1.0 / np.arange(1, V) ** 0.9
    p /= p.sum()
    sets = [np.unique(rng.choice(np.arange(1, V), size=int(n), p=p)).astype(np.uint32)
            for n in rng.integers(1, 600, size=60)]
    out["degree_zipf"] = fmt.from_sets(sets, universe=V)
    return out


def run(cmd, cwd=None):
    r = subprocess.run(cmd, capture_output=True, text=True, cwd=cwd)
    if r.returncode != 0:
        raise SystemExit(f"{cmd} failed: {r.stdout}\n{r.stderr}")
    return r.stdout


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def main():
    for exe in ("stdintersection", "serial_intersect", "boost_bitset", "ref_elements", "txt2bin", "bin2txt",
                "degree_cdf"):
        if not os.access(os.path.join(REF, exe), os.X_OK):
            raise SystemExit(f"oracle/_ref/{exe} missing: run `make -C oracle ref` first")
    manifest = {}
    for name, ds in datasets().items():
        binp = os.path.join(HERE, f"{name}.bin")
        fmt.write_dataset(binp, ds)
        files = [binp]
        for exe, tag in (("stdintersection", "std"), ("serial_intersect", "serial"), ("boost_bitset", "bitset")):
            if tag == "bitset" and ds.universe >= 0xffffffff:
                continue  # boost_bitset sizes its bitset with universe + 1 (src/boost_bitset.cpp:49)
            outp = os.path.join(HERE, f"{name}.{tag}.txt")
            run([os.path.join(REF, exe), "--input", binp, "--output", outp, "--threads", "3"])
            files.append(outp)
        elp = os.path.join(HERE, f"{name}.elements.bin")
        run([os.path.join(REF, "ref_elements"), binp, elp])
        files.append(elp)
        manifest[name] = {os.path.basename(f): sha(f) for f in files}
    # text <-> binary tools
    txt = os.path.join(HERE, "text_sets.txt")
    rng = np.random.default_rng(7)
    with open(txt, "w") as f:
        for n in (5, 1, 9, 3):
            s = np.sort(rng.choice(np.arange(1, 100), size=n, replace=False))
            f.write(" ".join(str(int(x)) for x in s) + "\n")
    run([os.path.join(REF, "txt2bin"), txt, "text_sets"], cwd=HERE)
    run([os.path.join(REF, "bin2txt"), "text_sets_asc.bin", "text_roundtrip"], cwd=HERE)
    manifest["text_tools"] = {f: sha(os.path.join(HERE, f)) for f in
                              ("text_sets.txt", "text_sets_asc.bin", "text_sets_desc.bin", "text_roundtrip.txt")}
    # dataset statistics
    for name, ds in degree_datasets().items():
        binp = os.path.join(HERE, f"{name}.bin")
        fmt.write_dataset(binp, ds)
        run([os.path.join(REF, "degree_cdf"), binp, name], cwd=HERE)
        manifest[name] = {f: sha(os.path.join(HERE, f)) for f in
                          [f"{name}.bin"] + [f"{name}_{t}.txt" for t in
                                             ("degree_set", "degree_element", "set_cdf", "element_cdf")]}
    with open(os.path.join(HERE, "MANIFEST.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print(json.dumps({k: len(v) for k, v in manifest.items()}))


if __name__ == "__main__":
    main()
