#!/usr/bin/env python
"""Benchmark of the set-intersection hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload W] [--technique T]

Workloads: sisi_large (default), sisi_mid, sisi_plain, sisi_skewed (single
pair, Gelem/s); misi_dense, misi_dense_small (all pairs on tensor cores or the
plain popcount kernel, pairs/s); misi_powerlaw, misi_powerlaw_small (all pairs,
ip/obs/hi/bitmap, pairs/s); batch_pairs, batch_pairs_small (1M pairs of a
100000-set pool in one CUDA graph, pairs/s).  A default run (SISI, one GPU)
also runs each other configuration briefly in a subprocess and adds a summary
of each line under "other_workloads" (--no-extras skips them).

One "step" is one pass of the single-pair (SISI) hot path over one pair of
sets: the workload by default is |A| = |B| = 2^28 sorted unique uint32 drawn
from [0, 2^31), technique auto (for two sets of similar size: the bitmap
engine over value-pivot tiles), count + materialised elements.
Metric: Gelem/s = (|A| + |B|) / step time.

  value   device-timed (CUDA events on the launching stream), inputs resident
          in HBM; 2 GiB of input per step > 126 MB L2, so no L2 flush.
  e2e     the same metric through the host-buffer C-ABI call si_sisi_host
          (via api.intersect_host): pinned host sets -> H2D -> kernels ->
          count + elements D2H, per step, pipelined over 8 value ranges.
  roofline  live per-launch time of the dominant kernel (the tile kernel) from the
          library's phase timer, against measured HBM; phase_avg_ms lists every
          phase of the step (set-up, stream/tiles, copy).  The phase events are
          recorded in a second pass of the same steps (phase_pass): between the
          launches they hold back the programmatic dependent launches, so the
          value pass runs without them.
  cpu_baseline  the reference's own CPU executable (oracle/_ref/stdintersection,
          built from the reference sources) on value-range slices of the same
          pair, timed by the reference's HostTimer.
  --impl reference  the same executable on slices of the same pair, built
          in that process by the oracle's restatement of the engine's seeded
          generator (the engine's library is never loaded there).
  techniques  (SISI, one GPU) every technique on the same pair after the timed
          region, 20 steps each, with whether its count and elements equal the
          benchmarked call's.

Multi-GPU: the single-pair path is replicas only -- each rank runs its own
independent pair (no data-path collective); value is the whole-job aggregate.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
FALLBACK_BF16_TFLOPS = 1590.0
CACHE_DIR = os.environ.get("SI_BENCH_CACHE", os.path.join(tempfile.gettempdir(), "si_bench_cache"))

WORKLOADS = {
    "sisi_large": dict(desc="SISI |A|=|B|=2^28 uint32 uniform w/o replacement from [0,2^31), seeds 3,4",
                       n=1 << 28, universe=1 << 31, seeds=(3, 4)),
    "sisi_mid": dict(desc="SISI |A|=|B|=2^25 uint32 uniform w/o replacement from [0,2^28), seeds 3,4 "
                          "(same density as sisi_large, 256 MiB > L2; profiling size)",
                     n=1 << 25, universe=1 << 28, seeds=(3, 4)),
    "sisi_plain": dict(desc="SISI |A|=|B|=2^20 uint32 uniform w/o replacement from [0,2^24), seeds 1,2",
                       n=1 << 20, universe=1 << 24, seeds=(1, 2)),
    "sisi_skewed": dict(desc="SISI |A|=2^16, |B|=2^26 from [0,2^30), 20% of A planted into B, seed 5",
                        n=None, universe=1 << 30, seeds=(5,)),
    "misi_dense": dict(desc="MISI all pairs: 16384 sets over values [0,65536), Bernoulli(0.05) membership, seed 6",
                       k=16384, n_values=65536, p=0.05, seeds=(6,)),
    "misi_powerlaw": dict(desc="MISI all pairs: 8192 sets, sizes ~ n^-1.1 on [16,65536], distinct values of "
                               "[1,2^20] with Zipf(0.8) popularity, seed 7",
                          kind="powerlaw", k=8192, n_min=16, n_max=65536, size_exp=1.1, universe=1 << 20,
                          value_exp=0.8, seeds=(7,)),
    "misi_powerlaw_small": dict(desc="MISI all pairs: the first 2048 sets of the power-law collection "
                                     "(profiling size)",
                                kind="powerlaw", k=2048, n_min=16, n_max=65536, size_exp=1.1, universe=1 << 20,
                                value_exp=0.8, seeds=(7,)),
    "batch_pairs": dict(desc="Batched pairs: pool of 100000 sets, sizes log-uniform on [32,2^18], distinct values of "
                             "[0,2^26); 1M pairs (i,j), i != j, uniform over the pool; counts only; seeds 8, 9",
                        kind="batch", k=100000, npairs=1000000, seeds=(8,)),
    "batch_pairs_small": dict(desc="Batched pairs: a tenth of the batched workload (10000 sets, 100000 pairs; "
                                   "profiling size)",
                              kind="batch", k=10000, npairs=100000, seeds=(8,)),
    "misi_dense_small": dict(desc="MISI all pairs: 4096 sets over values [0,65536), Bernoulli(0.05), seed 6 "
                                  "(incidence 256 MiB > L2; profiling size)",
                             k=4096, n_values=65536, p=0.05, seeds=(6,)),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


SKEW_RATIO = 64  # SI_TECH_AUTO: obs when one set is more than this many times the other

# DRAM bytes (read + write) per launch of the dominant kernel, from ncu
# captures summarised in profiles/: the bitmap engine's bp_stream_kernel
# measured at full size (a one-pass dram__bytes capture of the 2^28 x 2^28
# launch); the ip tile kernel from its 2^25 x 2^25 capture scaled by 8 (tiles,
# inputs and matches grow in proportion).
TRAFFIC_PER_LAUNCH = {
    "bitmap/sisi_large/out": 2.246e9 + 121.53e6,   # one-pass dram__bytes capture of the 2^28 stream kernel
    "bitmap/sisi_mid/out": 321.59e6 + 5.21e6,      # from the 2^25 full capture
    "ip/sisi_large/out": 8 * (268.727808e6 + 13.220096e6),
    "ip/sisi_mid/out": 268.727808e6 + 13.220096e6,
}


# ----------------------------------------------------------------- inputs --
def make_pair(name: str):
    from set_intersection_b200 import generate
    os.makedirs(CACHE_DIR, exist_ok=True)
    path = os.path.join(CACHE_DIR, f"{name}.npz")
    if os.path.exists(path):
        try:
            z = np.load(path)
            return z["a"], z["b"]
        except Exception:
            pass
    w = WORKLOADS[name]
    if name == "sisi_skewed":
        a, b = generate.sisi_skewed(seed=w["seeds"][0])
    else:
        a = generate.uniform(w["seeds"][0], w["n"], w["universe"])
        b = generate.uniform(w["seeds"][1], w["n"], w["universe"])
    tmp = path + f".{os.getpid()}.tmp.npz"
    np.savez(tmp, a=a, b=b)
    os.replace(tmp, path)
    return a, b


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML while running."""

    REASONS = {
        0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
        0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown", 0x2: "applications_clocks_setting",
    }

    def __init__(self, torch_dev: int = 0, period_s: float = 0.005):
        self.period = period_s
        self.samples, self.reasons = [], set()
        self.ok = False
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            self.nvml = pynvml
            uuid = str(torch.cuda.get_device_properties(torch_dev).uuid)
            try:
                self.h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + uuid)
            except Exception:
                vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
                idx = int(vis.split(",")[torch_dev]) if vis and vis.split(",")[0].isdigit() else torch_dev
                self.h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception as e:  # pragma: no cover - depends on the box
            log(f"clock sampling unavailable: {e}")
            self.max_mhz = None
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        nv = self.nvml
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.ok:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *exc):
        if self._t:
            self._stop.set()
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": float(statistics.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# -------------------------------------------------------------- reference --
def ref_pair(name: str):
    """The workload's pair as the reference arm builds it: the oracle's
    restatement of the engine's seeded generator (oracle.gen_uniform yields the
    very same sets), so this process never loads the engine's library."""
    import oracle
    w = WORKLOADS[name]
    os.makedirs(CACHE_DIR, exist_ok=True)
    path = os.path.join(CACHE_DIR, f"{name}.npz")  # the same sets as the engine arm's cache
    if os.path.exists(path):
        try:
            z = np.load(path)
            return z["a"], z["b"]
        except Exception:
            pass
    a = oracle.gen_uniform(w["seeds"][0], w["n"], w["universe"])
    b = oracle.gen_uniform(w["seeds"][1], w["n"], w["universe"])
    tmp = path + f".{os.getpid()}.tmp.npz"
    np.savez(tmp, a=a, b=b)
    os.replace(tmp, path)
    return a, b


def ref_slices(a, b, n_slices: int, per_set: int):
    """n_slices value-range slices of the pair, evenly spaced over it: slice j
    holds per_set consecutive elements of a from position j |a| / n_slices and
    the elements of b in the same value range (same density as the pair)."""
    out = []
    per_set = min(per_set, a.size // n_slices)
    for j in range(n_slices):
        i0 = j * a.size // n_slices
        i1 = i0 + per_set
        lo = int(a[i0])
        j0 = int(np.searchsorted(b, lo, "left"))
        j1 = int(np.searchsorted(b, int(a[i1]), "left")) if i1 < a.size else b.size
        out.append((a[i0:i1], b[j0:j1]))
    return out


def ref_sisi_measure(a, b, steps: int, warmup: int, budget_s: float):
    """The reference's own stdintersection (oracle/_ref, built from
    src/std_set_intersection.cpp) timed by its HostTimer on slices of the pair:
    step i runs slice i mod 8, sized so the whole run takes about budget_s.
    Returns (kind, Gelem/s over the timed steps, description)."""
    import oracle
    exe = oracle.ref_binary("stdintersection")
    # about 35 ns per element per run (the reference reads its dataset
    # element by element, then intersects on one thread)
    total = int(budget_s / max(1, steps + warmup) / 35e-9)
    per_set = 1 << max(16, min(27, (total // 2).bit_length() - 1))
    while per_set > 1 and per_set > a.size // 8:
        per_set >>= 1
    slices = ref_slices(a, b, 8, per_set)
    elems, ms_sum = 0, 0.0
    with tempfile.TemporaryDirectory() as td:
        for i in range(warmup + steps):
            sa, sb = slices[i % len(slices)]
            if exe:
                path = os.path.join(td, f"slice{i % len(slices)}.bin")
                if not os.path.exists(path):
                    oracle.write_dataset(path, [sa, sb], int(max(sa[-1], sb[-1]) if sb.size else sa[-1]))
                ms = oracle.run_ref("stdintersection", path, threads=os.cpu_count())["host_ms"]["std::set intersection"]
            else:
                t0 = time.perf_counter()
                oracle.count(sa, sb, "std")
                ms = (time.perf_counter() - t0) * 1e3
            if i >= warmup:
                elems += sa.size + sb.size
                ms_sum += ms
    kind = "reference" if exe else "port"
    desc = (f"step i: value-range slice i mod 8 of the workload's pair (8 slices evenly spaced over it, "
            f"2^{per_set.bit_length() - 1} elements of A each plus B's elements in the same range: the same "
            f"sets and density), {'oracle/_ref/stdintersection --threads nproc (src/std_set_intersection.cpp:58-76; with 2 sets one thread has work), its HostTimer' if exe else 'oracle std::set_intersection port'}; "
            f"Gelem/s = elements of the timed steps / their summed time")
    return kind, elems / (ms_sum * 1e-3) / 1e9, desc


def sisi_config(args, n_a: int, n_b: int, world: int) -> dict:
    """The workload's description, the same in both arms' lines."""
    return {"workload": args.workload, "desc": WORKLOADS[args.workload]["desc"], "materialize": bool(args.materialize),
            "n_a": int(n_a), "n_b": int(n_b),
            "l2": "inputs 2 GiB per step > 126 MB L2; no flush" if args.workload == "sisi_large"
                  else "inputs resident; no flush",
            "parallelism": f"replicas{world}"}


def run_reference_arm(args, rank: int):
    if rank != 0:
        return
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.workload == "sisi_skewed":
        a, b = make_pair(args.workload)  # planted pair: the engine's generator
    else:
        a, b = ref_pair(args.workload)
    kind, value, desc = ref_sisi_measure(a, b, args.steps, args.warmup, budget_s=150.0)
    line = {
        "impl": "reference", "metric": "SISI Gelem/s", "value": value, "unit": "Gelem/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": (a.size + b.size) / (value * 1e9) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": sisi_config(args, a.size, b.size, world),
        "technique": "std::set_intersection",
        "cpu_baseline": {"value": value, "unit": "Gelem/s", "cores": 1, "kind": kind, "sample": desc},
        "e2e": {"value": value, "unit": "Gelem/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------------- ours --
def run_ours(args, rank: int, world: int):
    import torch
    from set_intersection_b200 import api
    from set_intersection_b200._lib import lib
    import ctypes

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    from set_intersection_b200.replicas import Replicas
    rep = Replicas("nccl", dev)

    # inputs: rank 0 generates (or loads the cache), the others load the cache
    if rank == 0:
        a, b = make_pair(args.workload)
    rep.barrier()
    if rank != 0:
        a, b = make_pair(args.workload)

    n_a, n_b = a.size, b.size
    stream = torch.cuda.Stream(dev)
    da = torch.from_numpy(a.view(np.int32)).to(dev)
    db = torch.from_numpy(b.view(np.int32)).to(dev)
    ws = api.Workspace(dev)
    count = torch.zeros(1, dtype=torch.int64, device=dev)
    out = torch.empty(max(1, min(n_a, n_b)), dtype=torch.int32, device=dev) if args.materialize else None

    # parity of the benchmarked call, once, before timing
    api.sisi_into(da, db, count, out, ws, args.technique, stream)
    ws.check(stream)
    c = int(count.item())
    parity = None
    if rank == 0 and not args.no_parity:
        import oracle
        want = oracle.set_intersection(a, b)
        parity = bool(want.size == c and (out is None or np.array_equal(out[:c].cpu().numpy().view(np.uint32), want)))
        log(f"parity vs oracle: {parity} (count {c})")

    def step():
        api.sisi_into(da, db, count, out, ws, args.technique, stream)

    for _ in range(args.warmup):
        step()
    stream.synchronize()
    rep.barrier()
    torch.cuda.synchronize()

    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            step()
        stop.record(stream)
        stop.synchronize()
    ms_total = start.elapsed_time(stop)
    # per-kernel times: a second pass of the same steps with the library's
    # phase events recorded around every launch.  Those records sit between
    # the launches (a kernel launched as a programmatic dependent then waits
    # for the one before it to finish), so value comes from the pass without
    # them.
    phase_steps = max(1, min(args.steps, 50))
    lib.si_timer_reset()
    lib.si_timer_enable(1)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for _ in range(phase_steps):
        step()
    p1.record(stream)
    p1.synchronize()
    lib.si_timer_enable(0)
    phase_pass_ms = p0.elapsed_time(p1) / phase_steps
    tile_ms, tile_n = ctypes.c_double(0), ctypes.c_uint64(0)
    lib.si_timer_read(b"sisi_tile", ctypes.byref(tile_ms), ctypes.byref(tile_n))
    phases = {}
    for ph in ("sisi_split", "sisi_tile", "sisi_scan", "sisi_copy", "obs_sample", "obs_search",
               "obs_compact"):
        p_ms, p_n = ctypes.c_double(0), ctypes.c_uint64(0)
        lib.si_timer_read(ph.encode(), ctypes.byref(p_ms), ctypes.byref(p_n))
        if p_n.value:
            phases[ph] = p_ms.value / p_n.value
    lib.si_timer_reset()
    ws.check(stream)
    torch.cuda.synchronize()
    rep.barrier()
    ms_total = rep.max(ms_total)

    ms_step = ms_total / args.steps
    value = rep.rate(n_a + n_b, ms_step) / 1e9

    # ---- end to end through the public host API ----
    e2e = None
    if not args.no_e2e:
        ha = torch.from_numpy(a.view(np.int32)).pin_memory()
        hb = torch.from_numpy(b.view(np.int32)).pin_memory()
        hout = torch.empty(max(1, min(n_a, n_b)), dtype=torch.int32).pin_memory()
        ctx = api.HostPair(dev)
        for _ in range(2):
            api.intersect_host(ha, hb, args.technique, hout, ctx, stream)
        e_steps = max(1, min(args.steps, args.e2e_steps))
        rep.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e_steps):
            ce, _ = api.intersect_host(ha, hb, args.technique, hout, ctx, stream)
        e1.record(stream)
        e1.synchronize()
        e_ms = e0.elapsed_time(e1)
        e_ms = rep.max(e_ms)
        e_step = e_ms / e_steps
        e2e = {"value": rep.rate(n_a + n_b, e_step) / 1e9, "unit": "Gelem/s",
               "h2d_bytes_per_step": 4 * (n_a + n_b), "d2h_bytes_per_step": 8 + 4 * ce,
               "ms_per_step": e_step, "steps": e_steps,
               "host_buffers": "pinned: the caller's sets and result buffer, pinned before the timed region"}
        assert ce == c
        # the same call from pageable host memory: the library stages the
        # inputs through its pinned buffers (host threads copy, the DMA engine
        # moves the previous pieces up)
        pa = torch.from_numpy(a.view(np.int32))
        pb = torch.from_numpy(b.view(np.int32))
        pout = torch.empty(max(1, min(n_a, n_b)), dtype=torch.int32)
        api.intersect_host(pa, pb, args.technique, pout, ctx, stream)
        p_steps = max(1, min(e_steps, 3))
        rep.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(p_steps):
            cp, _ = api.intersect_host(pa, pb, args.technique, pout, ctx, stream)
        e1.record(stream)
        e1.synchronize()
        p_step = rep.max(e0.elapsed_time(e1)) / p_steps
        e2e["pageable"] = {"value": rep.rate(n_a + n_b, p_step) / 1e9, "unit": "Gelem/s", "ms_per_step": p_step,
                           "steps": p_steps}
        assert cp == c

    # ---- every technique on the same pair (outside the timed region) ----
    techniques = None
    if world == 1 and not args.no_techniques:
        techniques = {}
        t_steps = max(1, min(args.steps, 20))
        want_out = out[:c].clone() if out is not None else None
        tcount = torch.zeros(1, dtype=torch.int64, device=dev)
        for tech in ("auto", "ip", "obs", "hi", "bitmap"):
            for _ in range(3):
                api.sisi_into(da, db, tcount, out, ws, tech, stream)
            ws.check(stream)
            same = int(tcount.item()) == c and (out is None or bool(torch.equal(out[:c], want_out)))
            t0e, t1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0e.record(stream)
            for _ in range(t_steps):
                api.sisi_into(da, db, tcount, out, ws, tech, stream)
            t1e.record(stream)
            t1e.synchronize()
            t_ms = t0e.elapsed_time(t1e) / t_steps
            techniques[tech] = {"ms_per_step": t_ms, "value": (n_a + n_b) / (t_ms * 1e6), "unit": "Gelem/s",
                                "steps": t_steps, "same_result": same}
            log(f"technique {tech}: {t_ms:.4f} ms per step, same result: {same}")
        del want_out

    if rank != 0:
        rep.close()
        return

    # ---- roofline of the dominant kernel ----
    peaks = json.load(open(PEAKS_PATH)) if os.path.exists(PEAKS_PATH) else {}
    peak = peaks.get("hbm_gbs", FALLBACK_HBM_GBS)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    alg_bytes = 4 * (n_a + n_b) + (4 * c if args.materialize else 0)
    # the engine that ran: auto searches a much smaller set in the larger (obs)
    # and streams pairs of similar size through the bitmap tiles
    engine = args.technique
    if engine == "auto":
        engine = "obs" if min(n_a, n_b) * SKEW_RATIO < max(n_a, n_b) else "bitmap"
    kernel, launches = {
        "ip": ("ip_tile_kernel<merge path>", 3),
        "hi": ("bh_stream_kernel", 2 if args.materialize else 1),
        "bitmap": ("bp_stream_kernel", 2 if args.materialize else 1),
        "obs": ("obs_search_kernel", 3 if args.materialize else 2),
    }[engine]
    if engine == "obs":
        tile_avg_ms = phases.get("obs_search")
        achieved = None  # dependent-load chains over a fraction of the larger set: latency-bound
    else:
        tile_avg_ms = tile_ms.value / max(1, tile_n.value)
        achieved = alg_bytes / (tile_avg_ms * 1e-3) / 1e9 if tile_n.value else None
    traffic = TRAFFIC_PER_LAUNCH.get(f"{engine}/{args.workload}/{'out' if args.materialize else 'count'}")

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        kind, cval, desc = ref_sisi_measure(a, b, steps=3, warmup=1, budget_s=20.0)
        cpu = {"value": cval, "unit": "Gelem/s", "cores": 1, "kind": kind, "sample": desc}

    line = {
        "metric": "SISI Gelem/s", "value": value, "unit": "Gelem/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": sisi_config(args, n_a, n_b, world),
        "technique": args.technique, "intersection": c, "parity_vs_oracle": parity,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "kernel": kernel, "engine": engine, "alg_bytes_per_launch": alg_bytes,
                     "avg_launch_ms": tile_avg_ms, "launches": int(tile_n.value), "peak_source": peak_src,
                     "phase_avg_ms": phases,
                     "phase_pass": {"steps": phase_steps, "ms_per_step": phase_pass_ms,
                                    "note": "launch and phase times from a second pass with the phase events "
                                            "recorded around every launch"}},
        "e2e": e2e,
        "gpu_launches": launches * args.steps,
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
    }
    if techniques is not None:
        line["techniques"] = techniques
    if world == 1 and not args.no_extras:
        line["other_workloads"] = other_workloads(args)
    print(json.dumps(line), flush=True)
    rep.close()


# ------------------------------------------------------- MISI, dense form --
def is_powerlaw(name: str) -> bool:
    return WORKLOADS[name].get("kind") == "powerlaw"


def misi_universe(name: str) -> int:
    """Largest value of the workload's collection (the dataset header's universe)."""
    w = WORKLOADS[name]
    return w["universe"] if is_powerlaw(name) else w["n_values"] - 1


def dense_collection(name: str):
    return dense_sample(name, WORKLOADS[name]["k"])


def dense_sample(name: str, k_sample: int):
    """The first k_sample sets of the workload (every set is drawn from its own
    stream, so these are exactly the workload's first sets)."""
    from set_intersection_b200 import generate
    w = WORKLOADS[name]
    if is_powerlaw(name):
        return generate.powerlaw(w["seeds"][0], k_sample, w["n_min"], w["n_max"], w["size_exp"], w["universe"],
                                 w["value_exp"])
    return generate.bernoulli(w["seeds"][0], k_sample, w["n_values"], w["p"])


# CPU reference per all-pairs workload: executable, its HostTimer interval,
# the oracle technique of the same algorithm, the sample size in sets
CPU_REF = {
    "dense": ("boost_bitset", "Boost bitset intersection", "bitset", 1024, "src/boost_bitset.cpp:60-84"),
    "powerlaw": ("stdintersection", "std::set intersection", "std", 640, "src/std_set_intersection.cpp:58-76"),
}


def dense_reference_ms(el, off, universe: int, tmpdir: str, threads: int, exe: str, interval: str) -> float:
    """One run of a reference CPU executable (all pairs, OpenMP) on a dataset
    file; its own HostTimer figure for the intersection phase."""
    import oracle
    from set_intersection_b200 import dataset as fmt
    path = os.path.join(tmpdir, "misi.bin")
    if not os.path.exists(path):
        sizes = np.diff(off).astype(np.uint32)
        fmt.write_dataset(path, fmt.Dataset(len(sizes), universe, sizes, el))
    r = oracle.run_ref(exe, path, threads=threads)
    return r["host_ms"][interval]


def dense_port_ms(el, off, universe: int, threads: int, tech: str) -> float:
    import oracle
    k = off.size - 1
    t0 = time.perf_counter()
    oracle.all_pairs(el, off, k, universe, tech, threads=threads)
    return (time.perf_counter() - t0) * 1e3


def dense_cpu_measure(name: str, k_sample: int | None, steps: int, warmup: int):
    import oracle
    exe, interval, port_tech, k_default, cite = CPU_REF["powerlaw" if is_powerlaw(name) else "dense"]
    k_sample = k_sample or k_default
    el, off = dense_sample(name, k_sample)
    universe = misi_universe(name)
    threads = os.cpu_count() or 1
    kind = "reference" if oracle.ref_binary(exe) else "port"
    times = []
    with tempfile.TemporaryDirectory() as td:
        for i in range(warmup + steps):
            ms = (dense_reference_ms(el, off, universe, td, threads, exe, interval) if kind == "reference"
                  else dense_port_ms(el, off, universe, threads, port_tech))
            if i >= warmup:
                times.append(ms)
    ms = statistics.median(times)
    pairs = k_sample * (k_sample - 1) // 2
    desc = (f"first {k_sample} sets of the workload ({pairs} pairs), {exe} --threads {threads} "
            f"({cite}), median of {steps} runs timed by its HostTimer")
    return kind, threads, pairs / (ms * 1e-3), desc, ms


def run_reference_dense(args, rank: int):
    if rank != 0:
        return
    kind, threads, value, desc, ms = dense_cpu_measure(args.workload, None, args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": "MISI pairs/s", "value": value, "unit": "pairs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": args.workload, "desc": WORKLOADS[args.workload]["desc"],
                   "technique": CPU_REF["powerlaw" if is_powerlaw(args.workload) else "dense"][0]},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": kind, "sample": desc},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours_dense(args, rank: int, world: int):
    import ctypes
    import torch
    from set_intersection_b200 import api
    from set_intersection_b200._lib import lib

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    from set_intersection_b200.replicas import Replicas
    rep = Replicas("nccl", dev)
    powerlaw = is_powerlaw(args.workload)
    if powerlaw:
        tech = args.technique if args.technique in ("ip", "obs", "hi", "bitmap", "auto") else "bitmap"
    else:
        tech = args.technique if args.technique in ("mm", "bitmap_naive") else "mm"
    dtype = args.dtype
    w = WORKLOADS[args.workload]
    el, off = dense_collection(args.workload)
    k, universe = off.size - 1, misi_universe(args.workload)
    pairs = k * (k - 1) // 2
    stream = torch.cuda.Stream(dev)
    col = api.Collection(torch.from_numpy(el.view(np.int32)).to(dev), torch.from_numpy(off).to(dev), universe)
    ws = api.Workspace(dev)
    counts = torch.empty(pairs, dtype=torch.int32, device=dev)

    def step(t=tech, d=dtype, out=counts):
        if t in ("mm", "bitmap_naive"):
            api.misi_dense_into(col, out, t, d, ws, stream)
        else:
            api.misi_into(col, out, t, workspace=ws, stream=stream)

    # parity of the benchmarked call, once, before timing: against the plain
    # popcount kernel on every pair and the oracle on sampled pairs
    step()
    ws.check(stream)
    parity = None
    if rank == 0 and not args.no_parity:
        import oracle
        plain = torch.empty_like(counts)
        step(t="ip" if powerlaw else "bitmap_naive", d="int8", out=plain)
        ws.check(stream)
        same = bool(torch.equal(plain, counts))
        rng = np.random.default_rng(1)
        a = rng.integers(0, k - 1, 20000)
        b = a + 1 + (rng.random(20000) * (k - 1 - a)).astype(np.int64)
        want = oracle.pairs(el, off, k, np.stack([a, b], 1))
        idx = pairs - (k - a) * (k - a - 1) // 2 + b - a - 1
        got = counts.cpu().numpy().view(np.uint32)[idx]
        parity = same and bool(np.array_equal(got, want))
        log(f"parity: all pairs vs {'ip' if powerlaw else 'plain'} kernel {same}, "
            f"20000 sampled pairs vs oracle {np.array_equal(got, want)}")
        del plain

    for _ in range(args.warmup):
        step()
    stream.synchronize()
    rep.barrier()
    torch.cuda.synchronize()

    gemm_phase = b"misi_probe" if powerlaw else b"mm_gemm" if tech == "mm" else b"naive_popcount"
    lib.si_timer_reset()
    lib.si_timer_enable(1)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            step()
        stop.record(stream)
        stop.synchronize()
    lib.si_timer_enable(0)
    ms_total = start.elapsed_time(stop)
    k_ms, k_n = ctypes.c_double(0), ctypes.c_uint64(0)
    lib.si_timer_read(gemm_phase, ctypes.byref(k_ms), ctypes.byref(k_n))
    lib.si_timer_reset()
    ws.check(stream)
    torch.cuda.synchronize()
    rep.barrier()
    ms_total = rep.max(ms_total)
    ms_step = ms_total / args.steps
    value = rep.rate(pairs, ms_step)

    # the plain AND-popcount kernel on the same GPU, for the speed-up
    plain_ms = None
    if tech == "mm" and not args.no_plain:
        step(t="bitmap_naive", d="int8")
        stream.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n_plain = max(1, min(3, args.steps))
        p0.record(stream)
        for _ in range(n_plain):
            step(t="bitmap_naive", d="int8")
        p1.record(stream)
        p1.synchronize()
        plain_ms = p0.elapsed_time(p1) / n_plain

    e2e = None
    if not args.no_e2e:
        h_el = torch.from_numpy(el.view(np.int32)).pin_memory()
        h_off = torch.from_numpy(off).pin_memory()
        h_counts = torch.empty(pairs, dtype=torch.int32).pin_memory()
        ctx = api.HostCollection(dev)
        if powerlaw:
            api.misi_host(h_el, h_off, universe, tech, h_counts, ctx, stream)
        else:
            api.misi_dense_host(h_el, h_off, universe, tech, dtype, h_counts, ctx, stream)
        e_steps = max(1, min(args.steps, args.e2e_steps))
        rep.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e_steps):
            if powerlaw:
                api.misi_host(h_el, h_off, universe, tech, h_counts, ctx, stream)
            else:
                api.misi_dense_host(h_el, h_off, universe, tech, dtype, h_counts, ctx, stream)
        e1.record(stream)
        e1.synchronize()
        e_ms = e0.elapsed_time(e1)
        e_ms = rep.max(e_ms)
        e_step = e_ms / e_steps
        e2e = {"value": rep.rate(pairs, e_step), "unit": "pairs/s",
               "h2d_bytes_per_step": int(4 * el.size + 8 * off.size), "d2h_bytes_per_step": int(4 * pairs),
               "ms_per_step": e_step, "steps": e_steps}

    if rank != 0:
        rep.close()
        return

    peaks = json.load(open(PEAKS_PATH)) if os.path.exists(PEAKS_PATH) else {}
    avg_ms = k_ms.value / max(1, k_n.value)
    if tech == "mm":
        # algorithmic work: one multiply-add per (pair a < b, value)
        ops = 2.0 * pairs * w["n_values"]
        bf16 = peaks.get("bf16_tflops", FALLBACK_BF16_TFLOPS)
        peak = 2.0 * bf16
        achieved = ops / (avg_ms * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": None, "kernel": f"tc_gemm_kernel<{dtype}>", "alg_ops_per_launch": ops,
                "avg_launch_ms": avg_ms, "launches": int(k_n.value),
                "peak_source": ("2 x measured dense bf16 (8-bit operands run at twice the 16-bit rate)"
                                if "bf16_tflops" in peaks else "2 x fallback bf16")}
        i8 = cublas_int8_tops(dev) if not args.no_plain else None
        if i8:
            roof["cublas_int8_tops_measured"] = i8
            roof["frac_of_cublas_int8"] = achieved / i8
    elif powerlaw:
        # algorithmic bytes: every pair reads its smaller set once (4 B per
        # probe), each set is read once more as the staged side, and every
        # pair writes its count
        sizes = np.sort(np.diff(off))[::-1]
        suffix = np.cumsum(sizes[::-1])[::-1]
        probes = int(suffix[1:].sum())
        alg_bytes = 4 * probes + 4 * int(el.size) + 4 * pairs
        peak = peaks.get("hbm_gbs", FALLBACK_HBM_GBS)
        achieved = alg_bytes / (avg_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": f"misi_probe_kernel<{tech}>", "alg_bytes_per_launch": alg_bytes,
                "probes_per_launch": probes, "avg_launch_ms": avg_ms, "launches": int(k_n.value),
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "note": "probe reads of the smaller sets are mostly served by L2; HBM is the conservative peak"}
    else:
        roof = {"bound": "alu", "achieved": None, "peak": None, "unit": None, "frac": None, "traffic": None,
                "kernel": "popcount_gemm_kernel", "avg_launch_ms": avg_ms, "launches": int(k_n.value)}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        kind, threads, cval, desc, _ = dense_cpu_measure(args.workload, None, steps=3, warmup=1)
        cpu = {"value": cval, "unit": "pairs/s", "cores": threads, "kind": kind, "sample": desc}

    line = {
        "metric": "MISI pairs/s", "value": value, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "u32" if powerlaw else "u8" if dtype == "int8" else "e4m3",
        "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"], "technique": tech,
                   "operand": None if powerlaw else dtype,
                   "k": k, "universe": universe, "pairs": pairs, "elements": int(el.size),
                   "l2": ("collection and counts per step > 126 MB L2 at 8192 sets; no flush" if powerlaw else
                          f"incidence operand {w['k'] * w['n_values'] >> 20} MiB per step > 126 MB L2; no flush"),
                   "parallelism": f"replicas{world}", "parity_vs_oracle": parity,
                   "plain_popcount_ms_per_step": plain_ms,
                   "speedup_vs_plain": (plain_ms / ms_step) if plain_ms else None},
        "roofline": roof,
        "e2e": e2e,
        "gpu_launches": (4 if powerlaw else 2) * args.steps,
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    rep.close()


def cublas_int8_tops(dev, n: int = 8192, reps: int = 10):
    """cuBLAS's own dense INT8 GEMM (torch._int_mm, s32 accumulation) on this
    GPU, best of `reps` CUDA-event-timed runs of an n^3 product: an 8-bit
    denominator measured beside the kernel."""
    import torch
    try:
        a = torch.randint(-3, 4, (n, n), dtype=torch.int8, device=dev)
        b = torch.randint(-3, 4, (n, n), dtype=torch.int8, device=dev)
        for _ in range(3):
            torch._int_mm(a, b)
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        del a, b
        return 2.0 * n ** 3 / (best * 1e-3) / 1e12
    except Exception as e:  # not fatal: the bf16-derived peak stands
        log(f"cuBLAS int8 measurement unavailable: {e}")
        return None


# ------------------------------------------------------------ batched pairs --
def batch_data(name: str):
    from set_intersection_b200 import generate
    w = WORKLOADS[name]
    return generate.batch_pool(seed=w["seeds"][0], k=w["k"], npairs=w["npairs"])


def batch_cpu_measure(el, off, pairs, n_sample: int, steps: int, warmup: int):
    """The oracle's per-pair std::set_intersection count (the reference's
    std_set_intersection loop body, src/std_set_intersection.cpp:58-76, run on
    a pair list with OpenMP) on the first n_sample pairs: the reference has no
    pair-list executable, so this is a port."""
    import oracle
    threads = os.cpu_count() or 1
    sample = pairs[:n_sample]
    k = off.size - 1
    times = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        oracle.pairs(el, off, k, sample, threads=threads)
        if i >= warmup:
            times.append((time.perf_counter() - t0) * 1e3)
    ms = statistics.median(times)
    desc = (f"first {n_sample} pairs of the workload, std::set_intersection per pair, {threads} threads, "
            f"median of {steps} runs")
    return "port", threads, n_sample / (ms * 1e-3), desc, ms


def run_reference_batch(args, rank: int):
    if rank != 0:
        return
    el, off, pairs = batch_data(args.workload)
    kind, threads, value, desc, ms = batch_cpu_measure(el, off, pairs, 20000, args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": "batched pairs/s", "value": value, "unit": "pairs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": args.workload, "desc": WORKLOADS[args.workload]["desc"],
                   "technique": "std::set_intersection per pair"},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": kind, "sample": desc},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours_batch(args, rank: int, world: int):
    import ctypes
    import torch
    from set_intersection_b200 import api
    from set_intersection_b200._lib import lib

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    from set_intersection_b200.replicas import Replicas
    rep = Replicas("nccl", dev)
    w = WORKLOADS[args.workload]
    el, off, pairs = batch_data(args.workload)
    k, npairs = off.size - 1, len(pairs)
    stream = torch.cuda.Stream(dev)
    col = api.Collection(torch.from_numpy(el.view(np.int32)).to(dev), torch.from_numpy(off).to(dev), (1 << 26) - 1)
    dpairs = torch.from_numpy(pairs.view(np.int32)).to(dev)
    counts = torch.empty(npairs, dtype=torch.int32, device=dev)
    ws = api.Workspace(dev)
    tech = args.technique if args.technique in ("ip", "obs", "hi", "bitmap", "auto") else "auto"

    t0 = time.perf_counter()
    table = api.batch_tune(col, dpairs, workspace=ws, stream=stream) if tech == "auto" else None
    tune_s = time.perf_counter() - t0
    graph = api.BatchGraph(col, dpairs, counts, tech, table, workspace=api.Workspace(dev))

    graph.launch(stream)
    graph.check(stream)
    parity = None
    if rank == 0 and not args.no_parity:
        import oracle
        idx = np.random.default_rng(3).choice(npairs, 20000, replace=False)
        got = counts.cpu().numpy().view(np.uint32)
        parity = bool(np.array_equal(got[idx], oracle.pairs(el, off, k, pairs[idx])))
        log(f"parity: 20000 sampled pairs vs oracle {parity}")

    for _ in range(args.warmup):
        graph.launch(stream)
    stream.synchronize()
    rep.barrier()
    torch.cuda.synchronize()
    lib.si_timer_reset()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            graph.launch(stream)
        stop.record(stream)
        stop.synchronize()
    ms_total = start.elapsed_time(stop)
    graph.check(stream)
    rep.barrier()
    ms_total = rep.max(ms_total)
    ms_step = ms_total / args.steps
    value = rep.rate(npairs, ms_step)

    # the batch kernel alone (phase timer on a direct call, outside the graph)
    lib.si_timer_enable(1)
    for _ in range(3):
        api.batch_count_into(col, dpairs, counts, tech, table, ws, stream)
    stream.synchronize()
    lib.si_timer_enable(0)
    k_ms, k_n = ctypes.c_double(0), ctypes.c_uint64(0)
    lib.si_timer_read(b"batch_count", ctypes.byref(k_ms), ctypes.byref(k_n))
    lib.si_timer_reset()
    kern_ms = k_ms.value / max(1, k_n.value)

    # every populated bucket alone, each technique code (a table holding that
    # code for every bucket): what the tuner measures, on all of a bucket's pairs
    bucket_times = None
    if args.bucket_times and rank == 0:
        bk = api.batch_buckets(el, off, pairs)
        cbuf = torch.empty(npairs, dtype=torch.int32, device=dev)
        bucket_times = []
        for b in np.unique(bk):
            idx = np.nonzero(bk == b)[0]
            if len(idx) < 200:
                continue
            sub = dpairs[torch.from_numpy(idx).to(dev)].contiguous()
            row = {"bucket": int(b), "density": int(b >> 8), "log2_small": int((b >> 4) & 15),
                   "log2_ratio": int(b & 15), "pairs": int(len(idx)), "ms": []}
            for code in range(api.BATCH_CODES):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                for _ in range(2):  # the second run is timed
                    e0.record(stream)
                    api.batch_count_into(col, sub, cbuf, "auto", bytes([code]) * api.BATCH_TABLE_SIZE, ws, stream)
                    e1.record(stream)
                e1.synchronize()
                row["ms"].append(round(e0.elapsed_time(e1), 4))
            bucket_times.append(row)
            log(f"bucket {row['log2_small']},{row['log2_ratio']} d{row['density']} n={row['pairs']}: {row['ms']}")

    # plain: one single-pair call per pair (3 launches each), on a sample
    plain = None
    if not args.no_plain:
        n_plain = 2000
        a_t = [col.elements[int(off[i]):int(off[i + 1])] for i in range(k)]
        cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        pws = api.Workspace(dev)
        for i in range(50):
            api.sisi_into(a_t[pairs[i, 0]], a_t[pairs[i, 1]], cnt, None, pws, "ip", stream)
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for i in range(n_plain):
            api.sisi_into(a_t[pairs[i, 0]], a_t[pairs[i, 1]], cnt, None, pws, "ip", stream)
        p1.record(stream)
        p1.synchronize()
        pms = p0.elapsed_time(p1)
        plain = {"pairs_per_s": n_plain / (pms * 1e-3), "sample_pairs": n_plain,
                 "desc": "si_sisi(ip) per pair on the first 2000 pairs, one call (3 launches) each"}

    e2e = None
    if not args.no_e2e:
        h_pairs = torch.from_numpy(pairs.view(np.int32)).pin_memory()
        h_counts = torch.empty(npairs, dtype=torch.int32).pin_memory()
        e_steps = max(1, min(args.steps, args.e2e_steps))

        def e2e_step():
            with torch.cuda.stream(stream):
                dpairs.copy_(h_pairs, non_blocking=True)
                graph.launch(stream)
                h_counts.copy_(counts, non_blocking=True)
            stream.synchronize()

        e2e_step()
        rep.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e_steps):
            e2e_step()
        e1.record(stream)
        e1.synchronize()
        e_ms = e0.elapsed_time(e1)
        e_ms = rep.max(e_ms)
        e_step = e_ms / e_steps
        e2e = {"value": rep.rate(npairs, e_step), "unit": "pairs/s", "h2d_bytes_per_step": int(8 * npairs),
               "d2h_bytes_per_step": int(4 * npairs), "ms_per_step": e_step, "steps": e_steps,
               "note": "pool resident in HBM (the indexed collection); per step the query pairs go H2D and "
                       "the counts D2H through the graph"}
    graph.close()

    if rank != 0:
        rep.close()
        return
    peaks = json.load(open(PEAKS_PATH)) if os.path.exists(PEAKS_PATH) else {}
    sizes = np.diff(off)
    merge_elems = int(sizes[pairs[:, 0]].sum() + sizes[pairs[:, 1]].sum())
    alg_bytes = 4 * merge_elems + 12 * npairs
    peak = peaks.get("hbm_gbs", FALLBACK_HBM_GBS)
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": None, "kernel": "batch_kernel", "alg_bytes_per_launch": alg_bytes,
            "avg_launch_ms": kern_ms, "launches": int(k_n.value),
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "note": "algorithmic bytes of a full merge of every pair (4 B per element of both sets, pairs and "
                    "counts); search-technique pairs read less, so frac can exceed what a merge could reach"}
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        kind, threads, cval, desc, _ = batch_cpu_measure(el, off, pairs, 20000, steps=3, warmup=1)
        cpu = {"value": cval, "unit": "pairs/s", "cores": threads, "kind": kind, "sample": desc}
    codes_used = None
    if table is not None:
        tb = np.frombuffer(table, np.uint8)
        per_pair = tb[api.batch_buckets(el, off, pairs)]
        names = ["merge", "search", "hash_1024", "hash_512", "bitmap_16k", "bitmap_32k"]
        codes_used = {names[c]: int((per_pair == c).sum()) for c in range(api.BATCH_CODES) if (per_pair == c).any()}
    line = {
        "metric": "batched pairs/s", "value": value, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"], "technique": tech, "k": k, "pairs": npairs,
                   "elements": int(el.size), "merge_elements": merge_elems,
                   "l2": f"pool {el.size * 4 >> 20} MiB > 126 MB L2; no flush",
                   "graph": "one CUDA graph per step: key kernel, radix sort of the queue, the merge/search and "
                            "hash/bitmap batch kernels",
                   "autotune_s": tune_s if table is not None else None,
                   "pairs_per_technique": codes_used,
                   "parallelism": f"replicas{world}", "parity_vs_oracle": parity,
                   "plain_per_pair": plain,
                   "speedup_vs_plain": (value / world / plain["pairs_per_s"]) if plain else None},
        "roofline": roof,
        "e2e": e2e,
        # ours per step: the key kernel and one or two batch kernels (the sort is CUB's)
        "gpu_launches": (2 if tech in ("ip", "obs") else 3) * args.steps,
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
    }
    if bucket_times is not None:
        line["bucket_times"] = {"codes": ["merge", "search", "hash_1024", "hash_512", "bitmap_16k", "bitmap_32k"],
                                "buckets": bucket_times}
    print(json.dumps(line), flush=True)
    rep.close()


# Short runs of the other configurations, for the record of a default run.
EXTRAS = [  # workload, arguments, timed steps
    ("misi_dense", ["--technique", "mm", "--dtype", "int8"], 5),
    ("misi_dense", ["--technique", "mm", "--dtype", "fp8", "--no-plain"], 5),
    ("misi_powerlaw", ["--technique", "bitmap"], 5),
    ("batch_pairs", ["--technique", "auto"], 5),
    ("sisi_skewed", ["--technique", "auto"], 200),  # 0.03 ms steps
]


def other_workloads(args) -> list:
    out = []
    for wl, extra, steps in EXTRAS:
        cmd = [sys.executable, os.path.abspath(__file__), "--workload", wl, "--steps", str(steps), "--warmup", "3",
               "--no-e2e", "--no-cpu-baseline", "--no-extras", *extra]
        t0 = time.time()
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
            d = json.loads(r.stdout.strip().splitlines()[-1])
        except Exception as e:  # recorded, not fatal: the headline line stands on its own
            out.append({"workload": wl, "args": extra, "error": str(e)[:200]})
            continue
        roof = d.get("roofline") or {}
        cfg = d.get("config") or {}
        keep = {k: cfg[k] for k in ("technique", "operand", "parity_vs_oracle", "speedup_vs_plain",
                                     "plain_popcount_ms_per_step", "plain_per_pair") if k in cfg}
        keep.update({k: d[k] for k in ("technique", "parity_vs_oracle", "techniques") if k in d})
        out.append({"workload": wl, "metric": d["metric"], "value": d["value"], "unit": d["unit"],
                    "ms_per_step": d["ms_per_step"], "steps": d["steps"],
                    "roofline": {k: roof.get(k) for k in ("bound", "achieved", "peak", "unit", "frac", "kernel",
                                                           "avg_launch_ms", "cublas_int8_tops_measured",
                                                           "frac_of_cublas_int8") if k in roof},
                    "clocks": d.get("clocks"), **keep, "wall_s": round(time.time() - t0, 1)})
        log(f"{wl} {' '.join(extra)}: {d['value']:.4g} {d['unit']}")
    return out


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=sorted(WORKLOADS), default="sisi_large")
    p.add_argument("--technique", default="auto")
    p.add_argument("--count-only", dest="materialize", action="store_false")
    p.add_argument("--e2e-steps", type=int, default=10)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-parity", action="store_true")
    p.add_argument("--bucket-times", action="store_true",
                   help="batch: also time every technique code on every bucket of 200 pairs or more")
    p.add_argument("--no-plain", action="store_true",
                   help="dense / batch: skip timing the plain kernel (popcount / one call per pair)")
    p.add_argument("--dtype", choices=["int8", "fp8"], default="int8", help="dense: tensor-core operand type")
    p.add_argument("--no-techniques", action="store_true",
                   help="SISI: skip timing every technique on the workload's pair (outside the timed region)")
    p.add_argument("--no-extras", action="store_true",
                   help="SISI at N=1: skip the short runs of the other workloads added to the line")
    args = p.parse_args()
    if args.warmup < 3:
        p.error("--warmup must be >= 3")
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    kind = "misi" if args.workload.startswith("misi_") else "batch" if args.workload.startswith("batch_") else "sisi"
    if args.impl == "reference":
        {"misi": run_reference_dense, "batch": run_reference_batch, "sisi": run_reference_arm}[kind](args, rank)
    else:
        {"misi": run_ours_dense, "batch": run_ours_batch, "sisi": run_ours}[kind](args, rank, world)


if __name__ == "__main__":
    main()
