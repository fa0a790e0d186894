#!/usr/bin/env python3
"""Benchmark of the LDE + Poseidon2-Merkle commit (one JSON line on rank 0).

Default workload: one AIR instance of 2^22 rows x 256 base columns of uniform Goldilocks
elements, blowup 2 (LDE 2^23 rows), Poseidon2 width-16 row sponge and arity-4 tree — the
reference's production (W16, arity 4) pairing.  A step is one full commit: row-major trace in
HBM -> column-major LDE -> leaf digests -> every tree level -> root read back to the host.

  value  GElem/s = NExt * nCols / step time, inputs resident in HBM, CUDA events on the
         launching stream, max over ranks; every rank commits its own instance (weak scaling).
  e2e    the same metric through the reference-compatible C ABI (commit_witness /
         get_stream_proofs) from pinned host memory: each step copies its 8.6 GB trace to the
         device and reads its root back; the library's two stream slots overlap one step's copy
         with the previous step's kernels.

--impl reference times the reference's own CPU implementation (NTT_Goldilocks::LDE +
Poseidon2Goldilocks<16>::merkletree, compiled unmodified under oracle/_ref) with every host
thread, on the same full workload and the same seeded trace, in the same unit; that process loads
only the reference build.  Every arm checks its root against the reference CPU root of that trace
recorded in tests/golden/full_size.json.
"""
import argparse
import ctypes
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))

WORKLOADS = {
    "c2": dict(desc="single AIR 2^22 x 256 base columns, blowup 2, Poseidon2 W16 arity-4 tree",
               nbits=22, nbits_ext=23, ncols=256, arity=4),
    "c1": dict(desc="single AIR 2^16 x 32 base columns, blowup 2, Poseidon2 W16 arity-4 tree",
               nbits=16, nbits_ext=17, ncols=32, arity=4),
    # stage-2-style commit: 600 base + 60 cubic-extension columns (3 limbs each, hashed in row-major
    # limb order) = 780 words per row, blowup 4 (LDE 2^22 rows, 26 GB)
    "c4": dict(desc="stage-2 AIR 2^20 x (600 base + 60 cubic = 780 limbs), blowup 4, Poseidon2 W16 arity-4 tree",
               nbits=20, nbits_ext=22, ncols=780, arity=4),
    # profiling case of the 256-column workload: LDE 2.1 GB (larger than L2), ~4.3 GB on the device
    "c2s": dict(desc="single AIR 2^19 x 256 base columns, blowup 2, Poseidon2 W16 arity-4 tree",
                nbits=19, nbits_ext=20, ncols=256, arity=4),
}
METRIC = "LDE+Merkle commit GElem/s (NExt x nCols per second), bit-exact roots"
UNIT = "GElem/s"
P2_MULS = {8: 8 * 8 * 4 + 22 * (4 + 8), 12: 8 * 12 * 4 + 22 * (4 + 12), 16: 8 * 16 * 4 + 22 * (4 + 16)}
# Poseidon1: x^7 on every word of 8 full rounds, the dense pre-partial matrix P (W^2), and per partial
# round x0^7, a W-term dot product and W-1 products; the small-entry MDS M adds 32x64 products only
P1_MULS = {w: 8 * w * 4 + w * w + 22 * (4 + w + w - 1) for w in (8, 12, 16)}
HASH_NAME = {1: "Poseidon1", 2: "Poseidon2"}
IMAD_PER_MUL = 8  # four 32x32->64 partial products, two IMAD-pipe ops each


def load_package():
    name = "pil2_proofman_b200"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(REPO, "pil2-proofman_b200", "__init__.py")
    spec = importlib.util.spec_from_file_location(name, path, submodule_search_locations=[os.path.dirname(path)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except OSError:
        return {"hbm_gbs": 6650.0}, "fallback (6.65 TB/s, an earlier copy measurement on B200; MEASURED_PEAKS.json absent)"


def ncu_traffic(kernel, workload):
    """dram read+write bytes per launch from a committed ncu summary (profiles/traffic.txt)."""
    path = os.path.join(REPO, "profiles", "traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 3 and parts[0] == kernel and parts[1] == workload and not line.startswith("#"):
                    return float(parts[2])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", "b200_clocks_%d_%d.csv" % (os.getpid(), gpu_index))

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        power = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows), "power_w_max": max(power) if power else None}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_ram_gb():
    try:
        return os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") / 1e9
    except (ValueError, OSError, AttributeError):
        return 0.0


TRACE_SEED = 1000  # seed of the benchmarked trace on every rank (tests/golden/full_size.json pins its root)


def full_size_fixture(wl, family):
    """The reference CPU build's root for this workload's seeded trace under this hash family, if
    make_full_size.py recorded it."""
    path = os.path.join(REPO, "tests", "golden", "full_size.json")
    try:
        with open(path) as f:
            for s in json.load(f)["shapes"]:
                if (s["nBits"], s["nBitsExt"], s["nCols"], s["arity"], s["seed"], s.get("family", 2)) == (
                        wl["nbits"], wl["nbits_ext"], wl["ncols"], wl["arity"], TRACE_SEED, family):
                    return s
    except (OSError, KeyError, ValueError):
        pass
    return None


def bench_config(args, wl, world):
    """The config object both arms print (identical, so the two lines describe the same workload)."""
    nbits, nbe, ncols, arity = wl["nbits"], wl["nbits_ext"], wl["ncols"], wl["arity"]
    return {"workload": wl["desc"], "nBits": nbits, "nBitsExt": nbe, "nCols": ncols, "arity": arity,
            "hash": "%s W%d" % (HASH_NAME[args.hash_family], 4 * arity),
            "parallelism": "instance per GPU" if world > 1 else "single GPU",
            "trace_seed": TRACE_SEED,
            "l2": ("inputs (%.1f GB) larger than L2; no flush" if (1 << nbits) * ncols * 8 > 126e6 else
                   "inputs (%.3f GB) fit in L2; no flush") % ((1 << nbits) * ncols * 8 / 1e9)}


REF_MAX_STEPS = 6


def time_reference_cpu(wl, reps, warmup, family=2):
    """The reference's CPU commit (NTT_Goldilocks::LDE + merkletree, compiled unmodified under oracle/_ref)
    of the full workload shape, with every host thread, as commit_witness_cpu runs it
    (starks_api.cpp:683-721: LDE into the extended buffer with a caller work buffer, then the tree).
    The trace is the benchmarked one (seeded rule of ref_fill_random == the product's generator), so the
    root is the one the GPU arm must produce.  Returns (GElem/s, seconds per rep, threads, sample, root)."""
    sys.path.insert(0, REPO)
    import oracle  # CPU baseline / reference legs only

    threads = cpu_threads()
    ref = oracle.RefCPU(threads=threads, family=family)
    nb, nbe = wl["nbits"], wl["nbits_ext"]
    ncols, arity = wl["ncols"], wl["arity"]
    N, NExt = 1 << nb, 1 << nbe
    # the reference's LDE work buffer is NExt x ncols (nblock 1); on a host with less memory than the
    # trace, LDE, buffer and tree need, the buffer is split over column blocks (same values)
    need_gb = (N + 2 * NExt) * ncols * 8 / 1e9
    nblock = 1 if host_ram_gb() > 1.6 * need_gb else 4
    trace = ref.fill_random(N * ncols, TRACE_SEED).reshape(N, ncols)
    lde = np.empty((NExt, ncols), dtype=np.uint64)
    buf = np.empty(NExt * -(-ncols // nblock), dtype=np.uint64)
    tree = np.empty(oracle.tree_num_elements(NExt, arity), dtype=np.uint64)
    times = []
    for i in range(warmup + reps):
        t0 = time.perf_counter()
        ref.lde_raw(trace, nbe, out=lde, buffer=buf, nblock=nblock)
        ref.merkletree_raw(lde, arity, tree=tree)
        t1 = time.perf_counter()
        if i >= warmup:
            times.append(t1 - t0)
    root = oracle.RefCPU.canon(tree[-4:])
    sec = sum(times) / len(times)
    sample = ("full workload: %d x %d trace -> %d x %d LDE + %s W%d arity-%d tree, %s build, %d warm-up + %d "
              "timed commits, LDE work buffer in %d column block(s), %s" % (
                  N, ncols, NExt, ncols, HASH_NAME[family], 4 * arity, arity, ref.variant, warmup, reps, nblock,
                  cpu_model()))
    return NExt * ncols / sec / 1e9, sec, threads, sample, root


def run_reference(args, wl):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    # every step is one full commit of the workload (~15 s at C2 on 16 cores): at most
    # REF_MAX_STEPS timed and one warm-up, so that the arm ends within a few minutes
    reps, warm = max(1, min(args.steps, REF_MAX_STEPS)), min(args.warmup, 1)
    val, sec, threads, sample, root = time_reference_cpu(wl, reps, warm, args.hash_family)
    fx = full_size_fixture(wl, args.hash_family)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 6), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded uniform Goldilocks)",
        "config": bench_config(args, wl, args.gpus),
        "cpu_baseline": {"value": round(val, 6), "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(val, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "root": [hex(int(v)) for v in root],
        "root_matches_fixture": None if fx is None else [int(v) for v in root] == fx["root"],
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, wl):
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    pkg = load_package()
    pkg.init(local)
    pkg.set_native_hash_family(args.hash_family)
    nbits, nbe, ncols, arity = wl["nbits"], wl["nbits_ext"], wl["ncols"], wl["arity"]
    N, NExt = 1 << nbits, 1 << nbe
    elems = NExt * ncols
    dev = torch.device("cuda", local)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- resident-input path (value) -------------------------------------------------
    stream = torch.cuda.current_stream()
    trace = torch.empty(N * ncols, dtype=torch.int64, device=dev)
    scratch = torch.empty(pkg.lde_scratch_words(nbits, ncols), dtype=torch.int64, device=dev)
    lde = torch.empty(elems, dtype=torch.int64, device=dev)
    tree = torch.empty(pkg.tree_num_elements(NExt, arity), dtype=torch.int64, device=dev)
    pkg.fill_random_device(trace, N * ncols, TRACE_SEED, stream)
    tuned = None
    if args.autotune:  # untimed set-up: pick the NTT window plan for this shape
        t_ms, kf, kr = pkg.autotune_lde(nbits, nbe, ncols)
        tuned = {"kfirst": kf, "krest": kr, "probe_ms": round(t_ms, 3)}
    args.tuned_plan = tuned
    roots = []
    for _ in range(args.warmup):
        roots.append(pkg.commit_device(lde, tree, trace, nbits, nbe, ncols, arity, scratch, stream=stream))
    assert all((r == roots[0]).all() for r in roots)

    pkg.timing_enable(True)
    pkg.timing_reset()
    launches0 = pkg.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            pkg.commit_device(lde, tree, trace, nbits, nbe, ncols, arity, scratch, stream=stream)
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1)
    launches = pkg.launch_count() - launches0
    cats = pkg.timing()
    pkg.timing_enable(False)
    clocks = clk.summary()
    ms = max_over_ranks(ms)
    value = world * elems * args.steps / (ms * 1e-3) / 1e9

    # ---- roofline of the dominant kernel and of the NTT passes ------------------------
    peaks, peak_kind = measured_peaks()
    imad = pkg.probe_imad()
    w = 4 * arity
    perms_per_row = max(1, -(-ncols // (w - 4)))
    leaf_ms = cats["leaf_hash"][0] / max(1, cats["leaf_hash"][1])
    mul_table = P1_MULS if args.hash_family == 1 else P2_MULS
    muls = NExt * perms_per_row * mul_table[w]
    achieved_gmul = muls / (leaf_ms * 1e-3) / 1e9
    peak_gmul = imad / IMAD_PER_MUL
    ntt_ms = sum(cats[c][0] for c in ("transpose", "ntt_inverse", "ntt_forward")) / args.steps
    ntt_bytes = 8 * ncols * (N + NExt)
    ntt_gbs = ntt_bytes / (ntt_ms * 1e-3) / 1e9
    # the NTT windows are integer-issue bound: radix-2 butterflies of the iNTT (N) and of the NTT
    # (NExt, without its first log2(blowup) copy stages), one Goldilocks multiplication each
    butterflies = ncols * ((N // 2) * nbits + (NExt // 2) * nbits)
    ntt_kernel_ms = sum(cats[c][0] for c in ("ntt_inverse", "ntt_forward")) / args.steps
    ntt_gmul = butterflies / (ntt_kernel_ms * 1e-3) / 1e9
    ntt_int = {"bound": "int32_imad", "achieved": round(ntt_gmul, 2), "peak": round(peak_gmul, 2),
               "unit": "G butterfly-mul/s", "frac": round(ntt_gmul / peak_gmul, 4),
               "algorithmic": "nCols x (N/2 x log2 N + NExt/2 x log2 N) radix-2 butterflies, one multiplication "
                              "each; time = NTT window kernels only"}
    # the row-major -> column-major transpose in front of the LDE is the one pure HBM pass
    transpose_roof = None
    if cats["transpose"][1] and cats["transpose"][0] > 0:
        tr_ms = cats["transpose"][0] / cats["transpose"][1]
        tr_gbs = 16 * N * ncols / (tr_ms * 1e-3) / 1e9
        transpose_roof = {"bound": "hbm", "achieved": round(tr_gbs, 1), "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                          "frac": round(tr_gbs / peaks.get("hbm_gbs", 6650.0), 4),
                          "algorithmic_bytes": "16 x N x nCols per commit (read the row-major trace, write it "
                                               "column-major)"}
    roofline = {
        "kernel": "leaf_hash_kernel<%d,%d>" % (w, args.hash_family),
        "bound": "int32_imad",
        "achieved": round(achieved_gmul, 2), "peak": round(peak_gmul, 2), "unit": "G Goldilocks-mul/s",
        "frac": round(achieved_gmul / peak_gmul, 4),
        "traffic": ncu_traffic("leaf_hash_kernel", args.workload) if args.hash_family == 2 else None,
        "algorithmic": "%d permutations/row x %d muls (W%d) per row, %d IMAD-pipe ops per mul; peak = "
                       "measured IMAD probe %.0f G/s / %d" % (perms_per_row, mul_table[w], w, IMAD_PER_MUL, imad,
                                                             IMAD_PER_MUL),
        "ntt": {"bound": "hbm", "achieved": round(ntt_gbs, 1), "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                "frac": round(ntt_gbs / peaks.get("hbm_gbs", 6650.0), 4),
                "peak_kind": peak_kind,
                "algorithmic_bytes": "8 x nCols x (N + NExt) per commit (read trace once, write LDE once)",
                "traffic": ncu_traffic("ntt_lde", args.workload),
                "int": ntt_int},
        "transpose": transpose_roof,
    }
    kernel_ms = {k: round(v[0] / args.steps, 3) for k, v in cats.items()}

    # ---- end to end through the reference C ABI from pinned host memory ---------------
    if args.no_e2e:
        e2e = None
        return finish(args, wl, pkg, dist, rank, world, value, ms, launches, kernel_ms, roofline, clocks, roots,
                      None)
    host = torch.empty(N * ncols, dtype=torch.int64, pin_memory=True)
    host.copy_(trace)
    del trace, scratch, lde, tree
    torch.cuda.empty_cache()
    lib = pkg.load()
    pkg.set_hash_family(args.hash_family)
    bufs = pkg.DeviceBuffers(arity=arity, n_streams=2)
    shape = pkg.StarkShape(nbits, nbe, ncols, arity)
    params = pkg.StepsParams()
    params.trace = host.data_ptr()
    root_bufs = [np.zeros(4, dtype=np.uint64) for _ in range(args.warmup + args.steps)]
    for i in range(args.warmup):
        lib.commit_witness(shape.setup_ptr, ctypes.addressof(params), i, 0, 0, root_bufs[i].ctypes.data, bufs.ptr, b"")
    lib.get_stream_proofs(bufs.ptr)
    barrier()
    t0 = time.perf_counter()
    for i in range(args.warmup, args.warmup + args.steps):
        sid = lib.commit_witness(shape.setup_ptr, ctypes.addressof(params), i, 0, 0, root_bufs[i].ctypes.data, bufs.ptr,
                                 b"")
        if sid >= 2:
            raise RuntimeError(lib.b200_last_error().decode())
    lib.get_stream_proofs(bufs.ptr)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s)
    if bufs.error() != 0:
        raise RuntimeError("commit_witness failed: %s" % lib.b200_last_error().decode())
    if not all((r == roots[0]).all() for r in root_bufs):
        raise RuntimeError("e2e roots differ from the resident-path root")
    e2e = world * elems * args.steps / e2e_s / 1e9
    bufs.close()
    e2e_obj = {"value": round(e2e, 4), "unit": UNIT, "h2d_bytes_per_step": N * ncols * 8, "d2h_bytes_per_step": 32,
               "api": "commit_witness + get_stream_proofs, 2 stream slots, pinned host trace"}
    return finish(args, wl, pkg, dist, rank, world, value, ms, launches, kernel_ms, roofline, clocks, roots, e2e_obj)


def finish(args, wl, pkg, dist, rank, world, value, ms, launches, kernel_ms, roofline, clocks, roots, e2e_obj):
    nbits, nbe, ncols, arity = wl["nbits"], wl["nbits_ext"], wl["ncols"], wl["arity"]
    N = 1 << nbits
    w = 4 * arity
    fx = full_size_fixture(wl, args.hash_family)
    if fx is not None and [int(v) for v in roots[0]] != fx["root"]:
        raise RuntimeError("root %s differs from the reference CPU root %s of the same trace (full_size.json)"
                           % ([hex(int(v)) for v in roots[0]], [hex(v) for v in fx["root"]]))
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded uniform Goldilocks)",
        "config": bench_config(args, wl, world),
        "e2e": e2e_obj,
        "gpu_launches": int(launches),
        "kernel_ms_per_step": kernel_ms,
        "ntt_plan": getattr(args, "tuned_plan", None) or "default (first window <= 12 stages, later <= 11)",
        "roofline": roofline,
        "clocks": clocks,
        "root": [hex(int(v)) for v in roots[0]] if rank == 0 else None,
        "root_check": ("equal to the reference CPU build's root of the same seeded trace "
                       "(tests/golden/full_size.json)" if fx is not None else "no reference fixture for this shape"),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        val, sec, threads, sample, cpu_root = time_reference_cpu(wl, 1, 1, args.hash_family)
        line["cpu_baseline"] = {"value": round(val, 6), "unit": UNIT, "cores": threads, "kind": "reference",
                                "sample": sample, "root_equal": bool((cpu_root == roots[0]).all())}
        if not (cpu_root == roots[0]).all():
            raise RuntimeError("the reference CPU root of the benchmarked trace differs from the GPU root")
    if rank == 0 and world == 1 and args.workload == "c2" and not args.no_legs:
        # the metric's other two parts, measured in the same run: the batched mixed-size commit
        # against the plain per-instance path, and served-stream latency
        res = batched_vs_plain("c3", args.budget_gb)
        line["batched"] = {k: v for k, v in res.items() if k != "workload"}
        per_rate, npool = serve_rates([5.0], args.serve_seconds, args.pool, args.serve_budget_gb, args.slots,
                                      args.serve_timeout, serial=False)
        line["serve"] = dict(per_rate[0], workload="Poisson arrivals at 5 requests/s for %.0f s; shapes: %d drawn "
                             "from the 64-instance C3 distribution (80%%) and 2^20 x 780 blowup 4 (20%%)"
                             % (args.serve_seconds, npool - 1))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def c3_shapes(seed=3, n=64):
    """64 AIR instances: log2 rows uniform in 16..22, base columns uniform in [16, 512], blowup 2 for
    48 of them and 4 for 16, arity 4 (the reference's production W16 pairing)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nbits = rng.integers(16, 23, size=n)
    ncols = rng.integers(16, 513, size=n)
    blow = np.array([1] * 48 + [2] * 16)
    rng.shuffle(blow)
    return [(int(a), int(a + b), int(c)) for a, b, c in zip(nbits, blow, ncols)]


def c3small_shapes(seed=4, n=256):
    """256 small AIR instances: log2 rows uniform in 10..16, columns uniform in [8, 128], blowup 2
    for three quarters and 4 for a quarter: the regime where per-instance launches dominate."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nbits = rng.integers(10, 17, size=n)
    ncols = rng.integers(8, 129, size=n)
    blow = np.array([1] * (3 * n // 4) + [2] * (n - 3 * n // 4))
    rng.shuffle(blow)
    return [(int(a), int(a + b), int(c)) for a, b, c in zip(nbits, blow, ncols)]


BATCH_SETS = {
    "c3": (c3_shapes, "64 AIR instances, log2 rows U{16..22}, cols U[16,512], blowup 2 (48) / 4 (16)"),
    "c3small": (c3small_shapes, "256 AIR instances, log2 rows U{10..16}, cols U[8,128], blowup 2 (3/4) / 4 (1/4)"),
}


def instance_words(pkg, nb, nbe, nc, arity=4):
    N, NExt = 1 << nb, 1 << nbe
    return N * nc, N * nc, NExt * nc, pkg.tree_num_elements(NExt, arity)


def batched_vs_plain(workload, budget_gb, autotune=False):
    """Batched mixed-size commit vs the plain one-instance-at-a-time path on the same data and device,
    in waves bounded by a device-memory budget; roots compared bit for bit.  Returns a dict."""
    import torch

    pkg = load_package()
    pkg.init(0)
    lib = pkg.load()
    dev = torch.device("cuda", 0)
    make_shapes, shapes_desc = BATCH_SETS[workload]
    shapes = make_shapes()
    tuned = {}
    if autotune:  # untimed set-up: a plan per distinct (nBits, nBitsExt, column bucket)
        for nb, nbe, nc in shapes:
            key = (nb, nbe, 0 if nc <= 32 else 1 if nc <= 128 else 2 if nc <= 512 else 3)
            if key not in tuned:
                t_ms, kf, kr = pkg.autotune_lde(nb, nbe, nc)
                tuned[key] = (kf, kr)
    budget = int(budget_gb * 2**30) // 8  # words
    waves, cur, used = [], [], 0
    for i, (nb, nbe, nc) in enumerate(shapes):
        w = sum(instance_words(pkg, nb, nbe, nc))
        if cur and used + w > budget:
            waves.append(cur)
            cur, used = [], 0
        cur.append(i)
        used += w
    waves.append(cur)
    stream = torch.cuda.Stream()
    total_elems = sum((1 << nbe) * nc for _, nbe, nc in shapes)
    t_plain = t_batch = 0.0
    launches_plain = launches_batch = 0
    mismatches = 0
    for wave in waves:
        sizes = [instance_words(pkg, *shapes[i]) for i in wave]
        arena = torch.empty(sum(sum(s) for s in sizes) + 64 * len(wave), dtype=torch.int64, device=dev)
        base = arena.data_ptr()
        descs = (pkg.BatchInstance * len(wave))()
        off = 0
        for j, i in enumerate(wave):
            nb, nbe, nc = shapes[i]
            ptrs = []
            for words in sizes[j]:
                ptrs.append(base + 8 * off)
                off += words + 8  # keep 64-byte alignment slack
            d = descs[j]
            d.d_trace, d.d_scratch, d.d_lde, d.d_tree = ptrs
            d.nBits, d.nBitsExt, d.nCols, d.arity = nb, nbe, nc, 4
            pkg.fill_random_device(ptrs[0], (1 << nb) * nc, 5000 + i)
        torch.cuda.synchronize()
        # plain: one instance after another on one stream
        roots_plain = np.zeros((len(wave), 4), dtype=np.uint64)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            for rep in range(2):  # warm-up, then timed
                l0 = pkg.launch_count()
                ev0.record(stream)
                for j in range(len(wave)):
                    d = descs[j]
                    r = pkg.commit_device(d.d_lde, d.d_tree, d.d_trace, d.nBits, d.nBitsExt, d.nCols, 4, d.d_scratch,
                                          stream=stream)
                    roots_plain[j] = r
                ev1.record(stream)
                torch.cuda.synchronize()
            t_plain += ev0.elapsed_time(ev1)
            launches_plain += pkg.launch_count() - l0
            # batched: grouped kernels + persistent leaves, captured once in a CUDA graph
            plan = lib.b200_batch_plan_new(descs, len(wave))
            if not plan:
                raise RuntimeError(lib.b200_last_error().decode())
            roots_batch = np.zeros((len(wave), 4), dtype=np.uint64)
            for rep in range(2):
                ev0.record(stream)
                rc = lib.b200_batch_plan_run(plan, roots_batch.ctypes.data, stream.cuda_stream, 1)
                ev1.record(stream)
                torch.cuda.synchronize()
                if rc:
                    raise RuntimeError(lib.b200_last_error().decode())
            t_batch += ev0.elapsed_time(ev1)
            launches_batch += int(lib.b200_batch_plan_launches(plan))
            lib.b200_batch_plan_free(plan)
        mismatches += int((roots_plain != roots_batch).any(axis=1).sum())
        del arena
        torch.cuda.empty_cache()
    return {
        "workload": workload, "desc": shapes_desc + ", Poseidon2 W16 arity 4, device budget %.0f GiB per wave"
        % budget_gb,
        "value": round(total_elems / (t_batch * 1e-3) / 1e9, 4), "unit": UNIT,
        "plain_value": round(total_elems / (t_plain * 1e-3) / 1e9, 4),
        "batched_over_plain": round(t_plain / t_batch, 4),
        "ms_batched": round(t_batch, 2), "ms_plain": round(t_plain, 2),
        "instances": len(shapes), "waves": len(waves), "total_lde_elements": total_elems,
        "launches_plain": launches_plain, "launches_batched": launches_batch,
        "roots_bit_exact": mismatches == 0, "mismatched_roots": mismatches,
        "ntt_plans": {"%d/%d/%d" % k: list(v) for k, v in tuned.items()} if tuned else "default",
    }


def run_batched(args):
    res = batched_vs_plain(args.workload, args.budget_gb, args.autotune)
    line = {"metric": METRIC + " - batched vs plain", "workload": args.workload, "value": res["value"], "unit": UNIT,
            "config": {"workload": res["desc"]}, "n_gpus": 1, "higher_is_better": True, "dtype": "u64",
            "data": "synthetic (seeded uniform Goldilocks)"}
    line.update({k: v for k, v in res.items() if k not in ("value", "desc", "workload")})
    print(json.dumps(line), flush=True)
    return 0 if res["roots_bit_exact"] else 1


def serve_pool(lib, n_c3, seed=12):
    """Request shapes: n_c3 drawn from the 64-instance C3 distribution and the C4 shape (2^20 x 780,
    blowup 4), each with one seeded pinned host trace."""
    import torch

    pool = c3_shapes(seed=seed, n=n_c3) + [(20, 22, 780)]
    hosts = []
    for i, (nb, nbe, nc) in enumerate(pool):
        h = torch.empty((1 << nb) * nc, dtype=torch.int64, pin_memory=True)
        lib.b200_fill_random_host(h.data_ptr(), h.numel(), 7000 + i)
        hosts.append(h)
    return pool, hosts


def gpu_timeline(units):
    """Device timeline of a served stream from its units' (copies issued, copies done, kernels
    started, kernels done) times: ms with kernels running; the gaps between one unit's kernels and
    the next, split into the part before the next unit was issued (no request waiting, or the host
    admitted it late) and the part after (its host-to-device copy had not landed: the GPU waited
    for PCIe)."""
    spans = sorted((st, dn, iss) for iss, cp, st, dn in units if st >= 0 and dn >= 0)
    if not spans:
        return {}
    busy = sum(dn - st for st, dn, _ in spans)
    copy_wait = not_issued = 0.0
    for (_, prev_dn, _), (st, _, iss) in zip(spans, spans[1:]):
        gap = max(0.0, st - prev_dn)
        late = min(gap, max(0.0, iss - prev_dn))
        not_issued += late
        copy_wait += gap - late
    return {"gpu_kernels_ms": round(busy, 1), "gpu_waiting_for_copy_ms": round(copy_wait, 1),
            "gpu_idle_before_issue_ms": round(not_issued, 1), "gpu_span_ms": round(spans[-1][1] - spans[0][0], 1)}


def serve_stream(lib, pool, hosts, arrivals, picks, mode, budget_gb, slots, timeout_s):
    """Submit requests at the given arrival times to a commit server (mode 1 continuous batching,
    0 FIFO); returns (latencies ms, wall s, roots, stats)."""
    nreq = len(picks)
    srv = lib.b200_server_new(0, int(budget_gb * 2**30), slots)
    if not srv:
        raise RuntimeError(lib.b200_last_error().decode())
    roots = np.zeros((nreq, 4), dtype=np.uint64)
    ids, lat, done = [None] * nreq, [None] * nreq, 0
    lat_c = ctypes.c_double()
    try:
        if lib.b200_server_configure(srv, mode, 1 << 26, 64) != 0:
            raise RuntimeError(lib.b200_last_error().decode())
        t0 = time.perf_counter()
        nxt = 0
        while done < nreq:
            now = time.perf_counter() - t0
            while nxt < nreq and arrivals[nxt] <= now:
                nb, nbe, nc = pool[picks[nxt]]
                rid = lib.b200_server_submit(srv, hosts[picks[nxt]].data_ptr(), nb, nbe, nc, 4, roots[nxt].ctypes.data)
                if rid < 0:
                    raise RuntimeError(lib.b200_last_error().decode())
                ids[nxt] = rid
                nxt += 1
            for i in range(nxt):
                if lat[i] is None:
                    st = lib.b200_server_status(srv, ids[i], ctypes.byref(lat_c))
                    if st < 0:
                        raise RuntimeError("status %d: %s" % (st, lib.b200_last_error().decode()))
                    if st == 1:
                        lat[i] = lat_c.value
                        lib.b200_server_release(srv, ids[i])  # frees its device memory
                        done += 1
            if now > timeout_s:
                raise RuntimeError("served stream did not finish within %.0f s" % timeout_s)
            time.sleep(0.001)
        wall = time.perf_counter() - t0
        st = (ctypes.c_uint64 * 7)()
        lib.b200_server_stats(srv, st, 7)
        times, g = (ctypes.c_double * 3)(), (ctypes.c_double * 4)()
        waits, service, units = [], [], set()
        for rid in ids:
            lib.b200_server_request_times(srv, rid, times)
            waits.append(times[1] - times[0])
            service.append(times[2] - times[1])
            lib.b200_server_request_gpu_times(srv, rid, g)
            units.add(tuple(g))  # a batched unit's requests share its timeline
        stats = {"plain_units": st[0], "batched_units": st[1], "batched_requests": st[2], "waited_for_block": st[3],
                 "overtakes": st[4], "host_enqueue_ms": round(st[5] / 1e3, 1),
                 "host_alloc_ms": round(st[6] / 1e3, 1),
                 "mean_wait_to_admission_ms": round(float(np.mean(waits)), 2),
                 "mean_admission_to_done_ms": round(float(np.mean(service)), 2), **gpu_timeline(units)}
    finally:
        lib.b200_server_free(srv)
    return lat, wall, roots, stats


def serve_rates(rates, duration, n_c3, budget_gb, slots, timeout_s, serial=True, repeats=1):
    """Poisson request streams at each rate for `duration` seconds of arrivals, served by the
    continuous-batching server and by the FIFO server on the same arrivals; p50/p99 latency and
    GElem/s of each, and the GElem/s of serial plain commits of the same request list.  With
    repeats > 1 each mode serves the stream that many times, the modes alternating in mirrored order
    (batching, FIFO, FIFO, batching, ...) so that neither always runs first; the latencies reported
    are the means over a mode's runs, each run kept under "runs".  Near saturation a few percent of
    throughput moves the queueing delay a lot, so single runs of the two modes compare poorly."""
    import torch

    pkg = load_package()
    pkg.init(0)
    lib = pkg.load()
    # the server reserves its budget on the device when created: keep it within what is free
    torch.cuda.empty_cache()
    free_gb = torch.cuda.mem_get_info(0)[0] / 2**30
    budget_gb = min(budget_gb, free_gb - 4.0)
    pool, hosts = serve_pool(lib, n_c3)
    # untimed warm-up: every shape once through each mode (module loading, first device allocations)
    for mode in (1, 0):
        serve_stream(lib, pool, hosts, np.zeros(len(pool)), list(range(len(pool))), mode, budget_gb, slots, timeout_s)
    rng = np.random.Generator(np.random.PCG64(11))
    out = []
    for rate in rates:
        nreq = max(1, int(round(rate * duration)))
        picks = [len(pool) - 1 if rng.random() < 0.2 else int(rng.integers(0, len(pool) - 1)) for _ in range(nreq)]
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=nreq))
        elems = sum((1 << pool[p][1]) * pool[p][2] for p in picks)
        entry = {"rate_per_s": rate, "requests": nreq, "arrivals_s": round(float(arrivals[-1]), 2)}
        all_roots = []
        modes = ((1, "continuous_batching"), (0, "fifo"))
        runs = {name: [] for _, name in modes}
        for k in range(repeats):
            for mode, name in (modes if k % 2 == 0 else modes[::-1]):
                lat, wall, roots, stats = serve_stream(lib, pool, hosts, arrivals, picks, mode, budget_gb, slots,
                                                       timeout_s)
                all_roots.append(roots)
                runs[name].append({"wall_s": round(wall, 3), "throughput_gelem_s": round(elems / wall / 1e9, 4),
                                   "p50_ms": round(float(np.percentile(lat, 50)), 2),
                                   "p99_ms": round(float(np.percentile(lat, 99)), 2),
                                   "max_ms": round(float(np.max(lat)), 2), **stats})
        for name, rs in runs.items():
            if len(rs) == 1:
                entry[name] = rs[0]
            else:
                entry[name] = {key: round(float(np.mean([r[key] for r in rs])), 4 if key.startswith("through") else 2)
                               for key in ("wall_s", "throughput_gelem_s", "p50_ms", "p99_ms", "max_ms")}
                entry[name]["runs"] = rs
        if serial:
            # the same request list as plain commits one after another, all queued at time 0
            _, wall, roots, _ = serve_stream(lib, pool, hosts, np.zeros(nreq), picks, 0, budget_gb, 1, timeout_s)
            all_roots.append(roots)
            entry["serial_plain"] = {"wall_s": round(wall, 3), "throughput_gelem_s": round(elems / wall / 1e9, 4)}
        # every served root equals the root of the same trace served any other way
        for k in range(len(pool)):
            rk = [r[i] for r in all_roots for i in range(nreq) if picks[i] == k]
            if rk and not all((x == rk[0]).all() for x in rk):
                raise RuntimeError("served roots differ for one input")
        entry["roots_consistent"] = True
        entry["device_budget_gib"] = round(budget_gb, 1)
        out.append(entry)
    del hosts
    return out, len(pool)


def run_serving(args):
    """Served request stream (C5): Poisson arrivals at each rate, request shapes drawn from the C3
    distribution with a fifth shaped like C4, admitted by the commit server under a device-memory
    budget; each request's LDE and tree stay resident until it completes and is released."""
    rates = [float(r) for r in args.rates.split(",")]
    per_rate, npool = serve_rates(rates, args.duration, args.pool, args.serve_budget_gb, args.slots,
                                  args.serve_timeout, repeats=args.serve_repeats)
    line = {"metric": "served commit stream: request latency p50/p99 and throughput, continuous batching vs FIFO",
            "workload": "c5", "unit": "ms", "value": per_rate[0]["continuous_batching"]["p99_ms"],
            "higher_is_better": False, "per_rate": per_rate,
            "config": {"workload": "Poisson arrivals for %.0f s per rate; shapes: %d drawn from the 64-instance C3 "
                                   "distribution (80%%) and 2^20 x 780 blowup 4 (20%%); Poseidon2 W16 arity 4"
                                   % (args.duration, npool - 1),
                       "device_budget_gib": args.serve_budget_gb, "slots": args.slots,
                       "runs_per_mode": args.serve_repeats},
            "n_gpus": 1, "dtype": "u64", "data": "synthetic (seeded uniform Goldilocks)"}
    print(json.dumps(line), flush=True)
    return 0


def run_extras(args):
    """Throughput of the commit's consumers and variants at realistic sizes (one JSON line):
    Q-stage commit (computeQ + tree), FRI query openings from a resident commit, bit-packed,
    indexed and streaming commits.  Inputs resident on the device except the streaming commit,
    whose packed rows are read from pinned host memory as the reference's slot commit does."""
    import torch

    pkg = load_package()
    pkg.init(0)
    dev = torch.device("cuda", 0)
    s = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    spread = {}

    def timed(fn, reps, name=None):
        """mean ms per call over reps calls (CUDA events on s); per-call min/max kept in spread"""
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(reps + 1)]
        evs[0].record(s)
        for i in range(reps):
            fn()
            evs[i + 1].record(s)
        torch.cuda.synchronize()
        per = [evs[i].elapsed_time(evs[i + 1]) for i in range(reps)]
        if name:
            spread[name] = [round(min(per), 3), round(max(per), 3)]
        return evs[0].elapsed_time(evs[reps]) / reps

    def breakdown(fn):
        """per-category device ms of one untimed call (the unpack kernels count as transpose)"""
        torch.cuda.synchronize()
        pkg.timing_reset()
        pkg.timing_enable(True)
        try:
            fn()
            torch.cuda.synchronize()
            return {k: round(v[0], 3) for k, v in pkg.timing().items() if v[1]}
        finally:
            pkg.timing_enable(False)

    out = {}
    # Q stage: N = 2^22, NExt = 2^23, qDeg 2, qDim 3 (cubic extension limbs)
    nb, nbe, qdeg, qdim = 22, 23, 2, 3
    q = torch.empty((1 << nbe) * qdim, dtype=torch.int64, device=dev)
    pkg.fill_random_device(q, q.numel(), 11, s)
    cmq = torch.empty((1 << nbe) * qdeg * qdim, dtype=torch.int64, device=dev)
    qtree = torch.empty(pkg.tree_num_elements(1 << nbe, 4), dtype=torch.int64, device=dev)
    qscr = torch.empty(pkg.q_scratch_words(nbe, qdim), dtype=torch.int64, device=dev)
    ms = timed(lambda: pkg.commit_q_device(cmq, qtree, q, nb, nbe, qdeg, qdim, 4, qscr, stream=s), args.steps)
    out["q_stage"] = {"shape": "N 2^22 -> NExt 2^23, qDeg 2 x qDim 3, arity 4", "ms": round(ms, 3),
                      "gelem_s": round((1 << nbe) * qdeg * qdim / ms / 1e6, 3),
                      "kernel_ms": breakdown(lambda: pkg.commit_q_device(cmq, qtree, q, nb, nbe, qdeg, qdim, 4, qscr,
                                                                         stream=s))}
    del q, cmq, qtree, qscr
    # query openings: 2^19 x 256 commit, 2^20-row tree, 1024 queries
    nb, nbe, nc = 19, 20, 256
    tr = torch.empty((1 << nb) * nc, dtype=torch.int64, device=dev)
    pkg.fill_random_device(tr, tr.numel(), 12, s)
    lde = torch.empty((1 << nbe) * nc, dtype=torch.int64, device=dev)
    tree = torch.empty(pkg.tree_num_elements(1 << nbe, 4), dtype=torch.int64, device=dev)
    scr = torch.empty((1 << nb) * nc, dtype=torch.int64, device=dev)
    pkg.commit_device(lde, tree, tr, nb, nbe, nc, 4, scr, stream=s)
    nq = 1024
    rows = torch.from_numpy((np.random.default_rng(5).integers(0, 1 << nbe, nq)).astype(np.int64)).to(dev)
    words = pkg.query_proof_words(1 << nbe, nc, 4)
    opn = torch.empty(nq * words, dtype=torch.int64, device=dev)
    ms = timed(lambda: pkg.query_openings_device(opn, lde, 1 << nbe, nc, tree, 4, rows, nq, stream=s), 20)
    out["query_openings"] = {"shape": "1024 openings of 2^20-row x 256-column commit (%d words each)" % words,
                             "ms": round(ms, 4), "openings_per_s": round(nq / ms * 1e3, 1)}
    del tr, lde, tree, scr, opn
    # packed commit: 2^22 x 64 columns of 32 bits (half the plain trace's bytes)
    nb, nbe, nc, wbits = 22, 23, 64, 32
    bits = [wbits] * nc
    wpr = pkg.packed_words_per_row(bits)
    packed = torch.empty((1 << nb) * wpr, dtype=torch.int64, device=dev)
    pkg.fill_random_device(packed, packed.numel(), 13, s)
    lde = torch.empty((1 << nbe) * nc, dtype=torch.int64, device=dev)
    tree = torch.empty(pkg.tree_num_elements(1 << nbe, 4), dtype=torch.int64, device=dev)
    scr = torch.empty((1 << nb) * nc, dtype=torch.int64, device=dev)
    ms = timed(lambda: pkg.commit_packed_device(lde, tree, packed, wpr, bits, nb, nbe, 4, scr, stream=s), args.steps,
               "packed_commit")
    out["packed_commit"] = {"shape": "2^22 x 64 columns x 32 bits, blowup 2", "ms": round(ms, 3),
                            "gelem_s": round((1 << nbe) * nc / ms / 1e6, 3),
                            "kernel_ms": breakdown(lambda: pkg.commit_packed_device(lde, tree, packed, wpr, bits, nb,
                                                                                    nbe, 4, scr, stream=s))}
    tr = torch.empty((1 << nb) * nc, dtype=torch.int64, device=dev)
    pkg.fill_random_device(tr, tr.numel(), 17, s)
    ms = timed(lambda: pkg.commit_device(lde, tree, tr, nb, nbe, nc, 4, scr, stream=s), args.steps,
               "plain_commit_same_shape")
    out["plain_commit_same_shape"] = {"shape": "2^22 x 64 columns, row-major u64 trace, blowup 2", "ms": round(ms, 3),
                                      "gelem_s": round((1 << nbe) * nc / ms / 1e6, 3),
                                      "kernel_ms": breakdown(lambda: pkg.commit_device(lde, tree, tr, nb, nbe, nc, 4,
                                                                                       scr, stream=s))}
    del tr
    # indexed commit: same shape, half the columns from a 256-entry instruction table
    src = [c % 2 for c in range(nc)]
    ib, ent = 8, 256
    rt_bits = sum(b for b, x in zip(bits, src) if not x) + ib
    wpr_i = (rt_bits + 63) // 64
    wpe = (sum(b for b, x in zip(bits, src) if x) + 63) // 64
    rows_i = torch.empty((1 << nb) * wpr_i, dtype=torch.int64, device=dev)
    pkg.fill_random_device(rows_i, rows_i.numel(), 14, s)
    table = torch.empty(ent * wpe, dtype=torch.int64, device=dev)
    pkg.fill_random_device(table, table.numel(), 15, s)
    ms = timed(lambda: pkg.commit_indexed_device(lde, tree, rows_i, wpr_i, table, ent, wpe, ib, bits, src, nb, nbe,
                                                 4, scr, stream=s), args.steps, "indexed_commit")
    out["indexed_commit"] = {"shape": "2^22 x 64 columns x 32 bits (32 from a 256-entry table), blowup 2",
                             "ms": round(ms, 3), "gelem_s": round((1 << nbe) * nc / ms / 1e6, 3),
                             "kernel_ms": breakdown(lambda: pkg.commit_indexed_device(
                                 lde, tree, rows_i, wpr_i, table, ent, wpe, ib, bits, src, nb, nbe, 4, scr,
                                 stream=s))}
    del packed, lde, tree, scr, rows_i, table
    torch.cuda.empty_cache()
    # streaming slot commit (Poseidon1, as the reference's slot commit): 2^20 x 64 x 32 bits from host
    nb, nbe = 20, 21
    host_rows = torch.empty((1 << nb) * wpr, dtype=torch.int64, pin_memory=True)
    pkg.load().b200_fill_random_host(host_rows.data_ptr(), host_rows.numel(), 16)
    hp = host_rows.numpy().view(np.uint64).reshape(1 << nb, wpr)
    nbytes = pkg.stream_commit_slot_bytes(nb, nbe, nc, wpr)
    slot = torch.empty(nbytes // 8, dtype=torch.int64, device=dev)
    pkg.set_native_hash_family(1)
    try:
        ms = timed(lambda: pkg.stream_commit_packed(slot, nbytes // 8, hp, bits, nb, nbe, stream=s), args.steps)
    finally:
        pkg.set_native_hash_family(2)
    out["stream_commit"] = {"shape": "2^20 x 64 columns x 32 bits from pinned host rows, blowup 2, Poseidon1 W16, "
                                     "slot %.2f GB" % (nbytes / 1e9), "ms": round(ms, 3),
                            "gelem_s": round((1 << nbe) * nc / ms / 1e6, 3)}
    line = {"metric": "commit consumers and variants (Q stage, query openings, packed / indexed / streaming "
                      "commits)", "workload": "extras", "unit": "mixed", "results": out, "n_gpus": 1,
            "dtype": "u64", "data": "synthetic (seeded uniform words)", "per_call_min_max_ms": spread}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["c3", "c3small", "c5", "extras"], default="c2")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--budget-gb", type=float, default=120.0, help="device memory per wave (c3, c3small)")
    ap.add_argument("--autotune", action="store_true",
                    help="untimed NTT plan autotuning before the timed steps (default: the default plan)")
    ap.add_argument("--hash-family", type=int, choices=[1, 2], default=2,
                    help="1 = Poseidon1, 2 = Poseidon2 (single-instance workloads)")
    ap.add_argument("--rates", default="5,20,80", help="c5: Poisson arrival rates per second")
    ap.add_argument("--duration", type=float, default=60.0, help="c5: seconds of arrivals per rate")
    ap.add_argument("--pool", type=int, default=12, help="c5: distinct C3-distributed request shapes")
    ap.add_argument("--slots", type=int, default=4, help="c5: server slots (units admitted at once)")
    ap.add_argument("--serve-budget-gb", type=float, default=150.0, help="c5: server device-memory budget")
    ap.add_argument("--serve-timeout", type=float, default=1800.0, help="c5: give up after this many seconds")
    ap.add_argument("--serve-repeats", type=int, default=2,
                    help="c5: runs of each mode on the same stream, in mirrored order (batching, FIFO, FIFO, ...)")
    ap.add_argument("--no-legs", action="store_true",
                    help="default workload: skip the batched (c3) and served (c5) legs of the JSON line")
    ap.add_argument("--serve-seconds", type=float, default=30.0,
                    help="default workload: seconds of arrivals of its served leg (5 requests/s)")
    args = ap.parse_args()
    if args.workload in BATCH_SETS:
        return run_batched(args)
    if args.workload == "c5":
        return run_serving(args)
    if args.workload == "extras":
        return run_extras(args)
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference(args, wl)
    return run_ours(args, wl)


if __name__ == "__main__":
    sys.exit(main())
