"""Benchmark: in-place sort of 2^28 doubles (uniform [0,1)) on one B200.

One step = one Sort512::Sort of a fresh 2^28-double array resident in HBM
(a distinct input per step, 2 GiB each, so every step reads from DRAM, not
L2).  `value` is device throughput in Gkeys/s (CUDA events on the launching
stream, max over ranks); `e2e` is the same sort through the C ABI with a
pinned HOST buffer (host->device copy, sort, device->host copy inside the
timed region).  `roofline` reports the dominant kernel against the measured
HBM copy bandwidth, `cpu_baseline` the reference's own CPU sort on this host.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 (torchrun) every rank sorts its own array: replicas, no
collective on the data path ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
# DRAM bytes per key of one partition launch (read + write, ncu
# dram__bytes_read.sum + dram__bytes_write.sum, mean of the two levels of two
# 2^26-key double sorts: 1025.8, 1022.2, 1031.7 and 1032.0 MB for 67,108,864
# keys).  The algorithmic figure is 16 B/key: the capture is just below it
# because the last written lines are still in L2 when the launch ends (they
# reach DRAM with the next kernel).  Traffic grows with the keys, so the bench
# scales it to its own launch size.
PART_DRAM_BYTES_PER_KEY = 15.32
PKG = os.path.join(ROOT, "avx-512-sort_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")
sys.path.insert(0, PKG)
sys.path.insert(0, ROOT)

METRIC = "Gkeys/s at 2^28 int32/f64/kv; learned vs plain splitters; % of HBM roofline"
N_KEYS = 1 << 28
WORKLOAD = "Sort512::Sort, double, n=2^28, uniform [0,1) (splitmix64 seed per step), sampled splitters"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_KEYS)
    ap.add_argument("--no-extras", action="store_true", help="skip the per-distribution / int32 / kv extras")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--sharded", action="store_true",
                    help="with --gpus N > 1: one sorted array across the ranks (sample sort with one "
                         "all-to-all) instead of N independent sorts")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return

        def rd():
            for line in self.proc.stdout:
                self.samples.append([x.strip() for x in line.split(",")])

        self.thread = threading.Thread(target=rd, daemon=True)
        self.thread.start()

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = []
        smax = None
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[1]))
                smax = float(s[2])
                for nm, val in zip(names, s[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The slowest rank's time: every rank's number is replaced by the maximum."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# The reference's CPU path (compiled in place from its sources by oracle/Makefile)
def cpu_reference():
    """(checker, kind): the reference compiled in place when this host has
    AVX-512, else the C restatement (single-threaded `Sort` only)."""
    sys.path.insert(0, ORACLE_DIR)
    from oracle import REF_SO, Oracle, Reference, cpu_has_avx512
    if os.path.exists(REF_SO) and cpu_has_avx512():
        return Reference(), "reference"
    return Oracle(), "port"


REF_FUNCTIONS = {"sort_omp_partition": "Sort512::SortOmpPartition", "sort": "Sort512::Sort",
                 "kv_sort_omp_partition": "Sort512kv::SortOmpPartition"}


def time_reference(ref, kind, fn, base, threads, reps, vals=None, keep=None):
    """Seconds of each of `reps` runs of reference function `fn` on a fresh
    copy of `base` (copied outside the timed region); the last output is
    checked for sortedness (and left in `keep`, a list, when one is given).
    kv functions take `vals` too."""
    import numpy as np
    work = np.empty_like(base)
    vwork = np.empty_like(vals) if vals is not None else None
    times = []
    for _ in range(reps):
        np.copyto(work, base)
        if vwork is not None:
            np.copyto(vwork, vals)
        if kind == "reference":
            ref.set_threads(threads)
            t0 = time.perf_counter()
            if fn.startswith("kv_"):
                ref.call_kv(fn[3:], work, vwork)
            else:
                ref.call(fn, work)
        else:  # the restatement: one core, Sort
            t0 = time.perf_counter()
            if fn.startswith("kv_"):
                ref.sort_kv(work, vwork)
            else:
                ref.sort(work)
        times.append(time.perf_counter() - t0)
    if work.size > 1:
        assert bool(np.all(work[1:] >= work[:-1])), f"reference {fn} output not sorted"
    if keep is not None:
        keep.append(work)
    return times


def _median(v):
    v = sorted(v)
    return v[len(v) // 2]


def run_reference_arm(args, world, rank):
    """--impl reference: the reference's own CPU sort (SortOmpPartition on all
    host cores) on the full workload, one sort per step, the input restored
    from an untimed copy before each step."""
    if rank != 0:
        return
    import numpy as np

    import workloads
    threads = os.cpu_count() or 1
    n = args.n
    base = workloads.uniform01_np(n, 1)
    ref, kind = cpu_reference()
    cores = threads if kind == "reference" else 1
    if args.warmup:
        time_reference(ref, kind, "sort_omp_partition", base, threads, args.warmup)
    times = time_reference(ref, kind, "sort_omp_partition", base, threads, args.steps)
    tot = sum(times)
    val = n * len(times) / tot / 1e9
    fname = REF_FUNCTIONS["sort_omp_partition"] if kind == "reference" else "restated CoreSort (1 core)"
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 4), "unit": "Gkeys/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(tot / len(times) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": n, "function": fname,
                   "median_ms_per_step": round(_median(times) * 1e3, 3)},
        "cpu_baseline": {"value": round(val, 4), "unit": "Gkeys/s", "cores": cores, "kind": kind,
                         "sample": f"the full workload: {n} uniform doubles per step, {args.steps} steps "
                                   f"({fname}, {cores} threads)"},
        "e2e": {"value": round(val, 4), "unit": "Gkeys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_rows(n, dev):
    """The reference on this host's cores, same inputs as the GPU rows:
    SortOmpPartition (all cores, median of 5) and Sort (1 core) on the
    headline 2^28 doubles, the kv SortOmpPartition on 2^28 pairs, the normal
    distribution at 2^28, and the three distributions on which the
    reference's pivot rule is quadratic (ascending, descending, 256 distinct
    values) at the largest size that finishes under a per-run cap.  Returns
    (headline entry, rows)."""
    import numpy as np

    import workloads
    threads = os.cpu_count() or 1
    ref, kind = cpu_reference()
    cores = threads if kind == "reference" else 1
    rows = {}
    base = workloads.uniform01_torch(n, seed=1, device=dev).cpu().numpy()
    t = time_reference(ref, kind, "sort_omp_partition", base, threads, 5)
    head = {"value": round(n / _median(t) / 1e9, 4), "unit": "Gkeys/s", "cores": cores, "kind": kind,
            "sample": (f"{REF_FUNCTIONS['sort_omp_partition']} on the full workload ({n} uniform doubles), "
                       f"median of 5 runs, {threads} threads") if kind == "reference"
            else f"restated CoreSort on {n} uniform doubles, 1 core, median of 5 runs",
            "runs_ms": [round(x * 1e3, 1) for x in t]}
    if kind != "reference":
        return head, rows
    t = time_reference(ref, kind, "sort", base, 1, 1)
    rows["f64_uniform_sort_1core"] = {"n": n, "ms": round(t[0] * 1e3, 1), "gkeys_s": round(n / t[0] / 1e9, 4),
                                      "function": REF_FUNCTIONS["sort"], "cores": 1}
    del base
    x = workloads.double_dist_torch("normal", n, seed=2, device=dev).cpu().numpy()
    t = time_reference(ref, kind, "sort_omp_partition", x, threads, 3)
    rows["f64_normal"] = {"n": n, "ms_median": round(_median(t) * 1e3, 1),
                          "gkeys_s": round(n / _median(t) / 1e9, 4), "cores": threads}
    del x
    k = workloads.uniform_i32_torch(n, 9, dev).cpu().numpy()
    v = np.arange(n, dtype=np.int32)
    t = time_reference(ref, kind, "kv_sort_omp_partition", k, threads, 3, vals=v)
    rows["kv_uniform"] = {"n": n, "ms_median": round(_median(t) * 1e3, 1), "gkeys_s": round(n / _median(t) / 1e9, 4),
                          "function": REF_FUNCTIONS["kv_sort_omp_partition"], "cores": threads}
    del k, v
    cap_s = 4.0
    for dist in ("ascending", "descending", "distinct256"):
        m, done = 1 << 16, None
        while m <= n:
            x = workloads.double_dist_torch(dist, m, seed=3, device=dev).cpu().numpy()
            out = []
            t = time_reference(ref, kind, "sort_omp_partition", x, threads, 1, keep=out)[0]
            done = {"n": m, "ms": round(t * 1e3, 1), "gkeys_s": round(m / t / 1e9, 5),
                    "equal_to_np_sort": bool(np.array_equal(out[0], np.sort(x)))}
            if 4 * t > cap_s:  # the next size (quadratic) would pass the cap
                break
            m *= 2
        rows[f"f64_{dist}"] = dict(done, cap_s_per_run=cap_s,
                                   note=("finished at the full size" if done["n"] >= n else
                                         f"did not run at 2^{n.bit_length() - 1}: the next doubling "
                                         f"would exceed {cap_s} s (quadratic in the reference)"))
    return head, rows


# ---------------------------------------------------------------------------
def run_ours(args, world, rank, local):
    import torch

    import sort512cuda as s512
    import workloads

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    s512.lib()
    n = args.n
    stream = torch.cuda.current_stream(dev)
    s512.set_config(collect_stats=1)

    def make(seed):
        return workloads.uniform01_torch(n, seed=seed + 1000 * rank, device=dev)

    # warm-up (untimed)
    for w in range(args.warmup):
        x = make(900 + w)
        s512.sort(x, flags=s512.ASYNC, stream=stream)
        torch.cuda.synchronize()
        assert workloads.is_sorted_torch(x), "warm-up output not sorted"
        del x
    # distinct inputs for every timed step, generated before timing, with the
    # multiset fingerprint of each and a copy of the first (checked in full)
    inputs = [make(s) for s in range(args.steps)]
    fps = [workloads.multiset_fingerprint_torch(x) for x in inputs]
    first = inputs[0].clone()
    torch.cuda.synchronize()
    barrier(world)

    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    part_ms, part_keys, leaf_ms, samp_ms, launches, levels = [], [], [], [], 0, 0
    torch.cuda.synchronize()
    barrier(world)
    ev0.record(stream)
    for s in range(args.steps):
        s512.sort(inputs[s], flags=s512.ASYNC, stream=stream)
        st = s512.stats()
        part_ms.append(sum(st["partition_ms"]))
        part_keys.append(sum(st["partition_keys"]))
        leaf_ms.append(sum(st["leaf_ms"]))
        samp_ms.append(sum(st["sample_ms"]))
        launches += st["kernel_launches"]
        levels = st["levels"]
        last = st
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop() if sampler else None
    dev_ms = ev0.elapsed_time(ev1)
    dev_ms = max_over_ranks(dev_ms, world)
    # every step: sorted, and the same multiset as its input; the first step
    # also equal, key for key, to an independent sort of its input
    verify = {"sorted_every_step": all(workloads.is_sorted_torch(x) for x in inputs),
              "multiset_every_step": all(workloads.multiset_fingerprint_torch(x) == f
                                         for x, f in zip(inputs, fps)),
              "first_step_equal_to_torch_sort": bool(torch.equal(
                  workloads.order_keys_torch(inputs[0]), torch.sort(workloads.order_keys_torch(first)).values))}
    ok = all(verify.values())
    del inputs, first
    torch.cuda.empty_cache()
    ms_per_step = dev_ms / args.steps
    value = n * world / (ms_per_step * 1e-3) / 1e9

    # roofline of the partition kernel: algorithmic bytes = read + write of
    # every key it moves (8 B per double), per launch
    peak, peak_kind = peaks()
    tot_part_ms = sum(part_ms)
    tot_leaf_ms = sum(leaf_ms)
    part_bytes = 2 * 8 * sum(part_keys)
    part_gbs = part_bytes / (tot_part_ms * 1e-3) / 1e9 if tot_part_ms > 0 else None
    leaf_bytes = 2 * 8 * n * args.steps
    leaf_gbs = leaf_bytes / (tot_leaf_ms * 1e-3) / 1e9 if tot_leaf_ms > 0 else None
    dominant = "partition" if tot_part_ms >= tot_leaf_ms else "leaf"
    ach = part_gbs if dominant == "partition" else leaf_gbs
    roofline = {"bound": "hbm", "kernel": "partition_kernel" if dominant == "partition" else "leaf sorts",
                "achieved": round(ach, 1) if ach else None, "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4) if ach else None, "peak_source": peak_kind,
                "traffic": (round(PART_DRAM_BYTES_PER_KEY * n) if dominant == "partition" else None),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per partition launch on a "
                                  "2^26-key double sort (both levels), %.2f B/key, scaled to n keys per launch"
                                  % PART_DRAM_BYTES_PER_KEY,
                "partition_kernel": {"achieved": round(part_gbs, 1) if part_gbs else None,
                                     "frac": round(part_gbs / peak, 4) if part_gbs else None,
                                     "ms_per_step": round(tot_part_ms / args.steps, 3),
                                     "launches_per_step": levels,
                                     "algorithmic_bytes_per_step": part_bytes // args.steps},
                "leaf_sorts": {"achieved": round(leaf_gbs, 1) if leaf_gbs else None,
                               "frac": round(leaf_gbs / peak, 4) if leaf_gbs else None,
                               "ms_per_step": round(tot_leaf_ms / args.steps, 3)},
                "sampling_ms_per_step": round(sum(samp_ms) / args.steps, 3)}
    if rank != 0:
        return

    # e2e through the C ABI with page-locked HOST buffers
    try:
        e2e = e2e_host(n, dev)
    except Exception as e:  # noqa: BLE001
        e2e = {"value": None, "unit": "Gkeys/s", "error": str(e)[:200]}
    torch.cuda.empty_cache()

    # CPU baseline: the reference's SortOmpPartition on all host cores, on
    # the full workload, with the reference's other rows beside it
    cpu = None
    if not args.no_cpu and world == 1:
        try:
            cpu, rows = cpu_baseline_rows(n, dev)
            cpu["rows"] = rows
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "Gkeys/s", "error": str(e)[:200]}

    extras = {}
    if not args.no_extras:
        extras = run_extras(n, dev, stream)

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Gkeys/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": n, "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "inputs larger than L2: a distinct 2 GiB input per step",
                   "levels": levels},
        "clocks": clocks, "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu,
        "gpu_launches": launches, "sorted_ok": ok, "verify": verify, "stats_last_step": last, "extras": extras,
    }
    print(json.dumps(line), flush=True)


E2E_STEPS = 6


def e2e_host(n, dev, steps=E2E_STEPS):
    """The headline sort through the C ABI from page-locked host memory: every
    step copies its own 2 GiB input in (host->device), sorts it and copies the
    result back (device->host) inside the timed region.

    value: `steps` sorts issued back to back as asynchronous host-pointer calls
    (S512_ASYNC) alternating between two streams, timed by the host clock from
    the first call to the end of the last copy back: one step's copy back
    overlaps the next step's copy in (PCIe carries both directions at once).
    single_call_ms: one blocking call (the drop-in Sort512::Sort on a host
    array), median of 3.  Every output is checked on the device: sorted, and
    the same multiset as its input."""
    import torch

    import sort512cuda as s512
    import workloads
    ins = [workloads.uniform01_torch(n, seed=4242 + s, device=dev) for s in range(steps)]
    fps = [workloads.multiset_fingerprint_torch(x) for x in ins]
    hosts = []
    for x in ins:
        h = torch.empty(n, dtype=torch.float64, pin_memory=True)
        h.copy_(x)
        hosts.append(h)
    del ins
    torch.cuda.empty_cache()
    streams = [torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)]
    # warm-up: each stream's scratch pool sized, kernels loaded (untimed)
    warm = torch.empty(n, dtype=torch.float64, pin_memory=True)
    for st in streams:
        for _ in range(2):
            warm.copy_(hosts[0])
            s512.sort(warm.numpy(), flags=s512.ASYNC, stream=st)
            st.synchronize()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in range(steps):
        s512.sort(hosts[s].numpy(), flags=s512.ASYNC, stream=streams[s % 2])
    for st in streams:
        st.synchronize()
    t1 = time.perf_counter()
    ok = True
    for h, fp in zip(hosts, fps):
        d = h.to(dev)
        ok = ok and workloads.is_sorted_torch(d) and workloads.multiset_fingerprint_torch(d) == fp
        del d
    single = []
    for _ in range(3):
        warm.copy_(workloads.uniform01_torch(n, seed=77, device=dev))
        torch.cuda.synchronize()
        c0 = time.perf_counter()
        s512.sort(warm.numpy())  # blocking: copy in, sort, copy back, return
        single.append((time.perf_counter() - c0) * 1e3)
    ok = ok and workloads.is_sorted_torch(warm.to(dev))
    ms = (t1 - t0) * 1e3 / steps
    del hosts, warm
    s512.release_scratch()
    return {"value": round(n / (ms * 1e-3) / 1e9, 4), "unit": "Gkeys/s", "h2d_bytes_per_step": n * 8,
            "d2h_bytes_per_step": n * 8, "ms_per_step": round(ms, 3), "steps": steps,
            "timing": "host clock, first call to last copy back; asynchronous host-pointer calls on two streams "
                      "(page-locked buffers, one per step)",
            "single_call_ms": round(_median(single), 3),
            "single_call_gkeys_s": round(n / (_median(single) * 1e-3) / 1e9, 4),
            "verified": ok}


def run_sharded(args, world, rank, local):
    """--sharded: each rank holds n doubles of one array; the sort across
    ranks (dist_sort.sort_sharded: local sort, regular sample, splitters, one
    all-to-all over NCCL, merge of the received runs) is timed on the device,
    max over ranks.  value = n * N / time (weak scaling)."""
    import torch

    import dist_sort
    import sort512cuda as s512
    import workloads

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    s512.lib()
    n = args.n
    stream = torch.cuda.current_stream(dev)

    def make(seed):
        return workloads.uniform01_torch(n, seed=seed + 7919 * rank, device=dev)

    for w in range(args.warmup):
        dist_sort.sort_sharded(make(900 + w))
    torch.cuda.synchronize()
    inputs = [make(s) for s in range(args.steps)]
    torch.cuda.synchronize()
    barrier(world)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    out = None
    for s in range(args.steps):
        out = dist_sort.sort_sharded(inputs[s])
    ev1.record(stream)
    torch.cuda.synchronize()
    outs_ok = bool((out[1:] >= out[:-1]).all()) if out is not None and out.numel() > 1 else True
    del out
    barrier(world)
    ms = max_over_ranks(ev0.elapsed_time(ev1), world) / args.steps
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(n * world / (ms * 1e-3) / 1e9, 3), "unit": "Gkeys/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "one array of n doubles per rank, sorted across the ranks", "n_per_rank": n,
                   "parallelism": f"sample sort over {world} ranks (one all-to-all)"},
        "sorted_ok": outs_ok, "e2e": None, "roofline": None, "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)


def _timed(fn, stream):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


EXTRA_REPS = 10


def _median_timed(run, restore, stream, reps=EXTRA_REPS, warm=2):
    """Median device time (ms) of `reps` timed runs, each on a fresh input
    (restore() copies it back, untimed), after `warm` untimed runs."""
    import torch
    for _ in range(warm):
        restore()
        run()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        restore()
        times.append(_timed(run, stream))
    return _median(times), times


def run_extras(n, dev, stream):
    """The other workloads at full size, each the median of EXTRA_REPS timed
    runs on a restored input, each output checked: sorted and the same
    multiset as its input (key/value: the same (key, value) pairs)."""
    import torch

    import sort512cuda as s512
    import workloads
    out = {}

    def verified(x, fp, *more):
        return workloads.is_sorted_torch(x) and workloads.multiset_fingerprint_torch(x, *more) == fp

    for dist in workloads.DOUBLE_DISTS:
        x0 = workloads.double_dist_torch(dist, n, seed=6, device=dev)
        fp = workloads.multiset_fingerprint_torch(x0)
        x = torch.empty_like(x0)
        ms, _ = _median_timed(lambda: s512.sort(x, flags=s512.ASYNC, stream=stream), lambda: x.copy_(x0), stream)
        st = s512.stats()
        out[f"f64_{dist}"] = {"gkeys_s": round(n / ms / 1e6, 3), "ms": round(ms, 3), "verified": verified(x, fp),
                              "levels": st["levels"], "fallbacks": st["fallbacks"], "reps": EXTRA_REPS}
        del x, x0
    x0 = workloads.uniform_i32_torch(n, seed=8, device=dev)
    fp = workloads.multiset_fingerprint_torch(x0)
    x = torch.empty_like(x0)
    ms, _ = _median_timed(lambda: s512.sort(x, flags=s512.ASYNC, stream=stream), lambda: x.copy_(x0), stream)
    out["i32_uniform"] = {"gkeys_s": round(n / ms / 1e6, 3), "ms": round(ms, 3), "verified": verified(x, fp),
                          "reps": EXTRA_REPS}
    del x, x0
    for kname in ("uniform", "zipf"):
        k0 = workloads.uniform_i32_torch(n, 9, dev) if kname == "uniform" else workloads.zipf_i32_torch(n, seed=9,
                                                                                                          device=dev)
        v0 = torch.arange(n, dtype=torch.int32, device=dev)
        fp = workloads.multiset_fingerprint_torch(k0, v0)
        k, v = torch.empty_like(k0), torch.empty_like(v0)

        def restore():
            k.copy_(k0)
            v.copy_(v0)

        ms, _ = _median_timed(lambda: s512.sort_kv(k, v, flags=s512.ASYNC, stream=stream), restore, stream)
        out[f"kv_{kname}"] = {"gkeys_s": round(n / ms / 1e6, 3), "ms": round(ms, 3), "verified": verified(k, fp, v),
                              "reps": EXTRA_REPS}
        del k, v, k0, v0
    torch.cuda.empty_cache()
    out["int32_2p20_latency"] = extra_c1(dev, stream)
    out["learned_vs_plain"] = extra_learned(dev, stream)
    out["segmented_200k"] = extra_segsort(dev, stream)
    torch.cuda.empty_cache()
    return out


def extra_c1(dev, stream):
    """int32, n = 2^20, uniform over the full range, seed 0: device latency,
    the host-pointer call, exactness against the reference's output digest,
    and the reference's single-core Sort on the same array."""
    import hashlib

    import numpy as np
    import torch

    import sort512cuda as s512
    import workloads
    n = 1 << 20
    a = workloads.uniform_i32_np(n, 0)
    d = torch.from_numpy(a).to(dev)
    times = []
    for _ in range(23):
        x = d.clone()
        torch.cuda.synchronize()
        times.append(_timed(lambda: s512.sort(x, flags=s512.ASYNC, stream=stream), stream))
    dev_ms = float(np.median(times[3:]))
    host_times = []
    for _ in range(7):  # host pointer (pageable numpy memory): copy in, sort, copy out
        h = a.copy()
        t0 = time.perf_counter()
        s512.sort(h)
        host_times.append((time.perf_counter() - t0) * 1e3)
    host_ms = _median(host_times[2:])
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        want = json.load(f)["c1"]["sorted"]
    exact = hashlib.sha256(h.tobytes()).hexdigest()[:32] == want
    cpu_ms = None
    try:
        ref, kind = cpu_reference()
        cpu_ms = _median(time_reference(ref, kind, "sort", a, 1, 5)) * 1e3
    except Exception:  # noqa: BLE001
        kind = "unavailable"
    return {"n": n, "device_ms_median": round(dev_ms, 4), "gkeys_s": round(n / dev_ms / 1e6, 3),
            "host_pointer_call_ms": round(host_ms, 3), "exact_vs_reference_digest": exact,
            "reference_sort_1core_ms_median": round(cpu_ms, 3) if cpu_ms else None, "reference_kind": kind}


def extra_learned(dev, stream):
    """Learned vs sampled splitters on the same GPU: int32 n = 2^29 (Zipf 1.1
    over 2^24 values; mixture of 8 Gaussians) and double n = 2^28 (lognormal
    mu=0 sigma=2; mixture of 8 Gaussians): whole-sort and partition-pass
    times, bucket imbalance, levels the model routed and models rejected."""
    import torch

    import sort512cuda as s512
    import workloads
    rows = {}
    cases = (("i32_zipf_2p29", lambda: workloads.zipf_i32_torch(1 << 29, s=1.1, ranks=1 << 24, seed=21, device=dev)),
             ("i32_gauss_mix_2p29", lambda: workloads.gauss_mix_i32_torch(1 << 29, seed=22, device=dev)),
             ("f64_lognormal_2p28", lambda: workloads.double_dist_torch("lognormal", 1 << 28, seed=23, device=dev)),
             ("f64_gauss_mix_2p28", lambda: workloads.double_dist_torch("gauss_mix", 1 << 28, seed=24, device=dev)))
    for name, make in cases:
        x0 = make()
        n = x0.numel()
        fp = workloads.multiset_fingerprint_torch(x0)
        row = {"n": n}
        for mode, flag in (("plain", s512.SPLIT_PLAIN), ("learned", s512.SPLIT_LEARNED)):
            x = x0.clone()
            for _ in range(2):  # warm: scratch sized and kernels loaded for this mode
                x.copy_(x0)
                s512.sort(x, flags=flag | s512.ASYNC, stream=stream)
            times = []
            for _ in range(EXTRA_REPS):
                x.copy_(x0)
                times.append(_timed(lambda: s512.sort(x, flags=flag | s512.ASYNC, stream=stream), stream))
            ms = _median(times)
            st = s512.stats()
            row[mode] = {"gkeys_s": round(n / ms / 1e6, 3), "ms": round(ms, 3),
                         "partition_ms": round(sum(st["partition_ms"]), 3),
                         "partition_ms_per_level": [round(v, 3) for v in st["partition_ms"]],
                         "keys_per_level": st["partition_keys"],
                         "leaf_ms": round(sum(st["leaf_ms"]), 3),
                         "sample_and_fit_ms": round(sum(st["sample_ms"]), 3),
                         "levels": st["levels"], "model_levels": st["learned_levels"],
                         "models_rejected": st["learned_rejected"], "fallbacks": st["fallbacks"],
                         "max_bucket_over_mean": [round(v, 2) for v in st["max_bucket_over_mean"]],
                         "bucket_cv": [round(v, 3) for v in st["bucket_cv"]],
                         "verified": workloads.is_sorted_torch(x) and
                         workloads.multiset_fingerprint_torch(x) == fp, "reps": EXTRA_REPS}
            del x
        rows[name] = row
        del x0
        torch.cuda.empty_cache()
    return rows


def extra_segsort(dev, stream):
    """200,000 segments, lognormal lengths (mu=5, sigma=1.5, clipped 1..65536):
    int32 uniform, double U[0,1) and int32 key/value, one graph-captured
    persistent launch (plus partition levels for segments above a block),
    against a loop of single-array sorts over a sample of the segments and the
    reference's loop (SmallSort16V / Sort) on the host for the same sample."""
    import numpy as np
    import torch

    import sort512cuda as s512
    import workloads
    nseg = 200_000
    lens = workloads.segment_lengths_np(nseg, 31)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    total = int(off[-1])
    d_off = torch.from_numpy(off.view(np.int64)).to(dev)
    seg_id = torch.repeat_interleave(torch.arange(nseg, device=dev), torch.from_numpy(lens).to(dev))
    res = {"segments": nseg, "keys": total}
    tuned = {}
    for dt in (s512.DTYPE_I32, s512.DTYPE_F64, s512.DTYPE_KV_I32):
        tuned[dt] = s512.segsort_tune(dt, d_off)[1]
    for name, dt in (("i32", s512.DTYPE_I32), ("f64", s512.DTYPE_F64), ("kv_i32", s512.DTYPE_KV_I32)):
        if dt == s512.DTYPE_F64:
            keys0 = workloads.uniform01_torch(total, 32, dev)
        else:
            keys0 = workloads.uniform_i32_torch(total, 33, dev)
        vals0 = torch.arange(total, dtype=torch.int32, device=dev) if dt == s512.DTYPE_KV_I32 else None
        keys = keys0.clone()
        vals = vals0.clone() if vals0 is not None else None
        plan = s512.SegsortPlan(dt, keys, d_off, values=vals)
        def restore():
            keys.copy_(keys0)
            if vals is not None:
                vals.copy_(vals0)

        ms, _ = _median_timed(lambda: plan.launch(stream), restore, stream)
        plan.close()
        # every segment: equal to a segment-wise sort of its input (two
        # stable torch sorts: by key, then by segment)
        if dt == s512.DTYPE_KV_I32:
            key0 = keys0.to(torch.int64) * (1 << 32) + (vals0.to(torch.int64) + (1 << 31))
            got = keys.to(torch.int64) * (1 << 32) + (vals.to(torch.int64) + (1 << 31))
        else:
            key0 = workloads.order_keys_torch(keys0)
            got = workloads.order_keys_torch(keys)
        p1 = torch.sort(key0, stable=True).indices
        p2 = torch.sort(seg_id[p1], stable=True).indices
        every_segment_ok = bool(torch.equal(got, key0[p1[p2]]))
        del key0, got, p1, p2
        # a loop of single-array sorts over every 100th segment, scaled up
        idx = list(range(0, nseg, 100))
        sub = keys0.clone()
        loop_ms = _timed(lambda: [s512.sort(sub[int(off[i]):int(off[i + 1])], flags=s512.ASYNC, stream=stream)
                                  if dt != s512.DTYPE_KV_I32 else
                                  s512.sort_kv(sub[int(off[i]):int(off[i + 1])],
                                               vals0[int(off[i]):int(off[i + 1])].clone(), flags=s512.ASYNC,
                                               stream=stream)
                                  for i in idx], stream)
        sample_keys = int(sum(int(off[i + 1] - off[i]) for i in idx))
        loop_est_ms = loop_ms * total / max(sample_keys, 1)
        row = {"gkeys_s": round(total / ms / 1e6, 3), "ms": round(ms, 3), "launch_shape": tuned[dt],
               "loop_of_sorts_est_ms": round(loop_est_ms, 1), "every_segment_verified": every_segment_ok,
               "reps": EXTRA_REPS}
        # the reference's loop on the host for the same sample of segments
        try:
            sys.path.insert(0, ORACLE_DIR)
            from oracle import REF_SO, Reference, cpu_has_avx512
            if os.path.exists(REF_SO) and cpu_has_avx512():
                ref = Reference()
                ref.set_threads(1)
                host = keys0.cpu().numpy()
                hv = vals0.cpu().numpy() if vals0 is not None else None
                lim = 256 if dt != s512.DTYPE_F64 else 128
                t0 = time.perf_counter()
                for i in idx:
                    a = host[int(off[i]):int(off[i + 1])]
                    if dt == s512.DTYPE_KV_I32:
                        ref.call_kv("smallsort" if a.size <= lim else "sort", a, hv[int(off[i]):int(off[i + 1])])
                    else:
                        ref.call("smallsort" if a.size <= lim else "sort", a)
                cpu_s = time.perf_counter() - t0
                row["reference_loop_1core_est_ms"] = round(cpu_s * 1e3 * total / max(sample_keys, 1), 1)
        except Exception as e:  # noqa: BLE001
            row["reference_loop_error"] = str(e)[:120]
        res[name] = row
        del keys, keys0, vals, vals0, sub
        torch.cuda.empty_cache()
    return res


def main():
    args = parse()
    world, rank, local = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference_arm(args, world, rank)
        elif args.sharded and world > 1:
            run_sharded(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
