#!/usr/bin/env python
"""Benchmark of the batched small-array sort on B200 GPUs.

Metric: sorted keys per second over the whole job.  Default workload: 4096
independent arrays x 1024 int32 keys, i.i.d. uniform over the full int32
range (one batch per rank; ranks are independent replicas, weak scaling).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

One step = one sort of one batch already resident in HBM (out of place).
Steps rotate over enough input/output sets that every step reads inputs
evicted from the 126 MB L2.  Rank 0 prints one JSON line.

--impl reference times the reference's own CPU path on this host (one
std::sort per array over all host threads, compiled from the reference's
headers into oracle/_ref/) on the same workload; only rank 0 runs it.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "cuda-sort_b200"),):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

import b200sort as bs  # noqa: E402
import workloads  # noqa: E402

METRIC = "sorted keys/s"
UNIT = "keys/s"
L2_BYTES = 126 * 1024 * 1024
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    "int32_4096x1024": dict(dtype=bs.I32, n=1024, arrays=4096, dist="uniform", flags=0),
    "records_n4096": dict(dtype=bs.I32_I32, n=4096, arrays=1024, dist="uniform", flags=0),
    "records_n1000": dict(dtype=bs.I32_I32, n=1000, arrays=4194, dist="uniform", flags=0),
    "records_n32": dict(dtype=bs.I32_I32, n=32, arrays=131072, dist="uniform", flags=0),
}
DTYPE_NAMES = {bs.I32: "int32", bs.I32_I32: "int32+int32", bs.U64: "uint64", bs.U64_I32: "uint64+int32"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--workload", default="int32_4096x1024", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--preroll", type=float, default=1.5,
                    help="seconds of untimed sorting before the timed region, so clocks settle")
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def traffic_for(workload):
    """DRAM bytes per launch of the sort kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and parts[0] == workload and not line.startswith("#"):
                    return int(float(parts[1]))
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling while the GPU is under load."""

    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_uuid):
        self.proc = None
        self.lines = []
        self.uuid = device_uuid

    def start(self):
        cmd = ["nvidia-smi", "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits", "-lms", "100"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for name, val in zip(names, f[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_sort(data, n, arrays, threads):
    """The reference's own per-array std::sort (oracle/_ref), or the oracle port."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_oracle as orc

    if orc.ref_cpu_available() and data.dtype in (bs.NP_DTYPES[bs.I32], bs.NP_DTYPES[bs.I32_I32]):
        code = 0 if data.dtype == bs.NP_DTYPES[bs.I32] else 1
        return (lambda buf: orc.ref_cpu_sort_inplace(code, buf, n, arrays, threads)), "reference"

    def port(buf):
        dtype = {v: k for k, v in bs.NP_DTYPES.items()}[buf.dtype]
        buf[:] = orc.sort_packed(dtype, buf, n, arrays, orc.MODE_STD, threads)
    return port, "port"


def time_cpu(data, n, arrays, threads, budget_s=8.0, min_reps=2, max_reps=50):
    run, kind = cpu_reference_sort(data, n, arrays, threads)
    times = []
    t_total = 0.0
    while len(times) < max_reps and (len(times) < min_reps or t_total < budget_s):
        buf = data.copy()
        t0 = time.perf_counter()
        run(buf)
        dt = time.perf_counter() - t0
        times.append(dt)
        t_total += dt
    return statistics.median(times), kind, len(times)


def reference_arm(args, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n, arrays, dtype = wl["n"], wl["arrays"], wl["dtype"]
    data = workloads.make_packed(dtype, n, arrays, wl["dist"], seed=1234)
    threads = os.cpu_count() or 1
    run, kind = cpu_reference_sort(data, n, arrays, threads)
    for _ in range(args.warmup):
        buf = data.copy()
        run(buf)
    total = 0.0
    for _ in range(args.steps):
        buf = data.copy()
        t0 = time.perf_counter()
        run(buf)
        total += time.perf_counter() - t0
    sec = total / max(1, args.steps)
    value = n * arrays / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": DTYPE_NAMES[dtype], "data": "synthetic",
        "config": config_of(args, wl),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": "the full batch (%d arrays x %d) per step, std::sort per array over %d "
                                   "host threads" % (arrays, n, threads)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def config_of(args, wl):
    return {"workload": args.workload, "arrays_per_gpu": wl["arrays"], "n": wl["n"],
            "key_dtype": DTYPE_NAMES[wl["dtype"]], "distribution": wl["dist"],
            "stable": bool(wl["flags"] & bs.STABLE), "parallelism": "replicas",
            "l2": "inputs rotate over sets larger than L2 (126 MB)"}


def main():
    args = parse()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        return reference_arm(args, wl)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    dtype, n, arrays, flags = wl["dtype"], wl["n"], wl["arrays"], wl["flags"]
    eb = bs.ELEM_BYTES[dtype]
    batch_bytes = n * arrays * eb
    data = workloads.make_packed(dtype, n, arrays, wl["dist"], seed=1234 + rank)
    sets = max(2, math.ceil(2 * L2_BYTES / batch_bytes) + 1)
    host = torch.from_numpy(data.view(np.uint8).copy())
    d_in = [host.to(dev) for _ in range(sets)]
    d_out = [torch.empty_like(d_in[0]) for _ in range(sets)]
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    def step(i):
        k = i % sets
        bs.sort_packed(dtype, d_in[k].data_ptr(), d_out[k].data_ptr(), n, arrays, flags, None, sh)

    for i in range(max(3, args.warmup)):
        step(i)
    torch.cuda.synchronize(dev)

    sampler = ClockSampler(None)
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        sampler = ClockSampler(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
    except Exception:
        pass
    sampler.start()
    # Pre-roll so that the clocks settle under load before the timed region.
    t_end = time.perf_counter() + args.preroll
    i = 0
    while time.perf_counter() < t_end:
        for _ in range(50):
            step(i)
            i += 1
        torch.cuda.synchronize(dev)

    barrier()
    torch.cuda.synchronize(dev)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for j in range(args.steps):
        step(j)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    ms_total = ev0.elapsed_time(ev1)
    sampler.stop()
    ms_total = max_over_ranks(ms_total)
    ms_step = ms_total / args.steps

    # correctness of the last timed output (outside timing)
    k = (args.steps - 1) % sets
    got = d_out[k].cpu().numpy().view(bs.NP_DTYPES[dtype])
    if dtype in (bs.I32, bs.U64):
        verified = bool(np.array_equal(got.reshape(arrays, n), np.sort(data.reshape(arrays, n), axis=1)))
    else:
        verified = bool(np.array_equal(got["key"].reshape(arrays, n),
                                       np.sort(data["key"].reshape(arrays, n), axis=1)))

    keys_per_step = n * arrays
    value = keys_per_step * world / (ms_step * 1e-3)
    hbm, peak_src = peaks()
    algo_bytes = 2 * batch_bytes
    achieved = algo_bytes / (ms_step * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "peak_source": peak_src + " (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured"
                else "fallback 6.65 TB/s",
                "traffic": traffic_for(args.workload), "algorithmic_bytes_per_launch": algo_bytes,
                "kernel": "k_sort_packed", "launch_us": ms_step * 1e3}

    e2e = None
    if not args.no_e2e:
        pin_in = host.pin_memory()
        pin_out = torch.empty_like(pin_in).pin_memory()
        esteps = max(3, min(args.steps, 30))
        with bs.Session(local) as sess:
            for _ in range(2):
                sess.sort_host(dtype, pin_in.data_ptr(), pin_out.data_ptr(), n, arrays, flags)
            barrier()
            t0 = time.perf_counter()
            for _ in range(esteps):
                sess.sort_host(dtype, pin_in.data_ptr(), pin_out.data_ptr(), n, arrays, flags)
            dt = time.perf_counter() - t0
            barrier()
        dt = max_over_ranks(dt)
        e2e = {"value": keys_per_step * world * esteps / dt, "unit": UNIT, "h2d_bytes_per_step": batch_bytes,
               "d2h_bytes_per_step": batch_bytes, "steps": esteps,
               "path": "b200s_sort_packed_host (pinned host buffers, chunked copy/sort overlap)"}
        out = pin_out.numpy().view(bs.NP_DTYPES[dtype])
        if dtype in (bs.I32, bs.U64):
            verified = verified and bool(np.array_equal(out, got))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sec, kind, reps = time_cpu(data, n, arrays, threads)
        cpu = {"value": keys_per_step / sec, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": "the full batch (%d arrays x %d), %d repetitions, std::sort per array"
                         % (arrays, n, reps)}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": DTYPE_NAMES[dtype], "data": "synthetic",
        "config": config_of(args, wl), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": args.steps, "clocks": sampler.summary(), "verified": verified,
        "library": bs.version(),
    }
    print(json.dumps(line))
    return 0 if verified else 1


if __name__ == "__main__":
    sys.exit(main())
