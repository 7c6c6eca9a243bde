#!/usr/bin/env python
"""Benchmark of the batched small-array sort on B200 GPUs.

Metric: sorted keys per second over the whole job.  Default workload: 4096
independent arrays x 1024 int32 keys, i.i.d. uniform over the full int32
range (one batch per rank; ranks are independent replicas, weak scaling).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

One step = one sort of one batch already resident in HBM (out of place).
Steps rotate over enough input/output sets that every step reads inputs
evicted from the 126 MB L2 (batches larger than L2 use one set).  Rank 0
prints one JSON line.

Workloads: int32_4096x1024 (default), records_n{32,129,256,1000,2048,4096}
(IntAndData records, 4194304 per batch; --distribution picks one of the
nine seeded distributions, --sorted-check sets B200S_SORTED_CHECK),
ragged_200000 (200000 CSR arrays,
lengths log-uniform in [1, 8192], records; the plan's launch sequence
replayed from its CUDA graph, with one launch per length class and the
plain per-length launches timed beside it), cluster_256x65536 /
cluster_u64_256x65536 (256 arrays of 65536 records with int32 / uint64
keys, one thread-block cluster per array: 4 CTAs of 1024 threads / 8 CTAs
of 512),
serving (a stream of sort requests of 16 .. 65536 records into the
continuous-batching server under a 16 GB device budget: peak sustained keys/s
in closed loop, then Poisson arrival rates with p50/p99/p99.9 latency, each
beside per-request plain launches; --duration seconds per point).

--impl reference times the reference's own CPU path on this host (one
std::sort per array over all host threads, compiled from the reference's
headers into oracle/_ref/) on the same workload; only rank 0 runs it.
"""
import argparse
import ctypes
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
    "int32_4096x1024": dict(kind="packed", dtype=bs.I32, n=1024, arrays=4096, dist="uniform", flags=0),
    "ragged_200000": dict(kind="ragged", dtype=bs.I32_I32, arrays=200000, max_len=8192, dist="uniform", flags=0),
    "ragged_20000": dict(kind="ragged", dtype=bs.I32_I32, arrays=20000, max_len=8192, dist="uniform", flags=0),
}
for _n in (32, 129, 256, 1000, 2048, 4096):
    WORKLOADS["records_n%d" % _n] = dict(kind="packed", dtype=bs.I32_I32, n=_n, arrays=4194304 // _n,
                                         dist="uniform", flags=0)
# arrays larger than one CTA: thread-block clusters
WORKLOADS["cluster_256x65536"] = dict(kind="packed", dtype=bs.I32_I32, n=65536, arrays=256, dist="uniform",
                                      flags=0)
WORKLOADS["cluster_u64_256x65536"] = dict(kind="packed", dtype=bs.U64_I32, n=65536, arrays=256,
                                          dist="uniform", flags=0)
# request stream into the server: 2048 device-resident requests reused cyclically
WORKLOADS["serving"] = dict(kind="serving", dtype=bs.I32_I32, arrays=2048, min_len=16, max_len=65536,
                            dist="uniform", flags=0, budget=16 << 30)
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
    ap.add_argument("--no-plain", action="store_true", help="ragged workloads: skip the per-length comparison")
    ap.add_argument("--no-baselines", action="store_true",
                    help="packed workloads: skip the plain-form, CUB and reference-V6 timings")
    ap.add_argument("--preroll", type=float, default=1.5,
                    help="seconds of untimed sorting before the timed region, so clocks settle")
    ap.add_argument("--form", default="table", choices=["table", "0", "1", "2", "3"],
                    help="packed workloads: launch form of the tabled tile (0 one-shot, 1 register prefetch, "
                         "2 TMA pipeline, 3 transposed network); 'table' uses the tile table's choice")
    ap.add_argument("--tile", default=None, help="packed workloads: tile shape log2_items,log2_lanes,log2_warps "
                                                  "instead of the table's")
    ap.add_argument("--distribution", default=None, choices=list(workloads.DISTRIBUTIONS),
                    help="packed workloads: key distribution instead of the workload's (uniform)")
    ap.add_argument("--sorted-check", action="store_true",
                    help="packed workloads: B200S_SORTED_CHECK (test each array first, skip it when in order); "
                         "the reference-V6 baseline then runs with Sorted=true")
    ap.add_argument("--duration", type=float, default=10.0, help="serving: seconds per rate point")
    ap.add_argument("--rates", default="1e4,3e4,1e5,3e5,1e6", help="serving: Poisson arrival rates (req/s)")
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def layer_counts(lk, lg, lw, lc=0):
    """Comparator layers of the reflection network by where the partner lives:
    (registers, lanes, warps through shared memory, cluster CTAs)."""
    counts = [0, 0, 0, 0]
    logw = lk + lg + lw + lc
    for st in range(logw):
        for hb in [st] + list(range(st - 1, -1, -1)):
            counts[0 if hb < lk else 1 if hb < lk + lg else 2 if hb < lk + lg + lw else 3] += 1
    return counts


# ALU instructions per element and layer: int32 keys take one min or max per
# element inside a thread and both (one kept per lane) across threads; records
# take a compare and four selects per pair inside a thread and about five
# instructions per element across threads.
ALU_PER_ELEM = {bs.I32: (1.0, 2.0), bs.I32_I32: (2.5, 5.0), bs.U64: (2.5, 5.0), bs.U64_I32: (2.5, 5.0)}


def alu_roofline(dtype, tile, elements, seconds, sm_mhz, form=0):
    """Integer-ALU bound of the network: modelled instructions per element x
    element slots over the B200's ALU rate (16 lanes per clock per SM
    sub-partition, 4 per SM, 148 SMs).  Launch form 3 (the transposed network)
    runs every layer inside one thread's registers."""
    reg, lane, warp, cta = layer_counts(tile.log2_items, tile.log2_lanes, tile.log2_warps, tile.log2_ctas)
    if form == 3:
        reg, lane, warp = reg + lane + warp, 0, 0
    inside, across = ALU_PER_ELEM[dtype]
    per_elem = reg * inside + (lane + warp + cta) * across
    sms = 148
    mhz = sm_mhz or 1965.0
    peak = 64 * sms * mhz * 1e6           # ALU lane-instructions per second
    achieved = per_elem * elements / seconds
    return {"ops_per_element": per_elem, "layers": {"registers": reg, "lanes": lane, "warps": warp, "ctas": cta},
            "achieved_tops": achieved / 1e12, "peak_tops": peak / 1e12, "frac": achieved / peak,
            "sm_mhz": mhz, "model": "int32: 1 ALU op per element per in-thread layer, 2 across threads; "
                                    "records: 2.5 and 5 (compare + selects)"}


_ONCHIP = {}


def onchip_peaks(device, cluster=0):
    """Shared-memory (and, for cluster > 1, distributed-shared-memory) bandwidth
    of this device in GB/s, measured once per process by the probes of
    cuda-sort_b200/harness/onchip_peak.cu."""
    key = (device, cluster)
    if key not in _ONCHIP:
        lib = ctypes.CDLL(os.path.join(ROOT, "cuda-sort_b200", "libb200sort_onchip.so"))
        rd, cp = ctypes.c_double(0), ctypes.c_double(0)
        out = {}
        if lib.onchip_smem_gbs(device, ctypes.byref(rd), ctypes.byref(cp)) == 0:
            out.update(smem_read_gbs=rd.value, smem_copy_gbs=cp.value)
        if cluster > 1:
            ds = ctypes.c_double(0)
            if lib.onchip_dsmem_gbs(device, cluster, ctypes.byref(ds)) == 0:
                out["dsmem_read_gbs"] = ds.value
        _ONCHIP[key] = out
    return _ONCHIP[key]


def onchip_roofline(widths, elem_bytes, seconds, t_hbm, device, lc=0, arrays=0):
    """On-chip bound: every bitonic stage whose span leaves a 1024-element
    window costs at least one write and one read of the tile, so
    bytes = sum 2 * W * elem_bytes * max(0, log2 W - 10) over the arrays,
    against the measured shared-memory copy rate; fraction = the larger of the
    HBM and on-chip times over the measured time.  For cluster kernels also the
    distributed-shared-memory reads: every cross-CTA layer reads the whole tile
    from peers once."""
    widths = np.asarray(widths, dtype=np.int64)
    logw = np.log2(widths).astype(np.int64)
    r = np.maximum(0, logw - 10)
    nbytes = float(np.sum(2 * widths * elem_bytes * r))
    pk = onchip_peaks(device, 1 << lc if lc else 0)
    out = {"bytes": nbytes, "model": "sum 2*W*elem_bytes*max(0, log2 W - 10) at the measured shared-memory copy rate"}
    if "smem_copy_gbs" in pk:
        t_on = nbytes / (pk["smem_copy_gbs"] * 1e9)
        out.update(pk, t_us=t_on * 1e6, frac=t_on / seconds, frac_max_hbm_onchip=max(t_hbm, t_on) / seconds)
    if lc and "dsmem_read_gbs" in pk:
        layers = lc * (lc + 1) // 2
        dbytes = float(arrays) * layers * float(widths.max()) * elem_bytes
        t_ds = dbytes / (pk["dsmem_read_gbs"] * 1e9)
        out["dsmem"] = {"bytes": dbytes, "cross_cta_layers": layers, "t_us": t_ds * 1e6, "frac": t_ds / seconds}
    return out


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


# ---- CPU baseline: the reference's own std::sort per array (oracle/_ref) ------------

def _cpu_runner(data, wl, threads, off=None):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_oracle as orc

    dtype = wl["dtype"]
    if orc.ref_cpu_available() and dtype in (bs.I32, bs.I32_I32):
        code = 0 if dtype == bs.I32 else 1
        if off is None:
            return (lambda buf: orc.ref_cpu_sort_inplace(code, buf, wl["n"], wl["arrays"], threads)), "reference"
        return (lambda buf: orc.ref_cpu_sort_ragged_inplace(code, buf, off, threads)), "reference"
    if off is None:
        def port(buf):
            buf[:] = orc.sort_packed(dtype, buf, wl["n"], wl["arrays"], orc.MODE_STD, threads)
    else:
        def port(buf):
            buf[:] = orc.sort_ragged(dtype, buf, off, orc.MODE_STD, threads)
    return port, "port"


def time_cpu(data, wl, threads, off=None, budget_s=8.0, min_reps=2, max_reps=50):
    run, kind = _cpu_runner(data, wl, threads, off)
    times, total = [], 0.0
    while len(times) < max_reps and (len(times) < min_reps or total < budget_s):
        buf = data.copy()
        t0 = time.perf_counter()
        run(buf)
        dt = time.perf_counter() - t0
        times.append(dt)
        total += dt
    return statistics.median(times), kind, len(times)


def make_input(wl, seed):
    if wl["kind"] == "packed":
        return workloads.make_packed(wl["dtype"], wl["n"], wl["arrays"], wl["dist"], seed=seed), None
    if "min_len" in wl:
        lengths = workloads.log_uniform_lengths(wl["arrays"], wl["min_len"], wl["max_len"], seed=seed)
    else:
        lengths = workloads.ragged_lengths(wl["arrays"], max_len=wl["max_len"], seed=seed)
    return workloads.make_ragged(wl["dtype"], lengths, wl["dist"], seed=seed)


def config_of(args, wl, data):
    c = {"workload": args.workload, "kind": wl["kind"], "arrays_per_gpu": wl["arrays"],
         "key_dtype": DTYPE_NAMES[wl["dtype"]], "distribution": wl["dist"],
         "stable": bool(wl["flags"] & bs.STABLE), "sorted_check": bool(wl["flags"] & bs.SORTED_CHECK),
         "parallelism": "replicas (arrays are independent)",
         "keys_per_gpu": int(len(data))}
    if wl["kind"] == "packed":
        c["n"] = wl["n"]
        c["l2"] = "inputs rotate over sets larger than L2 (126 MB)"
    else:
        c["lengths"] = "log-uniform in [%d, %d], CSR int32 offsets" % (wl.get("min_len", 1), wl["max_len"])
        c["l2"] = "input %.2f GB, larger than L2" % (data.nbytes / 1e9)
    return c


def reference_arm(args, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    data, off = make_input(wl, 1234)
    threads = os.cpu_count() or 1
    run, kind = _cpu_runner(data, wl, threads, off)
    for _ in range(args.warmup):
        run(data.copy())
    total = 0.0
    for _ in range(args.steps):
        buf = data.copy()
        t0 = time.perf_counter()
        run(buf)
        total += time.perf_counter() - t0
    sec = total / max(1, args.steps)
    value = len(data) / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": DTYPE_NAMES[wl["dtype"]], "data": "synthetic",
        "config": config_of(args, wl, data),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": "the full batch (%d arrays, %d keys) per step, std::sort per array over %d "
                                   "host threads" % (wl["arrays"], len(data), threads)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---- ranks ------------------------------------------------------------------------
# One process per GPU; ranks are independent replicas (arrays are independent),
# so the only cross-rank operations are barriers and the maximum of the
# per-rank device times.

def reduce_max(dist, world, x, device):
    """Maximum of x over the ranks (x itself for a single rank)."""
    if world == 1:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_value(keys_per_rank, world, ms_max):
    """Whole-job keys/s: every rank sorted keys_per_rank keys; the job took the slowest rank's time."""
    return keys_per_rank * world / (ms_max * 1e-3)


# ---- GPU arm ---------------------------------------------------------------------

class Ctx:
    def __init__(self):
        import torch
        import torch.distributed as dist

        self.torch, self.dist = torch, dist
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(self.local)
        self.dev = torch.device("cuda", self.local)
        if self.world > 1:
            import datetime
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=self.dev)
        self.stream = torch.cuda.current_stream(self.dev)
        self.sh = self.stream.cuda_stream

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max_over_ranks(self, x):
        return reduce_max(self.dist, self.world, x, self.dev)

    def sync(self):
        self.torch.cuda.synchronize(self.dev)

    def event_time(self, step, count):
        """Device time of `count` back-to-back steps, between a barrier and a sync on both sides."""
        torch = self.torch
        self.barrier()
        self.sync()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(self.stream)
        for j in range(count):
            step(j)
        ev1.record(self.stream)
        self.sync()
        self.barrier()
        return self.max_over_ranks(ev0.elapsed_time(ev1))


def timed_region(ctx, step, args):
    for i in range(max(3, args.warmup)):
        step(i)
    ctx.sync()
    sampler = ClockSampler(None)
    try:
        uuid = str(ctx.torch.cuda.get_device_properties(ctx.dev).uuid)
        sampler = ClockSampler(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
    except Exception:
        pass
    sampler.start()
    t_end = time.perf_counter() + args.preroll
    i = 0
    while time.perf_counter() < t_end:
        for _ in range(10):
            step(i)
            i += 1
        ctx.sync()
    ms_total = ctx.event_time(step, args.steps)
    sampler.stop()
    return ms_total / args.steps, sampler.summary()


# ---- GPU baselines on the same inputs (packed workloads, one GPU) ------------------
# Three baselines the headline is compared with, each timed exactly like the
# product here: in place on BASELINE_SETS separate copies of the batch, restored
# and then evicted from L2 by a 256 MB write before every timed pass, one
# launch per copy back to back between two CUDA events (per launch = the pass
# time / BASELINE_SETS), median of the passes.  The best configuration of each
# family comes from a sweep at one pass each, then is re-timed.
#   plain      this library's launch form 0 of the same tile (one launch, one
#              array group per CTA slot, no persistence, TMA or transposes);
#   cub        CUB BlockMergeSort, the block-sort sequence the reference's
#              bench times (bench.cu:406-423), built into libb200sort_cub.so,
#              every thread count;
#   ref_v6     the reference's own V6 kernel (cusort_v6.hpp:144-184) compiled
#              unmodified for sm_100a (oracle/_ref/), over the reference's own
#              sweep of threads and Sorted / Shared / Async (bench.cu:497-552).
BASELINE_SETS = 24
CUB_LIB = os.path.join(ROOT, "cuda-sort_b200", "libb200sort_cub.so")


def _batched_inplace_us(ctx, launch, sets, pristine, flush, passes):
    torch = ctx.torch
    times = []
    for r in range(passes):
        for s in sets:
            s.copy_(pristine)
        flush.fill_(r & 0xFF)
        ctx.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ctx.stream)
        for s in sets:
            if launch(s.data_ptr()) not in (0, None):
                ctx.sync()
                return None
        e1.record(ctx.stream)
        ctx.sync()
        times.append(e0.elapsed_time(e1) * 1e3 / len(sets))
    return statistics.median(times)


def gpu_baselines(ctx, wl, data, host, ours_tile):
    torch = ctx.torch
    dtype, n, arrays, flags = wl["dtype"], wl["n"], wl["arrays"], wl["flags"]
    npd = bs.NP_DTYPES[dtype]
    keys_in = data if dtype in (bs.I32, bs.U64) else data["key"]
    want = np.sort(keys_in.reshape(arrays, n), axis=1).reshape(-1)
    pristine = host.to(ctx.dev)
    sets = [torch.empty_like(pristine) for _ in range(BASELINE_SETS)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=ctx.dev)
    w = 32
    while w < n:
        w *= 2
    out = {"method": "in place on %d copies of the batch restored and evicted from L2 before each pass, "
                     "%d back-to-back launches between two CUDA events, median of 5 passes "
                     "(best configuration of each family from a one-pass sweep)" % (BASELINE_SETS, BASELINE_SETS)}

    def check():
        got = sets[0].cpu().numpy().view(npd)
        k = got if dtype in (bs.I32, bs.U64) else got["key"]
        return bool(np.array_equal(k, want))

    def family(name, candidates):
        best = None
        for cfg, launch in candidates:
            us = _batched_inplace_us(ctx, launch, sets, pristine, flush, 1)
            if us is not None and (best is None or us < best[1]):
                best = (cfg, us, launch)
        if best is None:
            return
        us = _batched_inplace_us(ctx, best[2], sets, pristine, flush, 5)
        out[name] = {"us": us, "config": best[0], "verified": us is not None and check()}

    st = ctx.sh
    family("ours", [(repr(ours_tile), lambda p: bs.sort_packed_status(dtype, p, p, n, arrays, flags, ours_tile, st))])
    plain = ours_tile.with_form(0)
    family("plain", [(repr(plain), lambda p: bs.sort_packed_status(dtype, p, p, n, arrays, flags, plain, st))])
    plain_flags = flags & ~bs.SORTED_CHECK
    if dtype in (bs.I32, bs.I32_I32) and not plain_flags and os.path.exists(CUB_LIB) and w <= 4096:
        cub = ctypes.CDLL(CUB_LIB)
        cub.cub_block_merge_sort.restype = ctypes.c_int
        cub.cub_block_merge_sort.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        family("cub", [("threads=%d items=%d" % (th, w // th),
                        lambda p, th=th: cub.cub_block_merge_sort(dtype, p, n, arrays, w, th, st))
                       for th in (32, 64, 128, 256, 512, 1024) if th <= w and w // th <= 32])
    if dtype in (bs.I32, bs.I32_I32) and not plain_flags:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import cpu_oracle as orc
        if orc.ref_gpu_available() and w <= (4096 if dtype == bs.I32 else 2048):
            suffix = "int" if dtype == bs.I32 else "rec"
            fn = getattr(orc.ref_gpu(suffix), "ref_v6_" + suffix)
            cands = []
            for th in (32, 64, 128, 256, 512, 1024):
                if th > w or w // th > 16:
                    continue
                # with the sortedness check, the reference's own Sorted switch (Sorted=true
                # compiles with Shared=Async=false only in its sweep)
                combos = ((1, 0, 0),) if flags & bs.SORTED_CHECK else ((0, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1),
                                                                        (1, 0, 0))
                for so, sh, asy in combos:
                    cands.append(("threads=%d sorted=%d shared=%d async=%d" % (th, so, sh, asy),
                                  lambda p, th=th, so=so, sh=sh, asy=asy: fn(p, n, arrays, w, th, so, sh, asy, st)))
            family("ref_v6", cands)
    base = out.get("ours", {}).get("us")
    for name in ("plain", "cub", "ref_v6"):
        if base and name in out and out[name]["us"]:
            out["vs_" + name] = out[name]["us"] / base
    del sets, flush, pristine
    torch.cuda.empty_cache()
    return out


def bucket_breakdown(ctx, wl, data, off):
    """Per power-of-two length class: the persistent graph form on a batch
    holding only that class's arrays of the same input (device time, median
    of 5 batched passes), its arrays and elements, and its share of the sum."""
    torch = ctx.torch
    dtype, flags = wl["dtype"], wl["flags"]
    lens = np.diff(off)
    cls = np.where(lens > 0, np.ceil(np.log2(np.maximum(lens, 1))).astype(np.int64), -1)
    rows = []
    for L in sorted(set(cls[cls >= 0].tolist())):
        ids = np.nonzero(cls == L)[0]
        sub_len = lens[ids]
        sub_off = np.zeros(len(ids) + 1, dtype=np.int64)
        np.cumsum(sub_len, out=sub_off[1:])
        idx = np.concatenate([np.arange(off[a], off[a + 1]) for a in ids])
        sub = data[idx]
        d_in = torch.from_numpy(sub.view(np.uint8).copy()).to(ctx.dev)
        d_out = torch.empty_like(d_in)
        d_off = torch.from_numpy(sub_off.astype(np.int32)).to(ctx.dev)
        with bs.Plan(dtype, len(ids), flags, ctx.local) as plan:
            def step(i):
                plan.sort(d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), len(ids), ctx.sh)
            step(0)
            times = [ctx.event_time(step, 5) / 5 for _ in range(5)]
            # the same class through the plain form (one launch of the tabled tile of W)
            plan.prepare_plain(sub_off.astype(np.int32), by_bucket=True)

            def plain(i):
                plan.sort_plain(d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), ctx.sh)
            plain(0)
            ptimes = [ctx.event_time(plain, 5) / 5 for _ in range(5)]
        rows.append({"working_length": 1 << L, "arrays": int(len(ids)), "elements": int(sub_len.sum()),
                     "ms": statistics.median(times), "plain_ms": statistics.median(ptimes)})
    total = sum(r["ms"] for r in rows)
    for r in rows:
        r["share"] = r["ms"] / total if total else 0.0
    return {"method": "each length class alone through its own plan (graph replay) and through the plain form "
                      "(one launch of the tabled tile), 5 back-to-back steps between CUDA events, median of 5; "
                      "shares of the sum of the classes", "classes": rows, "sum_ms": total,
            "plain_sum_ms": sum(r["plain_ms"] for r in rows)}


def verify_ragged(dtype, data, off, got):
    """Size-independent checks: sorted within every array, per-array key sums
    equal, and (records) every payload is the position of an equal key of the
    same array, each position used once."""
    keys_in = data if dtype in (bs.I32, bs.U64) else data["key"]
    keys = got if dtype in (bs.I32, bs.U64) else got["key"]
    starts = off[:-1]
    nonempty = off[1:] > starts
    boundary = np.zeros(len(keys), dtype=bool)
    boundary[starts[nonempty]] = True
    ok = bool(np.all((keys[1:] >= keys[:-1]) | boundary[1:]))
    s_in = np.add.reduceat(keys_in.astype(np.int64), starts[nonempty]) if nonempty.any() else 0
    s_out = np.add.reduceat(keys.astype(np.int64), starts[nonempty]) if nonempty.any() else 0
    ok = ok and bool(np.array_equal(s_in, s_out))
    if dtype in (bs.I32_I32, bs.U64_I32):
        pos = got["data"].astype(np.int64)
        arr = np.repeat(np.arange(len(off) - 1), np.diff(off))
        ok = ok and bool(np.all((pos >= off[arr]) & (pos < off[arr + 1])))
        ok = ok and bool(np.array_equal(keys_in[pos], keys))
        ok = ok and bool(np.all(np.bincount(pos, minlength=len(keys)) == 1))
    return ok


def run_gpu(args, wl):
    ctx = Ctx()
    torch = ctx.torch
    dtype, flags = wl["dtype"], wl["flags"]
    eb = bs.ELEM_BYTES[dtype]
    data, off = make_input(wl, 1234 + ctx.rank)
    total_keys = len(data)
    batch_bytes = data.nbytes
    host = torch.from_numpy(data.view(np.uint8).copy())
    extra = {}

    if wl["kind"] == "packed":
        n, arrays = wl["n"], wl["arrays"]
        sets = max(2, math.ceil(2 * L2_BYTES / batch_bytes) + 1) if batch_bytes < 2 * L2_BYTES else 1
        d_in = [host.to(ctx.dev) for _ in range(sets)]
        d_out = [torch.empty_like(d_in[0]) for _ in range(sets)]

        tile = None
        if args.form != "table" or args.tile:
            t = bs.default_tile(dtype, n, flags)
            shape = [int(x) for x in args.tile.split(",")] if args.tile else [t.log2_items, t.log2_lanes, t.log2_warps]
            form = t.persistent if args.form == "table" else int(args.form)
            tile = bs.Tile(shape[0], shape[1], shape[2], 0, form, 0 if args.tile else t.log2_ctas)
        eff = tile if tile is not None else bs.default_tile(dtype, n, flags)
        extra["tile"] = repr(eff)
        tma_ok = (n * eb) % 128 == 0 and n * eb // 128 <= 256 and eff.log2_warps == 0 and eff.log2_ctas == 0
        form = eff.persistent if (eff.persistent != 2 or tma_ok) else 0

        def step(i):
            k = i % sets
            bs.sort_packed(dtype, d_in[k].data_ptr(), d_out[k].data_ptr(), n, arrays, flags, tile, ctx.sh)

        ms_step, clocks = timed_region(ctx, step, args)
        got = d_out[(args.steps - 1) % sets].cpu().numpy().view(bs.NP_DTYPES[dtype])
        keys_in = data if dtype in (bs.I32, bs.U64) else data["key"]
        keys_out = got if dtype in (bs.I32, bs.U64) else got["key"]
        verified = bool(np.array_equal(keys_out.reshape(arrays, n), np.sort(keys_in.reshape(arrays, n), axis=1)))
        info = bs.tile_info(dtype, n, flags, eff)
        cluster = info.arrays_per_cta == 0
        if form == 3 and not info.xpose_form:
            form = 0
        if form == 3:
            kernel = "k_sort_cluster_xc" if cluster else "k_sort_packed_xc" if eff.log2_warps > 0 else "k_sort_xpose"
        else:
            kernel = "k_sort_cluster" if cluster else {0: "k_sort_packed", 1: "k_sort_packed_pf",
                                                       2: "k_sort_packed_tma"}[form]
        launches = args.steps
        if ctx.world == 1 and not args.no_baselines:
            extra["baselines"] = gpu_baselines(ctx, wl, data, host, eff)
    else:
        arrays = wl["arrays"]
        d_in = host.to(ctx.dev)
        d_out = torch.empty_like(d_in)
        d_off = torch.from_numpy(off.astype(np.int32)).to(ctx.dev)
        plan = bs.Plan(dtype, arrays, flags, ctx.local)

        def step(i):
            plan.sort(d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), arrays, ctx.sh)

        ms_step, clocks = timed_region(ctx, step, args)
        got = d_out.cpu().numpy().view(bs.NP_DTYPES[dtype])
        verified = verify_ragged(dtype, data, off, got) and plan.too_long(ctx.sh) == 0
        kernel = "k_sort_ragged"
        launches = 3 * args.steps   # bin count, bin scatter, sort (one graph per step)
    if wl["kind"] == "ragged" and not args.no_plain:
        # the plain per-length launches on the same input
        plain_launches = plan.prepare_plain(off.astype(np.int32))
        d_out.zero_()

        def plain(i):
            plan.sort_plain(d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), ctx.sh)

        for i in range(2):
            plain(i)
        psteps = max(2, min(args.steps, 5))
        ms_plain = ctx.event_time(plain, psteps) / psteps
        verified = verified and verify_ragged(dtype, data, off, d_out.cpu().numpy().view(bs.NP_DTYPES[dtype]))
        # the same kernels launched once per power-of-two length class
        bucket_launches = plan.prepare_plain(off.astype(np.int32), by_bucket=True)
        for i in range(2):
            plain(i)
        ms_bucket = ctx.event_time(plain, psteps) / psteps
        verified = verified and verify_ragged(dtype, data, off, d_out.cpu().numpy().view(bs.NP_DTYPES[dtype]))
        extra["baselines"] = {
            "plain_per_length": {
                "ms_per_step": ms_plain, "value": total_keys * ctx.world / (ms_plain * 1e-3), "unit": UNIT,
                "launches_per_step": plain_launches, "persistent_graph_speedup": ms_plain / ms_step},
            "plain_per_bucket": {
                "ms_per_step": ms_bucket, "value": total_keys * ctx.world / (ms_bucket * 1e-3), "unit": UNIT,
                "launches_per_step": bucket_launches, "persistent_graph_speedup": ms_bucket / ms_step}}
        if ctx.world == 1:
            extra["bucket_breakdown"] = bucket_breakdown(ctx, wl, data, off)

    value = weak_value(total_keys, ctx.world, ms_step)
    hbm, peak_src = peaks()
    algo_bytes = 2 * batch_bytes
    achieved = algo_bytes / (ms_step * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "peak_source": peak_src, "traffic": traffic_for(args.workload),
                "algorithmic_bytes_per_launch": algo_bytes, "kernel": kernel, "launch_us": ms_step * 1e3}
    t_hbm = algo_bytes / (hbm * 1e9)
    if wl["kind"] == "packed":
        w = 1 << (eff.log2_items + eff.log2_lanes + eff.log2_warps + eff.log2_ctas)
        roofline["alu"] = alu_roofline(dtype, eff, wl["arrays"] * w, ms_step * 1e-3, clocks.get("sm_mhz"), form)
        wmin = 1 << max(5, int(wl["n"] - 1).bit_length())
        roofline["onchip"] = onchip_roofline(np.full(wl["arrays"], wmin), bs.ELEM_BYTES[dtype], ms_step * 1e-3,
                                             t_hbm, ctx.local, lc=eff.log2_ctas, arrays=wl["arrays"])
    else:
        lens = np.diff(off).astype(np.int64)
        lens = lens[lens > 0]
        widths = np.left_shift(1, np.maximum(5, np.ceil(np.log2(np.maximum(lens, 1))).astype(np.int64)))
        roofline["onchip"] = onchip_roofline(widths, bs.ELEM_BYTES[dtype], ms_step * 1e-3, t_hbm, ctx.local)

    e2e = None
    if not args.no_e2e:
        pin_in = host.pin_memory()
        pin_out = torch.empty_like(pin_in).pin_memory()
        esteps = max(3, min(args.steps, 30 if wl["kind"] == "packed" else 5))
        if wl["kind"] == "packed":
            with bs.Session(ctx.local) as sess:
                def e2e_step():
                    sess.sort_host(dtype, pin_in.data_ptr(), pin_out.data_ptr(), wl["n"], wl["arrays"], flags)
                e2e_step()
                ctx.barrier()
                t0 = time.perf_counter()
                for _ in range(esteps):
                    e2e_step()
                dt = time.perf_counter() - t0
            path = "b200s_sort_packed_host (pinned host buffers, chunked copy/sort overlap)"
            h2d = batch_bytes
        else:
            pin_off = torch.from_numpy(off.astype(np.int32)).pin_memory()

            def e2e_step():
                d_in.copy_(pin_in, non_blocking=True)
                d_off.copy_(pin_off, non_blocking=True)
                plan.sort(d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), wl["arrays"], ctx.sh)
                pin_out.copy_(d_out, non_blocking=True)
                ctx.sync()
            e2e_step()
            ctx.barrier()
            t0 = time.perf_counter()
            for _ in range(esteps):
                e2e_step()
            dt = time.perf_counter() - t0
            path = "pinned copies + b200s_sort_ragged (plan graph) + pinned copy back"
            h2d = batch_bytes + pin_off.numel() * 4
        ctx.barrier()
        dt = ctx.max_over_ranks(dt)
        e2e = {"value": total_keys * ctx.world * esteps / dt, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": batch_bytes, "steps": esteps, "path": path}
        out = pin_out.numpy().view(bs.NP_DTYPES[dtype])
        verified = verified and bool(np.array_equal(out["key"] if dtype in (bs.I32_I32, bs.U64_I32) else out,
                                                    got["key"] if dtype in (bs.I32_I32, bs.U64_I32) else got))

    cpu = None
    if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sec, kind, reps = time_cpu(data, wl, threads, off)
        cpu = {"value": total_keys / sec, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": "the full batch (%d arrays, %d keys), %d repetitions, std::sort per array"
                         % (wl["arrays"], total_keys, reps)}

    if ctx.world > 1:
        ctx.dist.destroy_process_group()
    if ctx.rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ctx.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": DTYPE_NAMES[dtype], "data": "synthetic",
        "config": config_of(args, wl, data), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": launches, "clocks": clocks, "verified": verified, "library": bs.version(),
    }
    line.update(extra)
    print(json.dumps(line))
    return 0 if verified else 1


# ---- serving: request stream into the continuous-batching server -------------------

class LgResult(ctypes.Structure):
    """lg_result of the load generator (cuda-sort_b200/harness/loadgen.cpp)."""
    _fields_ = [(n, ctypes.c_int64) for n in ("submitted", "completed", "rejected", "batches", "peak_arena_bytes")] + \
        [(n, ctypes.c_double) for n in ("p50_us", "p99_us", "p999_us", "max_us", "mean_us", "span_s", "keys_per_s",
                                        "req_per_s", "offered_req_per_s", "max_lag_us", "mean_batch")] + \
        [("overloaded", ctypes.c_int32)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


def run_serving(args, wl):
    ctx = Ctx()
    torch = ctx.torch
    if ctx.world > 1:
        ctx.dist.destroy_process_group()   # replicas: every rank serves its own stream
    dtype = wl["dtype"]
    lens = workloads.log_uniform_lengths(wl["arrays"], wl["min_len"], wl["max_len"], seed=4321 + ctx.rank)
    data, off = workloads.make_ragged(dtype, lens, wl["dist"], seed=4321 + ctx.rank)
    d_all = torch.from_numpy(data.view(np.uint8).copy()).to(ctx.dev)
    o_all = torch.empty_like(d_all)
    eb = bs.ELEM_BYTES[dtype]
    P = len(lens)
    src = (ctypes.c_void_p * P)(*[d_all.data_ptr() + int(off[i]) * eb for i in range(P)])
    dst = (ctypes.c_void_p * P)(*[o_all.data_ptr() + int(off[i]) * eb for i in range(P)])
    c_lens = (ctypes.c_int32 * P)(*[int(x) for x in lens])
    lg = ctypes.CDLL(os.path.join(ROOT, "cuda-sort_b200", "libb200sort_loadgen.so"))
    lg.lg_run.restype = ctypes.c_int
    lg.lg_run.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                          ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                          ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(LgResult)]
    SERVER_OPEN, PLAIN_OPEN, SERVER_CLOSED, PLAIN_CLOSED = 0, 1, 2, 3
    srv = bs.Server(dtype, budget_bytes=wl["budget"], max_inflight=4, max_batch=4096, max_queue=1 << 20,
                    device=ctx.local)

    def run(mode, rate=0.0, window=0, duration=args.duration, seed=1):
        r = LgResult()
        rc = lg.lg_run(mode, srv._h if mode in (SERVER_OPEN, SERVER_CLOSED) else None, dtype, src, dst, c_lens, P,
                       rate, duration, window, seed, 1.0, ctypes.byref(r))
        if rc != 0:
            raise RuntimeError("load generator mode %d failed with %d: %s" % (mode, rc, bs.lib().b200s_last_error()))
        return r

    clocks_sampler = ClockSampler(None)
    try:
        uuid = str(torch.cuda.get_device_properties(ctx.dev).uuid)
        clocks_sampler = ClockSampler(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
    except Exception:
        pass
    # warm-up: every kernel and both paths once, untimed
    run(SERVER_CLOSED, window=1024, duration=0.5)
    run(PLAIN_CLOSED, window=256, duration=0.3)
    clocks_sampler.start()
    peak = run(SERVER_CLOSED, window=8192)
    plain_peak = run(PLAIN_CLOSED, window=1024)
    rates = [float(x) for x in args.rates.split(",") if x]
    half = 0.5 * peak.req_per_s
    points = []
    for rate in rates + [half]:
        srv_r = run(SERVER_OPEN, rate=rate, seed=int(rate) + 7)
        pl_r = run(PLAIN_OPEN, rate=rate, seed=int(rate) + 7)
        points.append({"offered_req_per_s": rate, "server": srv_r.as_dict(), "plain": pl_r.as_dict(),
                       "is_half_peak": rate == half})
    clocks_sampler.stop()
    torch.cuda.synchronize()
    srv.close()
    # every pool entry holds the sort of its own input (the last request that used it)
    got = o_all.cpu().numpy().view(bs.NP_DTYPES[dtype])
    verified = verify_ragged(dtype, data, off, got)
    value = peak.keys_per_s * ctx.world
    hp = points[-1]["server"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ctx.world, "steps": len(points) + 2,
        "warmup": 2, "ms_per_step": args.duration * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": DTYPE_NAMES[dtype], "data": "synthetic",
        "config": {"workload": "serving", "kind": "serving", "requests_in_pool": P,
                   "lengths": "log-uniform in [%d, %d] records" % (wl["min_len"], wl["max_len"]),
                   "key_dtype": DTYPE_NAMES[dtype], "distribution": wl["dist"], "budget_bytes": wl["budget"],
                   "max_inflight_batches": 4, "seconds_per_point": args.duration,
                   "l2": "pool of %.0f MB inputs + outputs, larger than L2" % (2 * data.nbytes / 1e6)},
        "serving": {"peak_closed_loop": peak.as_dict(), "plain_closed_loop": plain_peak.as_dict(),
                    "peak_speedup_vs_plain": peak.keys_per_s / max(plain_peak.keys_per_s, 1.0),
                    "half_peak_req_per_s": half, "half_peak_p99_us": hp["p99_us"],
                    "half_peak_p99_target_met": bool(hp["p99_us"] <= 1000.0 and not hp["overloaded"]),
                    "poisson": points},
        "roofline": None, "cpu_baseline": None,
        "e2e": None, "gpu_launches": int(peak.batches * 5), "clocks": clocks_sampler.summary(),
        "verified": verified, "library": bs.version(),
    }
    if ctx.rank == 0:
        print(json.dumps(line))
    return 0 if verified else 1


def main():
    args = parse()
    wl = dict(WORKLOADS[args.workload])
    if args.distribution and wl["kind"] == "packed":
        wl["dist"] = args.distribution
    if args.sorted_check and wl["kind"] == "packed":
        wl["flags"] = wl["flags"] | bs.SORTED_CHECK
    if args.impl == "reference":
        return reference_arm(args, wl)
    if wl["kind"] == "serving":
        return run_serving(args, wl)
    return run_gpu(args, wl)


if __name__ == "__main__":
    sys.exit(main())
