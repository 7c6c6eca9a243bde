"""Side-by-side kernel timing on one B200: the new kernels, CUB BlockMergeSort
and the reference's own V6 kernel (compiled from its headers into
oracle/_ref/), on identical inputs.  Measurement infrastructure, not a test:

  python tests/perf_baselines.py [--out FILE.json] [--reps R]

Every timed launch starts from a freshly restored input and an L2 flushed by
a 512 MB write, so no kernel reads a warm cache.  Times are CUDA-event
medians per launch.  For each family the best configuration is reported:
the reference's own sweep (bench.cu:497-521: Threads and the Sorted /
Shared / Async switches) for V6, every thread count for CUB, every compiled
tile for the new kernels, in each launch form.  Outputs are checked against numpy/the oracle.
"""
import argparse
import ctypes
import json
import os
import statistics
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "cuda-sort_b200")]

import numpy as np  # noqa: E402
import torch  # noqa: E402

import b200sort as bs  # noqa: E402
import cpu_oracle as orc  # noqa: E402
import workloads  # noqa: E402

CUB_LIB = os.path.join(ROOT, "cuda-sort_b200", "libb200sort_cub.so")


def working(n):
    w = 32
    while w < n:
        w *= 2
    return w


class Timer:
    def __init__(self, data):
        self.src = torch.from_numpy(data.view(np.uint8).copy()).cuda()
        self.work = torch.empty_like(self.src)
        self.out = torch.empty_like(self.src)
        self.flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
        self.st = torch.cuda.current_stream()

    def time(self, launch, reps, inplace):
        times = []
        for r in range(reps + 2):
            self.work.copy_(self.src)
            self.flush.fill_(r & 0xFF)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(self.st)
            rc = launch(self.work.data_ptr(), (self.work if inplace else self.out).data_ptr())
            e1.record(self.st)
            torch.cuda.synchronize()
            if rc not in (0, None):
                return None, None
            if r >= 2:
                times.append(e0.elapsed_time(e1) * 1e3)
        res = (self.work if inplace else self.out).cpu().numpy()
        return statistics.median(times), res


def run_case(dtype, n, arrays, dist, reps, results):
    data = workloads.make_packed(dtype, n, arrays, dist, seed=99)
    npd = bs.NP_DTYPES[dtype]
    if dtype == bs.I32:
        want = np.sort(data.reshape(arrays, n), axis=1).reshape(-1)
    else:
        want = orc.sort_packed(dtype, data, n, arrays, orc.MODE_NETWORK, threads=os.cpu_count())
    timer = Timer(data)
    st = timer.st.cuda_stream
    w = working(n)
    case = {"dtype": dtype, "n": n, "arrays": arrays, "distribution": dist, "keys": n * arrays,
            "hbm_bytes": 2 * n * arrays * bs.ELEM_BYTES[dtype], "configs": []}

    def record(family, cfg, us, res):
        ok = None
        if res is not None:
            got = res.view(npd)
            ok = bool(np.array_equal(got["key"] if dtype else got, want["key"] if dtype else want))
        case["configs"].append({"family": family, "config": cfg, "us": us, "ok": ok})

    for base in bs.tiles(dtype):
        tw = 1 << sum(base.as_tuple())
        if tw < n or tw > 4 * w:
            continue
        forms = [base, base.with_persistent()]
        if bs.tile_info(dtype, n, 0, base).tma_form:
            forms.append(base.with_form(2))
        for tile in forms:
            us, res = timer.time(lambda i, o, t=tile: bs.sort_packed(dtype, i, o, n, arrays, 0, t, st), reps,
                                 False)
            record("b200sort", repr(tile), us, res)

    if os.path.exists(CUB_LIB):
        cub = ctypes.CDLL(CUB_LIB)
        cub.cub_block_merge_sort.restype = ctypes.c_int
        cub.cub_block_merge_sort.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        for th in (32, 64, 128, 256, 512, 1024):
            if th > w or w // th > 32:
                continue
            us, res = timer.time(lambda i, o, th=th: cub.cub_block_merge_sort(dtype, i, n, arrays, w, th, st),
                                 reps, True)
            if us is not None:
                record("cub_block_merge", "threads=%d items=%d" % (th, w // th), us, res)

    if orc.ref_gpu_available() and dtype in (bs.I32, bs.I32_I32):
        suffix = "int" if dtype == bs.I32 else "rec"
        fn = getattr(orc.ref_gpu(suffix), "ref_v6_" + suffix)
        for th in (32, 64, 128, 256, 512, 1024):
            if th > w or w // th > 16:
                continue
            for sh, asy in ((0, 0), (1, 0), (0, 1), (1, 1)):
                us, res = timer.time(lambda i, o, th=th, sh=sh, asy=asy: fn(i, n, arrays, w, th, 0, sh, asy, st),
                                     reps, True)
                if us is not None:
                    record("reference_v6", "threads=%d shared=%d async=%d" % (th, sh, asy), us, res)

    best = {}
    for c in case["configs"]:
        if c["us"] is None or not c["ok"]:
            continue
        if c["family"] not in best or c["us"] < best[c["family"]]["us"]:
            best[c["family"]] = c
    case["best"] = best
    results.append(case)
    line = "dtype=%d n=%d arrays=%d: " % (dtype, n, arrays) + ", ".join(
        "%s %.2f us (%s)" % (f, b["us"], b["config"]) for f, b in sorted(best.items()))
    print(line, flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--reps", type=int, default=15)
    ap.add_argument("--quick", action="store_true")
    args = ap.parse_args()
    results = []
    run_case(bs.I32, 1024, 4096, "uniform", args.reps, results)
    if not args.quick:
        for n in (32, 129, 256, 1000, 2048, 4096):
            run_case(bs.I32_I32, n, 4194304 // n, "uniform", args.reps, results)
    bad = [(c["n"], x["family"], x["config"]) for c in results for x in c["configs"] if x["ok"] is False]
    if args.out:
        with open(args.out, "w") as f:
            json.dump({"device": torch.cuda.get_device_name(), "results": results, "mismatches": bad}, f, indent=1)
    if bad:
        print("MISMATCHES:", bad)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
