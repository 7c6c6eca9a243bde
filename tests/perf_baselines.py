"""Side-by-side kernel timing on one B200: the new kernels, CUB BlockMergeSort
and the reference's own V6 kernel (compiled from its headers into
oracle/_ref/), on identical inputs.  Measurement infrastructure, not a test:

  python tests/perf_baselines.py [--out FILE.json] [--passes P]

Every configuration is timed the same way (cuda-sort_b200/devtime.py): in
place on several copies of the batch (together at least twice the 126 MB L2),
restored from a pristine copy before each pass and then evicted from L2, one
launch per copy back to back between two CUDA events; per-launch time = pass
time / copies, median of the passes.  For each family the best configuration
is reported: the reference's own sweep (bench.cu:497-521: Threads and the
Sorted / Shared / Async switches) for V6, every thread count for CUB, every
compiled tile in each launch form for the new kernels.  Outputs are checked
against numpy / the oracle.
"""
import argparse
import ctypes
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "cuda-sort_b200")]

import numpy as np  # noqa: E402
import torch  # noqa: E402

import b200sort as bs  # noqa: E402
import cpu_oracle as orc  # noqa: E402
import devtime  # noqa: E402
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
        self.sets = [torch.empty_like(self.src) for _ in range(devtime.sets_for(self.src.numel(), 20))]
        self.flush = devtime.Flusher()

    def restore(self):
        for s in self.sets:
            s.copy_(self.src)

    def time(self, launch, passes):
        """launch(ptr) sorts the batch at ptr in place; returns (us, spread, result of set 0)."""
        us, spread = devtime.batched_us([lambda p=s.data_ptr(): launch(p) for s in self.sets], self.flush, passes,
                                        before_pass=self.restore)
        if us is None:
            return None, None, None
        return us, spread, self.sets[0].cpu().numpy()


def run_case(dtype, n, arrays, dist, passes, results, flags=0):
    data = workloads.make_packed(dtype, n, arrays, dist, seed=99)
    npd = bs.NP_DTYPES[dtype]
    if dtype == bs.I32:
        want = np.sort(data.reshape(arrays, n), axis=1).reshape(-1)
    else:
        want = orc.sort_packed(dtype, data, n, arrays, orc.MODE_NETWORK, threads=os.cpu_count())
    timer = Timer(data)
    st = torch.cuda.current_stream().cuda_stream
    w = working(n)
    case = {"dtype": dtype, "n": n, "arrays": arrays, "distribution": dist, "keys": n * arrays,
            "hbm_bytes": 2 * n * arrays * bs.ELEM_BYTES[dtype], "configs": []}

    def record(family, cfg, timing):
        us, spread, res = timing
        ok = None
        if res is not None:
            got = res.view(npd)
            ok = bool(np.array_equal(got["key"] if dtype else got, want["key"] if dtype else want))
        case["configs"].append({"family": family, "config": cfg, "us": us, "spread": spread, "ok": ok})

    for base in bs.tiles(dtype):
        tw = 1 << sum(base.as_tuple())
        if tw < n or tw > 4 * w:
            continue
        info = bs.tile_info(dtype, n, 0, base)
        forms = [base, base.with_persistent()] + ([base.with_form(2)] if info.tma_form else []) + \
            ([base.with_form(3)] if info.xpose_form else [])
        for tile in forms:
            record("b200sort", repr(tile),
                   timer.time(lambda p, t=tile: bs.sort_packed_status(dtype, p, p, n, arrays, flags, t, st), passes))

    if os.path.exists(CUB_LIB) and not flags:
        cub = ctypes.CDLL(CUB_LIB)
        cub.cub_block_merge_sort.restype = ctypes.c_int
        cub.cub_block_merge_sort.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        for th in (32, 64, 128, 256, 512, 1024):
            if th > w or w // th > 32:
                continue
            t = timer.time(lambda p, th=th: cub.cub_block_merge_sort(dtype, p, n, arrays, w, th, st), passes)
            if t[0] is not None:
                record("cub_block_merge", "threads=%d items=%d" % (th, w // th), t)

    if orc.ref_gpu_available() and dtype in (bs.I32, bs.I32_I32):
        suffix = "int" if dtype == bs.I32 else "rec"
        fn = getattr(orc.ref_gpu(suffix), "ref_v6_" + suffix)
        # with B200S_SORTED_CHECK the reference runs its own Sorted switch
        combos = ((1, 0, 0),) if flags & bs.SORTED_CHECK else ((0, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1))
        for th in (32, 64, 128, 256, 512, 1024):
            if th > w or w // th > 16:
                continue
            for so, sh, asy in combos:
                t = timer.time(lambda p, th=th, so=so, sh=sh, asy=asy: fn(p, n, arrays, w, th, so, sh, asy, st),
                               passes)
                if t[0] is not None:
                    record("reference_v6", "threads=%d sorted=%d shared=%d async=%d" % (th, so, sh, asy), t)

    best = {}
    for c in case["configs"]:
        if c["us"] is None or not c["ok"]:
            continue
        if c["family"] not in best or c["us"] < best[c["family"]]["us"]:
            best[c["family"]] = c
    case["best"] = best
    results.append(case)
    line = "dtype=%d n=%d arrays=%d dist=%s flags=%d: " % (dtype, n, arrays, dist, flags) + ", ".join(
        "%s %.2f us (%s)" % (f, b["us"], b["config"]) for f, b in sorted(best.items()))
    print(line, flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--passes", type=int, default=5)
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--dist", default="uniform", help="key distribution (workloads.DISTRIBUTIONS)")
    ap.add_argument("--sorted-check", action="store_true",
                    help="B200S_SORTED_CHECK against the reference's Sorted=true (records, n = 1000 and 2048)")
    args = ap.parse_args()
    results = []
    if args.sorted_check:
        for n in (1000, 2048):
            run_case(bs.I32_I32, n, 4194304 // n, args.dist, args.passes, results, bs.SORTED_CHECK)
    else:
        run_case(bs.I32, 1024, 4096, args.dist, args.passes, results)
        if not args.quick:
            for n in (32, 129, 256, 1000, 2048, 4096):
                run_case(bs.I32_I32, n, 4194304 // n, args.dist, args.passes, results)
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
