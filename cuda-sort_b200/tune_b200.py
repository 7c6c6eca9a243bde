"""Autotuner for the tile table (tune/b200_table.csv, loaded by the library
at first use from beside libb200sort.so).

  python cuda-sort_b200/tune_b200.py [--out PATH] [--reps R]

For every element type, stable flag and working length W = 2^L it times each
compiled single-CTA tile of that W in each launch form (one slot per array /
persistent with register prefetch / persistent TMA pipeline) on a full-length batch of about 4 M elements and
keeps the fastest as the packed row.  For the ragged kernel it times, per
bucket L, a batch whose lengths all fall in that bucket with the bucket's
shape family A and with family B, and keeps the faster as the ragged row.
Every launch starts from an L2 flushed by a 512 MB write; times are CUDA-event
medians.  Requires a GPU.
"""
import argparse
import datetime
import os
import statistics
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402
import torch  # noqa: E402

import b200sort as bs  # noqa: E402
import workloads  # noqa: E402

TARGET_ELEMS = 1 << 22


def timed(fn, flush, reps):
    st = torch.cuda.current_stream()
    times = []
    for r in range(reps + 1):
        flush.fill_(r & 0xFF)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        torch.cuda.synchronize()
        if r:
            times.append(e0.elapsed_time(e1) * 1e3)
    return statistics.median(times)


def tune_packed(dtype, flags, flush, reps, log):
    rows = []
    tiles = [t for t in bs.tiles(dtype, flags) if t.log2_ctas == 0 and t.cta_threads > 0]
    by_w = {}
    for t in tiles:
        by_w.setdefault(sum(t.as_tuple()), []).append(t)
    for L in sorted(by_w):
        n = 1 << L
        arrays = max(1, TARGET_ELEMS // n)
        data = workloads.make_packed(dtype, n, arrays, "uniform", seed=L)
        d_in = torch.from_numpy(data.view(np.uint8).copy()).cuda()
        d_out = torch.empty_like(d_in)
        st = torch.cuda.current_stream().cuda_stream
        best = None
        for base in by_w[L]:
            forms = [base, base.with_persistent()]
            if bs.tile_info(dtype, n, flags, base).tma_form:
                forms.append(base.with_form(2))   # TMA pipeline, where compiled for this tile
            for tile in forms:
                us = timed(lambda t=tile: bs.sort_packed(dtype, d_in.data_ptr(), d_out.data_ptr(), n, arrays, flags,
                                                         t, st), flush, reps)
                log("packed dtype=%d flags=%d W=%d %r: %.2f us" % (dtype, flags, n, tile, us))
                if best is None or us < best[0]:
                    best = (us, tile)
        t = best[1]
        rows.append("%d,%d,%d,%d,%d,%d,%d  # %.2f us, %d arrays" % (dtype, flags, L, t.log2_items, t.log2_lanes,
                                                                  t.log2_warps, t.persistent, best[0], arrays))
    return rows


def tune_ragged(dtype, flags, flush, reps, log):
    rows = []
    top = bs.ragged_max_length(dtype, flags)
    L = 3
    while (1 << L) <= top:
        lo, hi = (1 << (L - 1)) + 1 if L > 3 else 1, 1 << L
        arrays = max(16, TARGET_ELEMS // hi)
        rng = np.random.default_rng(L)
        lengths = rng.integers(lo, hi, size=arrays, endpoint=True)
        data, off = workloads.make_ragged(dtype, lengths, "uniform", seed=L)
        d_in = torch.from_numpy(data.view(np.uint8).copy()).cuda()
        d_out = torch.empty_like(d_in)
        d_off = torch.from_numpy(off.astype(np.int32)).cuda()
        st = torch.cuda.current_stream().cuda_stream
        res = {}
        for fam in (0, 1):
            with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as f:
                f.write("r,%d,%d,%d,%d\n" % (dtype, flags, L, fam))
            bs.load_tile_table(f.name)
            os.unlink(f.name)
            with bs.Plan(dtype, arrays, flags) as plan:
                res[fam] = timed(lambda p=plan: p.sort(d_in.data_ptr(), d_out.data_ptr(), d_off.data_ptr(), arrays, st),
                                 flush, reps)
            log("ragged dtype=%d flags=%d W=%d family=%d: %.2f us" % (dtype, flags, 1 << L, fam, res[fam]))
        fam = min(res, key=res.get)
        rows.append("r,%d,%d,%d,%d  # %.2f us vs %.2f us" % (dtype, flags, L, fam, res[fam], res[1 - fam]))
        L += 1
    # leave the process's table as tuned
    with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as f:
        f.write("\n".join(r.split("#")[0] for r in rows) + "\n")
    bs.load_tile_table(f.name)
    os.unlink(f.name)
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "tune", "b200_table.csv"))
    ap.add_argument("--reps", type=int, default=7)
    args = ap.parse_args()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    lines = []
    log = lambda s: print(s, flush=True)  # noqa: E731
    for dtype in (bs.I32, bs.I32_I32, bs.U64, bs.U64_I32):
        for flags in ((0,) if dtype in (bs.I32, bs.U64) else (0, bs.STABLE)):
            lines += tune_packed(dtype, flags, flush, args.reps, log)
            lines += tune_ragged(dtype, flags, flush, args.reps, log)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    with open(args.out, "w") as f:
        f.write("# b200sort tile table, written by cuda-sort_b200/tune_b200.py\n")
        f.write("# device: %s; %s; library: %s\n" % (torch.cuda.get_device_name(),
                                                     datetime.datetime.now(datetime.timezone.utc).strftime(
                                                         "%Y-%m-%d %H:%M UTC"), bs.version()))
        f.write("# packed rows: dtype,flags,log2_w,log2_items,log2_lanes,log2_warps,form (0 one-shot, 1 prefetch, 2 TMA)\n")
        f.write("# ragged rows: r,dtype,flags,log2_w,family (0: larger per-thread tile, 1: smaller)\n")
        for ln in lines:
            f.write(ln + "\n")
    print("wrote", args.out, len(lines), "rows")


if __name__ == "__main__":
    main()
