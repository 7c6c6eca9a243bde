"""Autotuner for the tile table (tune/b200_table.csv, loaded by the library
at first use from beside libb200sort.so).

  python cuda-sort_b200/tune_b200.py [--out PATH] [--summary PATH] [--passes P]

For every element type, stable flag and working length W = 2^L it times each
compiled tile of that W (single-CTA and cluster tiles) in each launch form it
has (0 one slot per array, 1 persistent with register prefetch, 2 persistent
TMA pipeline, 3 transposed network) on a full-length batch of about 4 M
elements, checks the output, and keeps the fastest as the packed row.  For the ragged kernel it
times, per bucket L, a batch whose lengths all fall in that bucket in the
persistent kernel with the bucket's shape family A, with family B, and as a
launch of its own (the tabled tile of its working length, beside the
persistent kernel), and keeps the fastest as the ragged row.

Timing (devtime.batched_us): each pass evicts L2, then runs one launch on
each of several buffer sets (at least twice the L2 in total) back to back
between two CUDA events; the per-launch time is the median over the passes.
Every row records the best and the runner-up with the best's spread over the
passes; --summary writes that table as markdown.  Requires a GPU.
"""
import argparse
import datetime
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402
import torch  # noqa: E402

import b200sort as bs  # noqa: E402
import devtime  # noqa: E402
import workloads  # noqa: E402

TARGET_ELEMS = 1 << 22
FORM_NAMES = {0: "one-shot", 1: "prefetch", 2: "TMA", 3: "transposed"}
# ragged rows: 0 / 1 run the bucket in the persistent kernel with shape family
# A / B; 2 gives the bucket a launch of its own, in the tile and form the row
# names (the tuner searches them)
FAMILY_NAMES = {0: "persistent A", 1: "persistent B", 2: "own launch"}


def _keys(dtype, arr):
    return arr if dtype in (bs.I32, bs.U64) else arr["key"]


def tune_packed(dtype, flags, flush, passes, log, summary):
    rows = []
    tiles = [t for t in bs.tiles(dtype, flags) if t.cta_threads > 0]   # single-CTA and cluster tiles
    by_w = {}
    for t in tiles:
        by_w.setdefault(sum(t.as_tuple()), []).append(t)
    st = torch.cuda.current_stream().cuda_stream
    for L in sorted(by_w):
        n = 1 << L
        arrays = max(1, TARGET_ELEMS // n)
        data = workloads.make_packed(dtype, n, arrays, "uniform", seed=L)
        want = np.sort(_keys(dtype, data).reshape(arrays, n), axis=1).reshape(-1)
        sets = devtime.sets_for(data.nbytes, 8)
        src = torch.from_numpy(data.view(np.uint8).copy()).cuda()
        ins = [src.clone() for _ in range(sets)]
        outs = [torch.empty_like(src) for _ in range(sets)]
        cands = []
        for base in by_w[L]:
            info = bs.tile_info(dtype, n, flags, base)
            # cluster tiles (no arrays per CTA) have one launch besides form 3
            forms = ([0] if info.arrays_per_cta == 0 else [0, 1]) + ([2] if info.tma_form else []) + \
                ([3] if info.xpose_form else [])
            cands += [base.with_form(f) for f in forms]
        results = []
        for tile in cands:
            launches = [lambda i=i, t=tile: bs.sort_packed_status(dtype, ins[i].data_ptr(), outs[i].data_ptr(), n,
                                                                  arrays, flags, t, st) for i in range(sets)]
            us, spread = devtime.batched_us(launches, flush, passes)
            if us is None:
                continue
            ok = bool(np.array_equal(_keys(dtype, outs[0].cpu().numpy().view(bs.NP_DTYPES[dtype])), want))
            log("packed dtype=%d flags=%d W=%d %r: %.2f us (spread %.1f %%)%s"
                % (dtype, flags, n, tile, us, 100 * spread, "" if ok else " WRONG OUTPUT"))
            if ok:
                results.append((us, spread, tile))
        results.sort(key=lambda r: r[0])
        (us, spread, t) = results[0]
        second = results[1] if len(results) > 1 else None
        tail = (", runner-up %.2f us %s" % (second[0], _shape(second[2]))) if second else ""
        lc = (",%d" % t.log2_ctas) if t.log2_ctas else ""
        rows.append("%d,%d,%d,%d,%d,%d,%d%s  # %.2f us (spread %.1f %%)%s, %d arrays"
                    % (dtype, flags, L, t.log2_items, t.log2_lanes, t.log2_warps, t.persistent, lc, us, 100 * spread,
                       tail, arrays))
        summary.append(("packed", dtype, flags, n, arrays, _shape(t), us, spread,
                        _shape(second[2]) if second else "-", second[0] if second else None))
        del ins, outs, src
        torch.cuda.empty_cache()
    # the ragged rows are timed with these packed rows in force (a launch of
    # its own runs the tabled tile in its tabled form)
    with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as f:
        f.write("\n".join(r.split("#")[0] for r in rows) + "\n")
    bs.load_tile_table(f.name)
    os.unlink(f.name)
    return rows


def _shape(t):
    c = ".C%d" % (1 << t.log2_ctas) if t.log2_ctas else ""
    return "K%d.G%d.W%d%s/%s" % (1 << t.log2_items, 1 << t.log2_lanes, 1 << t.log2_warps, c, FORM_NAMES[t.persistent])


def tune_ragged(dtype, flags, flush, passes, log, summary):
    rows = []
    top = bs.ragged_max_length(dtype, flags)
    st = torch.cuda.current_stream().cuda_stream
    L = 3
    while (1 << L) <= top:
        lo, hi = (1 << (L - 1)) + 1 if L > 3 else 1, 1 << L
        arrays = max(16, TARGET_ELEMS // hi)
        rng = np.random.default_rng(L)
        lengths = rng.integers(lo, hi, size=arrays, endpoint=True)
        data, off = workloads.make_ragged(dtype, lengths, "uniform", seed=L)
        sets = devtime.sets_for(data.nbytes, 6)
        src = torch.from_numpy(data.view(np.uint8).copy()).cuda()
        ins = [src.clone() for _ in range(sets)]
        outs = [torch.empty_like(src) for _ in range(sets)]
        d_off = torch.from_numpy(off.astype(np.int32)).cuda()
        def time_row(row):
            with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as f:
                f.write(row + "\n")
            bs.load_tile_table(f.name)
            os.unlink(f.name)
            plans = [bs.Plan(dtype, arrays, flags) for _ in range(sets)]   # one captured graph per buffer set
            launches = [lambda i=i: plans[i].sort(ins[i].data_ptr(), outs[i].data_ptr(), d_off.data_ptr(), arrays, st)
                        for i in range(sets)]
            for fn in launches:
                fn()   # capture each plan's graph outside the timed passes
            r = devtime.batched_us(launches, flush, passes)
            for p in plans:
                p.close()
            return r

        # families 0 and 1: the persistent kernel; family 2: a launch of its
        # own, in each single-CTA tile of W and each of its id-list forms
        # (form 0, and form 3 where compiled; a cluster of one CTA has form 3
        # only); the row keeps the fastest tile
        cands = [("r,%d,%d,%d,%d" % (dtype, flags, L, fam), FAMILY_NAMES[fam]) for fam in (0, 1)]
        for base in bs.tiles(dtype, flags):
            if sum(base.as_tuple()) != L or base.log2_ctas != 0:
                continue
            info = bs.tile_info(dtype, 1 << L, flags, base)
            forms = ([] if info.arrays_per_cta == 0 else [0]) + ([3] if info.xpose_form else [])
            for form in forms:
                cands.append(("r,%d,%d,%d,2,%d,%d,%d,%d" % (dtype, flags, L, base.log2_items, base.log2_lanes,
                                                             base.log2_warps, form),
                              "own launch " + _shape(base.with_form(form))))
        res = []
        for row, name in cands:
            us, spread = time_row(row)
            if us is None:
                continue
            log("ragged dtype=%d flags=%d W=%d %s: %.2f us (spread %.1f %%)"
                % (dtype, flags, 1 << L, name, us, 100 * spread))
            res.append((us, spread, row, name))
        res.sort(key=lambda r: r[0])
        (us, spread, row, name), second = res[0], res[1]
        time_row(row)   # the class keeps its best row while the next ones are timed
        rows.append("%s  # %.2f us (spread %.1f %%) vs %.2f us (%s)" % (row, us, 100 * spread, second[0], second[3]))
        summary.append(("ragged", dtype, flags, 1 << L, arrays, name, us, spread, second[3], second[0]))
        del ins, outs, src
        torch.cuda.empty_cache()
        L += 1
    # leave the process's table as tuned
    with tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False) as f:
        f.write("\n".join(r.split("#")[0] for r in rows) + "\n")
    bs.load_tile_table(f.name)
    os.unlink(f.name)
    return rows


def write_summary(path, summary, argv):
    names = {bs.I32: "int32", bs.I32_I32: "int32+int32", bs.U64: "uint64", bs.U64_I32: "uint64+int32"}
    with open(path, "w") as f:
        f.write("# Tile table tuning on %s\n\n" % torch.cuda.get_device_name())
        f.write("Command: `python cuda-sort_b200/tune_b200.py %s`\n\n" % " ".join(argv))
        f.write("Per row: the fastest configuration and the runner-up, per-launch microseconds from batched CUDA "
                "events (devtime.batched_us: L2 evicted, one launch per buffer set, median of the passes), the best's "
                "spread over the passes, and the margin (runner-up / best - 1).\n\n")
        f.write("| path | dtype | stable | W | arrays | best | us | spread | runner-up | us | margin |\n")
        f.write("|---|---|---|---|---|---|---|---|---|---|---|\n")
        for kind, d, fl, w, arrays, best, us, spread, second, us2 in summary:
            margin = "%.1f %%" % (100 * (us2 / us - 1)) if us2 else "-"
            f.write("| %s | %s | %s | %d | %d | %s | %.2f | %.1f %% | %s | %s | %s |\n"
                    % (kind, names[d], "yes" if fl else "no", w, arrays, best, us, 100 * spread, second,
                       "%.2f" % us2 if us2 else "-", margin))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "tune", "b200_table.csv"))
    ap.add_argument("--summary", default=None, help="markdown table of best and runner-up per row")
    ap.add_argument("--passes", type=int, default=5)
    ap.add_argument("--only", default=None, help="comma-separated dtype codes to tune (default all)")
    args = ap.parse_args()
    flush = devtime.Flusher()
    lines, summary = [], []
    log = lambda s: print(s, flush=True)  # noqa: E731
    dtypes = [int(x) for x in args.only.split(",")] if args.only else [bs.I32, bs.I32_I32, bs.U64, bs.U64_I32]
    for dtype in dtypes:
        for flags in ((0,) if dtype in (bs.I32, bs.U64) else (0, bs.STABLE)):
            lines += tune_packed(dtype, flags, flush, args.passes, log, summary)
            lines += tune_ragged(dtype, flags, flush, args.passes, log, summary)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    with open(args.out, "w") as f:
        f.write("# b200sort tile table, written by cuda-sort_b200/tune_b200.py\n")
        f.write("# device: %s; %s; library: %s\n" % (torch.cuda.get_device_name(),
                                                     datetime.datetime.now(datetime.timezone.utc).strftime(
                                                         "%Y-%m-%d %H:%M UTC"), bs.version()))
        f.write("# packed rows: dtype,flags,log2_w,log2_items,log2_lanes,log2_warps,form (0 one-shot, 1 prefetch, 2 TMA, "
                "3 transposed)\n")
        f.write("# ragged rows: r,dtype,flags,log2_w,family[,log2_items,log2_lanes,log2_warps,form] (0: persistent, "
                "larger per-thread tile; 1: persistent, smaller; 2: a launch of its own, in the tile and form given)\n")
        for ln in lines:
            f.write(ln + "\n")
    if args.summary:
        write_summary(args.summary, summary, sys.argv[1:])
    print("wrote", args.out, len(lines), "rows")


if __name__ == "__main__":
    main()
