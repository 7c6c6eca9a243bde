"""CPU checks of the C ABI: the library loads, exports every declared entry
point, and rejects bad arguments before touching a GPU."""
import ctypes
import os
import re

import pytest

import b200sort as bs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


def _declared():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(b200s_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    names = _declared()
    assert "b200s_sort_packed" in names and len(names) >= 10
    handle = ctypes.CDLL(bs.LIB_PATH)
    missing = [n for n in names if not hasattr(handle, n)]
    assert not missing, missing


def test_version_and_status_strings():
    assert "sm_100a" in bs.version()
    # every value of b200s_status has its own string
    strings = [bs.lib().b200s_status_string(s) for s in range(9)]
    assert all(strings) and b"unknown status" not in strings
    assert len(set(strings)) == 9
    assert bs.lib().b200s_status_string(99) == b"unknown status"


@pytest.mark.parametrize("args,status", [
    ((9, 16, 16, 10, 1, 0), bs.STATUS_NAMES and 1),     # unknown dtype
    ((bs.I32, 16, 16, -1, 1, 0), 1),                     # negative n
    ((bs.I32, 16, 16, 10, -1, 0), 1),                    # negative arrays
    ((bs.I32, 16, 16, 10, 1, 0x80), 1),                  # unknown flag
    ((bs.I32, 0, 16, 10, 1, 0), 1),                      # null input
    ((bs.I32, 16, 0, 10, 1, 0), 1),                      # null output
    ((bs.I32, 16, 16, 1 << 30, 1, 0), 2),                # longer than any tile
    ((bs.I32, 0, 0, 0, 5, 0), 0),                        # empty arrays: nothing to do
    ((bs.I32, 0, 0, 7, 0, 0), 0),                        # no arrays: nothing to do
])
def test_argument_checks_need_no_gpu(args, status):
    dtype, pin, pout, n, arrays, flags = args
    assert bs.sort_packed_status(dtype, pin, pout, n, arrays, flags) == status


def test_explicit_tile_must_cover_n():
    t = bs.default_tile(bs.I32, 100)
    assert (1 << sum(t.as_tuple())) >= 100
    short = bs.Tile(3, 0, 0, 0, 0, 0)
    assert bs.sort_packed_status(bs.I32, 16, 16, 100, 1, 0, short) == 2
    bogus = bs.Tile(9, 9, 9, 0, 0, 0)
    assert bs.sort_packed_status(bs.I32, 16, 16, 10, 1, 0, bogus) == 2


def test_tile_registry_covers_every_length_up_to_the_maximum():
    for dtype in (bs.I32, bs.I32_I32, bs.U64, bs.U64_I32):
        for flags in (0, bs.STABLE):
            top = bs.max_length(dtype, flags)
            assert top >= 4096
            assert len(bs.tiles(dtype, flags)) >= 8
            for n in [1, 2, 3, 31, 32, 33, 1000, 1024, 1025, top // 2 + 1, top]:
                t = bs.default_tile(dtype, n, flags)
                w = 1 << sum(t.as_tuple())
                assert w >= n and t.cta_threads % 32 == 0


def test_tile_table_file_round_trip(tmp_path):
    t = bs.tiles(bs.I32)[0]
    p = tmp_path / "table.csv"
    p.write_text("# dtype,flags,log2_w,log2_items,log2_lanes,log2_warps\n0,0,%d,%d,%d,%d\n"
                 % (sum(t.as_tuple()), t.log2_items, t.log2_lanes, t.log2_warps))
    assert bs.load_tile_table(str(p)) == 1
    bad = tmp_path / "bad.csv"
    bad.write_text("0,0,3,9,9,9\n")
    with pytest.raises(bs.B200SortError):
        bs.load_tile_table(str(bad))


def _shipped_table():
    return os.path.join(os.path.dirname(bs.LIB_PATH), "tune", "b200_table.csv")


def test_tile_table_rows_name_cluster_tiles_and_forms(tmp_path):
    # a packed row may give a cluster tile (8th column: log2 CTAs per array)
    # and launch form 3; the default choice for that length then reports both
    try:
        for dtype in (bs.I32_I32, bs.U64_I32):
            clusters = [t for t in bs.tiles(dtype) if t.log2_ctas > 0]
            assert clusters, dtype
            t = clusters[0]
            w = sum(t.as_tuple())
            p = tmp_path / ("cluster%d.csv" % dtype)
            p.write_text("%d,0,%d,%d,%d,%d,3,%d\n" % (dtype, w, t.log2_items, t.log2_lanes, t.log2_warps,
                                                      t.log2_ctas))
            assert bs.load_tile_table(str(p)) == 1
            d = bs.default_tile(dtype, 1 << w)
            assert (d.as_tuple(), d.persistent) == (t.as_tuple(), 3)
        # a CTA count no tile of that shape has is rejected
        t = [t for t in bs.tiles(bs.I32_I32) if t.log2_ctas > 0][0]
        bad = tmp_path / "bad_ctas.csv"
        bad.write_text("1,0,%d,%d,%d,%d,3,7\n" % (sum(t.as_tuple()), t.log2_items, t.log2_lanes, t.log2_warps))
        with pytest.raises(bs.B200SortError):
            bs.load_tile_table(str(bad))
        # without the column a row names a single-CTA tile (log2 CTAs 0)
        one = [t for t in bs.tiles(bs.I32_I32) if t.log2_ctas == 0 and t.log2_warps > 0][0]
        p = tmp_path / "one.csv"
        p.write_text("1,0,%d,%d,%d,%d,3\n" % (sum(one.as_tuple()), one.log2_items, one.log2_lanes, one.log2_warps))
        assert bs.load_tile_table(str(p)) == 1
        d = bs.default_tile(bs.I32_I32, 1 << sum(one.as_tuple()))
        assert (d.as_tuple(), d.persistent) == (one.as_tuple(), 3)
    finally:
        bs.load_tile_table(_shipped_table())


def test_hinted_ragged_sort_checks_its_plan():
    # a null plan is an argument error, reported before any GPU work
    fn = bs.declare("b200s_sort_ragged_hinted", ctypes.c_int,
                    [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                     ctypes.c_int64, ctypes.c_void_p])
    assert fn(None, None, None, None, None, 1, None) == 1


def test_ragged_rows_name_the_tile_of_a_launch_of_its_own(tmp_path):
    # r,dtype,flags,log2_w,2,log2_items,log2_lanes,log2_warps,form: a
    # single-CTA tile of W in form 0 or 3; anything else is rejected
    tiles = [t for t in bs.tiles(bs.I32_I32) if t.log2_ctas == 0 and sum(t.as_tuple()) == 10]
    assert len(tiles) >= 2
    try:
        good = tmp_path / "own.csv"
        good.write_text("".join("r,1,0,10,2,%d,%d,%d,%d\n" % (t.log2_items, t.log2_lanes, t.log2_warps, f)
                                for t in tiles for f in (0, 3)))
        assert bs.load_tile_table(str(good)) == 2 * len(tiles)
        t = tiles[0]
        for line in ("r,1,0,10,1,%d,%d,%d,0\n" % (t.log2_items, t.log2_lanes, t.log2_warps),   # not family 2
                     "r,1,0,10,2,%d,%d,%d,2\n" % (t.log2_items, t.log2_lanes, t.log2_warps),   # form 2
                     "r,1,0,11,2,%d,%d,%d,0\n" % (t.log2_items, t.log2_lanes, t.log2_warps),   # tile of another W
                     "r,1,0,10,2,9,9,9,0\n",                                                     # no such tile
                     "r,1,0,10,2,%d,%d\n" % (t.log2_items, t.log2_lanes)):                      # incomplete
            bad = tmp_path / "bad_own.csv"
            bad.write_text(line)
            with pytest.raises(bs.B200SortError):
                bs.load_tile_table(str(bad))
    finally:
        bs.load_tile_table(_shipped_table())
