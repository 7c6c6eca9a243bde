"""b200sort_bench: the reference's bench command line (bench.cu:66-136) and CSV
schema (bench.cu:249-252) over b200sort.  Option handling is checked on the
host; --check-only sweeps and timed CSV runs on the GPU."""
import csv
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "cuda-sort_b200", "b200sort_bench")

# the reference's columns, in its order (bench.cu:249-252)
REFERENCE_COLUMNS = ("method,distribution,N,arrays,total_values,working_values,threads,items_per_thread,"
                     "testsorted,fullsm,asynccpy,shared_bytes,trial,E_s,X_s,E_wall_s,wall_X_s,time_per_array_s,"
                     "time_per_value_s,validated,cuda_runtime,thrust_version,cub_version,registers_per_thread,"
                     "active_blocks_per_sm,local_bytes_per_thread").split(",")


def run(*args, timeout=600):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=timeout)


@pytest.mark.parametrize("args,message", [
    (["--methods", "bogus"], "Unknown --methods entry: bogus"),
    (["--methods", "b200_bitonic,"], "Empty name in --methods"),
    (["--mode", "huge"], "Invalid --mode"),
    (["--type", "float"], "Invalid --type"),
    (["--max-threads", "48"], "--max-threads must be a multiple of 32 in [32,1024]"),
    (["--min-size", "10", "--max-size", "5"], "--min-size exceeds --max-size"),
    (["--arrays", "0"], "Invalid positive integer for --arrays"),
    (["--arrays"], "Missing value for --arrays"),
    (["--frobnicate", "3"], "Unknown option: --frobnicate"),
])
def test_option_errors_match_the_reference(args, message):
    r = run(*args)
    assert r.returncode == 1
    assert message in r.stderr


def test_help_lists_the_reference_options():
    r = run("--help")
    assert r.returncode == 0
    for opt in ("--mode", "--type", "--min-size", "--max-size", "--max-threads", "--arrays", "--batch-elements",
                "--repetitions", "--output", "--methods", "--check-only"):
        assert opt in r.stdout


@pytest.mark.gpu
def test_check_only_passes_every_configuration(tmp_path):
    prefix = str(tmp_path / "chk")
    r = run("--check-only", "--max-size", "40", "--output", prefix, timeout=900)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("PASS ")]
    methods = {ln.split()[1] for ln in lines}
    assert {"b200_bitonic", "b200_tiles", "b200_ragged", "cub_block_merge", "thrust_segment_loop"} <= methods
    assert any(" EXTREMES" in ln for ln in lines)
    for t in ("int", "record"):
        with open(prefix + "_%s_small.csv" % t) as f:
            header = f.readline().strip().split(",")
        assert header[:len(REFERENCE_COLUMNS)] == REFERENCE_COLUMNS


@pytest.mark.gpu
def test_timed_csv_rows(tmp_path):
    prefix = str(tmp_path / "t")
    r = run("--type", "record", "--min-size", "1000", "--max-size", "1024", "--repetitions", "2",
            "--methods", "b200_bitonic,bitonic_v6_register,cub_block_merge", "--output", prefix)
    assert r.returncode == 0, r.stderr
    with open(prefix + "_record_small.csv") as f:
        rows = list(csv.DictReader(f))
    assert rows
    assert {row["method"] for row in rows} == {"b200_bitonic", "bitonic_v6_register", "cub_block_merge"}
    for row in rows:
        assert row["validated"] == "1"
        assert float(row["E_s"]) > 0 and float(row["keys_per_s"]) > 0
        assert int(row["N"]) in (1000, 1023, 1024)
    b200 = [row for row in rows if row["method"] == "b200_bitonic"]
    assert all(int(row["registers_per_thread"]) > 0 and row["tile"] for row in b200)


@pytest.mark.gpu
def test_large_mode_single_arrays(tmp_path):
    prefix = str(tmp_path / "l")
    r = run("--mode", "large", "--type", "record", "--max-size", "16384", "--check-only", "--methods",
            "large_merge,large_hybrid", "--output", prefix)
    assert r.returncode == 0, r.stderr
    passes = [ln for ln in r.stdout.splitlines() if ln.startswith("PASS ")]
    assert any("N=16384" in ln and "large_merge" in ln for ln in passes)
    assert any("large_hybrid" in ln for ln in passes)
