"""Build recipe for the b200sort CUDA library (sm_100a only).

Compiles every translation unit under csrc/ to an object with nvcc, in
parallel, and links them into libb200sort.so beside this file.  Objects are
rebuilt only when a source or header is newer than the object.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libb200sort.so")
BASELINES = os.path.join(HERE, "baselines")
CUB_LIB = os.path.join(HERE, "libb200sort_cub.so")
HARNESS = os.path.join(HERE, "harness")
LOADGEN_LIB = os.path.join(HERE, "libb200sort_loadgen.so")
BENCH_CLI = os.path.join(HERE, "b200sort_bench")
ONCHIP_LIB = os.path.join(HERE, "libb200sort_onchip.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps_mtime(obj, path):
    """Newest modification time among the source and the headers it included
    at its last compile (nvcc -MD writes them to obj.d); every header when the
    dependency file is missing."""
    newest = os.path.getmtime(path)
    dep = obj[:-2] + ".d"
    if os.path.exists(dep):
        with open(dep) as f:
            text = f.read().replace("\\\n", " ")
        for tok in text.split(":", 1)[-1].split():
            if os.path.exists(tok):
                newest = max(newest, os.path.getmtime(tok))
        return newest
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cuh", ".h", ".hpp")):
                newest = max(newest, os.path.getmtime(os.path.join(d, f)))
    return newest


def _compile(src, extra):
    obj = os.path.join(OBJ, src[:-3] + ".o")
    path = os.path.join(CSRC, src)
    if os.path.exists(obj) and os.path.getmtime(obj) >= _deps_mtime(obj, path):
        return obj, None
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-MD", "-MF", obj[:-2] + ".d", "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "$ " + " ".join(cmd) + "\n" + r.stdout + r.stderr
    return obj, None


def build(verbose=False, extra=None, jobs=None):
    """Compile csrc/*.cu for sm_100a and link libb200sort.so; return its path."""
    os.makedirs(OBJ, exist_ok=True)
    extra = list(extra or [])
    jobs = jobs or max(1, min(len(_sources()), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, extra), _sources()))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    objs = [o for o, _ in results]
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    build_cub_baseline()
    build_loadgen()
    build_bench_cli()
    build_onchip()
    if verbose:
        print("built", LIB, CUB_LIB, LOADGEN_LIB, BENCH_CLI)
    return LIB


def build_cub_baseline():
    """The CUB BlockMergeSort baseline library (timed beside the product, never linked into it)."""
    src = os.path.join(BASELINES, "cub_block_merge.cu")
    if os.path.exists(CUB_LIB) and os.path.getmtime(CUB_LIB) >= os.path.getmtime(src):
        return CUB_LIB
    cmd = [NVCC] + ARCH + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", src, "-o", CUB_LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("CUB baseline build failed:\n" + r.stdout + r.stderr)
    return CUB_LIB


def build_loadgen():
    """The serving load generator (benchmark harness over the library's C ABI)."""
    src = os.path.join(HARNESS, "loadgen.cpp")
    if os.path.exists(LOADGEN_LIB) and os.path.getmtime(LOADGEN_LIB) >= max(
            os.path.getmtime(src), os.path.getmtime(LIB), os.path.getmtime(os.path.join(ROOT, "include", "b200sort.h"))):
        return LOADGEN_LIB
    cmd = [NVCC, "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-I" + os.path.join(ROOT, "include"),
           "-x", "cu", src, "-o", LOADGEN_LIB, "-L" + HERE, "-lb200sort", "-Xlinker", "-rpath,$ORIGIN"] + ARCH
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("load generator build failed:\n" + r.stdout + r.stderr)
    return LOADGEN_LIB


def build_onchip():
    """Shared-memory and distributed-shared-memory bandwidth probes (the on-chip roofline's peaks)."""
    src = os.path.join(HARNESS, "onchip_peak.cu")
    if os.path.exists(ONCHIP_LIB) and os.path.getmtime(ONCHIP_LIB) >= os.path.getmtime(src):
        return ONCHIP_LIB
    cmd = [NVCC] + ARCH + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", src, "-o", ONCHIP_LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("on-chip probe build failed:\n" + r.stdout + r.stderr)
    return ONCHIP_LIB


def build_bench_cli():
    """b200sort_bench: the reference's bench command line and CSV over the library and the baselines."""
    src = os.path.join(HARNESS, "bench_cli.cu")
    deps = [src, LIB, CUB_LIB, os.path.join(ROOT, "include", "b200sort.h")]
    if os.path.exists(BENCH_CLI) and os.path.getmtime(BENCH_CLI) >= max(os.path.getmtime(d) for d in deps):
        return BENCH_CLI
    cmd = [NVCC] + ARCH + ["-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), src, "-o", BENCH_CLI,
                           "-L" + HERE, "-lb200sort", "-l:libb200sort_cub.so", "-Xlinker", "-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("bench CLI build failed:\n" + r.stdout + r.stderr)
    return BENCH_CLI


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
