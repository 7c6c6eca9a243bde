"""The C++ wrappers (include/b200sort.hpp) compile against the reference's
names and forward argument errors as status codes, without a GPU."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "cuda-sort_b200")

SRC = r'''
#include <cstdio>
#include "b200sort.hpp"
struct IntAndDataLike { int val; int data; };
int main() {
    int bad = 0;
    // n beyond the working length: the reference asserts on the device, here a status
    bad += b200sort::Sort_1Block_v6_register<int, 1024, 128, false, false, false>(nullptr, nullptr, 1025)
           != B200S_ERR_INVALID_ARGUMENT;
    bad += b200sort::Sort_1Warp_SM_le32<IntAndDataLike, true, false>(nullptr, nullptr, 33)
           != B200S_ERR_INVALID_ARGUMENT;
    bad += b200sort::Sort_1Block_v4_xor<int, false, true, false>(nullptr, nullptr, 10, 48)
           != B200S_ERR_INVALID_ARGUMENT;
    // an empty batch is a no-op that touches no device
    bad += b200sort::Sort_1Block_v6_register<IntAndDataLike, 2048, 256, true, true, true>(nullptr, nullptr, 100, 0)
           != B200S_OK;
    // the partition leaf under the reference kernel's name: no partitions, nothing to do;
    // a negative count is an argument error
    bad += b200sort::SortPartitionsAdaptive_outofplace<IntAndDataLike>(nullptr, nullptr, nullptr, nullptr, 0)
           != B200S_OK;
    bad += b200sort::SortPartitionsAdaptive_outofplace<int, true, true>(nullptr, nullptr, nullptr, nullptr, -1)
           != B200S_ERR_INVALID_ARGUMENT;
    bad += b200sort::dtype_of<IntAndDataLike>::value != B200S_I32_I32;
    bad += b200sort::dtype_of<unsigned long>::value != B200S_U64;
    std::printf("%d\n", bad);
    return bad;
}
'''


def test_cpp_wrappers_compile_and_check_arguments(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(SRC)
    exe = tmp_path / "t"
    cmd = ["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
           "-L", LIBDIR, "-lb200sort", "-Wl,-rpath," + LIBDIR]
    subprocess.run(cmd, check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
