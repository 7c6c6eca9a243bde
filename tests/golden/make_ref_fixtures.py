"""Record the reference's own GPU output as fixtures (tests/golden/ref_network.json).

Runs on a machine with a B200 and the reference kernels built into
oracle/_ref/ (oracle/Makefile `ref`).  Inputs: IntAndData records with many
equal keys (payload = global index) at lengths 1..2048; the output is what
the reference's V6 kernel (cusort_v6.hpp) returns for them, i.e. its exact
record order including ties.  The CPU test test_oracle_pins.py checks the
oracle's network restatement against this file on machines without a GPU.

Usage: python tests/golden/make_ref_fixtures.py OUT.json
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "cuda-sort_b200"), os.path.join(ROOT, "tests")]

import numpy as np  # noqa: E402
import torch  # noqa: E402

import b200sort as bs  # noqa: E402
import cpu_oracle as orc  # noqa: E402
import workloads  # noqa: E402


def main(out_path):
    lib = orc.ref_gpu("rec")
    cases = []
    for n in (1, 3, 16, 31, 32, 33, 64, 100, 129, 256, 500, 1000, 1024, 1500, 2048):
        for dist in ("distinct16", "equal", "swap8"):
            arrays = 2
            data = workloads.make_packed(bs.I32_I32, n, arrays, dist, seed=n * 31 + len(dist), extremes=True)
            w = 32
            while w < n:
                w *= 2
            d = torch.from_numpy(data.view(np.uint8).copy()).cuda()
            threads = max(32, w // 16)
            rc = lib.ref_v6_rec(d.data_ptr(), n, arrays, w, threads, 0, 0, 0,
                                torch.cuda.current_stream().cuda_stream)
            assert rc == 0
            torch.cuda.synchronize()
            got = d.cpu().numpy().view(bs.NP_DTYPES[bs.I32_I32])
            cases.append({"n": n, "arrays": arrays, "distribution": dist, "threads": threads,
                          "input": [[int(k), int(v)] for k, v in zip(data["key"], data["data"])],
                          "reference_v6_output": [[int(k), int(v)] for k, v in zip(got["key"], got["data"])]})
    with open(out_path, "w") as f:
        json.dump({"generator": "reference cusort_v6::Sort via oracle/_ref/libref_gpu_rec.so on a B200",
                   "cases": cases}, f, separators=(",", ":"))
    print("wrote", out_path, len(cases))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "ref_network.json"))
