"""Record the reference's own GPU output as a fixture (tests/golden/ref_network.json).

Runs on a machine with a B200 and the reference kernels built into
oracle/_ref/ (oracle/Makefile `ref`).  For every case of ref_inputs.cases()
it sorts the records with the reference's V6 kernel (cusort_v6.hpp:144-184,
compiled unmodified for sm_100a) and stores the SHA-256 of the output bytes
and, for short batches, the output payload order itself (the payload is the
input index, so it fixes the whole output).  test_oracle_pins.py checks the
oracle's network restatement against it on machines without a GPU.

Usage: python tests/golden/make_ref_fixtures.py [OUT.json]
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [HERE, os.path.join(ROOT, "oracle")]

import numpy as np  # noqa: E402
import torch  # noqa: E402

import cpu_oracle as orc  # noqa: E402
import ref_inputs  # noqa: E402

FULL_LIMIT = 1024   # store the payload order itself up to this many records


def main(out_path):
    fn = orc.ref_gpu("rec").ref_v6_rec
    rows = []
    for n, arrays, dist, seed, threads, sorted_ in ref_inputs.cases():
        data = ref_inputs.records(n, arrays, dist, seed)
        w = 32
        while w < n:
            w *= 2
        d = torch.from_numpy(data.view(np.uint8).copy()).cuda()
        rc = fn(d.data_ptr(), n, arrays, w, threads, sorted_, 0, 0, torch.cuda.current_stream().cuda_stream)
        if rc != 0:
            raise RuntimeError("reference V6 failed (%d) for n=%d threads=%d" % (rc, n, threads))
        torch.cuda.synchronize()
        got = d.cpu().numpy().view(ref_inputs.REC)
        row = {"n": n, "arrays": arrays, "distribution": dist, "seed": seed, "threads": threads,
               "sorted": sorted_, "sha256": hashlib.sha256(got.tobytes()).hexdigest()}
        if n * arrays <= FULL_LIMIT:
            row["payload"] = [int(x) for x in got["data"]]
        rows.append(row)
    with open(out_path, "w") as f:
        json.dump({"generator": "reference cusort_v6::Sort (oracle/_ref/libref_gpu_rec.so, sm_100a) on "
                                + torch.cuda.get_device_name(),
                   "inputs": "tests/golden/ref_inputs.py", "cases": rows}, f, separators=(",", ":"))
    print("wrote", out_path, len(rows), "cases")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_network.json"))
