"""The oracle's network restatement against the reference's own output (CPU).

tests/golden/ref_network.json holds what the reference's V6 kernel
(cusort_v6.hpp:144-184, compiled unmodified for sm_100a and run on a B200 by
tests/golden/make_ref_fixtures.py) returned for tie-heavy IntAndData batches
(inputs: tests/golden/ref_inputs.py), including its Sorted early-exit
variant.  The oracle's MODE_NETWORK must give the same records in the same
order, bit for bit, so the oracle is pinned to the reference on machines
without a GPU too.
"""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

import cpu_oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import ref_inputs  # noqa: E402

FIXTURE = os.path.join(HERE, "golden", "ref_network.json")
I32_I32 = 1


def _cases():
    with open(FIXTURE) as f:
        return json.load(f)["cases"]


def test_fixture_covers_every_generated_case():
    rows = _cases()
    keys = {(r["n"], r["arrays"], r["distribution"], r["seed"], r["threads"], r["sorted"]) for r in rows}
    assert keys == set(ref_inputs.cases())
    assert any(r["sorted"] for r in rows) and any("payload" in r for r in rows)


@pytest.mark.parametrize("row", _cases(), ids=lambda r: "n%d-%s-t%d-s%d" % (r["n"], r["distribution"],
                                                                             r["threads"], r["sorted"]))
def test_oracle_network_equals_reference_output(row):
    data = ref_inputs.records(row["n"], row["arrays"], row["distribution"], row["seed"])
    got = orc.sort_packed(I32_I32, data, row["n"], row["arrays"], orc.MODE_NETWORK)
    if "payload" in row:
        assert [int(x) for x in got["data"]] == row["payload"]
        assert np.array_equal(got["key"], data["key"][np.asarray(row["payload"])])
    assert hashlib.sha256(got.view(ref_inputs.REC).tobytes()).hexdigest() == row["sha256"]
