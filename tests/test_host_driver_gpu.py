"""The C++ host side (io::DataSet, tree::B200Index, the qcp_eval driver)
reads the reference's binary file formats and returns the same hit lists as
the oracle.  Needs a GPU."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR, assert_same_hits

pytestmark = pytest.mark.gpu


def read_hits(path):
    raw = open(path, "rb").read()
    q = int(np.frombuffer(raw[:8], np.uint64)[0])
    offs = np.frombuffer(raw[8:8 + 8 * (q + 1)], np.uint64)
    ids = np.frombuffer(raw[8 + 8 * (q + 1):], np.int32)
    return offs, ids


@pytest.mark.parametrize("index_type", ["b200", "b200-plain"])
def test_qcp_eval_matches_oracle(qcp, oracle, cases, tmp_path, index_type):
    exe = PKG_DIR / "qcp_eval"
    if not exe.exists():
        subprocess.run(["make", "-s", "-C", str(PKG_DIR)], check=True)
    objs, boxes, dims = cases.COUNT_CASES["g3"]()
    data = tmp_path / "data.bin"
    query = tmp_path / "query.bin"
    objs.astype(np.float32).tofile(data)
    # reference query file: two rows of D floats per query (lo row, hi row)
    boxes.astype(np.float32).tofile(query)
    out = tmp_path / "hits.bin"
    r = subprocess.run([str(exe), "-d", str(len(objs)), "-q", str(len(boxes)), "-D", str(data),
                        "-Q", str(query), "-k", "3", "-i", index_type, "-o", str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    want_offs, want_ids = oracle.ids(objs, dims, False, boxes)
    assert f"Hit : {int(want_offs[-1])}" in r.stdout
    offs, ids = read_hits(out)
    assert_same_hits(offs, ids, want_offs, want_ids)
