"""The FP64 oracle against its committed outputs (tests/golden/oracle_small.npz,
written by tests/golden/make_golden.py): a change that moves the parity
reference's results -- a different transform, a changed rounding -- shows up
here before it silently shifts every GPU parity test."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))


def test_oracle_reproduces_its_golden_outputs():
    import make_golden
    want = np.load(os.path.join(HERE, "golden", "oracle_small.npz"))
    got = make_golden.cases()
    assert sorted(got) == sorted(want.files)
    for k in want.files:
        assert np.array_equal(got[k], want[k], equal_nan=True), k
    assert (want["strack_type"] > 0).mean() > 0.9 and (want["amp_type"] > 0).mean() > 0.9
    assert (want["strackw_type"] > 0).any()
