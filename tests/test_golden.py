"""The oracle restatement against golden outputs of the reference's own
sources (tests/golden/, made by tests/golden/make_golden.py): bit-for-bit.
Runs without the reference checkout."""
import glob
import json
import os

import numpy as np
import pytest

from oracle.oracle import restatement
from tests.golden.make_golden import run_case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(glob.glob(os.path.join(GOLDEN, "*.json")))


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(c)[:-5] for c in CASES])
def test_restatement_matches_reference_golden(path):
    case = json.load(open(path))
    want = np.load(path[:-5] + ".npz")
    got = run_case(restatement(), case)
    for name in want.files:
        assert np.array_equal(got[name], want[name], equal_nan=True), name


def test_golden_present():
    assert len(CASES) >= 5
