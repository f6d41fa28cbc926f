"""The smoothing schedule's host side: variants per axis, set/get round trip,
range checks, and the autotuner's persisted file (when present) naming a
valid variant for every axis and bucket."""
import json
import os

import pytest

import libapr_b200 as A
from libapr_b200 import _lib


def test_variants_and_round_trip():
    n = A.smoothing_variants()
    assert n == {"y": 3, "x": 5, "z": 5}
    old = A.smoothing_schedule()
    try:
        new = {a: [(i + k) % n[a] for i in range(len(A.SCHEDULE_BUCKETS))] for k, a in enumerate("yxz")}
        A.set_smoothing_schedule(new)
        assert A.smoothing_schedule() == new
    finally:
        A.set_smoothing_schedule(old)


@pytest.mark.parametrize("axis,bucket,variant", [(0, 0, 3), (1, 0, 5), (2, 6, 0), (3, 0, 0), (-1, 0, 0), (0, -1, 0)])
def test_out_of_range_is_rejected(axis, bucket, variant):
    assert _lib.lib().aprb_smoothing_schedule_set(axis, bucket, variant) == 1  # APRB_ERR_INVALID_ARGUMENT


@pytest.mark.skipif(not os.path.exists(_lib.SCHEDULE_FILE), reason="no autotuned schedule persisted")
def test_persisted_schedule_is_valid():
    with open(_lib.SCHEDULE_FILE) as f:
        doc = json.load(f)
    n = A.smoothing_variants()
    for a in "yxz":
        row = doc["schedule"][a]
        assert len(row) == len(A.SCHEDULE_BUCKETS)
        assert all(0 <= v < n[a] for v in row)
