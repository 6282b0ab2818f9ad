"""The learned scheduler's decision step (tc_sched_from_costs, host only; tc_sched_learned runs
it on the network's outputs): per degree cell, the fixed rule's strategy unless the predicted cost
of another is at least 5 % lower. Static count: table entry = network output (0 warp, 1 lane,
2 packed), rule lane for b <= lane_max_deg, packed for b <= packed_max_deg, else warp. Streaming
delta: table entries 0 (search) and 1 (merge) read outputs 1 and 2."""
import ctypes
import math

import numpy as np
import pytest

from custingeralg_b200 import native as N

OUT = N.MLP_OUT


def decide(kind, costs, sched=None, feat=None):
    s = sched or N.default_sched()
    c = np.ascontiguousarray(costs, dtype=np.float32).reshape(256, OUT)
    f = None if feat is None else np.ascontiguousarray(feat, dtype=np.float32)
    st = N.lib().tc_sched_from_costs(kind, f.ctypes.data if f is not None else None, c.ctypes.data, ctypes.byref(s))
    assert st == N.TC_OK
    assert s.use_table == 1
    return np.array([[s.table[i][j] for j in range(16)] for i in range(16)])


def nominal_b(j):
    return round(1.5 * 2 ** j)   # the cells' nominal degrees when no features are given


def rule(bi, lane_max=8, packed_max=32):
    return 1 if bi <= lane_max else 2 if bi <= packed_max else 0


def test_equal_costs_keep_the_fixed_rule():
    t = decide(0, np.zeros((256, OUT)))
    for i in range(16):
        for j in range(16):
            assert t[i, j] == rule(nominal_b(j)), (i, j)
    d = N.default_sched()
    assert (d.lane_max_deg, d.packed_max_deg) == (8, 32)


@pytest.mark.parametrize("cheaper,switch", [(0.04, False), (0.06, True), (0.5, True)])
def test_margin(cheaper, switch):
    costs = np.zeros((256, OUT))
    # every cell: the strategy after the rule's one (mod 3) is `cheaper` cheaper
    want = np.zeros((16, 16), dtype=int)
    for c in range(256):
        r = rule(nominal_b(c % 16))
        other = (r + 1) % 3
        costs[c, other] = math.log2(1.0 - cheaper)
        want[c // 16, c % 16] = other if switch else r
    assert np.array_equal(decide(0, costs), want)


def test_packed_threshold_and_no_packed_rule():
    s = N.default_sched()
    s.packed_max_deg = 0
    t = decide(0, np.zeros((256, OUT)), sched=s)
    assert set(np.unique(t[:, 5:])) == {0} and set(np.unique(t[:, :3])) == {1}
    s = N.default_sched()
    s.lane_max_deg, s.packed_max_deg = 0, 1 << 20
    assert set(np.unique(decide(0, np.zeros((256, OUT)), sched=s))) == {2}


def test_streaming_reads_outputs_one_and_two():
    costs = np.zeros((256, OUT))
    costs[:, 0] = -100.0           # output 0 is no streaming strategy: never picked
    t = decide(1, costs)
    assert set(np.unique(t)) <= {0, 1}
    costs[:, 2] = -1.0             # merge (entry 1) far cheaper everywhere
    assert set(np.unique(decide(1, costs))) == {1}
    costs[:, 2] = 0.0
    costs[:, 1] = -1.0             # search (entry 0) far cheaper everywhere
    assert set(np.unique(decide(1, costs))) == {0}


def test_features_drive_the_rule():
    """With explicit cell features the rule reads the mean degrees from them."""
    feat = np.zeros((256, 4), dtype=np.float32)
    feat[:, 0] = math.log2(1 + 100)   # a = 100 everywhere
    feat[:, 1] = math.log2(1 + 20)    # b = 20 everywhere: packed by the rule
    feat[:, 2] = 0.2
    feat[:, 3] = np.arange(256) / 255.0
    assert set(np.unique(decide(0, np.zeros((256, OUT)), feat=feat))) == {2}


def test_invalid_arguments():
    s = N.default_sched()
    c = np.zeros((256, OUT), dtype=np.float32)
    assert N.lib().tc_sched_from_costs(2, None, c.ctypes.data, ctypes.byref(s)) == N.TC_ERR_INVALID_ARG
    assert N.lib().tc_sched_from_costs(0, None, None, ctypes.byref(s)) == N.TC_ERR_INVALID_ARG
