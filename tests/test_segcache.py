"""Segment cache bookkeeping (host-pool mode: no GPU needed): admission, the three
eviction policies, pinning by the running query, epoch replacement by weights."""
import numpy as np
import pytest

from mordred_b200 import _lib as L
from mordred_b200.segcache import SegmentCache

SEG = 1024


def _cols(ncol, nseg, seed=0):
    rng = np.random.default_rng(seed)
    return [rng.integers(-2**31, 2**31 - 1, nseg * SEG, dtype=np.int64).astype(np.int32) for _ in range(ncol)]


def test_admission_copies_and_maps():
    cols = _cols(2, 5)
    c = SegmentCache(4, SEG, 2, 5, "lru", device=-1)
    c.begin_query()
    s = c.admit(1, 3, cols[1][3 * SEG:].ctypes.data, SEG)
    assert c.slot(1, 3) == s and c.slot(0, 3) == -1
    assert np.array_equal(c.host_slot_view(s), cols[1][3 * SEG: 4 * SEG])
    assert c.admit(1, 3, cols[1][3 * SEG:].ctypes.data, SEG) == s  # already resident: no copy
    idx = c.col_idx(1)
    assert idx[3] == s and (np.delete(idx, 3) == -1).all()
    st = c.stats()
    assert st["admissions"] == 1 and st["resident"] == 1 and st["bytes_h2d"] == SEG * 4


@pytest.mark.parametrize("policy", ["lru", "lfu", "weight"])
def test_eviction_policies(policy):
    cols = _cols(1, 6)
    c = SegmentCache(3, SEG, 1, 6, policy, device=-1)
    # three segments resident, used with different recency / frequency / weight
    for seg, uses, w in [(0, 5, 3.0), (1, 1, 1.0), (2, 3, 2.0)]:
        c.begin_query()
        c.admit(0, seg, cols[0][seg * SEG:].ctypes.data, SEG)
        for _ in range(uses - 1):
            c.touch(0, seg)
        c.set_weight(0, seg, w)
    c.begin_query()
    c.touch(0, 1)  # segment 1 is now the most recent; it is also the least used and lightest
    c.begin_query()
    c.admit(0, 5, cols[0][5 * SEG:].ctypes.data, SEG)
    evicted = [s for s in range(3) if c.slot(0, s) == -1]
    assert evicted == {"lru": [0], "lfu": [1], "weight": [1]}[policy]
    assert c.stats()["evictions"] == 1


def test_running_query_segments_are_pinned():
    cols = _cols(1, 4)
    c = SegmentCache(2, SEG, 1, 4, "lru", device=-1)
    c.begin_query()
    c.admit(0, 0, cols[0].ctypes.data, SEG)
    c.admit(0, 1, cols[0][SEG:].ctypes.data, SEG)
    with pytest.raises(L.MbError) as e:
        c.admit(0, 2, cols[0][2 * SEG:].ctypes.data, SEG)
    assert e.value.code == 6
    c.begin_query()
    c.touch(0, 1)  # pin 1 in the new query: 0 is the only victim
    c.admit(0, 2, cols[0][2 * SEG:].ctypes.data, SEG)
    assert c.slot(0, 0) == -1 and c.slot(0, 1) >= 0 and c.slot(0, 2) >= 0


def test_epoch_replacement_keeps_heaviest():
    cols = _cols(3, 4, seed=1)
    c = SegmentCache(5, SEG, 3, 4, "weight", device=-1)
    c.begin_query()
    c.admit(2, 3, cols[2][3 * SEG:].ctypes.data, SEG)  # weight 0 below: evicted
    w = np.zeros((3, 4))
    w[0, 0], w[0, 1], w[1, 2], w[2, 0], w[2, 1], w[1, 1] = 9, 8, 7, 6, 5, 4
    rows = np.full(4, SEG, np.int32)
    c.replace(w, [x.ctypes.data for x in cols], rows)
    resident = {(col, seg) for col in range(3) for seg in range(4) if c.slot(col, seg) >= 0}
    assert resident == {(0, 0), (0, 1), (1, 2), (2, 0), (2, 1)}
    for col, seg in resident:
        assert np.array_equal(c.host_slot_view(c.slot(col, seg)), cols[col][seg * SEG:(seg + 1) * SEG])


def test_bad_arguments():
    with pytest.raises(L.MbError):
        SegmentCache(4, 1000, 1, 4, device=-1)  # segment size not a power of two
    c = SegmentCache(1, SEG, 1, 2, device=-1)
    with pytest.raises(L.MbError):
        c.touch(1, 0)


def test_admit_segments_in_order_until_full():
    cols = _cols(3, 6)
    c = SegmentCache(7, SEG, 3, 6, "lru", device=-1)
    rows = np.full(6, SEG, np.int32)
    c.begin_query()
    done, copied = c.admit_segments([0, 2], [4, 1, 5, 0], [x.ctypes.data for x in cols], rows)
    assert done == 3 and copied == 7  # the fourth segment gets one column in; the second does not fit
    for seg in (4, 1, 5):
        for col in (0, 2):
            assert np.array_equal(c.host_slot_view(c.slot(col, seg)), cols[col][seg * SEG:(seg + 1) * SEG])
    c.begin_query()
    done, copied = c.admit_segments([0, 2], [5, 0], [x.ctypes.data for x in cols], rows)
    assert done == 2 and copied == 1  # segment 5 resident; segment 0's first column was copied before


def test_reserved_staging_slots_are_never_used_by_the_cache():
    cols = _cols(1, 10)
    c = SegmentCache(6, SEG, 1, 10, "lru", device=-1)
    c.begin_query()
    for seg in range(6):
        c.admit(0, seg, cols[0][seg * SEG:].ctypes.data, SEG)
    first = c.reserve(2)               # evicts what the top two slots held
    assert first == 4
    assert c.stats()["resident"] == 4
    assert all(s < 4 for s in c.col_idx(0) if s >= 0)
    # admissions and epoch replacement stay within the four managed slots
    for seg in range(6, 10):
        c.begin_query()
        assert c.admit(0, seg, cols[0][seg * SEG:].ctypes.data, SEG) < 4
    w = np.arange(10, dtype=np.float64)[None, :] + 1.0
    c.replace(w, [cols[0].ctypes.data], np.full(10, SEG, np.int32))
    idx = c.col_idx(0)
    assert sorted(np.nonzero(idx >= 0)[0].tolist()) == [6, 7, 8, 9] and all(s < 4 for s in idx if s >= 0)
    with pytest.raises(L.MbError):
        c.reserve(4)                   # would leave no managed slot


def test_stage_copies_into_reserved_slots_only():
    cols = _cols(1, 4)
    c = SegmentCache(5, SEG, 1, 4, "lru", device=-1)
    first = c.reserve(2)
    c.stage(first + 1, cols[0][2 * SEG:].ctypes.data, SEG)
    assert np.array_equal(c.host_slot_view(first + 1), cols[0][2 * SEG: 3 * SEG])
    assert (c.col_idx(0) == -1).all()           # staging leaves the map alone
    with pytest.raises(L.MbError):
        c.stage(0, cols[0].ctypes.data, SEG)     # a managed slot
