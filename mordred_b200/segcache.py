"""Python handle on the library's GPU segment cache (``mb_segcache_*`` in
``include/mordred_b200.h``): fact columns in fixed-size segments, a device pool of
segment slots, admission with LRU / LFU / benefit-weight eviction, and epoch
replacement by benefit weights (the reference's CacheManager)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

POLICIES = {"lru": L.MB_CACHE_LRU, "lfu": L.MB_CACHE_LFU, "weight": L.MB_CACHE_WEIGHT}


class SegmentCache:
    def __init__(self, num_slots: int, segment_size: int, num_columns: int, num_segments: int,
                 policy: str = "lru", device: int = 0):
        self.segment_size, self.num_columns, self.num_segments = segment_size, num_columns, num_segments
        self.num_slots, self.device = num_slots, device
        h = L.lib().mb_segcache_create(device, num_slots, segment_size, num_columns, num_segments, POLICIES[policy])
        if not h:
            raise L.MbError("mb_segcache_create", L.MB_ERR_ARG, "bad arguments or the slot pool could not be allocated")
        self.h = C.c_void_p(h)

    def close(self) -> None:
        if self.h:
            L.lib().mb_segcache_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def pool(self) -> int:
        return int(L.lib().mb_segcache_pool(self.h))

    def slot(self, col: int, seg: int) -> int:
        return int(L.lib().mb_segcache_slot(self.h, col, seg))

    def col_idx(self, col: int) -> np.ndarray:
        out = np.empty(self.num_segments, np.int32)
        L.call("mb_segcache_col_idx", self.h, col, out.ctypes.data)
        return out

    def begin_query(self) -> None:
        L.lib().mb_segcache_begin_query(self.h)

    def touch(self, col: int, seg: int) -> None:
        L.call("mb_segcache_touch", self.h, col, seg)

    def set_weight(self, col: int, seg: int, w: float) -> None:
        L.call("mb_segcache_set_weight", self.h, col, seg, float(w))

    def admit(self, col: int, seg: int, host_ptr: int, rows: int, stream: int = 0) -> int:
        slot = C.c_int(-1)
        L.call("mb_segcache_admit", self.h, col, seg, host_ptr, rows, stream, C.byref(slot))
        return slot.value

    def admit_segments(self, cols, segs, host_cols: list, seg_rows: np.ndarray, stream: int = 0) -> tuple[int, int]:
        """Admit every column in `cols` of every segment in `segs`, in order; returns
        (segments fully admitted, column segments copied). Stops at the first segment that
        does not fit beside the pinned ones."""
        cols = np.ascontiguousarray(cols, dtype=np.int32)
        segs = np.ascontiguousarray(segs, dtype=np.int32)
        ptrs = (C.c_void_p * self.num_columns)(*host_cols)
        rows = np.ascontiguousarray(seg_rows, dtype=np.int32)
        done, copied = C.c_int(0), C.c_ulonglong(0)
        code = L.lib().mb_segcache_admit_segments(self.h, cols.ctypes.data, len(cols), segs.ctypes.data, len(segs),
                                                  ptrs, rows.ctypes.data, stream, C.byref(done), C.byref(copied))
        if code not in (L.MB_OK, L.MB_ERR_SIZE):
            L.check("mb_segcache_admit_segments", code)
        return done.value, int(copied.value)

    def evict(self, col: int, seg: int) -> None:
        L.call("mb_segcache_evict", self.h, col, seg)

    def replace(self, weights: np.ndarray, host_cols: list, segment_rows: np.ndarray, stream: int = 0) -> None:
        w = np.ascontiguousarray(weights, dtype=np.float64).reshape(-1)
        assert w.size == self.num_columns * self.num_segments
        ptrs = (C.c_void_p * self.num_columns)(*[p for p in host_cols])
        rows = np.ascontiguousarray(segment_rows, dtype=np.int32)
        L.call("mb_segcache_replace", self.h, w.ctypes.data, ptrs, rows.ctypes.data, stream)

    def reserve(self, nslots: int) -> int:
        """Take the top `nslots` unreserved slots out of management (a staging area the
        caller copies into); returns the first reserved slot."""
        first = C.c_int64(0)
        L.call("mb_segcache_reserve", self.h, nslots, C.byref(first))
        return int(first.value)

    def stage(self, slot: int, host_ptr: int, rows: int, stream: int = 0) -> None:
        """Copy a segment's rows into reserved slot `slot` (asynchronous on `stream`)."""
        L.call("mb_segcache_stage", self.h, slot, host_ptr, rows, stream)

    def stats(self) -> dict:
        s = L.MbSegcacheStats()
        L.call("mb_segcache_get_stats", self.h, C.byref(s))
        return {k: int(getattr(s, k)) for k, _ in L.MbSegcacheStats._fields_}

    def host_slot_view(self, slot: int) -> np.ndarray:
        """The slot's ints (host-pool caches only, device < 0)."""
        assert self.device < 0
        buf = (C.c_int * self.segment_size).from_address(self.pool + slot * self.segment_size * 4)
        return np.ctypeslib.as_array(buf)
