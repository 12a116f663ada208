"""Randomised dimension builds against the oracle, slot for slot.

Each case draws a dimension of 1..300,000 rows with distinct keys (shifted by whole
table lengths now and then, so keys wrap onto their slot), a key_min, a slot count at
or above the key range, an optional filter of every mode, and a payload column; it
builds the Crystal layouts (`mb_build_pht`: keys only with a presence bitmap, or
{key, val}), the engine layout (`mb_build_GPU2`: {val, row + 1}) and the CPU builds
(`mb_cpu_build_pht`, all three layouts), and compares every table word with the oracle.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from mordred_b200 import _lib as L
from mordred_b200 import cpu, ssb
from oracle import oracle as O


def make_build(seed: int) -> dict:
    rng = np.random.default_rng(seed)
    n = int(rng.choice([1, 100, 4097, 40_000, 300_000]))
    kmin = int(rng.choice([1, 7, 19920101]))
    slots = n + int(rng.choice([0, 0, 5, n]))
    keys = kmin + rng.choice(slots, size=n, replace=False).astype(np.int64)
    if rng.random() < 0.3:
        keys += slots * rng.integers(0, 2, n)  # (key - key_min) % slots: the same slot
    val = rng.integers(-10**6, 10**6, n).astype(np.int32)
    mode = int(rng.integers(-1, 3))  # -1: no filter
    c1, c2 = int(rng.integers(0, 10)), int(rng.integers(0, 10))
    if mode == L.MB_FILTER_BETWEEN:
        c1, c2 = min(c1, c2), max(c1, c2)
    flt = rng.integers(0, 10, n).astype(np.int32) if mode >= 0 else None
    return dict(n=n, kmin=kmin, slots=slots, key=keys.astype(np.int32), val=val, flt=flt,
                mode=max(mode, 0), c1=c1, c2=c2)


def oracle_table(b, layout):
    ht = np.zeros(b["slots"] if layout == L.MB_HT_KEY else 2 * b["slots"], np.int32)
    pres = np.zeros((b["slots"] + 31) // 32, np.uint32) if layout == L.MB_HT_KEY else None
    st = O.build_ht(b["flt"], b["mode"], b["c1"], b["c2"], b["key"], None if layout == L.MB_HT_KEY else b["val"],
                    ht, b["slots"], b["kmin"], layout, presence=pres)
    assert st == 0
    return ht, pres


@pytest.mark.parametrize("seed", range(30))
def test_cpu_builds_match_oracle(seed):
    b = make_build(300 + seed)
    for layout in (L.MB_HT_KEY, L.MB_HT_KEY_VAL, L.MB_HT_VAL_OFF):
        exp, _ = oracle_table(b, layout)
        ht = np.zeros_like(exp)
        assert cpu.build_pht(b["flt"], b["mode"], b["c1"], b["c2"], b["key"],
                             None if layout == L.MB_HT_KEY else b["val"], ht, b["slots"], b["kmin"], layout) == 0
        assert np.array_equal(ht, exp), layout


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(40))
def test_gpu_builds_match_oracle(seed):
    b = make_build(700 + seed)
    torch.cuda.set_device(0)
    L.call("mb_init", 0)
    L.device_status(0, clear=True)
    st = ssb._stream()
    key = torch.from_numpy(b["key"]).cuda()
    val = torch.from_numpy(b["val"]).cuda()
    flt = torch.from_numpy(b["flt"]).cuda() if b["flt"] is not None else None
    for layout in (L.MB_HT_KEY, L.MB_HT_KEY_VAL):
        exp, exp_pres = oracle_table(b, layout)
        ht = torch.zeros(exp.size, dtype=torch.int32, device="cuda")
        pres = torch.zeros((b["slots"] + 31) // 32, dtype=torch.int32, device="cuda") \
            if layout == L.MB_HT_KEY else None
        L.call("mb_build_pht", ssb._p(flt), b["mode"], b["c1"], b["c2"], ssb._p(key),
               ssb._p(val) if layout == L.MB_HT_KEY_VAL else None, b["n"], ssb._p(ht), b["slots"], b["kmin"],
               ssb._p(pres), st)
        assert np.array_equal(ht.cpu().numpy(), exp), layout
        if pres is not None:
            assert np.array_equal(pres.cpu().numpy().view(np.uint32), exp_pres)
    # engine layout {val, row + 1}
    exp, _ = oracle_table(b, L.MB_HT_VAL_OFF)
    ht = torch.zeros(exp.size, dtype=torch.int32, device="cuda")
    f = L.MbFilterArgsGPU(ssb._p(flt), None, b["c1"], b["c2"], 0, 0, b["mode"], 0)
    ba = L.MbBuildArgsGPU(ssb._p(key), ssb._p(val), b["slots"], b["kmin"], 0)
    L.call("mb_build_GPU2", None, C.byref(f), C.byref(ba), b["n"], ssb._p(ht), 0, None, st)
    assert np.array_equal(ht.cpu().numpy(), exp)
    assert L.device_status(0, clear=True) == 0
