"""Cost models for placing fact segments on the CPU or the GPU: the reference's analytic
bandwidth model and the learned MLP, behind one interface.

A planner maps the candidate segments of a query to predicted CPU and GPU milliseconds
per segment, plus each device's fixed cost for the query (its hash-table builds and
launches, paid once if the device takes any segment); :func:`place` then splits the
segments between the devices to minimise the query's makespan
(``mb_place_segments``). Features are computed per (query, segment) from the query's
constants, the segment's min/max statistics and the segment cache's residency, the
quantities the reference's optimizer reads (segment_min/max, CacheManager.h:156-157;
selectivities, KernelArgs.h:121-122; residency, segment_bitmap CacheManager.h:153; join
count; hash-table bytes).

* :class:`AnalyticPlanner` — src/gpudb/CostModel.cu:283-440 restated in C++
  (``mb_cost_segments``, ``mb_cost_build_ms``): CPU cost from 42 GB/s scans and 64-byte
  line probes, plus the CPU hash-table builds; GPU cost zero when resident
  (CostModel.cu:341-343) plus the 12 GB/s PCIe transfer of the segment's missing columns.
* :class:`LearnedPlanner` — the 24 -> 64 -> 64 -> 2 MLP of ``mb_mlp_*`` (CUDA forward,
  backward and Adam) trained on logged per-segment timings; it predicts log CPU ms and
  log GPU ms per segment; its fixed costs per query form are the logged medians. Its
  weights, feature scaling, fixed costs and training record persist as a small binary
  file plus a JSON manifest.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from . import ssb

NUM_FEATURES = L.MB_MLP_IN
FEATURE_NAMES = [
    "is_agg", "is_qa", "is_qb", "log2_rows", "date_sel", "discount_sel", "quantity_sel", "s_sel", "c_sel", "p_sel",
    "log10_sel", "num_probes", "num_filters", "log2_groups", "needed_cols", "resident_frac", "log2_missing_mb",
    "log2_ht_mb", "log2_out_rows", "agg_op", "log2_cpu_threads", "log_analytic_cpu_ms", "log_analytic_gpu_ms",
    "cache_free_frac"]
assert len(FEATURE_NAMES) == NUM_FEATURES
MIN_MS = 1e-3
TEMPLATES = ("agg", "qa", "qb")


@dataclass
class QueryContext:
    """What the planners see of a query's candidate segments (arrays over segments)."""
    template: str
    rows: np.ndarray           # float64
    date_sel: np.ndarray       # share of each segment's rows inside the query's date range
    small_sel: dict            # discount, quantity, s, c, p selectivities (1.0 where unconstrained)
    needed_cols: int
    resident_cols: np.ndarray  # int32, needed columns resident per segment
    ht_bytes: int
    dim_rows: int              # dimension rows the query's hash-table builds scan
    groups: int
    cpu_threads: int
    cache_free_frac: float

    def __len__(self) -> int:
        return len(self.rows)

    def subset(self, idx) -> "QueryContext":
        return QueryContext(self.template, self.rows[idx], self.date_sel[idx], self.small_sel, self.needed_cols,
                            self.resident_cols[idx], self.ht_bytes, self.dim_rows, self.groups, self.cpu_threads,
                            self.cache_free_frac)


def pipeline(ctx: QueryContext) -> L.MbCostPipeline:
    """The query's operator pipeline (the date filter first) for the analytic model."""
    p = L.MbCostPipeline()
    s = ctx.small_sel
    if ctx.template == "agg":
        fs, ps, aggr = [1.0, s["discount"], s["quantity"]], [], 2
    elif ctx.template == "qa":
        fs, ps, aggr = [1.0], [s["s"], s["p"], 1.0], 1
    else:
        fs, ps, aggr = [1.0], [s["s"], s["c"], s["p"], 1.0], 2
    p.num_filters, p.num_probes, p.group_by, p.num_aggr = len(fs), len(ps), 1, aggr
    for i, v in enumerate(fs):
        p.filter_sel[i] = v
    for i, v in enumerate(ps):
        p.probe_sel[i] = v
    return p


def analytic_ms(ctx: QueryContext) -> tuple[np.ndarray, np.ndarray]:
    n = len(ctx)
    cpu, gpu = np.zeros(n), np.zeros(n)
    rows = np.ascontiguousarray(ctx.rows, dtype=np.float64)
    sel = np.ascontiguousarray(ctx.date_sel, dtype=np.float64)
    miss = np.ascontiguousarray(ctx.needed_cols - ctx.resident_cols, dtype=np.int32)
    L.call("mb_cost_segments", C.byref(pipeline(ctx)), n, rows.ctypes.data, sel.ctypes.data, miss.ctypes.data,
           cpu.ctypes.data, gpu.ctypes.data)
    return np.maximum(cpu, MIN_MS), np.maximum(gpu, MIN_MS)


def features(ctx: QueryContext) -> np.ndarray:
    n = len(ctx)
    s = ctx.small_sel
    small = s["discount"] * s["quantity"] * s["s"] * s["c"] * s["p"]
    sel = ctx.date_sel * small
    nprobe = {"agg": 0, "qa": 3, "qb": 4}[ctx.template]
    nfilt = {"agg": 3, "qa": 1, "qb": 1}[ctx.template]
    op = {"agg": L.MB_AGG_MUL, "qa": L.MB_AGG_SUM, "qb": L.MB_AGG_SUB}[ctx.template]
    missing = (ctx.needed_cols - ctx.resident_cols) * ctx.rows * 4
    a_cpu, a_gpu = analytic_ms(ctx)
    f = np.empty((n, NUM_FEATURES), np.float32)
    const = [ctx.template == "agg", ctx.template == "qa", ctx.template == "qb"]
    f[:, 0:3] = np.array(const, np.float32)
    f[:, 3] = np.log2(np.maximum(ctx.rows, 1))
    f[:, 4] = ctx.date_sel
    f[:, 5:10] = [s["discount"], s["quantity"], s["s"], s["c"], s["p"]]
    f[:, 10] = np.log10(sel + 1e-7)
    f[:, 11], f[:, 12] = nprobe, nfilt
    f[:, 13] = math.log2(ctx.groups)
    f[:, 14] = ctx.needed_cols
    f[:, 15] = ctx.resident_cols / max(ctx.needed_cols, 1)
    f[:, 16] = np.log2(1 + missing / 1e6)
    f[:, 17] = math.log2(1 + ctx.ht_bytes / 1e6)
    f[:, 18] = np.log2(1 + sel * ctx.rows)
    f[:, 19] = op
    f[:, 20] = math.log2(max(ctx.cpu_threads, 1))
    f[:, 21] = np.log(a_cpu)
    f[:, 22] = np.log(a_gpu)
    f[:, 23] = ctx.cache_free_frac
    return f


_NPROBE = {"agg": 0, "qa": 3, "qb": 4}
_NFILT = {"agg": 3, "qa": 1, "qb": 1}
_OP = {"agg": L.MB_AGG_MUL, "qa": L.MB_AGG_SUM, "qb": L.MB_AGG_SUB}
_TPL = {"agg": 0, "qa": 1, "qb": 2}


def features_many(ctxs: list[QueryContext]) -> np.ndarray:
    """features() of many contexts, stacked in order: the per-segment columns are computed
    once over all of them (the per-query constants repeated), which for a window of
    thousands of queries replaces thousands of small array programs by one."""
    ctxs = [c for c in ctxs if len(c)]
    if not ctxs:
        return np.zeros((0, NUM_FEATURES), np.float32)
    lens = np.array([len(c) for c in ctxs])
    rep = lambda vals, dtype=np.float64: np.repeat(np.asarray(vals, dtype), lens)
    rows = np.concatenate([np.asarray(c.rows, np.float64) for c in ctxs])
    date_sel = np.concatenate([np.asarray(c.date_sel, np.float64) for c in ctxs])
    resident = np.concatenate([np.asarray(c.resident_cols, np.float64) for c in ctxs])
    sm = np.array([[c.small_sel[k] for k in ("discount", "quantity", "s", "c", "p")] for c in ctxs])
    small = rep(np.prod(sm, axis=1))
    sel = date_sel * small
    needed = rep([c.needed_cols for c in ctxs])
    missing = (needed - resident) * rows * 4
    a = [analytic_ms(c) for c in ctxs]
    a_cpu = np.concatenate([x[0] for x in a])
    a_gpu = np.concatenate([x[1] for x in a])
    tpl = rep([_TPL[c.template] for c in ctxs], np.int64)
    f = np.empty((len(rows), NUM_FEATURES), np.float32)
    f[:, 0:3] = np.eye(3, dtype=np.float32)[tpl]
    f[:, 3] = np.log2(np.maximum(rows, 1))
    f[:, 4] = date_sel
    f[:, 5:10] = np.repeat(sm, lens, axis=0)
    f[:, 10] = np.log10(sel + 1e-7)
    f[:, 11] = rep([_NPROBE[c.template] for c in ctxs])
    f[:, 12] = rep([_NFILT[c.template] for c in ctxs])
    f[:, 13] = rep([math.log2(c.groups) for c in ctxs])
    f[:, 14] = needed
    f[:, 15] = resident / np.maximum(needed, 1)
    f[:, 16] = np.log2(1 + missing / 1e6)
    f[:, 17] = rep([math.log2(1 + c.ht_bytes / 1e6) for c in ctxs])
    f[:, 18] = np.log2(1 + sel * rows)
    f[:, 19] = rep([_OP[c.template] for c in ctxs])
    f[:, 20] = rep([math.log2(max(c.cpu_threads, 1)) for c in ctxs])
    f[:, 21] = np.log(a_cpu)
    f[:, 22] = np.log(a_gpu)
    f[:, 23] = rep([c.cache_free_frac for c in ctxs])
    return f


def place(cpu_ms: np.ndarray, gpu_ms: np.ndarray, cpu_fixed: float = 0.0, gpu_fixed: float = 0.0):
    """Split segments between the devices (mb_place_segments): returns (on_gpu, makespan)."""
    cpu_ms = np.ascontiguousarray(cpu_ms, dtype=np.float64)
    gpu_ms = np.ascontiguousarray(gpu_ms, dtype=np.float64)
    on = np.zeros(len(cpu_ms), np.uint8)
    span = C.c_double(0)
    L.call("mb_place_segments", len(cpu_ms), cpu_ms.ctypes.data, gpu_ms.ctypes.data, float(cpu_fixed),
           float(gpu_fixed), on.ctypes.data, C.byref(span))
    return on.astype(bool), span.value


class AnalyticPlanner:
    name = "analytic"

    def predict(self, ctx: QueryContext):
        cpu, gpu = analytic_ms(ctx)
        return cpu, gpu, float(L.lib().mb_cost_build_ms(float(ctx.dim_rows))), 0.0

    def predict_many(self, ctxs: list[QueryContext]) -> list:
        return [self.predict(c) for c in ctxs]


class LearnedPlanner:
    """The cost MLP on the GPU. `params` is the flat fp32 parameter vector (5,890)."""
    name = "learned"

    def __init__(self, params: np.ndarray | None = None, mean=None, std=None, seed: int = 0, device="cuda",
                 fixed_ms: dict | None = None):
        self.device = device
        if params is None:
            params = init_params(seed)
        self.params = torch.tensor(np.asarray(params, np.float32), device=device)
        self.mean = np.zeros(NUM_FEATURES, np.float32) if mean is None else np.asarray(mean, np.float32)
        self.std = np.ones(NUM_FEATURES, np.float32) if std is None else np.asarray(std, np.float32)
        self.fixed_ms = fixed_ms or {t: [0.0, 0.0] for t in TEMPLATES}
        self.record: dict = {}
        self.manifest: dict = {}

    def _x(self, feats: np.ndarray) -> torch.Tensor:
        z = (np.asarray(feats, np.float32) - self.mean) / self.std
        return torch.tensor(z, dtype=torch.float32, device=self.device)

    def predict_log(self, feats: np.ndarray) -> np.ndarray:
        x = self._x(feats)
        y = torch.empty(len(feats), 2, dtype=torch.float32, device=self.device)
        L.call("mb_mlp_forward", self.params.data_ptr(), x.data_ptr(), len(feats), y.data_ptr(), ssb._stream())
        return y.cpu().numpy().astype(np.float64)

    def predict(self, ctx: QueryContext):
        fc, fg = self.fixed_ms.get(ctx.template, [0.0, 0.0])
        if len(ctx) == 0:
            return np.zeros(0), np.zeros(0), fc, fg
        y = np.exp(self.predict_log(features(ctx)))
        return y[:, 0], y[:, 1], fc, fg

    def predict_log_host(self, feats: np.ndarray) -> np.ndarray:
        """The same network evaluated on the host (fp32, numpy). For callers that must not
        wait on the device: a forward launch queues behind whatever occupies the SMs (a
        persistent batch kernel holds every SM until it ends). Agrees with the kernel to
        fp32 rounding (the summation order differs)."""
        w = self._host_params()
        x = (np.asarray(feats, np.float32) - self.mean) / self.std
        h1 = np.maximum(x @ w["W1"] + w["b1"], 0.0)
        h2 = np.maximum(h1 @ w["W2"] + w["b2"], 0.0)
        return (h2 @ w["W3"] + w["b3"]).astype(np.float64)

    def predict_host(self, ctx: QueryContext):
        """predict() with the host forward pass."""
        fc, fg = self.fixed_ms.get(ctx.template, [0.0, 0.0])
        if len(ctx) == 0:
            return np.zeros(0), np.zeros(0), fc, fg
        y = np.exp(self.predict_log_host(features(ctx)))
        return y[:, 0], y[:, 1], fc, fg

    def _host_params(self) -> dict:
        key = id(self.params), self.params._version
        if getattr(self, "_host_key", None) != key:
            p = self.params.detach().cpu().numpy()
            i, h, o = L.MB_MLP_IN, L.MB_MLP_HIDDEN, L.MB_MLP_OUT
            w, off = {}, 0
            for name, shape in (("W1", (i, h)), ("b1", (h,)), ("W2", (h, h)), ("b2", (h,)), ("W3", (h, o)),
                                ("b3", (o,))):
                n = int(np.prod(shape))
                w[name] = p[off: off + n].reshape(shape)
                off += n
            self._host_w, self._host_key = w, key
        return self._host_w

    def predict_many(self, ctxs: list[QueryContext]) -> list:
        """predict() for many queries with one model call over all their segments."""
        feats = features_many(ctxs)
        y = np.exp(self.predict_log(feats)) if len(feats) else np.zeros((0, 2))
        out, off = [], 0
        for c in ctxs:
            fc, fg = self.fixed_ms.get(c.template, [0.0, 0.0])
            n = len(c)
            out.append((y[off: off + n, 0], y[off: off + n, 1], fc, fg))
            off += n
        return out

    def train(self, feats: np.ndarray, log_ms: np.ndarray, epochs: int = 40, batch: int = 256, lr: float = 2e-3,
              weight_decay: float = 1e-5, seed: int = 0) -> dict:
        """Fit on (features, [log cpu ms, log gpu ms]) with the CUDA backward and Adam
        kernels; feature scaling comes from these samples."""
        feats = np.asarray(feats, np.float32)
        self.mean = feats.mean(0)
        self.std = feats.std(0) + 1e-6
        x = self._x(feats)
        t = torch.tensor(np.asarray(log_ms, np.float32), device=self.device)
        n = len(feats)
        g, m, v = (torch.zeros(L.MB_MLP_PARAMS, dtype=torch.float32, device=self.device) for _ in range(3))
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        rng = np.random.default_rng(seed)
        st = ssb._stream()
        step = 0
        hist = []
        for ep in range(epochs):
            perm = torch.tensor(rng.permutation(n), device=self.device)
            xs, ts = x[perm].contiguous(), t[perm].contiguous()
            loss.zero_()
            lr_ep = lr * (0.5 * (1 + math.cos(math.pi * ep / epochs)))  # cosine decay
            for b0 in range(0, n, batch):
                nb = min(batch, n - b0)
                step += 1
                g.zero_()
                L.call("mb_mlp_backward", self.params.data_ptr(), xs[b0:].data_ptr(), ts[b0:].data_ptr(), nb,
                       g.data_ptr(), loss.data_ptr(), st)
                L.call("mb_mlp_adam", self.params.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(),
                       L.MB_MLP_PARAMS, lr_ep, 0.9, 0.999, 1e-8, step, weight_decay, st)
            hist.append(float(loss.item()) / n)
        self.record = {"epochs": epochs, "batch": batch, "lr": lr, "steps": step, "samples": n,
                       "train_loss_per_epoch": hist}
        return self.record

    def save(self, path_bin: str, manifest: dict | None = None) -> None:
        os.makedirs(os.path.dirname(path_bin) or ".", exist_ok=True)
        self.params.cpu().numpy().astype("<f4").tofile(path_bin)
        man = {"params": os.path.basename(path_bin), "num_params": L.MB_MLP_PARAMS, "layout":
               "W1[24][64] b1[64] W2[64][64] b2[64] W3[64][2] b3[2], float32 little-endian",
               "features": FEATURE_NAMES, "feature_mean": self.mean.tolist(), "feature_std": self.std.tolist(),
               "outputs": ["log_cpu_ms", "log_gpu_ms"], "fixed_ms": self.fixed_ms, "training": self.record}
        if manifest:
            man.update(manifest)
        with open(os.path.splitext(path_bin)[0] + ".json", "w") as f:
            json.dump(man, f, indent=1)

    @classmethod
    def load(cls, path_bin: str, device="cuda") -> "LearnedPlanner":
        man = json.load(open(os.path.splitext(path_bin)[0] + ".json"))
        p = np.fromfile(path_bin, dtype="<f4")
        if p.size != L.MB_MLP_PARAMS:
            raise ValueError(f"{path_bin}: {p.size} parameters, expected {L.MB_MLP_PARAMS}")
        out = cls(p, man["feature_mean"], man["feature_std"], device=device, fixed_ms=man.get("fixed_ms"))
        out.record = man.get("training", {})
        out.manifest = man
        return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised weights, zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((NUM_FEATURES, L.MB_MLP_HIDDEN), (L.MB_MLP_HIDDEN, L.MB_MLP_HIDDEN),
                            (L.MB_MLP_HIDDEN, L.MB_MLP_OUT)):
        parts.append(rng.normal(0, math.sqrt(2.0 / fan_in), fan_in * fan_out))
        parts.append(np.zeros(fan_out))
    return np.concatenate(parts).astype(np.float32)
