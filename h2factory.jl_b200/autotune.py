"""Autotuner for the serving parameters of a map: right-hand-side block width and requests in flight.

A server coalesces the waiting requests of one (map, orientation) into blocks of up to `max_block`
right-hand sides and keeps `slots` blocks of a map on the device at once (`serving.MatvecServer`).
Which pair gives the most right-hand sides per second depends on the map's shape and arithmetic:
the interpolation order p (coefficients per box, hence the far-field product sizes), the leaf size
(the near blocks' shape), the number of right-hand sides the clients can supply at once, and the
dtype (FP64 or FP32 far field, real or complex). The tuner times candidate pairs on the device
through the public API (`measure_on_device`), keeps the fastest whose per-request p99 latency meets
an optional budget, and caches the choice per key, (order, leaf size, RHS count, dtype), in a JSON
file, so that a server started later on a map of the same shape reuses it without timing again.
"""

from __future__ import annotations

import json
import os
import threading
from dataclasses import asdict, dataclass

import numpy as np


@dataclass(frozen=True)
class TuneKey:
    order: int       # moment extent per axis (p of a tensor interpolation)
    leaf_size: int   # largest number of points in a leaf
    nrhs: int        # right-hand sides the clients can supply at once (the largest block tried)
    dtype: str       # "<far-field precision>/<field>", e.g. "fp32/real"

    def text(self) -> str:
        return f"p{self.order}-leaf{self.leaf_size}-rhs{self.nrhs}-{self.dtype}"


def key_of(core, nrhs: int) -> TuneKey:
    """The tuning key of an H2Core for blocks of up to `nrhs` right-hand sides."""
    order = int(np.asarray(core.shape_test)[1:, 0].max())
    counts = np.diff(np.asarray(core.test.value_ptr))
    return TuneKey(order, int(counts.max()) if counts.size else 0, int(nrhs), f"{core.precision}/{core.field}")


def measure_on_device(core, block: int, inflight: int, steps: int = 20, warmup: int = 3,
                      device: int = 0, dcore=None) -> tuple[float, float]:
    """Right-hand sides per second and per-request p99 latency (ms) of `steps` products of
    `block` right-hand sides, forward/transpose alternating, `inflight` at a time on their own
    workspaces and streams (CUDA events)."""
    import torch

    from .core import DeviceCore, H2Workspace, mul_, transpose

    own = dcore is None
    if own:
        dcore = DeviceCore(core, device)
    dev = f"cuda:{device}"
    wss = [H2Workspace(dcore, max_nrhs=block) for _ in range(inflight)]
    n = max(core.size)
    dt = torch.complex128 if core.field == "complex" else torch.float64
    gen = torch.Generator(dev).manual_seed(0)
    x = torch.randn((block, n), dtype=dt, device=dev, generator=gen).t()
    ys = [torch.zeros((block, n), dtype=dt, device=dev).t() for _ in range(inflight)]
    streams = [torch.cuda.Stream(dev) for _ in range(inflight)]
    views = [[w, transpose(w)] for w in wss]
    rows, cols = core.size

    def enqueue(i):
        j = i % inflight
        nin = cols if i % 2 == 0 else rows
        nout = rows if i % 2 == 0 else cols
        mul_(ys[j][:nout], views[j][i % 2], x[:nin], stream=streams[j].cuda_stream)

    try:
        for i in range(warmup):
            enqueue(i)
        torch.cuda.synchronize(dev)
        main = torch.cuda.current_stream(dev)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        t0.record(main)
        for st in streams:
            st.wait_event(t0)
        for i in range(steps):
            st = streams[i % inflight]
            ev[i][0].record(st)
            enqueue(i)
            ev[i][1].record(st)
        for st in streams:
            main.wait_stream(st)
        t1.record(main)
        torch.cuda.synchronize(dev)
        total_ms = t0.elapsed_time(t1)
        lat = [a.elapsed_time(b) for a, b in ev]
    finally:
        for w in wss:
            w.close()
        if own:
            dcore.close()
    return block * steps / (total_ms * 1e-3), float(np.percentile(lat, 99))


class Autotuner:
    """Chooses (block width, requests in flight) per TuneKey and remembers the choice.

    `measure(core, block, inflight)` returns (RHS/s, p99 ms); by default `measure_on_device`.
    `cache_path`: a JSON file read at construction and rewritten after each new choice (None keeps
    the cache in memory only)."""

    def __init__(self, cache_path: str | None = None, measure=None):
        self.cache_path = cache_path
        self.measure = measure or measure_on_device
        self._lock = threading.Lock()
        self.cache = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.cache = json.load(f)

    def choose(self, core, nrhs: int, blocks=(1, 2, 4, 8, 16, 32), inflight=(1, 2, 3),
               p99_budget_ms: float | None = None) -> dict:
        """The fastest (block, inflight) with block <= nrhs whose p99 meets the budget (if none
        does, the one with the lowest p99); ties go to the smaller block, then fewer in flight."""
        key = key_of(core, nrhs)
        name = key.text() + ("" if p99_budget_ms is None else f"-p99le{p99_budget_ms:g}")
        with self._lock:
            if name in self.cache:
                return dict(self.cache[name])
        cands = [(b, f) for b in sorted(set(blocks)) if b <= nrhs for f in sorted(set(inflight))]
        if not cands:
            raise ValueError(f"no block width <= {nrhs} among {blocks}")
        trials = []
        for b, f in cands:
            rate, p99 = self.measure(core, b, f)
            trials.append({"block": b, "inflight": f, "rhs_per_s": float(rate), "p99_ms": float(p99)})
        ok = [t for t in trials if p99_budget_ms is None or t["p99_ms"] <= p99_budget_ms]
        if ok:
            best = max(ok, key=lambda t: (t["rhs_per_s"], -t["block"], -t["inflight"]))
        else:
            best = min(trials, key=lambda t: t["p99_ms"])
        choice = dict(best, key=asdict(key), budget_met=bool(ok), trials=trials)
        with self._lock:
            self.cache[name] = choice
            if self.cache_path:
                tmp = self.cache_path + ".tmp"
                with open(tmp, "w") as f:
                    json.dump(self.cache, f, indent=1, sort_keys=True)
                os.replace(tmp, self.cache_path)
        return dict(choice)

    def server_params(self, core, nrhs: int, **kw) -> dict:
        """`max_block` and `slots` for `serving.MatvecServer` from the choice for `core`."""
        c = self.choose(core, nrhs, **kw)
        return {"max_block": c["block"], "slots": c["inflight"]}
