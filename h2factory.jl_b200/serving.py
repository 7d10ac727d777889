"""Continuous-batching matvec server for resident H2 maps.

Iterative solvers (GMRES, CG, ...) issue one matvec at a time per client, forward, transpose or
adjoint, on a handful of maps. The server keeps each map's core (trees, plans, collections,
transfers, couplings, near blocks) resident in HBM under a memory budget and turns the request
stream into multi-RHS products:

* requests on the same (map, orientation) that are waiting when a slot frees up are coalesced into
  one block of up to `max_block` right-hand sides (one matvec reads the near blocks once for all);
  a request carries one right-hand side (a vector) or several (an n x k matrix, k <= max_block),
  and a block holds whole requests;
* every map has `slots` workspaces, each on its own CUDA stream, so blocks of different maps and
  orientations -- and consecutive blocks of one map -- run concurrently on the device; requests
  that arrive while blocks are in flight are admitted as soon as a slot is free (continuous
  batching, not a queue drained one block at a time);
* `max_inflight` caps the blocks on the device at once over all maps. With many resident maps an
  uncapped server launches a narrow block per map and orientation, the device's launch queues
  fill, and every block costs about as much as a full one (the dense M2L tiles 32 complex
  right-hand sides); capped, the waiting requests of a (map, orientation) coalesce into wide
  blocks, launched oldest request first;
* a map is admitted only if its core and workspaces fit the budget; idle maps are evicted least
  recently used first, and reloaded from their host description on the next request.

The workspace/core split is H2Factory's own model for concurrent products (one core, one
workspace per in-flight product: src/maps/workspace.jl:81-113, similarworkspace).

The scheduling logic is independent of the device: an executor performs loads and block launches.
`GpuExecutor` drives the C ABI; tests also run the scheduler against a dense CPU executor.
"""

from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

MODES = {"forward": 0, "transpose": 1, "adjoint": 2}


@dataclass
class Request:
    key: object
    mode: int
    x: np.ndarray
    future: Future
    t_submit: float
    t_done: float = 0.0
    ncols: int = 1          # right-hand sides carried (1 for a vector)


@dataclass
class _Resident:
    key: object
    handle: object
    nbytes: int
    slots: list
    last_used: float = 0.0
    busy: int = 0


@dataclass
class _Ticket:
    resident: _Resident
    slot: object
    requests: list
    handle: object


class AdmissionError(MemoryError):
    """A map does not fit the memory budget even after evicting every idle map."""


class MatvecServer:
    """Serve matvec requests on resident maps with continuous batching."""

    def __init__(self, executor, budget_bytes: float, max_block: int = 16, slots: int = 2,
                 max_inflight: int | None = None):
        self.executor = executor
        self.max_inflight = max_inflight
        self.budget = float(budget_bytes)
        self.max_block = int(max_block)
        self.nslots = int(slots)
        self.maps = {}                      # key -> host description (for reloads)
        self.resident = collections.OrderedDict()  # key -> _Resident, LRU order
        self.pending = collections.OrderedDict()   # (key, mode) -> deque[Request]
        self.inflight = []                  # _Ticket
        self.used = 0
        self.latencies = []                 # seconds, per completed request
        self.blocks = []                    # sizes of launched blocks
        self._lock = threading.Condition()
        self._stop = False
        self._error = None
        self._thread = threading.Thread(target=self._loop, name="h2b-server", daemon=True)
        self._thread.start()

    # -- public ---------------------------------------------------------------------------------
    def add_map(self, key, description) -> None:
        """Register a map; it is loaded on first use (or now, if it fits)."""
        with self._lock:
            self.maps[key] = description

    def submit(self, key, x, mode: str | int = "forward") -> Future:
        """Queue y = op(A_key) x for a vector x or an n x k block of right-hand sides (k <=
        max_block); the future resolves to y of the same shape (numpy, or a CUDA tensor for a
        CUDA x)."""
        m = MODES[mode] if isinstance(mode, str) else int(mode)
        fut = Future()
        xv = x if getattr(x, "is_cuda", False) else np.asarray(x)  # device tensors stay on the device
        k = 1 if xv.ndim == 1 else int(xv.shape[1])
        if xv.ndim > 2 or not 1 <= k <= self.max_block:
            raise ValueError(f"a request carries 1 to {self.max_block} right-hand sides, got shape {tuple(xv.shape)}")
        req = Request(key, m, xv, fut, time.perf_counter(), ncols=k)
        with self._lock:
            if key not in self.maps:
                raise KeyError(key)
            self.pending.setdefault((key, m), collections.deque()).append(req)
            self._lock.notify_all()
        return fut

    def close(self) -> None:
        with self._lock:
            self._stop = True
            self._lock.notify_all()
        self._thread.join()
        for r in list(self.resident.values()):
            self.executor.unload(r.handle, r.slots)
        self.resident.clear()

    def stats(self) -> dict:
        lat = np.array(self.latencies) if self.latencies else np.zeros(1)
        return {"requests": len(self.latencies), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_block": float(np.mean(self.blocks)) if self.blocks else 0.0,
                "resident_maps": len(self.resident), "used_bytes": self.used}

    # -- scheduling -----------------------------------------------------------------------------
    def _admit(self, key) -> _Resident:
        r = self.resident.get(key)
        if r is not None:
            self.resident.move_to_end(key)
            return r
        need = self.executor.footprint(self.maps[key], self.max_block, self.nslots)
        for victim in [k for k, v in self.resident.items() if v.busy == 0]:
            if self.used + need <= self.budget:
                break
            v = self.resident.pop(victim)
            self.executor.unload(v.handle, v.slots)
            self.used -= v.nbytes
        if self.used + need > self.budget:
            raise AdmissionError(f"map {key!r} needs {need} bytes; {self.budget - self.used:.0f} free")
        handle = self.executor.load(self.maps[key])
        slots = [self.executor.make_slot(handle, self.max_block) for _ in range(self.nslots)]
        r = _Resident(key, handle, need, slots)
        self.resident[key] = r
        self.used += need
        return r

    def _launch_ready(self) -> bool:
        launched = False
        order = list(self.pending.keys())
        if self.max_inflight is not None:
            order.sort(key=lambda km: self.pending[km][0].t_submit if self.pending[km] else 0.0)
        for (key, mode) in order:
            q = self.pending[(key, mode)]
            while q:
                if self.max_inflight is not None and len(self.inflight) >= self.max_inflight:
                    return launched
                try:
                    r = self._admit(key)
                except AdmissionError as exc:
                    while q:
                        f = q.popleft().future
                        if f.set_running_or_notify_cancel():
                            f.set_exception(exc)
                    break
                free = [s for s in r.slots if not getattr(s, "busy", False)]
                if not free:
                    break
                slot = free[0]
                block, cols = [], 0
                while q and cols + q[0].ncols <= self.max_block:
                    req = q.popleft()
                    # a request its client cancelled before it started is dropped here; once in a
                    # block it can no longer be cancelled
                    if req.future.set_running_or_notify_cancel():
                        block.append(req)
                        cols += req.ncols
                if not block:
                    continue
                slot.busy = True
                r.busy += 1
                r.last_used = time.perf_counter()
                handle = self.executor.launch(slot, mode, [b.x for b in block])
                self.inflight.append(_Ticket(r, slot, block, handle))
                self.blocks.append(cols)
                launched = True
            if not q:
                del self.pending[(key, mode)]
        return launched

    def _complete(self) -> bool:
        done_any = False
        keep = []
        for t in self.inflight:
            if self.executor.done(t.handle):
                ys = self.executor.results(t.slot, t.handle, [req.x.ndim == 2 and req.ncols for req in t.requests])
                now = time.perf_counter()
                for req, y in zip(t.requests, ys):
                    req.t_done = now
                    self.latencies.append(now - req.t_submit)
                    if not req.future.done():
                        req.future.set_result(y)
                t.slot.busy = False
                t.resident.busy -= 1
                done_any = True
            else:
                keep.append(t)
        self.inflight = keep
        return done_any

    def _loop(self):
        try:
            while True:
                with self._lock:
                    if self._stop and not self.pending and not self.inflight:
                        return
                    progressed = self._complete()
                    progressed |= self._launch_ready()
                    if not progressed:
                        if self.inflight:
                            self._lock.wait(timeout=20e-6)
                        else:
                            self._lock.wait(timeout=0.05)
        except BaseException as exc:  # surface scheduler failures on every waiting request
            self._error = exc
            with self._lock:
                for q in self.pending.values():
                    for req in q:
                        if not req.future.done():
                            req.future.set_exception(exc)
                for t in self.inflight:
                    for req in t.requests:
                        if not req.future.done():
                            req.future.set_exception(exc)
            raise


# ---------------------------------------------------------------------------------------------
# Executors
# ---------------------------------------------------------------------------------------------
class _GpuSlot:
    def __init__(self, ws, stream, x, y, event):
        self.ws, self.stream, self.x, self.y, self.event = ws, stream, x, y, event
        self.busy = False
        self.out = None


class GpuExecutor:
    """Runs blocks through the C ABI: one workspace and one CUDA stream per slot."""

    def __init__(self, device: int = 0):
        import torch

        self.torch = torch
        self.device = device
        self.dev = f"cuda:{device}"

    def footprint(self, core, max_block, nslots) -> int:
        """Core bytes (estimated from the host description) plus the slots' workspaces."""
        near = core.near_device.numel() * core.near_device.element_size() if core.near_device is not None \
            else core.near_data.nbytes
        per = 16 if core.field == "complex" else 8
        far = sum(np.asarray(v).nbytes for v in core.collections_test.values())
        ws = 4 * (core.test.nnodes * 64 * per) * max_block + 4 * core.test.npoints * per * max_block
        return int(2 * near + far + nslots * ws)

    def load(self, core):
        from .core import DeviceCore

        return DeviceCore(core, self.device)

    def unload(self, handle, slots):
        for s in slots:
            s.ws.close()
        handle.close()

    def make_slot(self, handle, max_block):
        from .core import H2Workspace

        torch = self.torch
        ws = H2Workspace(handle, max_nrhs=max_block)
        n = max(handle.core.size)
        dt = torch.complex128 if handle.core.field == "complex" else torch.float64
        x = torch.zeros((max_block, n), dtype=dt, device=self.dev)
        y = torch.zeros((max_block, n), dtype=dt, device=self.dev)
        return _GpuSlot(ws, torch.cuda.Stream(self.dev), x, y, torch.cuda.Event())

    def launch(self, slot, mode, xs):
        """Gather the block into the slot's x, multiply, and stage the outputs; asynchronous.

        Requests given as CUDA tensors are copied device to device (their producers must have
        finished, e.g. the client synchronised its stream before submitting) and answered with
        CUDA tensors; host requests are staged through the slot's stream and answered on the host.
        """
        from .core import OrientedMap, mul_

        torch = self.torch
        widths = [1 if xi.ndim == 1 else int(xi.shape[1]) for xi in xs]
        k = sum(widths)
        core = slot.ws.core
        nin = core.size[1] if mode == 0 else core.size[0]
        nout = core.size[0] if mode == 0 else core.size[1]
        on_device = getattr(xs[0], "is_cuda", False)
        with torch.cuda.stream(slot.stream):
            if on_device:
                c = 0
                for xi, w in zip(xs, widths):
                    # rows of slot.x are right-hand sides: a block's columns become rows
                    slot.x[c:c + w, :nin].copy_(xi.reshape(nin, w).t(), non_blocking=True)
                    c += w
            else:
                rows = [np.asarray(xi).reshape(nin, w).T for xi, w in zip(xs, widths)]
                host = torch.from_numpy(np.ascontiguousarray(np.concatenate(rows, axis=0)))
                slot.x[:k, :nin].copy_(host, non_blocking=False)
            X = slot.x[:k, :nin].t()
            Y = slot.y[:k, :nout].t()
            A = slot.ws if mode == 0 else OrientedMap(slot.ws, mode)
            mul_(Y, A, X, stream=slot.stream.cuda_stream)
            if on_device:
                out, c = [], 0
                for xi, w in zip(xs, widths):
                    out.append(slot.y[c, :nout].clone() if xi.ndim == 1 else slot.y[c:c + w, :nout].t().clone())
                    c += w
                slot.out = out
            else:
                slot.out = slot.y[:k, :nout].to("cpu", non_blocking=True)
            slot.event.record(slot.stream)
        return slot.event

    def done(self, event) -> bool:
        return event.query()

    def results(self, slot, event, shapes):
        """The block's outputs per request; `shapes` holds False for a vector request and the
        column count of a block request."""
        if isinstance(slot.out, list):
            return slot.out
        return _split_rows(slot.out.numpy(), shapes)


class DenseExecutor:
    """CPU stand-in: each 'map' is a dense matrix; used to test the scheduler without a GPU."""

    def __init__(self, delay: float = 0.0):
        self.delay = delay
        self.loads = 0

    def footprint(self, mat, max_block, nslots) -> int:
        return int(mat.nbytes + nslots * max_block * mat.shape[0] * mat.itemsize)

    def load(self, mat):
        self.loads += 1
        return mat

    def unload(self, handle, slots):
        pass

    def make_slot(self, handle, max_block):
        class S:
            busy = False
        s = S()
        s.mat = handle
        return s

    def launch(self, slot, mode, xs):
        A = slot.mat if mode == 0 else (slot.mat.T if mode == 1 else slot.mat.conj().T)
        X = np.concatenate([np.asarray(x).reshape(x.shape[0], -1) for x in xs], axis=1)
        return {"t": time.perf_counter() + self.delay, "Y": A @ X}

    def done(self, ticket) -> bool:
        return time.perf_counter() >= ticket["t"]

    def results(self, slot, ticket, shapes):
        return _split_rows(ticket["Y"].T, shapes)


def _split_rows(rows, shapes):
    """Rows of a block's output (one per right-hand side) back into per-request results."""
    out, c = [], 0
    for w in shapes:
        if w:
            out.append(np.ascontiguousarray(rows[c:c + w].T))
            c += w
        else:
            out.append(rows[c].copy())
            c += 1
    return out


# ---------------------------------------------------------------------------------------------
# Replicas: maps partitioned over devices
# ---------------------------------------------------------------------------------------------
class ReplicaRouter:
    """Serve many maps on several devices, one server per device, no collective on the data path.

    A single map's product does not shard (each level's I2O needs the moments of all boxes), but
    the serving workload -- many independent maps and requests -- does: each map is assigned to
    one device when it is added (the device with the fewest bytes assigned so far, by its server's
    footprint estimate), and its requests go to that device's server. `servers` are MatvecServer
    objects, typically one per GPU (GpuExecutor(device)); with one process per GPU, each process
    builds a router over its own device and the maps it owns.
    """

    def __init__(self, servers):
        self.servers = list(servers)
        if not self.servers:
            raise ValueError("at least one server")
        self.device_of = {}
        self.assigned = [0] * len(self.servers)

    def add_map(self, key, description) -> int:
        """Register a map on the least-loaded device; returns that device's index."""
        if key in self.device_of:
            raise KeyError(f"map {key!r} already added")
        sizes = []
        for d, srv in enumerate(self.servers):
            need = srv.executor.footprint(description, srv.max_block, srv.nslots)
            sizes.append((self.assigned[d] + need, d, need))
        _, d, need = min(sizes)
        self.servers[d].add_map(key, description)
        self.device_of[key] = d
        self.assigned[d] += need
        return d

    def submit(self, key, x, mode="forward"):
        return self.servers[self.device_of[key]].submit(key, x, mode)

    def stats(self) -> dict:
        per = [s.stats() for s in self.servers]
        lat = np.concatenate([np.asarray(s.latencies) for s in self.servers if s.latencies]) \
            if any(s.latencies for s in self.servers) else np.zeros(1)
        return {"devices": per, "requests": int(sum(p["requests"] for p in per)),
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "assigned_bytes": list(self.assigned)}

    def close(self) -> None:
        for s in self.servers:
            s.close()
