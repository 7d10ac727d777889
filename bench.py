"""Benchmark of the B200 H2 matvec on the Toeplitz far-field workload.

Workload (synthetic, seeded): Laplace kernel 1/(4 pi |x-y|), N = 262144 points uniform in the unit
cube, uniform octree of depth 5 (4096 leaves, ~64 points per leaf), equispaced interpolation p = 4
per axis with Toeplitz M2L (FFT on (2p-1)^3 = 7^3 padded grids), dense FP64 near blocks of adjacent
leaves (97,336 blocks, ~399 M entries). One step = one matvec on one right-hand-side block,
alternating forward and transpose. Two forms are timed: plain (FP64 everywhere, one right-hand
side per matvec) and served (FP32 far field, FP64 near field and final sum, R = 16 right-hand sides
coalesced per matvec); `value` is the served form's throughput, `plain` the plain form's. The near
blocks (3.2 GB) exceed L2 (126 MB), so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--nrhs R]

Rank 0 prints one JSON line. With N > 1 every rank runs an independent replica of the map (the
single-map product does not shard), timing is the max over ranks, and `value` is the total
right-hand sides of all ranks per second.
"""

from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "h2factory.jl_b200")
METRIC = "H2 matvec RHS/s + p50/p99 latency at <=1e-6 rel err vs FP64; served vs plain"
WORKLOAD = "toeplitz-laplace-N262144-depth5-p4"


def _package():
    if "h2factory_b200" in sys.modules:
        return sys.modules["h2factory_b200"]
    spec = importlib.util.spec_from_file_location(
        "h2factory_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["h2factory_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_table():
    """Per-launch DRAM bytes of kernels captured with ncu (profiles/ncu_traffic.txt)."""
    out = {}
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if os.path.exists(path):
        for line in open(path):
            parts = line.split()
            if len(parts) >= 3 and not line.startswith("#"):
                out[(parts[0], parts[1])] = float(parts[2])
    return out


# ---------------------------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------------------------
def build_core(n=262144, depth=5, p=4, seed=0, device="cuda:0", precision="fp64"):
    h2 = _package()
    from h2factory_b200 import assembly, methods, trees

    rng = np.random.default_rng(seed)
    pts = rng.random((n, 3))
    pts = pts[trees.morton_order(pts)]
    tree = trees.build_tree(pts, depth=depth, root_center=[0.5] * 3, root_halfsize=0.5)
    core = methods.interpolation_core(tree, methods.laplace, p, nodes="equispaced",
                                      couplings="toeplitz", transfers="dense", near="none",
                                      precision=precision)
    assembly.near_blocks_device(core, "laplace", device=device)
    return h2, core


def launches_per_step(core, mode: int, nrhs: int = 1) -> int:
    """Kernels one h2b_matvec enqueues (same node-list logic as the library)."""
    agg = core.plans.trial if mode == 0 else core.plans.test
    dis = core.plans.test if mode == 0 else core.plans.trial
    tree = core.trial if mode == 0 else core.test
    dtree = core.test if mode == 0 else core.trial
    count = 1  # near
    if core.field == "real" and nrhs >= 8:
        count += 1  # gather of the x rows for the tensor-core near kernel
    count += 1  # leaf aggregation
    for st in range(agg.agg_level.size):
        nodes = agg.agg_node[agg.agg_ptr[st]:agg.agg_ptr[st + 1]]
        if any(not tree.isleaf(int(n)) for n in nodes):
            count += 1
    toep = core.coupling_kind == "toeplitz"
    count += 1 + (2 if toep else 0)  # i2o (+ fft in / out)
    for st in range(dis.dis_level.size):
        nodes = dis.dis_node[dis.dis_ptr[st]:dis.dis_ptr[st + 1]]
        if any(int(n) != 0 and dis.dis_isnode[dtree.parent[int(n)]] for n in nodes):
            count += 1
    count += 1  # leaf disaggregation
    return count


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def time_loop(torch, fn, steps, warmup, stream):
    """Per-step device times (ms) from CUDA events on `stream`, and the total."""
    for i in range(warmup):
        fn(i)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for i in range(steps):
            fn(i)
            ev[i + 1].record(stream)
    torch.cuda.synchronize()
    per = [ev[i].elapsed_time(ev[i + 1]) for i in range(steps)]
    return per, ev[0].elapsed_time(ev[steps])


def max_over_ranks(torch, values, world, device):
    """Each value's maximum over the replicas (the job time is the slowest rank's)."""
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def job_rate(units_per_rank, world, total_ms):
    """Whole-job throughput of `world` replicas that each processed `units_per_rank` units."""
    return units_per_rank * world / (total_ms * 1e-3)


def pct(v, q):
    return float(np.percentile(np.asarray(v), q))


# ---------------------------------------------------------------------------------------------
# CPU arms
# ---------------------------------------------------------------------------------------------
def cpu_matvec_rate(core, seconds=15.0, nthreads=0):
    """The oracle (a CPU port of the reference algorithm) on the host cores: RHS/s over a bounded
    number of forward/transpose matvecs of the full workload."""
    sys.path.insert(0, ROOT)
    from oracle import oracle
    from h2factory_b200.core import flatten

    desc = flatten(core)
    threads = nthreads or oracle.max_threads()
    rng = np.random.default_rng(1)
    x = rng.standard_normal(core.trial.npoints)
    oracle.matvec(core, x, 0, nthreads=threads, desc=desc)  # warm
    done, t0, times = 0, time.perf_counter(), []
    while time.perf_counter() - t0 < seconds or done < 2:
        t1 = time.perf_counter()
        oracle.matvec(core, x, done % 2, nthreads=threads, desc=desc)
        times.append(time.perf_counter() - t1)
        done += 1
    wall = time.perf_counter() - t0
    return {"value": done / wall, "unit": "RHS/s", "cores": threads, "kind": "port",
            "sample": f"{done} full matvecs (alternating forward/transpose, 1 RHS) in {wall:.1f} s",
            "p50_ms": pct(times, 50) * 1e3, "p99_ms": pct(times, 99) * 1e3}


def reference_arm(args, rank, world):
    if rank != 0:
        return
    import torch

    device = "cuda:0" if torch.cuda.is_available() else "cpu"
    if device == "cpu":
        h2, core = build_core_cpu()
    else:
        h2, core = build_core(device=device)
        core.near_data = core.near_device.cpu().numpy()
        core.near_device = None
        torch.cuda.empty_cache()
    per = max(1, args.steps)
    sys.path.insert(0, ROOT)
    from oracle import oracle
    from h2factory_b200.core import flatten

    desc = flatten(core)
    threads = oracle.max_threads()
    rng = np.random.default_rng(1)
    x = rng.standard_normal(core.trial.npoints)
    for i in range(args.warmup):
        oracle.matvec(core, x, i % 2, nthreads=threads, desc=desc)
    times = []
    for i in range(per):
        t1 = time.perf_counter()
        oracle.matvec(core, x, i % 2, nthreads=threads, desc=desc)
        times.append(time.perf_counter() - t1)
    tot = sum(times)
    value = per / tot
    line = {"metric": METRIC, "value": value, "unit": "RHS/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": per, "warmup": args.warmup, "ms_per_step": tot / per * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "rhs_per_step": 1, "modes": "forward/transpose alternating"},
            "p50_ms": pct(times, 50) * 1e3, "p99_ms": pct(times, 99) * 1e3,
            "cpu_baseline": {"value": value, "unit": "RHS/s", "cores": threads, "kind": "port",
                             "sample": f"{per} full matvecs of the workload after {args.warmup} warm-up"},
            "e2e": {"value": value, "unit": "RHS/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference is Julia and cannot run here; this arm times the C restatement of its "
                    "CPU algorithm (oracle/) with OpenMP over node chunks"}
    print(json.dumps(line), flush=True)


def build_core_cpu():
    h2 = _package()
    from h2factory_b200 import methods, trees

    rng = np.random.default_rng(0)
    pts = rng.random((262144, 3))
    pts = pts[trees.morton_order(pts)]
    tree = trees.build_tree(pts, depth=5, root_center=[0.5] * 3, root_halfsize=0.5)
    core = methods.interpolation_core(tree, methods.laplace, 4, nodes="equispaced", couplings="toeplitz")
    return h2, core


# ---------------------------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------------------------
def form_run(torch, h2, core, nrhs, steps, warmup, device, seed):
    """Time `steps` matvecs (forward/transpose alternating) on an `nrhs` block; device events."""
    ws = h2.H2Workspace(core, max_nrhs=nrhs, device=int(device.split(":")[1]))
    n = core.trial.npoints
    rng = np.random.default_rng(seed)
    xh = rng.standard_normal((n, nrhs))
    x = torch.from_numpy(np.ascontiguousarray(xh.T)).to(device).t()
    ys = [torch.zeros((nrhs, n), dtype=torch.float64, device=device).t() for _ in range(2)]
    views = [ws, h2.transpose(ws)]
    stream = torch.cuda.current_stream(device)
    sptr = stream.cuda_stream

    def step(i):
        h2.mul_(ys[i % 2], views[i % 2], x, stream=sptr)

    per, total = time_loop(torch, step, steps, warmup, stream)
    return ws, x, xh, per, total


def served_run(torch, h2, core, nrhs, steps, warmup, device, seed, inflight):
    """The served form: `steps` requests of `nrhs` right-hand sides, forward/transpose alternating,
    `inflight` of them on the device at once (request i on workspace and stream i % inflight, as a
    serving loop runs them). Device events: per-request latency on its stream, and the total from
    one start event that every stream waits for to the last request's end."""
    dcore = h2.DeviceCore(core, int(device.split(":")[1]))  # one resident core, one workspace per request slot
    wss = [h2.H2Workspace(dcore, max_nrhs=nrhs) for _ in range(inflight)]
    n = core.trial.npoints
    rng = np.random.default_rng(seed)
    xh = rng.standard_normal((n, nrhs))
    x = torch.from_numpy(np.ascontiguousarray(xh.T)).to(device).t()
    ys = [torch.zeros((nrhs, n), dtype=torch.float64, device=device).t() for _ in range(inflight)]
    streams = [torch.cuda.Stream(device) for _ in range(inflight)]
    views = [[w, h2.transpose(w)] for w in wss]

    def enqueue(i):
        j = i % inflight
        h2.mul_(ys[j], views[j][i % 2], x, stream=streams[j].cuda_stream)

    per, total = time_streams(torch, enqueue, steps, warmup, streams, device)
    return wss, x, xh, per, total


def time_streams(torch, enqueue, steps, warmup, streams, device):
    """Per-request device times (ms) and the total of `steps` requests spread over `streams`."""
    for i in range(warmup):
        enqueue(i)
    torch.cuda.synchronize()
    main = torch.cuda.current_stream(device)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    t0.record(main)
    for st in streams:
        st.wait_event(t0)
    for i in range(steps):
        st = streams[i % len(streams)]
        ev[i][0].record(st)
        enqueue(i)
        ev[i][1].record(st)
    for st in streams:
        main.wait_stream(st)
    t1.record(main)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev], t0.elapsed_time(t1)


def gpu_arm(args, rank, world, local_rank):
    import copy

    import torch

    torch.cuda.set_device(local_rank)
    device = f"cuda:{local_rank}"
    h2, core = build_core(n=args.n, depth=args.depth, device=device, precision="fp64")
    core32 = copy.copy(core)
    core32.precision = "fp32"
    n = core.trial.npoints
    nserve = args.nrhs
    sptr = torch.cuda.current_stream(device).cuda_stream

    # accuracy, before timing: plain FP64 against the CPU oracle and the dense kernel; served FP32
    # far field against the FP64 GPU product on the same right-hand-side block
    acc, cpu = {}, None
    ws64 = h2.H2Workspace(core, max_nrhs=nserve, device=local_rank)
    ws32 = h2.H2Workspace(core32, max_nrhs=nserve, device=local_rank)
    rng = np.random.default_rng(100 + rank)
    xb = rng.standard_normal((n, nserve))
    xd = torch.from_numpy(np.ascontiguousarray(xb.T)).to(device).t()
    errs = []
    for mode, (a64, a32) in enumerate(((ws64, ws32), (h2.transpose(ws64), h2.transpose(ws32)))):
        y64 = torch.zeros((nserve, n), dtype=torch.float64, device=device).t()
        y32 = torch.zeros((nserve, n), dtype=torch.float64, device=device).t()
        h2.mul_(y64, a64, xd, stream=sptr)
        h2.mul_(y32, a32, xd, stream=sptr)
        torch.cuda.synchronize()
        d = (y32 - y64).norm(dim=0) / y64.norm(dim=0)
        errs.append(float(d.max()))
    acc["served_max_rel_err_vs_fp64"] = max(errs)
    if rank == 0 and not args.skip_check:
        sys.path.insert(0, ROOT)
        from oracle import oracle

        near_host = core.near_device.cpu().numpy()
        hc = core_with_host_near(core, near_host)
        want = oracle.matvec(hc, xb[:, 0], 0)
        y0 = torch.zeros(n, dtype=torch.float64, device=device)
        h2.mul_(y0, ws64, xd[:, 0].contiguous(), stream=sptr)
        got = y0.cpu().numpy()
        acc["plain_rel_err_vs_fp64_oracle"] = float(np.linalg.norm(got - want) / np.linalg.norm(want))
        rows = rng.choice(n, 512, replace=False)
        P = torch.from_numpy(core.test.points).to(device)
        dd = P[torch.from_numpy(rows).to(device)][:, None, :] - P[None, :, :]
        r = torch.sqrt((dd * dd).sum(-1))
        K = torch.where(r > 0, 1.0 / (4 * np.pi * torch.where(r > 0, r, torch.ones_like(r))), torch.zeros_like(r))
        exact = (K @ xd[:, 0].contiguous()).cpu().numpy()
        acc["method_rel_err_vs_dense_512rows"] = float(np.linalg.norm(got[rows] - exact) / np.linalg.norm(exact))
        del dd, r, K
        torch.cuda.empty_cache()
        cpu = cpu_matvec_rate(hc, seconds=args.cpu_seconds)
        del near_host, hc
    ws64.close()
    ws32.close()
    if world > 1:
        torch.distributed.barrier()

    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        wsp, xp, xhp, per_p, tot_p = form_run(torch, h2, core, 1, args.steps, args.warmup, device, 7 + rank)
        wsl, xs_, xhs, per_s, tot_s = served_run(torch, h2, core32, nserve, args.steps, args.warmup, device,
                                                 11 + rank, args.inflight)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        # dominant kernel: near field, timed alone on the same stream (plain form, 1 RHS)
        yn = torch.zeros(n, dtype=torch.float64, device=device)
        xn = xp[:, 0].contiguous()
        nper, ntotal = time_loop(torch, lambda i: h2.nearmul_(yn, wsp, xn, stream=sptr),
                                 max(args.steps, 5), 3, torch.cuda.current_stream(device))
    tot_p, tot_s = max_over_ranks(torch, [tot_p, tot_s], world, device)

    # end to end through the host-buffer C-ABI call (pinned host memory, copies inside the region):
    # each request copies its x block in and its y block out; with `inflight` workspaces on their
    # own streams (h2b_matvec_host_async) one request's copies overlap another's product
    streams = [torch.cuda.Stream(device) for _ in range(args.inflight)]
    xpin = [torch.from_numpy(np.asfortranarray(xhs)).pin_memory().numpy() for _ in range(args.inflight)]
    ypin = [torch.zeros((nserve, n), dtype=torch.float64).pin_memory().numpy().T for _ in range(args.inflight)]

    def host_request(i):
        j = i % args.inflight
        wsl[j].matvec_host_async(xpin[j], ypin[j], i % 2, stream=streams[j].cuda_stream)

    for i in range(3):
        host_request(i)
    torch.cuda.synchronize()
    te_dev, _ = time_streams(torch, host_request, args.steps, 0, streams, device)
    t1 = time.perf_counter()
    for i in range(args.steps):
        host_request(i)
    torch.cuda.synchronize()
    te_total = time.perf_counter() - t1

    serving = serving_leg(torch, h2, core32, local_rank, args) if args.serve_seconds > 0 else None

    # the serving autotuner's choice for this map (block width, requests in flight), timed on the
    # resident core; informational: the timed forms above use --nrhs and --inflight
    tuned = None
    if args.autotune:
        from h2factory_b200 import autotune

        tuner = autotune.Autotuner(measure=lambda c, b, f: autotune.measure_on_device(
            c, b, f, steps=12, warmup=2, device=local_rank, dcore=wsl[0].dcore))
        ch = tuner.choose(core32, nserve, blocks=(1, 4, 8, 16), inflight=(1, 2, 3))
        tuned = {"key": ch["key"], "block": ch["block"], "inflight": ch["inflight"],
                 "rhs_per_s": ch["rhs_per_s"], "p99_ms": ch["p99_ms"],
                 "trials": [(t["block"], t["inflight"], round(t["rhs_per_s"]), round(t["p99_ms"], 3))
                            for t in ch["trials"]]}

    # the same map with a matrix-free near field (entries recomputed from the points, no stored
    # blocks): its own form, reported beside the stored-block forms
    mf = None
    if args.matrix_free:
        free = copy.copy(core)
        free.set_near_kernel("laplace")
        free32 = copy.copy(free)
        free32.precision = "fp32"
        steps_mf = max(3, args.steps // 10)
        wfp, _, _, _, tfp = form_run(torch, h2, free, 1, steps_mf, args.warmup, device, 7 + rank)
        wfs, _, _, _, tfs = form_run(torch, h2, free32, nserve, steps_mf, args.warmup, device, 11 + rank)
        tfp, tfs = max_over_ranks(torch, [tfp, tfs], world, device)
        mf = {"plain_rhs_per_s": job_rate(steps_mf, world, tfp), "served_rhs_per_s": job_rate(steps_mf * nserve, world, tfs),
              "steps": steps_mf, "near_bytes_stored": 0, "device_bytes": int(wfp.dcore.info().device_bytes)}
        for w in (wfp, wfs):
            w.close()
            w.dcore.close()

    if rank != 0:
        return
    hbm, peak_kind = peaks()
    info = wsp.dcore.info()
    near_bytes = info.near_entries * 8 + 2 * n * 8
    near_ms = ntotal / len(nper)
    achieved = near_bytes / (near_ms * 1e-3) / 1e9
    workload = WORKLOAD if (args.n, args.depth) == (262144, 5) else f"toeplitz-laplace-N{args.n}-depth{args.depth}-p4"
    traffic = traffic_table().get(("near_rows_kernel", workload))
    launches = sum(launches_per_step(core, i % 2, 1) + launches_per_step(core, i % 2, nserve)
                   for i in range(args.steps))
    plain_rate = job_rate(args.steps, world, tot_p)
    served_rate = job_rate(args.steps * nserve, world, tot_s)
    line = {
        "metric": METRIC, "value": served_rate, "unit": "RHS/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 far / f64 near",
        "data": "synthetic (seeded uniform points in the unit cube)",
        "config": {"workload": workload, "form": "served: FP32 far field, FP64 near field and sum, "
                   f"{nserve} right-hand sides coalesced per matvec, {args.inflight} requests in flight",
                   "rhs_per_step": nserve,
                   "modes": "forward/transpose alternating", "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (3.2 GB near blocks); no flush",
                   "near_entries": int(info.near_entries), "i2o_pairs": int(info.npairs[0])},
        "p50_ms": pct(per_s, 50), "p99_ms": pct(per_s, 99),
        "plain": {"value": plain_rate, "unit": "RHS/s", "dtype": "f64", "rhs_per_step": 1,
                  "ms_per_step": tot_p / args.steps, "p50_ms": pct(per_p, 50), "p99_ms": pct(per_p, 99)},
        "served_over_plain": served_rate / plain_rate,
        "accuracy": acc,
        "e2e": {"value": nserve * args.steps / te_total, "unit": "RHS/s",
                "h2d_bytes_per_step": int(n * 8 * nserve), "d2h_bytes_per_step": int(n * 8 * nserve),
                "requests_in_flight": args.inflight, "clock": "host wall clock, enqueue to last copy out",
                "p50_ms": pct(te_dev, 50), "p99_ms": pct(te_dev, 99)},
        "roofline": {"kernel": "near_rows_kernel", "bound": "hbm", "achieved": achieved,
                     "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                     "traffic": traffic, "algorithmic_bytes": near_bytes, "avg_launch_ms": near_ms},
        "clocks": clk.summary(),
        "gpu_launches": launches,
    }
    if mf is not None:
        line["matrix_free_near"] = mf
    if cpu is not None:
        line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if serving is not None:
        line["serving"] = serving
    if tuned is not None:
        line["autotune"] = tuned
    print(json.dumps(line), flush=True)


def serving_leg(torch, h2, core, local_rank, args):
    """Closed-loop clients against the continuous-batching server on the served form's map.

    Each client (an iterative solver) keeps one request in flight: forward / transpose / adjoint in
    60 / 20 / 20 proportion on a device-resident vector, waits for the result, and submits the next.
    Reports completed right-hand sides per second and per-request latency (submit to result).
    """
    from h2factory_b200.serving import GpuExecutor, MatvecServer

    device = f"cuda:{local_rank}"
    srv = MatvecServer(GpuExecutor(local_rank), budget_bytes=150e9, max_block=args.nrhs, slots=2)
    srv.add_map("toeplitz", core)
    n = core.trial.npoints
    xs = [torch.randn(n, dtype=torch.float64, device=device) for _ in range(args.clients)]
    torch.cuda.synchronize()
    srv.submit("toeplitz", xs[0]).result(timeout=300)  # load the map and warm the slots
    stop = [False]
    counts = [0] * args.clients
    t_start = [0.0]

    def client(i):
        r = np.random.default_rng(1000 + i)
        while not stop[0]:
            u = r.random()
            mode = "forward" if u < 0.6 else ("transpose" if u < 0.8 else "adjoint")
            srv.submit("toeplitz", xs[i], mode).result(timeout=300)
            counts[i] += 1

    ts = [threading.Thread(target=client, args=(i,), daemon=True) for i in range(args.clients)]
    for t in ts:
        t.start()
    time.sleep(min(1.0, args.serve_seconds / 3))  # ramp up
    base = sum(counts)
    srv.latencies.clear()
    srv.blocks.clear()
    t0 = time.perf_counter()
    time.sleep(args.serve_seconds)
    done = sum(counts) - base
    wall = time.perf_counter() - t0
    stats = srv.stats()
    stop[0] = True
    for t in ts:
        t.join(timeout=60)
    srv.close()
    return {"clients": args.clients, "mode_mix": "60/20/20 forward/transpose/adjoint",
            "requests": done, "seconds": wall, "rhs_per_s": done / wall, "p50_ms": stats["p50_ms"],
            "p99_ms": stats["p99_ms"], "mean_block": stats["mean_block"], "max_block": args.nrhs,
            "requests_on_device": True}


def core_with_host_near(core, near_host):
    import copy

    c = copy.copy(core)
    c.near_data, c.near_device = near_host, None
    return c


def sphere_core(n, device, precision="fp64", transfers="dense"):
    """The sphere configuration's map at `n` points: Fibonacci sphere (radius 0.45 in the unit
    cube) with jitter 0.1 x spacing, leaves <= 128 points, Helmholtz k = 8 pi x 0.45 (the unit
    sphere's electrical size), Chebyshev p = 6, symmetry-reduced couplings, near blocks assembled
    on the device."""
    h2 = _package()
    from h2factory_b200 import assembly, methods, trees

    rng = np.random.default_rng(0)
    i = np.arange(n) + 0.5
    phi, th = np.arccos(1 - 2 * i / n), np.pi * (1 + 5 ** 0.5) * i
    p = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], axis=1)
    p = p + 0.1 * np.sqrt(4 * np.pi / n) * rng.standard_normal(p.shape)
    tree = trees.build_tree(0.5 + 0.45 * p, maxvalues=128, root_center=[0.5] * 3, root_halfsize=0.5)
    k = 8 * np.pi * 0.45
    core = methods.interpolation_core(tree, methods.helmholtz(k), 6, near="none", symmetry=True,
                                      precision=precision, transfers=transfers)
    assembly.near_blocks_device(core, "helmholtz", wavenumber=k, device=device)
    return h2, core


def batched_arm(args):
    """The batched-uneven configuration's shape: `--maps` maps drawn as that configuration draws them
    (point counts log-uniform in [2048, --nmax], unit-cube volume / sphere surface / 4:1:1 ellipsoid
    surface, Laplace or Helmholtz with k uniform in [1, 20], Chebyshev p in {4, 5, 6}, leaves of at
    most 64 points, 1-16 right-hand sides, orientations mixed), FP32 far field, near blocks
    assembled on the device. A pass is every map's product once; it is timed as eager launches
    (each map on its own stream) and as one replay of the batch captured in a CUDA graph."""
    import torch

    h2 = _package()
    from h2factory_b200 import assembly, batch, methods, trees

    device = "cuda:0"
    rng = np.random.default_rng(2026)
    cores, nrhs, modes, shapes = [], [], [], []
    for _ in range(args.maps):
        n = int(np.exp(rng.uniform(np.log(2048), np.log(args.nmax))))
        geometry = ("cube", "sphere", "ellipsoid")[rng.integers(3)]
        if geometry == "cube":
            pts = rng.random((n, 3))
        else:
            i = np.arange(n) + 0.5
            phi, th = np.arccos(1 - 2 * i / n), np.pi * (1 + 5 ** 0.5) * i
            sp = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], axis=1)
            sp = sp + 0.1 * np.sqrt(4 * np.pi / n) * rng.standard_normal(sp.shape)
            pts = 0.5 + sp * (np.array([0.45, 0.45, 0.45]) if geometry == "sphere" else np.array([0.45, 0.1125, 0.1125]))
        helm = rng.random() >= 0.5
        k = float(rng.uniform(1, 20)) if helm else 0.0
        p = int(rng.integers(4, 7))
        tree = trees.build_tree(pts, maxvalues=64, root_center=[0.5] * 3, root_halfsize=0.5)
        core = methods.interpolation_core(tree, methods.helmholtz(k) if helm else methods.laplace, p, near="none",
                                          symmetry=True, precision="fp32")
        assembly.near_blocks_device(core, "helmholtz" if helm else "laplace", wavenumber=k, device=device)
        cores.append(core)
        nrhs.append(int(rng.integers(1, 17)))
        modes.append(int(rng.integers(3)))
        shapes.append(n)
    b = batch.BatchedMaps(cores, nrhs, device=0, modes=modes)
    b.set_inputs([torch.randn(x.shape[1], x.shape[0], dtype=x.dtype, device=device).t() for x in b.inputs])
    stream = torch.cuda.current_stream(device)
    per_e, tot_e = time_loop(torch, lambda i: b.run_eager(), args.steps, args.warmup, stream)
    b.capture()
    per_g, tot_g = time_loop(torch, lambda i: b.replay(), args.steps, args.warmup, stream)
    rhs = b.rhs_total()
    print(json.dumps({
        "metric": METRIC, "value": rhs * args.steps / (tot_g * 1e-3), "unit": "RHS/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_g / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 far / f64 near", "data": "synthetic (seeded)",
        "config": {"workload": f"batched-uneven-{args.maps}maps-N2048-{args.nmax}", "maps": args.maps,
                   "points_total": int(sum(shapes)), "rhs_per_pass": rhs,
                   "step": "one pass: every map's product once",
                   "scale": "point counts up to --nmax (the configuration draws up to 262,144)"},
        "graph": {"rhs_per_s": rhs * args.steps / (tot_g * 1e-3), "ms_per_pass": tot_g / args.steps,
                  "p50_ms": pct(per_g, 50), "p99_ms": pct(per_g, 99)},
        "eager": {"rhs_per_s": rhs * args.steps / (tot_e * 1e-3), "ms_per_pass": tot_e / args.steps,
                  "p50_ms": pct(per_e, 50), "p99_ms": pct(per_e, 99)}}), flush=True)
    b.close()


def sphere_arm(args):
    """Dense (Chebyshev) far field on the sphere configuration's shape: FP64 and FP32 forms, 32
    complex right-hand sides per matvec, forward/adjoint alternating (device timing)."""
    import copy

    import torch

    device = "cuda:0"
    h2, core = sphere_core(args.n, device, transfers=args.transfers)
    n = core.trial.npoints
    stream = torch.cuda.current_stream(device)
    x = torch.randn((32, n), dtype=torch.complex128, device=device).t()
    out = {}
    ref = None
    for prec in ("fp64", "fp32"):
        c = copy.copy(core)
        c.precision = prec
        ws = h2.H2Workspace(c, max_nrhs=32)
        y = torch.zeros((32, n), dtype=torch.complex128, device=device).t()
        views = [ws, h2.adjoint(ws)]
        per, tot = time_loop(torch, lambda i: h2.mul_(y, views[i % 2], x, stream=stream.cuda_stream),
                             args.steps, args.warmup, stream)
        h2.mul_(y, ws, x, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        if ref is None:
            ref = y.clone()
        out[prec] = {"rhs_per_s": 32 * args.steps / (tot * 1e-3), "ms_per_step": tot / args.steps,
                     "p50_ms": pct(per, 50), "p99_ms": pct(per, 99),
                     "rel_err_vs_fp64": float(((y - ref).norm(dim=0) / ref.norm(dim=0)).max())}
        ws.close()
        ws.dcore.close()
    print(json.dumps({
        "metric": METRIC, "value": out["fp32"]["rhs_per_s"], "unit": "RHS/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": out["fp32"]["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64 far / c128 near", "data": "synthetic (seeded sphere)",
        "config": {"workload": f"sphere-helmholtz-cheb6-N{n}", "rhs_per_step": 32, "modes": "forward/adjoint",
                   "far_pairs": int(core.plans.far.shape[0]), "near_entries": int(core.near_device.numel()),
                   "l2": "near blocks larger than L2; no flush"},
        "fp64": out["fp64"], "fp32": out["fp32"]}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nrhs", type=int, default=16, help="right-hand sides per served block")
    ap.add_argument("--inflight", type=int, default=3,
                    help="served requests on the device at once (3: the autotuner's choice for this map)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="skip the autotuner's report of block width and requests in flight")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--skip-check", action="store_true")
    ap.add_argument("--n", type=int, default=262144, help="points (smaller cases are for profiling)")
    ap.add_argument("--depth", type=int, default=5)
    ap.add_argument("--clients", type=int, default=64, help="closed-loop clients of the serving leg")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="serving leg length (0: skip)")
    ap.add_argument("--no-matrix-free", dest="matrix_free", action="store_false",
                    help="skip the matrix-free near-field forms")
    ap.add_argument("--batched", action="store_true",
                    help="time the batched-uneven configuration's shape (eager vs one graph replay per pass)")
    ap.add_argument("--maps", type=int, default=96, help="maps of the batched mode")
    ap.add_argument("--nmax", type=int, default=16384, help="largest point count of the batched mode")
    ap.add_argument("--transfers", default="dense", choices=["dense", "separable"],
                    help="level transfers of the sphere mode's map")
    ap.add_argument("--sphere", action="store_true",
                    help="time the sphere configuration's shape at --n points instead (dense far field)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.sphere:
        sphere_arm(args)
        return
    if args.batched:
        batched_arm(args)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        gpu_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
