"""Benchmark of the B200 H2 matvec.

Default workload (the largest single-GPU configuration of the benchmark set; synthetic, seeded):
Helmholtz kernel exp(ik|x-y|)/(4 pi |x-y|) with k = 8 pi x 0.45 (eight wavelengths across the
sphere), N = 1,048,576 points quasi-uniform on a sphere of radius 0.45 (Fibonacci lattice with
seeded jitter of 0.1 spacing), octree split while a box holds more than 128 points, Chebyshev
interpolation p = 6 (216 coefficients per box) with separable level transfers and
symmetry-reduced dense M2L couplings, dense complex near blocks of adjacent leaves (1.11 G
entries, 17.8 GB, assembled on the device). One step = one matvec on a block of 32 complex
right-hand sides, alternating forward and adjoint.

Two forms of the same map are timed:
  * plain:  ComplexF64 everywhere, one request at a time;
  * served: ComplexF32 far field (moments, transfers, couplings; dense M2L on the tcgen05 tensor
            cores with a three-term TF32 split), FP64 near field and near + far sum, `--inflight`
            requests in flight on their own workspaces and streams, as the serving loop runs them.
`value` is the served form's right-hand sides per second (device time of all requests, max over
ranks), `plain` the plain form's. `e2e` is the served form through the host-buffer C-ABI call
(h2b_matvec_host_async: each request copies its x block in and its y block out, pinned memory,
copies inside the host-clocked region). The near blocks (17.8 GB) exceed L2, so no flush is needed.
A second leg times the Toeplitz configuration (Laplace, N = 262,144 uniform in the unit cube,
depth-5 octree, equispaced p = 4 with FFT'd M2L) in the same two forms (`toeplitz` in the line).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload sphere|toeplitz]
    python bench.py --serve [--maps 32] [--serve-n 65536] [--rates 1000,...,50000] [--serve-rhs 1,8]
    python bench.py --batched [--maps 96] [--nmax 16384]

`--serve` times the serving configuration's shape (resident sphere maps, open-loop Poisson request
stream swept over rates, 1- and 8-RHS requests, p50/p99 per rate); `--batched` the batched-uneven
configuration's shape (many uneven maps per pass, eager vs one CUDA-graph replay). Each prints its
own JSON line.

Rank 0 prints one JSON line. With N > 1 every rank runs an independent replica of the map (the
single-map product does not shard), timing is the max over ranks, and `value` is the total
right-hand sides of all ranks per second. `--impl reference` times the CPU port of the reference
algorithm (oracle/) on the same workload.
"""

from __future__ import annotations

import argparse
import copy
import importlib.util
import json
import math
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
SPHERE_K = 8 * np.pi * 0.45


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
    """(HBM GB/s, dense bf16 TFLOP/s burst, kind): the measured copy bandwidth and cuBLAS bf16 rate
    of this pool's B200s, else the recorded fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


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
# workloads
# ---------------------------------------------------------------------------------------------
def sphere_points(n, seed=0):
    """Fibonacci lattice on the unit sphere with seeded jitter of 0.1 x spacing, scaled to radius
    0.45 about the centre of the unit cube."""
    rng = np.random.default_rng(seed)
    i = np.arange(n) + 0.5
    phi, th = np.arccos(1 - 2 * i / n), np.pi * (1 + 5 ** 0.5) * i
    p = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], axis=1)
    p = p + 0.1 * np.sqrt(4 * np.pi / n) * rng.standard_normal(p.shape)
    return 0.5 + 0.45 * p


def sphere_core(n, device, precision="fp64", transfers="separable", near="device", seed=0):
    """The sphere configuration's map at `n` points: leaves <= 128 points, Helmholtz k = 8 pi x 0.45,
    Chebyshev p = 6, symmetry-reduced couplings, near blocks assembled on the device (or on the host
    with near="host", for CPU-only runs)."""
    h2 = _package()
    from h2factory_b200 import assembly, methods, trees

    tree = trees.build_tree(sphere_points(n, seed), maxvalues=128, root_center=[0.5] * 3, root_halfsize=0.5)
    core = methods.interpolation_core(tree, methods.helmholtz(SPHERE_K), 6, symmetry=True, precision=precision,
                                      transfers=transfers, near="host" if near == "host" else "none")
    if near == "device":
        assembly.near_blocks_device(core, "helmholtz", wavenumber=SPHERE_K, device=device)
    return h2, core


def toeplitz_core(n=262144, depth=5, p=4, seed=0, device="cuda:0", near="device"):
    """The Toeplitz configuration's map: Laplace, n points uniform in the unit cube (Morton ordered),
    uniform octree of `depth`, equispaced p = 4 with FFT'd Toeplitz couplings."""
    h2 = _package()
    from h2factory_b200 import assembly, methods, trees

    rng = np.random.default_rng(seed)
    pts = rng.random((n, 3))
    pts = pts[trees.morton_order(pts)]
    tree = trees.build_tree(pts, depth=depth, root_center=[0.5] * 3, root_halfsize=0.5)
    core = methods.interpolation_core(tree, methods.laplace, p, nodes="equispaced", couplings="toeplitz",
                                      transfers="dense", near="host" if near == "host" else "none")
    if near == "device":
        assembly.near_blocks_device(core, "laplace", device=device)
    return h2, core


def core_with_host_near(core, near_host):
    c = copy.copy(core)
    c.near_data, c.near_device = near_host, None
    return c


def fp32_twin(core):
    c = copy.copy(core)
    c.precision = "fp32"
    return c


def direct_rows(torch, pts, rows, x, wavenumber, chunk=64):
    """FP64 direct sum of the kernel rows `rows` against every column: K[rows, :] x on the device."""
    out = []
    for s in range(0, rows.numel(), chunk):
        r = torch.cdist(pts[rows[s:s + chunk]], pts, compute_mode="donot_use_mm_for_euclid_dist")
        safe = torch.where(r > 0, r, torch.ones_like(r))
        if wavenumber:
            k = torch.where(r > 0, torch.exp(1j * wavenumber * safe) / (4 * math.pi * safe),
                            torch.zeros_like(r, dtype=torch.complex128))
        else:
            k = torch.where(r > 0, 1.0 / (4 * math.pi * safe), torch.zeros_like(r))
        out.append(k.to(x.dtype) @ x)
        del r, safe, k
    return torch.cat(out)


# ---------------------------------------------------------------------------------------------
# GPU timing helpers
# ---------------------------------------------------------------------------------------------
def _view(h2, ws, mode):
    return ws if mode == 0 else (h2.transpose(ws) if mode == 1 else h2.adjoint(ws))


def requests_run(torch, h2, dcore, nrhs, steps, warmup, device, seed, inflight, modes):
    """`steps` requests of `nrhs` right-hand sides, orientation modes[i % len(modes)], `inflight`
    of them on the device at once (request i on workspace and stream i % inflight). Device events:
    per-request latency on its stream, and the total from one start event to the last end."""
    wss = [h2.H2Workspace(dcore, max_nrhs=nrhs) for _ in range(inflight)]
    n = dcore.core.size[1]
    cplx = dcore.core.field == "complex"
    dt = torch.complex128 if cplx else torch.float64
    g = torch.Generator(device=device).manual_seed(seed)
    x = torch.randn((nrhs, n), dtype=dt, device=device, generator=g).t()
    ys = [torch.zeros((nrhs, n), dtype=dt, device=device).t() for _ in range(inflight)]
    streams = [torch.cuda.Stream(device) for _ in range(inflight)]
    views = [[_view(h2, w, m) for m in modes] for w in wss]

    def enqueue(i):
        j = i % inflight
        h2.mul_(ys[j], views[j][i % len(modes)], x, stream=streams[j].cuda_stream)

    per, total = time_streams(torch, enqueue, steps, warmup, streams, device)
    return wss, x, per, total


def e2e_run(torch, wss, nrhs, steps, modes, seed):
    """The same requests through the host-buffer call (h2b_matvec_host_async) with pinned host
    buffers, one workspace and stream per request in flight; host wall clock from the first enqueue
    to the last copy out, plus per-request device times."""
    inflight = len(wss)
    core = wss[0].core
    n = core.size[1]
    dt = core.dtype
    device = f"cuda:{wss[0].dcore.device}"
    rng = np.random.default_rng(seed)
    xh = rng.standard_normal((n, nrhs))
    if dt == np.complex128:
        xh = xh + 1j * rng.standard_normal((n, nrhs))
    tdt = torch.complex128 if dt == np.complex128 else torch.float64
    xpin = [torch.from_numpy(np.asfortranarray(xh)).pin_memory().numpy() for _ in range(inflight)]
    ypin = [torch.zeros((nrhs, n), dtype=tdt).pin_memory().numpy().T for _ in range(inflight)]
    streams = [torch.cuda.Stream(device) for _ in range(inflight)]

    def host_request(i):
        j = i % inflight
        wss[j].matvec_host_async(xpin[j], ypin[j], modes[i % len(modes)], stream=streams[j].cuda_stream)

    for i in range(max(3, inflight)):
        host_request(i)
    torch.cuda.synchronize()
    per, _ = time_streams(torch, host_request, steps, 0, streams, device)
    t1 = time.perf_counter()
    for i in range(steps):
        host_request(i)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t1
    nbytes = int(n * nrhs * (16 if dt == np.complex128 else 8))
    return {"value": nrhs * steps / wall, "unit": "RHS/s", "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
            "requests_in_flight": inflight, "clock": "host wall clock, enqueue to last copy out",
            "steps": steps, "p50_ms": pct(per, 50), "p99_ms": pct(per, 99)}


def pass_times(h2, ws, x, modes, reps):
    """Average device time (ms) of each pass kind over `reps` profiled products per orientation
    (h2b_profile_matvec: CUDA events on the launching stream, passes serialised), and the number
    of far-pass launches per product."""
    acc, nfar = {}, 0
    for m in modes:
        for _ in range(reps):
            recs = h2.profilemul(_view(h2, ws, m), x)
            nfar = max(nfar, len(recs) - 1)
            per = {}
            for r in recs:
                per[r["pass"]] = per.get(r["pass"], 0.0) + r["ms"]
            for k, v in per.items():
                acc.setdefault(k, []).append(v)
    return {k: float(np.mean(v)) for k, v in acc.items()}, nfar


def near_launches(field, nrhs):
    """Kernels one stored-block near product launches (the dispatch of h2b_near.cu)."""
    n, r = 0, nrhs
    if field == "complex":
        while r >= 8:
            n += 2          # gather + tensor-core slab kernel per 16 right-hand sides
            r -= min(16, r)
        return n + (r + 15) // 16
    if nrhs >= 8:
        return 2 * ((nrhs + 15) // 16)
    return (nrhs + 15) // 16


def i2o_useful_flops(core, nrhs):
    """Real floating-point operations of one dense I2O pass: every far pair (r, t) is an
    ncoef(r) x ncoef(t) block times nrhs columns; a complex multiply-add is 8 flops."""
    far = core.plans.far

    def ncoef(sh, tree, nodes):
        lv = tree.level[nodes]
        return sh[lv, 0].astype(np.int64) * sh[lv, 1] * sh[lv, 2]

    per = ncoef(core.shape_test, core.test, far[:, 0]) * ncoef(core.shape_trial, core.trial, far[:, 1])
    return float(per.sum()) * nrhs * (8 if core.field == "complex" else 2)


# ---------------------------------------------------------------------------------------------
# the sphere configuration (headline)
# ---------------------------------------------------------------------------------------------
def sphere_leg(args, rank, world, local_rank):
    import torch

    h2 = _package()
    from h2factory_b200.core import flatten

    device = f"cuda:{local_rank}"
    q = args.nrhs
    modes = (0, 2)  # forward / adjoint
    t_build = time.perf_counter()
    _, core = sphere_core(args.n, device, transfers=args.transfers)
    core32 = fp32_twin(core)
    n = core.trial.npoints
    d64 = h2.DeviceCore(core, local_rank)
    d32 = h2.DeviceCore(core32, local_rank)
    near_host = core.near_device.cpu().numpy() if (rank == 0 and not args.skip_check) else None
    core.near_device = core32.near_device = None  # each device core holds its own copy
    torch.cuda.empty_cache()
    build_s = time.perf_counter() - t_build

    # ---- accuracy, before timing ----
    acc, cpu = {}, None
    ws64 = h2.H2Workspace(d64, max_nrhs=q)
    ws32 = h2.H2Workspace(d32, max_nrhs=q)
    rng = np.random.default_rng(100 + rank)
    xb = rng.standard_normal((n, q)) + 1j * rng.standard_normal((n, q))
    xd = torch.from_numpy(np.ascontiguousarray(xb.T)).to(device).t()
    sptr = torch.cuda.current_stream(device).cuda_stream
    errs, y_fwd = [], None
    for m in modes:
        y64 = torch.zeros((q, n), dtype=torch.complex128, device=device).t()
        y32 = torch.zeros((q, n), dtype=torch.complex128, device=device).t()
        h2.mul_(y64, _view(h2, ws64, m), xd, stream=sptr)
        h2.mul_(y32, _view(h2, ws32, m), xd, stream=sptr)
        torch.cuda.synchronize()
        errs.append(float(((y32 - y64).norm(dim=0) / y64.norm(dim=0)).max()))
        if m == 0:
            y_fwd = (y64, y32)
    acc["served_max_rel_err_vs_fp64"] = max(errs)
    if rank == 0 and not args.skip_check:
        # method error: rows of the FP64 direct sum over all N columns, on the device
        rows = torch.from_numpy(rng.choice(n, args.dense_rows, replace=False)).to(device)
        pts = torch.from_numpy(core.test.points).to(device)
        exact = direct_rows(torch, pts, rows, xd, SPHERE_K)
        for name, y in (("plain", y_fwd[0]), ("served", y_fwd[1])):
            acc[f"{name}_rel_err_vs_dense_{args.dense_rows}rows"] = float((y[rows] - exact).norm() / exact.norm())
        del exact, pts
        torch.cuda.empty_cache()
        # the CPU port of the reference algorithm on the same map, one right-hand side: parity of
        # the plain form and the CPU baseline (the port's loops do not amortise right-hand sides)
        sys.path.insert(0, ROOT)
        from oracle import oracle

        hc = core_with_host_near(core, near_host)
        desc = flatten(hc)
        threads = oracle.max_threads()
        t1 = time.perf_counter()
        want = oracle.matvec(hc, xb[:, 0], 0, nthreads=threads, desc=desc)
        cpu_s = time.perf_counter() - t1
        got64 = y_fwd[0][:, 0].cpu().numpy()
        got32 = y_fwd[1][:, 0].cpu().numpy()
        acc["plain_rel_err_vs_fp64_oracle"] = float(np.linalg.norm(got64 - want) / np.linalg.norm(want))
        acc["served_rel_err_vs_fp64_oracle"] = float(np.linalg.norm(got32 - want) / np.linalg.norm(want))
        cpu = {"value": 1.0 / cpu_s, "unit": "RHS/s", "cores": threads, "kind": "port",
               "sample": f"one full forward matvec of the workload with 1 right-hand side ({cpu_s:.1f} s; the "
                         "port's loops do not amortise right-hand sides, so RHS/s = 1 / matvec time)"}
        del desc, hc, near_host, want
    del y_fwd
    ws64.close()
    ws32.close()
    torch.cuda.empty_cache()
    if world > 1:
        torch.distributed.barrier()

    # ---- timed region: plain, served, and both end to end ----
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        wsp, xpd, per_p, tot_p = requests_run(torch, h2, d64, q, args.steps, args.warmup, device, 7 + rank, 1, modes)
        wss, xsd, per_s, tot_s = requests_run(torch, h2, d32, q, args.steps, args.warmup, device, 11 + rank,
                                              args.inflight, modes)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e2e = e2e_run(torch, wss, q, args.steps, modes, 13 + rank)
        e2e_plain = e2e_run(torch, wsp, q, max(3, args.steps // 2), modes, 17 + rank)
    tot_p, tot_s = max_over_ranks(torch, [tot_p, tot_s], world, device)

    # ---- dominant kernels, timed alone on the launching stream ----
    served_passes, nfar = pass_times(h2, wss[0], xsd, modes, args.profile_reps)
    plain_passes, _ = pass_times(h2, wsp[0], xpd, modes, args.profile_reps)
    if rank != 0:
        return None
    hbm, bf16, peak_kind = peaks()
    info64 = d64.info()
    i2o_flops = i2o_useful_flops(core, q)
    i2o_ms = served_passes["i2o"]
    i2o_tf = i2o_flops / (i2o_ms * 1e-3) / 1e12
    near_entries = int(info64.near_entries)
    near_bytes = near_entries * 16 + 2 * n * q * 16
    near_ms = plain_passes["near"]
    near_flops = near_entries * q * 8.0
    wl = f"sphere-helmholtz-cheb6-N{n}"
    per_step = nfar + near_launches("complex", q)
    e2e_steps = args.steps + max(3, args.inflight) + max(3, args.steps // 2) + 3
    launches = per_step * (2 * args.steps + e2e_steps)
    plain_rate = job_rate(args.steps * q, world, tot_p)
    served_rate = job_rate(args.steps * q, world, tot_s)
    line = {
        "metric": METRIC, "value": served_rate, "unit": "RHS/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64 far / c128 near",
        "data": "synthetic (seeded Fibonacci sphere with jitter, complex Gaussian right-hand sides)",
        "config": {"workload": wl, "kernel": "Helmholtz exp(ik|x-y|)/(4 pi |x-y|), k = 8 pi x 0.45",
                   "points": n, "leaf_max": 128, "order": 6, "transfers": args.transfers,
                   "couplings": "dense, symmetry-reduced", "rhs_per_step": q, "modes": "forward/adjoint alternating",
                   "form": f"served: ComplexF32 far field (tcgen05 TF32-split M2L), FP64 near field and sum, "
                           f"{q} right-hand sides per request, {args.inflight} requests in flight",
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (17.8 GB near blocks); no flush",
                   "near_entries": near_entries, "i2o_pairs": int(info64.npairs[0]), "build_s": round(build_s, 1)},
        "p50_ms": pct(per_s, 50), "p99_ms": pct(per_s, 99),
        "plain": {"value": plain_rate, "unit": "RHS/s", "dtype": "c128", "rhs_per_step": q,
                  "ms_per_step": tot_p / args.steps, "p50_ms": pct(per_p, 50), "p99_ms": pct(per_p, 99),
                  "e2e": e2e_plain},
        "served_over_plain": served_rate / plain_rate,
        "accuracy": acc,
        "e2e": e2e,
        "roofline": {"kernel": "i2o_umma_kernel<cfloat> (served form's dense M2L: tcgen05 kind::tf32, three-term split)",
                     "bound": "tensor", "achieved": i2o_tf, "peak": bf16, "unit": "TFLOP/s", "frac": i2o_tf / bf16,
                     "peak_kind": f"{peak_kind} dense bf16 (burst)",
                     "traffic": traffic_table().get(("i2o_umma_kernel", wl)),
                     "algorithmic_flops": i2o_flops, "avg_launch_ms": i2o_ms,
                     "issued_tf32_tflops": 3 * i2o_tf, "frac_issued_vs_half_bf16": 3 * i2o_tf / (bf16 / 2)},
        "roofline_near": {"kernel": "near_slab_mma_c_kernel (FP64 tensor cores; plain and served forms)",
                          "bound": "fp64 tensor", "achieved_tflops": near_flops / (near_ms * 1e-3) / 1e12,
                          "achieved_gbs": near_bytes / (near_ms * 1e-3) / 1e9, "hbm_peak": hbm,
                          "algorithmic_bytes": near_bytes, "algorithmic_flops": near_flops, "avg_ms": near_ms,
                          "passes_over_blocks": (q + 15) // 16,
                          "traffic_per_launch": traffic_table().get(("near_slab_mma_c_kernel", wl))},
        "passes_ms": {"served": served_passes, "plain": plain_passes},
        "clocks": clk.summary(),
        "gpu_launches": launches,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    return line


# ---------------------------------------------------------------------------------------------
# the Toeplitz configuration
# ---------------------------------------------------------------------------------------------
def toeplitz_leg(args, rank, world, local_rank, n=262144, depth=5, nrhs=16, inflight=3):
    import torch

    h2 = _package()
    device = f"cuda:{local_rank}"
    modes = (0, 1)  # forward / transpose
    _, core = toeplitz_core(n=n, depth=depth, device=device)
    core32 = fp32_twin(core)
    d64 = h2.DeviceCore(core, local_rank)
    d32 = h2.DeviceCore(core32, local_rank)
    near_host = core.near_device.cpu().numpy() if (rank == 0 and not args.skip_check) else None
    core.near_device = core32.near_device = None
    torch.cuda.empty_cache()
    acc, cpu = {}, None
    ws64, ws32 = h2.H2Workspace(d64, max_nrhs=nrhs), h2.H2Workspace(d32, max_nrhs=nrhs)
    rng = np.random.default_rng(200 + rank)
    xb = rng.standard_normal((n, nrhs))
    xd = torch.from_numpy(np.ascontiguousarray(xb.T)).to(device).t()
    errs, y64f = [], None
    for m in modes:
        y64 = torch.zeros((nrhs, n), dtype=torch.float64, device=device).t()
        y32 = torch.zeros((nrhs, n), dtype=torch.float64, device=device).t()
        h2.mul_(y64, _view(h2, ws64, m), xd)
        h2.mul_(y32, _view(h2, ws32, m), xd)
        torch.cuda.synchronize()
        errs.append(float(((y32 - y64).norm(dim=0) / y64.norm(dim=0)).max()))
        if m == 0:
            y64f = y64
    acc["served_max_rel_err_vs_fp64"] = max(errs)
    if near_host is not None:
        sys.path.insert(0, ROOT)
        from oracle import oracle

        hc = core_with_host_near(core, near_host)
        threads = oracle.max_threads()
        t1 = time.perf_counter()
        want = oracle.matvec(hc, xb[:, 0], 0, nthreads=threads)
        cpu_s = time.perf_counter() - t1
        got = y64f[:, 0].cpu().numpy()
        acc["plain_rel_err_vs_fp64_oracle"] = float(np.linalg.norm(got - want) / np.linalg.norm(want))
        cpu = {"value": 1.0 / cpu_s, "unit": "RHS/s", "cores": threads, "kind": "port",
               "sample": f"one forward matvec, 1 right-hand side ({cpu_s:.2f} s)"}
        del hc, near_host
    ws64.close()
    ws32.close()
    if world > 1:
        torch.distributed.barrier()
    wsp, xpd, per_p, tot_p = requests_run(torch, h2, d64, 1, args.steps, args.warmup, device, 7 + rank, 1, modes)
    wss, xsd, per_s, tot_s = requests_run(torch, h2, d32, nrhs, args.steps, args.warmup, device, 11 + rank,
                                          inflight, modes)
    torch.cuda.synchronize()
    e2e = e2e_run(torch, wss, nrhs, args.steps, modes, 23 + rank)
    tot_p, tot_s = max_over_ranks(torch, [tot_p, tot_s], world, device)
    served_passes, _ = pass_times(h2, wss[0], xsd, modes, args.profile_reps)
    plain_passes, _ = pass_times(h2, wsp[0], xpd, modes, args.profile_reps)
    if rank != 0:
        return None
    hbm, _, peak_kind = peaks()
    info = d64.info()
    near_bytes = int(info.near_entries) * 8 + 2 * n * 8
    near_ms = plain_passes["near"]
    wl = f"toeplitz-laplace-N{n}-depth{depth}-p4"
    out = {"workload": wl, "rhs_per_step": nrhs, "modes": "forward/transpose alternating",
           "served": {"value": job_rate(args.steps * nrhs, world, tot_s), "unit": "RHS/s",
                      "ms_per_step": tot_s / args.steps, "requests_in_flight": inflight,
                      "p50_ms": pct(per_s, 50), "p99_ms": pct(per_s, 99), "e2e": e2e},
           "plain": {"value": job_rate(args.steps, world, tot_p), "unit": "RHS/s", "rhs_per_step": 1,
                     "ms_per_step": tot_p / args.steps, "p50_ms": pct(per_p, 50), "p99_ms": pct(per_p, 99)},
           "accuracy": acc,
           "roofline_near": {"kernel": "near_rows_kernel (plain form, 1 RHS)", "bound": "hbm",
                             "achieved": near_bytes / (near_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                             "frac": near_bytes / (near_ms * 1e-3) / 1e9 / hbm, "peak_kind": peak_kind,
                             "traffic": traffic_table().get(("near_rows_kernel", wl)),
                             "algorithmic_bytes": near_bytes, "avg_launch_ms": near_ms},
           "passes_ms": {"served": served_passes, "plain": plain_passes},
           "near_entries": int(info.near_entries), "i2o_pairs": int(info.npairs[0])}
    out["served_over_plain"] = out["served"]["value"] / out["plain"]["value"]
    if cpu:
        out["cpu_baseline"] = cpu
    return out


# ---------------------------------------------------------------------------------------------
# reference arm: the CPU port of the reference algorithm on the headline workload
# ---------------------------------------------------------------------------------------------
def reference_arm(args, rank, world):
    if rank != 0:
        return
    import torch

    _package()
    sys.path.insert(0, ROOT)
    from oracle import oracle
    from h2factory_b200.core import flatten

    on_gpu = torch.cuda.is_available()
    if args.workload == "sphere":
        _, core = sphere_core(args.n, "cuda:0", transfers=args.transfers, near="device" if on_gpu else "host")
        modes, wl = (0, 2), f"sphere-helmholtz-cheb6-N{args.n}"
    else:
        _, core = toeplitz_core(n=args.n, device="cuda:0", near="device" if on_gpu else "host")
        modes, wl = (0, 1), f"toeplitz-laplace-N{args.n}-depth5-p4"
    if core.near_device is not None:
        core = core_with_host_near(core, core.near_device.cpu().numpy())
        torch.cuda.empty_cache()
    desc = flatten(core)
    threads = oracle.max_threads()
    rng = np.random.default_rng(1)
    x = rng.standard_normal(core.trial.npoints)
    if core.field == "complex":
        x = x + 1j * rng.standard_normal(core.trial.npoints)
    # warm-up and timed steps are whole 1-RHS matvecs; a step of the sphere map takes seconds, so
    # the run is bounded: one warm-up, and timed steps until --reference-seconds have passed
    for i in range(min(args.warmup, 1)):
        oracle.matvec(core, x, modes[i % 2], nthreads=threads, desc=desc)
    times, t0 = [], time.perf_counter()
    for i in range(args.steps):
        t1 = time.perf_counter()
        oracle.matvec(core, x, modes[i % 2], nthreads=threads, desc=desc)
        times.append(time.perf_counter() - t1)
        if time.perf_counter() - t0 > args.reference_seconds and len(times) >= 2:
            break
    tot = sum(times)
    done = len(times)
    value = done / tot
    line = {"metric": METRIC, "value": value, "unit": "RHS/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": done, "steps_requested": args.steps, "warmup": min(args.warmup, 1),
            "ms_per_step": tot / done * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128" if core.field == "complex" else "f64", "data": "synthetic (seeded)",
            "config": {"workload": wl, "rhs_per_step": 1,
                       "modes": "forward/adjoint alternating" if modes[1] == 2 else "forward/transpose alternating"},
            "p50_ms": pct(times, 50) * 1e3, "p99_ms": pct(times, 99) * 1e3,
            "cpu_baseline": {"value": value, "unit": "RHS/s", "cores": threads, "kind": "port",
                             "sample": f"{done} full matvecs of the workload, 1 right-hand side each (the port's "
                                       f"loops do not amortise right-hand sides), after one warm-up; steps stop "
                                       f"after {args.reference_seconds:.0f} s"},
            "e2e": {"value": value, "unit": "RHS/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference is Julia and cannot run here; this arm times the C restatement of its CPU "
                    "algorithm (oracle/) with OpenMP over node chunks on all host threads"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# serving and batched modes
# ---------------------------------------------------------------------------------------------
def serve_arm(args):
    """The serving configuration's shape: `--maps` maps from the sphere configuration's generator
    (`--serve-n` points each, jitter seeds 0..maps-1), served form (FP32 far field, FP64 near field)
    kept resident under a 150 GB budget by the continuous-batching server, two stream slots per map.

    Open loop: requests arrive as a Poisson stream (256 simulated solver clients, each a Poisson
    stream at rate / 256, superpose to one at `rate`), each for a uniformly drawn map, forward /
    transpose / adjoint in 60 / 20 / 20 proportion, carrying 1 or 8 device-resident right-hand
    sides. For every rate of `--rates` and request width of `--serve-rhs` the stream runs
    `--serve-seconds`; a request's latency runs from its scheduled arrival to its result (a late
    submission counts against the server: no coordinated omission). When the window closes, requests
    that have not started are cancelled (the server drops them), the blocks in flight finish, and
    the step reports what completed inside the window."""
    import torch

    h2 = _package()
    from h2factory_b200.serving import GpuExecutor, MatvecServer

    device = "cuda:0"
    n, nmaps = args.serve_n, args.maps
    t_build = time.perf_counter()
    cores = []
    for i in range(nmaps):
        _, core = sphere_core(n, device, seed=i)
        cores.append(core)
    build_s = time.perf_counter() - t_build
    max_block = 32
    srv = MatvecServer(GpuExecutor(0), budget_bytes=150e9, max_block=max_block, slots=2,
                       max_inflight=args.serve_inflight or None)
    for i, c in enumerate(cores):
        srv.add_map(i, fp32_twin(c))
    rng = np.random.default_rng(31)
    widths = [int(w) for w in args.serve_rhs.split(",")]
    xs = {}
    for i, c in enumerate(cores):
        npts = c.trial.npoints
        for w in widths:
            shape = (npts,) if w == 1 else (w, npts)
            x = torch.randn(shape, dtype=torch.complex128, device=device)
            xs[(i, w)] = x if w == 1 else x.t()
    torch.cuda.synchronize()
    for i in range(nmaps):  # load every map (residency check) and warm its slots
        srv.submit(i, xs[(i, widths[-1])], "forward").result(timeout=600)
    resident, used = len(srv.resident), srv.used

    # accuracy of the served form against the FP64 product, map 0, every orientation
    ws64 = h2.H2Workspace(h2.DeviceCore(cores[0]), max_nrhs=max(widths))
    errs = []
    for mode in ("forward", "transpose", "adjoint"):
        x = xs[(0, max(widths))]
        got = srv.submit(0, x, mode).result(timeout=600)
        want = torch.zeros_like(got)
        h2.mul_(want, _view(h2, ws64, {"forward": 0, "transpose": 1, "adjoint": 2}[mode]), x)
        torch.cuda.synchronize()
        errs.append(float(((got - want).norm(dim=0) / want.norm(dim=0)).max()))
    ws64.close()
    torch.cuda.empty_cache()

    sweep = []
    rates = [float(r) for r in args.rates.split(",")]
    for w in widths:
        for rate in rates:
            sweep.append(_open_loop(srv, xs, nmaps, w, rate, args.serve_seconds, rng))
    srv.close()
    best = max(sweep, key=lambda r: r["achieved_rhs_per_s"])
    print(json.dumps({
        "metric": METRIC, "value": best["achieved_rhs_per_s"], "unit": "RHS/s", "n_gpus": 1,
        "steps": len(sweep), "warmup": nmaps, "ms_per_step": args.serve_seconds * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64 far / c128 near",
        "data": "synthetic (seeded Fibonacci spheres with jitter, complex Gaussian right-hand sides)",
        "config": {"workload": f"serving-{nmaps}maps-sphere-N{n}", "maps": nmaps, "points_per_map": n,
                   "clients": 256, "arrivals": "open-loop Poisson", "mode_mix": "60/20/20 forward/transpose/adjoint",
                   "rhs_per_request": widths, "rates_req_per_s": rates, "seconds_per_rate": args.serve_seconds,
                   "budget_bytes": 150e9, "max_block": max_block, "slots_per_map": 2,
                   "max_inflight_blocks": args.serve_inflight or None,
                   "step": "one rate x request width for --serve-seconds",
                   "scale": "maps of --serve-n points (the configuration's generator draws 1,048,576)",
                   "build_s": round(build_s, 1)},
        "resident_maps": resident, "resident_bytes_estimate": used,
        "accuracy": {"served_max_rel_err_vs_fp64": max(errs)},
        "best": best, "sweep": sweep,
        "e2e": None, "e2e_note": "requests are device-resident solver vectors: no host copies on this path"}),
        flush=True)


def _open_loop(srv, xs, nmaps, width, rate, seconds, rng):
    """One open-loop window: Poisson arrivals at `rate` requests/s for `seconds`; see serve_arm."""
    import torch

    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * seconds * 1.2) + 16))
    arrivals = arrivals[arrivals < seconds]
    maps = rng.integers(nmaps, size=arrivals.size)
    u = rng.random(arrivals.size)
    modes = np.where(u < 0.6, 0, np.where(u < 0.8, 1, 2))
    done_t = np.full(arrivals.size, np.nan)
    live = {}  # requests not yet answered (answered ones drop their results at once)
    srv.latencies.clear()
    srv.blocks.clear()
    lag = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i, ta in enumerate(arrivals):
        now = time.perf_counter() - t0
        if ta > now:
            if ta - now > 2e-4:
                time.sleep(ta - now - 1e-4)
            while time.perf_counter() - t0 < ta:
                pass
        lag.append(time.perf_counter() - t0 - ta)
        f = srv.submit(int(maps[i]), xs[(int(maps[i]), width)], int(modes[i]))
        live[i] = f

        def answered(_f, i=i):
            if not _f.cancelled():
                done_t[i] = time.perf_counter() - t0
            live.pop(i, None)

        f.add_done_callback(answered)
    t_end = time.perf_counter() - t0
    rest = list(live.values())
    cancelled = sum(1 for f in rest if f.cancel())  # not started: dropped by the server
    deadline = time.perf_counter() + 120
    for f in rest:
        if not f.cancelled():
            f.result(timeout=max(1.0, deadline - time.perf_counter()))
    window = max(seconds, t_end)
    inside = np.isfinite(done_t) & (done_t <= window)
    lat = (done_t - arrivals)[np.isfinite(done_t)]
    blocks = list(srv.blocks)
    return {"rate_req_per_s": rate, "rhs_per_request": width, "offered_rhs_per_s": rate * width,
            "requests": int(arrivals.size), "completed": int(np.isfinite(done_t).sum()),
            "completed_in_window": int(inside.sum()), "cancelled": int(cancelled),
            "achieved_req_per_s": float(inside.sum() / window),
            "achieved_rhs_per_s": float(inside.sum() * width / window),
            "p50_ms": float(np.percentile(lat, 50) * 1e3) if lat.size else None,
            "p99_ms": float(np.percentile(lat, 99) * 1e3) if lat.size else None,
            "submit_lag_p99_ms": float(np.percentile(lag, 99) * 1e3) if lag else None,
            "mean_block_rhs": float(np.mean(blocks)) if blocks else 0.0, "blocks": len(blocks)}


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
    # where a pass goes: every map's product once more, each pass timed on its stream (after the
    # timed region), summed by pass over the maps and by the map's far-field shape
    by_pass, by_shape = {}, {}
    for k, ws in enumerate(b.ws):
        view = ws if modes[k] == 0 else (h2.transpose(ws) if modes[k] == 1 else h2.adjoint(ws))
        recs = h2.profilemul(view, b.inputs[k])
        tot = sum(rec["ms"] for rec in recs)
        for rec in recs:
            by_pass[rec["pass"]] = by_pass.get(rec["pass"], 0.0) + rec["ms"]
        c = cores[k]
        key = f"{c.field} p={int(round(c.collections_test[next(iter(c.collections_test))].shape[1] ** (1 / 3)))}" \
              f" nrhs {'1' if nrhs[k] == 1 else ('2-7' if nrhs[k] < 8 else '8-16')}"
        by_shape[key] = by_shape.get(key, 0.0) + tot
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
                  "p50_ms": pct(per_e, 50), "p99_ms": pct(per_e, 99)},
        "serialised_ms_by_pass": {k: round(v, 2) for k, v in sorted(by_pass.items(), key=lambda kv: -kv[1])},
        "serialised_ms_by_map_shape": {k: round(v, 2) for k, v in sorted(by_shape.items(), key=lambda kv: -kv[1])}}),
        flush=True)
    b.close()


def gpu_arm(args, rank, world, local_rank):
    import torch

    torch.cuda.set_device(local_rank)
    if args.workload == "sphere":
        line = sphere_leg(args, rank, world, local_rank)
        if args.toeplitz_leg:
            tl = toeplitz_leg(args, rank, world, local_rank)
            if line is not None:
                line["toeplitz"] = tl
    else:
        tl = toeplitz_leg(args, rank, world, local_rank, n=args.n)
        line = None
        if tl is not None:
            line = {"metric": METRIC, "value": tl["served"]["value"], "unit": "RHS/s", "n_gpus": world,
                    "steps": args.steps, "warmup": args.warmup, "ms_per_step": tl["served"]["ms_per_step"],
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                    "dtype": "f32 far / f64 near", "data": "synthetic (seeded uniform points in the unit cube)",
                    "config": {"workload": tl["workload"]}, "e2e": tl["served"]["e2e"], "toeplitz": tl}
    if line is not None:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="sphere", choices=["sphere", "toeplitz"])
    ap.add_argument("--n", type=int, default=None, help="points (default: the configuration's size)")
    ap.add_argument("--nrhs", type=int, default=32, help="right-hand sides per request of the sphere workload")
    ap.add_argument("--inflight", type=int, default=2, help="served requests on the device at once")
    ap.add_argument("--transfers", default="separable", choices=["dense", "separable"],
                    help="level transfers of the sphere map")
    ap.add_argument("--no-toeplitz", dest="toeplitz_leg", action="store_false",
                    help="skip the Toeplitz configuration's secondary leg")
    ap.add_argument("--skip-check", action="store_true", help="skip the oracle / direct-sum checks")
    ap.add_argument("--dense-rows", type=int, default=4096, help="rows of the FP64 direct-sum check")
    ap.add_argument("--profile-reps", type=int, default=2, help="profiled products per orientation")
    ap.add_argument("--reference-seconds", type=float, default=150.0,
                    help="time budget of the reference arm's timed steps")
    ap.add_argument("--serve", action="store_true",
                    help="run the serving configuration's shape (open-loop Poisson rate sweep over resident maps)")
    ap.add_argument("--serve-n", type=int, default=65536, help="points per map of the serving mode")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="window per rate of the serving mode")
    ap.add_argument("--rates", default="1000,2000,5000,10000,20000,50000", help="request rates of the serving mode")
    ap.add_argument("--serve-rhs", default="1,8", help="right-hand sides per request of the serving mode")
    ap.add_argument("--serve-inflight", type=int, default=4,
                    help="blocks on the device at once in the serving mode (0: one per free slot of every map)")
    ap.add_argument("--batched", action="store_true",
                    help="time the batched-uneven configuration's shape (eager vs one graph replay per pass)")
    ap.add_argument("--maps", type=int, default=None, help="maps of the batched (96) or serving (32) mode")
    ap.add_argument("--nmax", type=int, default=16384, help="largest point count of the batched mode")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.n is None:
        args.n = 1048576 if args.workload == "sphere" else 262144
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.batched:
        args.maps = args.maps or 96
        batched_arm(args)
        return
    if args.serve:
        args.maps = args.maps or 32
        serve_arm(args)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        gpu_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
