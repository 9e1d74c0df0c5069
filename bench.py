#!/usr/bin/env python
"""Benchmark of the plain FP64 HPR iteration on the large sparse SOCP
(n = 2,000,000, m = 1,500,000, nnz(A) = 25M, 20 x 5000 / 5k x 50 / 100k x 3
variable cones, 100k x 3 + 4k x 50 constraint cones; seeded synthetic data).

A step is one HPR iteration (x half-step over A' and y half-step over A, both
fused SpMV + projection + Halpern kernels).  `value` is iterations/s with all
data resident in HBM (A and A' are ~600 MB, far larger than the 126 MB L2, so
no flush is needed between steps); `e2e` is the same metric through the public
C ABI from host buffers: upload, scaling, eigenvalue estimate, K iterations
and the solution read-back all inside the timed region.

--impl reference times the CPU restatement of the reference solver (the
oracle, the only CPU implementation of this path that runs here) with every
host thread, on the same instance and metric.

Multi-GPU: the path does not shard (one solve per GPU); --gpus N runs N
independent replicas, one per rank, and reports the aggregate rate.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hpr-socp_b200"))

WORKLOAD = ("sparse SOCP n=2,000,000 m=1,500,000 nnz(A)=25M (A1 1M lognormal rows, A2 0.5M rows), "
            "var cones 100k x3 + 5k x50 + 20 x5000, con cones 100k x3 + 4k x50, Q=0")
METRIC = "HPR iters/s"

# --workload config2: the Q path at its configured size (one replica per GPU
# too); the default line above is the benchmark workload
WORKLOADS = {
    "config1": {"workload": WORKLOAD, "seed": 1,
                "l2": "inputs larger than L2 (A + A' ~ 600 MB)",
                "kernel": "engine_kernel (x half-step over A' + y half-step over A, per iteration)",
                "traffic_file": "engine_config1_dram_bytes.txt"},
    "config2": {"workload": "QP-SOCP (robust portfolio) n=200,000 m=212,001 nnz(A)=4.4M, Q = D + F'F with F "
                            "50 x n at 5% (never formed), box [0, 0.05], 2000 con cones x101",
                "seed": 2,
                "l2": "per-iteration streams ~186 MB (A + A' 106 MB) against the 126 MB L2: `value` is back to "
                      "back iterations; `l2_flushed` times single iterations after a 512 MB write",
                "kernel": "engine_kernel, 6 launches per iteration (F w; F'(.) + x/w step; F w_bar; "
                          "F'(.) + tempv; A tempv + y step; A' y_bar + w2 step)",
                "traffic_file": "engine_config2_dram_bytes.txt"},
}


def make_model(args):
    from hprsocp_b200 import instances
    gen = {"config1": instances.config1, "config2": instances.config2}[args.workload]
    return gen(WORKLOADS[args.workload]["seed"], scale=args.scale)


def measured_peak():
    """HBM copy bandwidth measured on this pool's B200s (MEASURED_PEAKS.json
    beside this file), else the pool's earlier fallback figure."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device=0):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_samples(self, count, timeout=5.0):
        """Block until `count` more samples than now have arrived (nvidia-smi
        takes a moment to start), so a short timed region is bracketed."""
        if not self.proc:
            return
        target = len(self.lines) + count
        t0 = time.perf_counter()
        while len(self.lines) < target and time.perf_counter() - t0 < timeout and self.proc.poll() is None:
            time.sleep(0.02)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, first=0):
        """Median SM clock and the throttle reasons seen in samples[first:]."""
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[first:]:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = max(smax, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(n_gpus, backend=None):
    """One process per GPU (torchrun): NCCL on GPUs, gloo for CPU tests."""
    if n_gpus <= 1 or "RANK" not in os.environ:
        return 0, 1, None
    import datetime
    import torch
    import torch.distributed as dist
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
    if backend == "nccl":
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", rank)))
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, world, dist


def dist_max(dist, v):
    """Max of a per-rank value over all ranks (device timing is max-over-ranks)."""
    if dist is None:
        return v
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def aggregate(world, steps, ms_max):
    """Whole-job rate of N replicas: all ranks' iterations over the slowest
    rank's device time."""
    return world * steps / (ms_max / 1e3)


def l2_flushed_iterations(ctx, dev, count):
    """Median device time (ms) of single partial iterations, each after a
    512 MB write that evicts the L2, for workloads whose per-iteration
    streams are within a small factor of the L2."""
    import torch
    buf = torch.empty(64 << 20, dtype=torch.float64, device=f"cuda:{dev}")
    times = []
    for i in range(count):
        buf.fill_(float(i))
        torch.cuda.synchronize(dev)
        ctx.iterate(1, False)
        times.append(ctx.last_iterate()[0])
    del buf
    return statistics.median(times)


def cpu_iteration_rate(model, iters=3, threads=0):
    """Oracle (CPU restatement) iterations/s on this host's cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle_ctx import OracleContext
    from hprsocp_b200 import HPRSOCP_parameters
    o = OracleContext(model, threads=threads)
    o.scale(HPRSOCP_parameters(verbose=False))
    o.set_sigma_lambda(1.0, 1.05 * 4000.0, 0.0)
    o.iterate(1, False)
    t = time.perf_counter()
    o.iterate(iters, True)
    dt = time.perf_counter() - t
    o.close()
    return iters / dt


def arm_config(args, world=1):
    """The `config` object both arms print (the driver compares them)."""
    w = WORKLOADS[args.workload]
    return {"workload": w["workload"], "precision": "fp64", "l2": w["l2"],
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU", "scale": args.scale}


def run_reference(args, model, budget_s=150.0):
    """CPU arm: the oracle (the CPU restatement of the reference solver) with
    every host thread, timed over the same phases as the GPU arm's `e2e`:
    copying the problem in, scaling, the power iteration (tolerance 1e-4,
    as the reference), K HPR iterations with the residual check every 150
    iterations, and the unscaled solution read-back.  `value` is the
    iteration rate of the HPR loop alone, the counterpart of the GPU arm's
    device-resident rate.  The solve stops at ``budget_s`` seconds (the
    reference's time_limit rule, which counts the power iteration) so the
    run stays bounded; the rates are over the iterations it completed."""
    cores = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle_ctx import OracleContext
    from hprsocp_b200 import HPRSOCP_parameters
    p = HPRSOCP_parameters(verbose=False, max_iter=args.steps, stoptol=0.0, check_iter=150,
                           print_frequency=10**9, time_limit=budget_s)
    t0 = time.perf_counter()
    o = OracleContext(model, threads=0)
    r = o.solve(p)  # scaling, power iteration, HPR loop, unscaled solution
    total = time.perf_counter() - t0
    o.close()
    loop_s = max(r.time - r.power_time, 1e-9)
    done = max(r.iter, 1)
    v = done / loop_s
    sample = f"{r.iter} of {args.steps} HPR iterations of the {args.workload} instance, one full solve" + (
        f" (stopped at the {budget_s:.0f} s bound)" if r.iter < args.steps else "")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "iter/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * loop_s / done,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": f"synthetic (seeded generator, seed {WORKLOADS[args.workload]['seed']})",
            "config": arm_config(args, args.gpus),
            "path": "CPU restatement of the reference solver (oracle port), all host threads; no JIT, so the "
                    "warm-up steps do not apply",
            "cpu_baseline": {"value": v, "unit": "iter/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": r.iter / total, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                    "seconds": total,
                    "what": "oracle solve from host arrays: problem copy + scaling + power iteration + "
                            f"{r.iter} iterations (checks every 150) + unscaled solution",
                    "phases_s": {"power_iteration": r.power_time, "hpr_loop_after_power": loop_s,
                                 "setup_scaling_readback": total - r.time}}}
    print(json.dumps(line))


def serving_measure(requests, slots=32, rate=0.0, baseline=60, resident=False, seed=11):
    """Serving stream: small SOCPs (n lognormal, median 400) with per-request
    tolerances 1e-4 / 1e-6 through the continuous-batching server, against
    the same requests solved one at a time with hpr_optimize."""
    # as many hardware work queues as slots can use (read at CUDA context creation)
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    import ctypes as C
    import numpy as np
    from hprsocp_b200 import HPRSOCP_parameters, _abi, instances
    from hprsocp_b200.serving import Server
    stream = instances.serving_stream(seed, requests, rate=rate, procs=os.cpu_count() or 1)
    params = [HPRSOCP_parameters(verbose=False, stoptol=tol, max_iter=200000) for _, tol, _ in stream]
    lib = _abi.load_library()
    # the server: requests submitted at their arrival times (all at t = 0 at
    # saturation), results polled in submission order
    with Server(slots=slots, resident=resident) as srv:
        for model, p in zip([m for m, _, _ in stream[:2]], params[:2]):   # warm the slots
            srv.poll(srv.submit(model, p))
        tickets = []
        t0 = time.perf_counter()
        for (model, _, arrival), p in zip(stream, params):
            delay = arrival - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            tickets.append(srv.submit(model, p))
        lats, iters, ok, loop_s = [], [], 0, []
        for t in tickets:
            r, lat = srv.poll(t)
            lats.append(lat)
            iters.append(r.iter)
            loop_s.append(r.time - r.power_time)
            ok += r.status == "OPTIMAL"
        wall = time.perf_counter() - t0
        phases = srv.phase_times()
    rate_s = len(stream) / wall
    # one at a time, after the server (so both run with the CUDA context up
    # and the schedule autotuner's choices made): the first `baseline`
    # requests, each a full hpr_optimize, after one untimed solve
    nb = min(baseline, len(stream))

    def solve_one(model, p):
        prob, pc = model.to_c(), p.to_c()
        x, y, z = np.zeros(model.n), np.zeros(model.m), np.zeros(model.n)
        r = _abi.hpr_results()
        r.x, r.y, r.z = _abi.dptr(x), _abi.dptr(y), _abi.dptr(z)
        if lib.hpr_optimize(C.byref(prob), C.byref(pc), C.byref(r)) != 0:
            raise RuntimeError("hpr_optimize failed")

    solve_one(stream[0][0], params[0])
    t0 = time.perf_counter()
    for (model, _, _), p in zip(stream[:nb], params[:nb]):
        solve_one(model, p)
    seq_rate = nb / (time.perf_counter() - t0)
    lats = np.sort(np.asarray(lats))
    return {"solves_per_s": rate_s, "requests": len(stream), "slots": slots,
            "device_resident_loop": bool(resident),
            "arrival_rate": rate or "saturation (all at t=0)",
            "latency_s": {"p50": float(np.percentile(lats, 50)), "p99": float(np.percentile(lats, 99)),
                          "max": float(lats[-1])},
            "optimal": ok, "mean_iterations": float(np.mean(iters)),
            "mean_phase_s": phases,
            "mean_loop_time_s": float(np.mean(loop_s)),
            "one_at_a_time": {"value": seq_rate, "unit": "solves/s", "requests": nb,
                              "how": "hpr_optimize per request, sequentially, after the server run "
                                     "and one untimed solve"},
            "speedup_vs_one_at_a_time": rate_s / seq_rate}


def serving_in_fresh_process(requests, slots=32, baseline=30, timeout=900):
    """`serving_measure` in a new process (``--mode serve``): the server
    must create the process's CUDA context to get a hardware work queue per
    slot and blocking waits, and this process already holds one."""
    cmd = [sys.executable, os.path.abspath(__file__), "--mode", "serve", "--requests", str(requests),
           "--slots", str(slots), "--baseline", str(baseline)]
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"error": f"serving run exceeded {timeout} s"}
    lines = [ln for ln in out.stdout.strip().splitlines() if ln.startswith("{")]
    if out.returncode != 0 or not lines:
        return {"error": f"serving run failed (rc {out.returncode}): {out.stderr.strip()[-300:]}"}
    d = json.loads(lines[-1])
    keep = ("latency_s", "optimal", "mean_iterations", "mean_phase_s", "mean_loop_time_s", "one_at_a_time",
            "speedup_vs_one_at_a_time")
    res = {"solves_per_s": d["value"], "requests": d["steps"], "slots": d["config"]["slots"],
           "device_resident_loop": d["config"]["device_resident_loop"], "arrival_rate": d["config"]["arrival_rate"]}
    res.update({k: d[k] for k in keep})
    return res


def run_serving(args):
    d = serving_measure(args.requests, args.slots, args.rate, args.baseline, resident=args.resident)
    line = {"metric": "solves/s", "value": d["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
            "steps": d["requests"], "warmup": 2, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded serving stream, seed 11)",
            "config": {"workload": "serving stream of small SOCPs: n lognormal (median 400, 50..20000), "
                                   "m = n/2, density 2-5%, 1-200 variable cones of 3-64, half with diagonal Q, "
                                   "tolerance 1e-4 or 1e-6 per request",
                       "slots": args.slots, "arrival_rate": d["arrival_rate"],
                       "device_resident_loop": d["device_resident_loop"]}}
    line.update({k: d[k] for k in ("latency_s", "optimal", "mean_iterations", "mean_phase_s", "mean_loop_time_s",
                                   "one_at_a_time", "speedup_vs_one_at_a_time")})
    print(json.dumps(line))


def run_tts(args):
    """Time to solution at 1e-6 KKT on the benchmark SOCP with the plain FP64
    stream and the reduced-precision streams (FP32 values and gathers; BF16
    values with FP32 accumulation), each with the FP64 finish, and the error
    of each result against the FP64 solution."""
    import numpy as np
    from hprsocp_b200 import Context, HPRSOCP_parameters, instances
    model = instances.config1(1, scale=args.scale)
    out = {}
    ref = None
    for prec in ("fp64", "fp32", "bf16"):
        p = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=200000, time_limit=600, precision=prec)
        with Context(model) as ctx:
            t0 = time.perf_counter()
            r = ctx.solve(p)
            wall = time.perf_counter() - t0
        d = {"status": r.status, "iterations": r.iter, "solve_s": r.time, "wall_s": wall, "kkt": r.residuals,
             "primal_obj": r.primal_obj}
        if ref is None:
            ref = r
        else:
            d["x_rel_err"] = float(np.max(np.abs(r.x - ref.x)) / max(1.0, np.max(np.abs(ref.x))))
            d["y_rel_err"] = float(np.max(np.abs(r.y - ref.y)) / max(1.0, np.max(np.abs(ref.y))))
            d["obj_rel_err"] = abs(r.primal_obj - ref.primal_obj) / max(1.0, abs(ref.primal_obj))
            d["speedup_vs_fp64"] = ref.time / r.time
        out[prec] = d
    line = {"metric": "time to 1e-6 KKT", "value": out["fp32"]["solve_s"], "unit": "s", "n_gpus": 1, "steps": 1,
            "warmup": 0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32/bf16",
            "data": "synthetic (seeded generator, seed 1)",
            "config": {"workload": WORKLOAD, "scale": args.scale,
                       "what": "solve() to stoptol 1e-6 per SpMV precision; residuals, restart and sigma in FP64"},
            "runs": out}
    print(json.dumps(line))


def run_spmv_baseline(args):
    """Library SpMV stand-in for the reference's GPU path: cuSPARSE CSR SpMV
    (through torch.sparse CSR matvec) on the benchmark's A and A', timed
    with CUDA events; the fused iteration does both products and every
    epilogue in one pass each."""
    import torch
    from hprsocp_b200 import instances
    model = instances.config1(1, scale=args.scale)
    dev = torch.device("cuda")
    out = {}
    for name, M in (("A", model.A), ("AT", model.AT)):
        T = torch.sparse_csr_tensor(torch.from_numpy(M.indptr.astype("int32")), torch.from_numpy(M.indices.astype("int32")),
                                    torch.from_numpy(M.data), size=M.shape, device=dev)
        x = torch.rand(M.shape[1], dtype=torch.float64, device=dev)
        for _ in range(5):
            y = T @ x
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(50):
            y = T @ x
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 50
        nbytes = M.nnz * 12 + (M.shape[0] + 1) * 4 + (M.shape[0] + M.shape[1]) * 8
        out[name] = {"ms": ms, "GBs": nbytes / ms / 1e6, "nnz": int(M.nnz)}
    print(json.dumps({"metric": "cuSPARSE CSR SpMV (torch.sparse matvec)", "config": {"workload": WORKLOAD},
                      "spmv": out, "sum_ms": out["A"]["ms"] + out["AT"]["ms"]}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="shrink the instance (testing only)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--mode", default="iterate", choices=["iterate", "serve", "tts", "spmv-baseline"],
                    help="serve: the small-SOCP serving stream; tts: time to 1e-6 per SpMV precision")
    ap.add_argument("--requests", type=int, default=400, help="serve: requests in the stream")
    ap.add_argument("--slots", type=int, default=32, help="serve: concurrent solver slots")
    ap.add_argument("--rate", type=float, default=0.0, help="serve: Poisson arrivals/s (0 = saturation)")
    ap.add_argument("--baseline", type=int, default=60, help="serve: requests solved one at a time")
    ap.add_argument("--resident", action="store_true",
                    help="serve: small problems' solve loops in the device-resident request loop")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving summary of the default line")
    ap.add_argument("--workload", default="config1", choices=sorted(WORKLOADS),
                    help="iterate: config1 (the benchmark) or config2 (the Q path at n=200k)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.mode == "serve":
        run_serving(args)
        return
    if args.mode == "tts":
        run_tts(args)
        return
    if args.mode == "spmv-baseline":
        run_spmv_baseline(args)
        return

    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return
        run_reference(args, make_model(args))
        return

    rank, world, dist = dist_init(args.gpus)
    import ctypes as C
    from hprsocp_b200 import Context, HPRSOCP_parameters, _abi
    model = make_model(args)
    has_q = model.Q is not None or model.F is not None or model.q_diag is not None
    if has_q:
        args.no_serve = True  # the serving summary belongs to the benchmark line
    dev = int(os.environ.get("LOCAL_RANK", "0")) if dist is not None else 0

    # ---- device-resident iterations
    ctx = Context(model, device=dev)
    info = ctx.scale(HPRSOCP_parameters(verbose=False))
    lam = ctx.power_A() * 1.05
    lamq = ctx.power_Q() * 1.05 if has_q else 0.0
    sigma = info["norm_b"] / info["norm_c"]
    ctx.set_sigma_lambda(sigma, lam, lamq)
    ctx.set_inner(0)
    with ClockSampler(dev) as clk:
        # clocks are sampled from the warm-up on; a timed region shorter than
        # the sampling period is followed by untimed iterations until two
        # samples have been taken under load
        clk.wait_samples(1)
        first = len(clk.lines)
        ctx.iterate(args.warmup, False)
        barrier(dist)
        ctx.iterate(args.steps, True)  # device-timed with CUDA events inside
        ms, launches = ctx.last_iterate()
        while clk.proc and clk.proc.poll() is None and len(clk.lines) - first < 2:
            ctx.iterate(20, False)
    clocks = clk.summary(first)
    flushed = None
    if has_q:
        flushed = l2_flushed_iterations(ctx, dev, min(args.steps, 200))
    ms = dist_max(dist, ms)
    bytes_iter = ctx.iteration_bytes()
    ctx.close()
    value = aggregate(world, args.steps, ms)
    per_iter_ms = ms / args.steps
    peak, peak_kind = measured_peak()
    achieved = bytes_iter / (per_iter_ms / 1e3) / 1e9

    # ---- end to end through the C ABI from host buffers
    e2e = None
    if not args.no_e2e:
        lib = _abi.load_library()
        prob = model.to_c()
        p = HPRSOCP_parameters(verbose=False, max_iter=args.steps, stoptol=0.0, check_iter=150,
                               print_frequency=10**9).to_c()
        m, n = model.m, model.n
        import numpy as np
        x, y, z = np.zeros(n), np.zeros(m), np.zeros(n)
        r = _abi.hpr_results()
        r.x, r.y, r.z = _abi.dptr(x), _abi.dptr(y), _abi.dptr(z)
        barrier(dist)
        t0 = time.perf_counter()
        rc = lib.hpr_optimize(C.byref(prob), C.byref(p), C.byref(r))
        dt = time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError(f"hpr_optimize failed: {rc}")
        dt = dist_max(dist, dt)
        h2d = model.nbytes()
        d2h = int(x.nbytes + y.nbytes + z.nbytes)
        e2e = {"value": world * r.iter / dt, "unit": "iter/s", "h2d_bytes_per_step": h2d / max(r.iter, 1),
               "d2h_bytes_per_step": d2h / max(r.iter, 1), "h2d_bytes_per_solve": h2d, "d2h_bytes_per_solve": d2h,
               "what": "hpr_optimize from host arrays: upload + scaling + power iteration + "
                       f"{r.iter} iterations (checks every 150) + unscaled solution read-back; "
                       "inputs are copied once per solve, so bytes per step = bytes per solve / iterations",
               "seconds": dt,
               # where the call's time went: the HPR loop (power iteration
               # included, as in the reference's solve time) and the rest
               # (upload, scaling, unscaled read-back)
               "phases_s": {"power_iteration": r.power_time, "hpr_loop_after_power": r.time - r.power_time,
                            "upload_scaling_readback": dt - r.time}}

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    serving = None
    if not args.no_serve:
        # a fixed 200-request sample of the serving stream (config 4) through
        # the server, against one-at-a-time solves (before the CPU baseline,
        # whose host threads would compete with the server's)
        serving = serving_in_fresh_process(200, slots=32, baseline=30)
    cpu = None
    if not args.no_cpu:
        iters = 3
        cpu_rate = cpu_iteration_rate(model, iters=iters, threads=0)
        cpu = {"value": cpu_rate, "unit": "iter/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"{iters} HPR iterations of the {args.workload} instance on the oracle (all host threads)",
               "one_thread": {"value": cpu_iteration_rate(model, iters=1, threads=1), "unit": "iter/s",
                              "cores": 1, "sample": "1 HPR iteration on one thread (the reference's CPU "
                                                    "path is single-threaded)"}}
    traffic = None
    tfile = os.path.join(ROOT, "profiles", WORKLOADS[args.workload]["traffic_file"])
    if os.path.exists(tfile):
        try:
            traffic = float(open(tfile).read().split()[0])
        except (ValueError, IndexError):
            traffic = None
    line = {
        "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_iter_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": f"synthetic (seeded generator, seed {WORKLOADS[args.workload]['seed']})",
        "config": arm_config(args, world),
        "hbm_gbs": achieved,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "algorithmic_bytes_per_iter": bytes_iter,
                     "kernel": WORKLOADS[args.workload]["kernel"]},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clocks,
        "serving": serving,
    }
    if flushed is not None:
        fl_ms = flushed / 1.0
        line["l2_flushed"] = {"ms_per_step": fl_ms, "value": 1e3 / fl_ms, "unit": "iter/s",
                              "hbm_gbs": bytes_iter / (fl_ms / 1e3) / 1e9,
                              "what": "single iterations, each after a 512 MB device write that evicts L2, "
                                      "timed with the iteration's CUDA events (launch latency included)"}
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
