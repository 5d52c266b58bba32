"""Benchmark of the B200 path tracker on the large single system:
n = 16 variables, all degrees 2, 24 distinct monomials (of 153) per
equation with complex normal coefficients, 65,536 total-degree paths.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one pass of the tracker over all 65,536 paths of the system
(start_solution + track + Cauchy end game + classify numerics), i.e. the
per-path work of one solve(). Metric: paths/s (higher is better).

  value   mixed-precision persistent tracker, inputs (the compiled sparse
          table) resident in device memory, timed with CUDA events on the
          launching stream, L2 flushed (256 MiB written) between timed steps
  e2e     the same metric through the public C ABI: phc_solve_sparse on one
          GPU (host table in; the kernel writes each path's results to mapped
          host memory and the host copies and books it in path order while
          later paths are tracked), wall clock per call; on N GPUs each
          rank calls phc_solve_paths on its path range with host buffers,
          the records are gathered to rank 0 and phc_finish_solve runs the
          bookkeeping there
  fp64    the plain all-FP64 tracker, same schedule and timing as value (the
          baseline of the mixed-precision target)

Under torchrun the system's paths are split into contiguous ranges, one per
rank (src/solve.f90:190-208: paths are independent), so the total work is
fixed (strong scaling); times are the max over ranks, and no collective
touches the data path. The key `replicas` times one whole system per rank
(weak scaling) beside it. --impl reference times the reference's CPU
algorithm (the C++ restatement under oracle/, all host threads) on the same
system, a bounded sample of its paths per step.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "paths/s mixed vs FP64 at <=1e-10 endpoint err"
WORKLOAD = ("large single system: n=16, degrees 2, 24 of 153 monomials per equation, complex "
            "normal coefficients, 65536 total-degree paths, end game on")
WORKLOAD_N10 = ("batched paths: n=10, degrees 2, 20 of 66 monomials per equation, complex "
                "normal coefficients, 1024 total-degree paths, end game on")
# paths of the restatement per step of the reference arm (a bounded sample
# of the 65,536: a window of consecutive paths, a different one each step)
REF_SAMPLE_PATHS = 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-n10", action="store_true",
                    help="skip the secondary n=10, 1024-path measurement")
    ap.add_argument("--serving-systems", type=int, default=4096,
                    help="systems in the serving stream (0 skips the serving leg)")
    ap.add_argument("--replica-steps", type=int, default=3,
                    help="N > 1: timed steps of the replicas key (one whole system per "
                         "rank); 0 skips it")
    ap.add_argument("--max-paths", type=int, default=0,
                    help="track only the first N paths of the system (a small case for "
                         "profiler captures; the line says so)")
    ap.add_argument("--configs", action="store_true",
                    help="instead of the benchmark line, measure the other single-system "
                         "configurations (n=4 dense quadratic; n=4 singular cubic; n=10 with "
                         "1024 paths; n=16 with 65536 paths): one JSON line each")
    ap.add_argument("--config-filter", default="",
                    help="with --configs: only the configurations whose description "
                         "contains this text")
    ap.add_argument("--no-tune", action="store_true",
                    help="default launch configuration instead of the autotuner's "
                         "(for profiling: the timed launches then follow the warm-up directly)")
    ap.add_argument("--serving-only", action="store_true",
                    help="only the serving leg (--serving-systems systems, one GPU): "
                         "one JSON line (for profiling the batch kernels)")
    ap.add_argument("--warps-per-block", type=int, default=0,
                    help="with --no-tune: warps per block of both arms (0: the default)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def workload():
    from polyhomocont_b200 import workloads as W
    return W.cfg5()


def sample_windows(npaths, count, nwin):
    """nwin windows of `count` consecutive 1-based paths, spread evenly over
    1..npaths (the first starts at path 1, the last ends at npaths)."""
    if nwin <= 1:
        return [1]
    span = npaths - count
    return [1 + (span * w) // (nwin - 1) for w in range(nwin)]


# ---------------------------------------------------------------------------
# CPU baseline: the C++ restatement of the reference (oracle/), all threads
# ---------------------------------------------------------------------------
def cpu_paths_per_s(min_seconds=10.0, max_windows=16):
    """The restatement on all host threads over windows of the system's
    paths (REF_SAMPLE_PATHS each, spread over the range) until about
    min_seconds have passed."""
    from oracle import oracle as O
    from polyhomocont_b200 import workloads as W
    O.build()
    n, eqs = workload()
    s = W.build(lambda: O.SparseSystem(fast=True), n, eqs)
    threads = os.cpu_count() or 1
    npaths = int(O.lib(fast=True).orc_bezout(s.h))
    wins = sample_windows(npaths, REF_SAMPLE_PATHS, max_windows)
    done, t0 = 0, time.perf_counter()
    for k0 in wins:
        O.solve_paths(s, k0=k0, count=REF_SAMPLE_PATHS, nthreads=threads)
        done += 1
        el = time.perf_counter() - t0
        if el >= min_seconds:
            break
    paths = done * REF_SAMPLE_PATHS
    return (paths / el, threads,
            f"{paths} of the {npaths} paths ({done} windows of {REF_SAMPLE_PATHS} consecutive "
            f"paths spread over the range), {threads} threads", el)


def cpu_serving_baseline(nsys_max=512, max_seconds=10.0):
    """The serving stream on the host cores: the C++ restatement of the
    reference solves one system per thread (each solve single-threaded, the
    systems spread over all cores), over the first systems of the stream
    until about max_seconds have passed."""
    import concurrent.futures as cf
    from oracle import oracle as O
    from polyhomocont_b200 import workloads as W
    O.build()
    threads = os.cpu_count() or 1
    systems = [W.build(lambda: O.SparseSystem(fast=True), *W.stream_system(i))
               for i in range(nsys_max)]
    done = paths = 0
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        for i0 in range(0, nsys_max, threads):
            batch = systems[i0:i0 + threads]
            for res, st in ex.map(lambda s: O.solve(s, nthreads=1), batch):
                done += 1
                paths += res.npaths
            if time.perf_counter() - t0 >= max_seconds:
                break
    el = time.perf_counter() - t0
    return {"systems_per_s": done / el, "paths_per_s": paths / el, "cores": threads,
            "kind": "port",
            "sample": f"first {done} systems of the stream, one system per thread, "
                      f"{threads} threads (C++ restatement of the reference, -O3)"}


def run_reference(args):
    """The reference's algorithm on the host cores (the C++ restatement,
    -O3, all threads; no Fortran compiler exists for the reference itself)
    on the same system: each step tracks a window of REF_SAMPLE_PATHS
    consecutive paths, the windows spread over the 65,536 paths."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    from polyhomocont_b200 import workloads as W
    O.build()
    n, eqs = workload()
    s = W.build(lambda: O.SparseSystem(fast=True), n, eqs)
    threads = os.cpu_count() or 1
    npaths = int(O.lib(fast=True).orc_bezout(s.h))
    steps = max(args.steps, 1)
    wins = sample_windows(npaths, REF_SAMPLE_PATHS, max(args.warmup, 0) + steps)
    for k0 in wins[:max(args.warmup, 0)]:
        O.solve_paths(s, k0=k0, count=REF_SAMPLE_PATHS, nthreads=threads)
    t0 = time.perf_counter()
    for k0 in wins[max(args.warmup, 0):]:
        O.solve_paths(s, k0=k0, count=REF_SAMPLE_PATHS, nthreads=threads)
    el = time.perf_counter() - t0
    v = REF_SAMPLE_PATHS * steps / el
    sample = (f"{REF_SAMPLE_PATHS} consecutive paths per step, windows spread over the "
              f"{npaths} paths, {threads} threads (C++ restatement of the reference, -O3; "
              "no Fortran compiler for the reference itself)")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "paths/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "paths": npaths,
                   "paths_per_step": REF_SAMPLE_PATHS, "threads": threads},
        "cpu_baseline": {"value": v, "unit": "paths/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "paths/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one
# mixed-precision launch of the tracker on the first 6,144 paths of the
# n = 16 system, from
#   ncu --set full --clock-control none -k regex:track_kernel -s 6 -c 2
#   python bench.py --max-paths 6144 --no-tune --steps 1 --warmup 3 --no-cpu
#       --no-e2e --no-n10 --serving-systems 0
# The kernel is compute- and latency-bound: its DRAM traffic is the table,
# the kernel's code and the path records, most of which stay in L2.
NCU_DRAM_BYTES = {"bytes": 204288, "paths": 6144}
SCHED_NAMES = {0: "grid", 1: "persistent"}


# ---------------------------------------------------------------------------
# serving: stream of random sparse systems (n ~ U{2..8}, d_i ~ U{2,3})
# ---------------------------------------------------------------------------


def serving(P, W, nsys, device, load=0.7, nslots=16, max_batch_systems=64,
            max_batch_paths=1 << 15):
    systems = [W.build(P.SparseSystem, *W.stream_system(i)) for i in range(nsys)]
    npaths = sum(s.bezout() for s in systems)
    cfg = dict(device=device, nslots=nslots, max_batch_systems=max_batch_systems,
               max_batch_paths=max_batch_paths)

    def drain(srv, tickets):
        lat = []
        for t in tickets:
            srv.wait(t, 600000)
            res, st, l = srv.result(t)
            if st != 0:
                raise RuntimeError(f"serving request failed with status {st}")
            lat.append(l)
        return np.asarray(lat)

    # capacity: everything submitted at once
    srv = P.Server(**cfg)
    t0 = time.perf_counter()
    tickets = [srv.submit(s)[0] for s in systems]
    drain(srv, tickets)
    cap = nsys / (time.perf_counter() - t0)
    srv.close()
    # Poisson arrivals at the given fraction of capacity
    rate = load * cap
    arrivals = W.poisson_arrivals(nsys, rate)
    srv = P.Server(**cfg)
    t0 = time.perf_counter()
    tickets = []
    for s, ta in zip(systems, arrivals):
        now = time.perf_counter() - t0
        if ta > now:
            time.sleep(ta - now)
        tickets.append(srv.submit(s)[0])
    lat = drain(srv, tickets)
    elapsed = time.perf_counter() - t0
    stats = srv.stats()
    srv.close()
    return {"systems": nsys, "paths": npaths, "capacity_systems_per_s": cap,
            "arrival_rate_per_s": rate, "load": load,
            "systems_per_s": nsys / elapsed, "paths_per_s": npaths / elapsed,
            "latency_p50_ms": 1e3 * float(np.percentile(lat, 50)),
            "latency_p99_ms": 1e3 * float(np.percentile(lat, 99)),
            "latency_max_ms": 1e3 * float(lat.max()), "batches": stats["batches"],
            "slots": cfg["nslots"]}


def run_serving_only(args):
    """The serving leg alone on GPU 0: one JSON line."""
    import torch
    import polyhomocont_b200 as P
    from polyhomocont_b200 import _abi
    from polyhomocont_b200 import workloads as W
    from polyhomocont_b200 import build as B

    if not os.path.exists(_abi.LIB_PATH):
        B.build()
    torch.cuda.set_device(0)
    serve = serving(P, W, max(args.serving_systems, 1), 0)
    print(json.dumps({"impl": "ours", "metric": "serving stream (systems/s, latency)",
                      "serving": serve}), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_configs(args):
    """Mixed against plain FP64 on the other single-system configurations,
    on one GPU: device-timed paths/s of both (each autotuned, L2 flushed
    between timed launches), endpoint agreement and classification, and for
    the singular cubic the error of the singular endpoints against the
    exactly known root r. One JSON line per configuration."""
    import torch
    import polyhomocont_b200 as P
    from polyhomocont_b200 import _abi
    from polyhomocont_b200 import workloads as W
    from polyhomocont_b200 import build as B

    if not os.path.exists(_abi.LIB_PATH):
        B.build()
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    n3, eqs3, r3 = W.singular_cubic()
    cases = [
        ("plain method: n=4, degrees 2, all 15 monomials of degree <= 2, 16 paths",
         W.dense_quadratic(), None),
        ("singular endpoints: n=4, degrees 3, (x_j - r_j)^2 and ^3 terms, 81 paths, "
         "16 ending at the known root r", (n3, eqs3), r3),
        (WORKLOAD_N10, W.cfg2(), None),
        ("large single system: n=16, degrees 2, 24 of 153 monomials per equation, "
         "65536 paths", W.cfg5(), None),
    ]
    for name, (n, eqs), root in cases:
        if args.config_filter and args.config_filter not in name:
            continue
        s = W.build(P.SparseSystem, n, eqs)
        npaths = s.bezout()
        if args.max_paths > 0:
            npaths = min(npaths, args.max_paths)
        arms = {}
        for prec, key in ((P.PHC_PREC_MIXED, "mixed"), (P.PHC_PREC_FP64, "fp64")):
            if args.no_tune:
                g = P.default_gpu_options(prec)
            else:
                g, _ = P.autotune(s, gpu=P.default_gpu_options(prec))
            plan = P.Plan(s, gpu=g)
            out = torch.zeros(npaths * 96, dtype=torch.uint8, device=dev)
            z = torch.zeros(npaths * (n + 1) * 2, dtype=torch.float64, device=dev)
            for _ in range(max(args.warmup, 3)):
                plan.launch(1, npaths, out.data_ptr(), z.data_ptr(), stream.cuda_stream)
            torch.cuda.synchronize()
            total = 0.0
            for _ in range(args.steps):
                flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                plan.launch(1, npaths, out.data_ptr(), z.data_ptr(), stream.cuda_stream)
                b.record(stream)
                b.synchronize()
                total += a.elapsed_time(b) * 1e-3
            paths = np.frombuffer(out.cpu().numpy().tobytes(), dtype=P.PATH_DTYPE)
            zz = z.cpu().numpy().view(np.complex128).reshape(npaths, n + 1)
            arms[key] = {"paths_per_s": npaths * args.steps / total,
                         "ms_per_launch": 1e3 * total / args.steps,
                         "schedule": SCHED_NAMES[g.schedule],
                         "warps_per_block": plan.config()["warps_per_block"],
                         "paths": paths, "z": zz}
            plan.close()
        pm, pd = arms["mixed"]["paths"], arms["fp64"]["paths"]
        same = all(np.array_equal(pm[k], pd[k]) for k in
                   ("status", "winding_number", "at_infinity", "singular", "is_real"))
        fin = (pd["status"] == 0) & (pd["at_infinity"] == 0) & (pd["singular"] == 0)
        xm = arms["mixed"]["z"][:, :n] / arms["mixed"]["z"][:, n:n + 1]
        xd = arms["fp64"]["z"][:, :n] / arms["fp64"]["z"][:, n:n + 1]
        err = 0.0
        if fin.any():
            err = float(np.max(np.max(np.abs(xm[fin] - xd[fin]), axis=1) /
                               np.maximum(1.0, np.max(np.abs(xd[fin]), axis=1))))
        line = {"impl": "ours", "config": {"workload": name, "paths": npaths,
                                           "paths_of_system": s.bezout(),
                                           "tuned": not args.no_tune},
                "metric": "paths/s, mixed vs plain FP64, device-timed, L2 flushed",
                "steps": args.steps, "warmup": args.warmup,
                "mixed": {k: v for k, v in arms["mixed"].items() if k not in ("paths", "z")},
                "fp64": {k: v for k, v in arms["fp64"].items() if k not in ("paths", "z")},
                "mixed_vs_fp64": arms["mixed"]["paths_per_s"] / arms["fp64"]["paths_per_s"],
                "classification_identical": bool(same),
                "regular_endpoint_max_rel_err_mixed_vs_fp64": err,
                "counts": {"regular": int(fin.sum()),
                           "singular": int(((pd["status"] == 0) & (pd["singular"] != 0)
                                            & (pd["at_infinity"] == 0)).sum()),
                           "infinite": int(((pd["status"] == 0) & (pd["at_infinity"] != 0)).sum()),
                           "failed": int((pd["status"] != 0).sum())}}
        if root is not None:
            def root_err(p, x):
                sing = (p["status"] == 0) & (p["singular"] != 0) & (p["at_infinity"] == 0)
                if not sing.any():
                    return None
                return float(np.max(np.max(np.abs(x[sing] - root[None, :]), axis=1)) /
                             max(1.0, float(np.max(np.abs(root)))))
            line["singular_endpoint_err_vs_exact_root"] = {"mixed": root_err(pm, xm),
                                                           "fp64": root_err(pd, xd)}
        print(json.dumps(line), flush=True)


def time_launches(stream, flush, launch, k):
    """Total device time (s) of k launches, each timed with CUDA events on
    the launching stream after an L2 flush (256 MiB written)."""
    import torch
    total = 0.0
    for _ in range(k):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        launch()
        b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b) * 1e-3
    return total


def endpoint_agreement(n, pm, zm, pd, zd):
    """(max relative error of the regular finite endpoints of two runs,
    whether their classification is identical)."""
    fin = (pd["status"] == 0) & (pd["at_infinity"] == 0)
    err = 0.0
    if fin.any():
        xm = zm[fin, :n] / zm[fin, n:n + 1]
        xd = zd[fin, :n] / zd[fin, n:n + 1]
        err = float(np.max(np.max(np.abs(xm - xd), axis=1) /
                           np.maximum(1.0, np.max(np.abs(xd), axis=1))))
    same = all(np.array_equal(pm[k], pd[k]) for k in
               ("status", "winding_number", "at_infinity", "singular", "is_real"))
    return err, same


def measure_n10(P, W, dev, stream, flush, steps, warmup, local):
    """The n=10, 1024-path system on one GPU: device-timed paths/s of both
    precisions, each autotuned (a secondary key of the line)."""
    import torch
    n, eqs = W.cfg2()
    s = W.build(P.SparseSystem, n, eqs)
    npaths = s.bezout()
    out = {}
    for prec, key in ((P.PHC_PREC_MIXED, "mixed"), (P.PHC_PREC_FP64, "fp64")):
        g, _ = P.autotune(s, gpu=P.default_gpu_options(prec, device=local))
        plan = P.Plan(s, gpu=g)
        o = torch.zeros(npaths * 96, dtype=torch.uint8, device=dev)
        z = torch.zeros(npaths * (n + 1) * 2, dtype=torch.float64, device=dev)

        def launch():
            plan.launch(1, npaths, o.data_ptr(), z.data_ptr(), stream.cuda_stream)
        for _ in range(max(warmup, 3)):
            launch()
        torch.cuda.synchronize()
        t = time_launches(stream, flush, launch, steps)
        out[key] = {"value": npaths * steps / t, "unit": "paths/s",
                    "ms_per_step": 1e3 * t / steps, "schedule": SCHED_NAMES[g.schedule],
                    "warps_per_block": plan.config()["warps_per_block"]}
        plan.close()
    out["mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["workload"] = WORKLOAD_N10
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.configs:
        run_configs(args)
        return
    if args.serving_only:
        run_serving_only(args)
        return
    rank, world, local = dist_env()
    import torch
    import polyhomocont_b200 as P
    from polyhomocont_b200 import _abi, flops, shard
    from polyhomocont_b200 import workloads as W
    from polyhomocont_b200 import build as B

    if not os.path.exists(_abi.LIB_PATH):
        B.build()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
        pg = dist

    def barrier():
        if pg is not None:
            pg.barrier()

    def reduce_over_ranks(x, op):
        if pg is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=op)
        return float(t.item())

    def max_over_ranks(x):
        return reduce_over_ranks(x, pg.ReduceOp.MAX if pg else None)

    def sum_over_ranks(x):
        return reduce_over_ranks(x, pg.ReduceOp.SUM if pg else None)

    L = _abi.lib()
    p64, p32 = ctypes.c_double(), ctypes.c_double()
    st = L.phc_measure_fma_peaks(local, ctypes.byref(p64), ctypes.byref(p32))
    if st != 0:
        raise RuntimeError(f"phc_measure_fma_peaks: {_abi.last_error()}")
    peak64, peak32 = p64.value, p32.value

    # one system; this rank's contiguous range of its paths
    n, eqs = workload()
    sysP = W.build(P.SparseSystem, n, eqs)
    npaths_sys = sysP.bezout()
    npaths = min(npaths_sys, args.max_paths) if args.max_paths > 0 else npaths_sys
    k0, count = shard.path_range(npaths, rank, world)
    t, _ = sysP.table()
    T = sysP.total_terms()
    hexps = np.ctypeslib.as_array(t.hexps, shape=(T * (n + 1),)).reshape(T, n + 1).copy()
    model = flops.unit_model(n, sysP.degrees(), hexps)

    # both arms get their launch configuration from the autotuner (timed on
    # a sample of the system's paths, before and outside the timed region);
    # the two arms then differ only in precision and in what the tuner chose
    if args.no_tune:
        wpb = {"warps_per_block": args.warps_per_block} if args.warps_per_block > 0 else {}
        g_mixed = P.default_gpu_options(P.PHC_PREC_MIXED, device=local, **wpb)
        g_fp64 = P.default_gpu_options(P.PHC_PREC_FP64, device=local, **wpb)
        tune_m = {"sample_paths": 0, "candidates": []}
    else:
        g_mixed, tune_m = P.autotune(sysP, gpu=P.default_gpu_options(P.PHC_PREC_MIXED,
                                                                     device=local))
        g_fp64, _ = P.autotune(sysP, gpu=P.default_gpu_options(P.PHC_PREC_FP64,
                                                               device=local))
    plan_m = P.Plan(sysP, gpu=g_mixed)
    plan_d = P.Plan(sysP, gpu=g_fp64)
    out_m = torch.zeros(max(count, 1) * 96, dtype=torch.uint8, device=dev)
    z_m = torch.zeros(max(count, 1) * (n + 1) * 2, dtype=torch.float64, device=dev)
    out_d = torch.zeros_like(out_m)
    z_d = torch.zeros_like(z_m)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream

    def launch_m():
        plan_m.launch(k0, count, out_m.data_ptr(), z_m.data_ptr(), sptr)

    def launch_d():
        plan_d.launch(k0, count, out_d.data_ptr(), z_d.data_ptr(), sptr)

    for _ in range(max(args.warmup, 3)):
        launch_m()
        launch_d()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    t_mixed = time_launches(stream, flush, launch_m, args.steps)
    torch.cuda.synchronize()
    barrier()
    t_fp64 = time_launches(stream, flush, launch_d, args.steps)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    t_mixed_max = max_over_ranks(t_mixed)
    t_fp64_max = max_over_ranks(t_fp64)

    value = npaths * args.steps / t_mixed_max
    v_fp64 = npaths * args.steps / t_fp64_max

    # results of the last runs: counters for the flop model, endpoints
    pm = np.frombuffer(out_m.cpu().numpy().tobytes(), dtype=P.PATH_DTYPE)[:count]
    pd = np.frombuffer(out_d.cpu().numpy().tobytes(), dtype=P.PATH_DTYPE)[:count]
    zm = z_m.cpu().numpy().view(np.complex128).reshape(-1, n + 1)[:count]
    zd = z_d.cpu().numpy().view(np.complex128).reshape(-1, n + 1)[:count]
    err, same_class = endpoint_agreement(n, pm, zm, pd, zd)
    err = max_over_ranks(err)
    same_class = max_over_ranks(0.0 if same_class else 1.0) == 0.0
    f64m, f32m = flops.path_flops(model, pm, mixed=True)
    f64d, _ = flops.path_flops(model, pd, mixed=False)
    per_launch_s = t_mixed / args.steps  # this rank's launch
    achieved = (f64m + f32m) / per_launch_s / 1e12
    t_at_peak = f64m / (peak64 * 1e12) + f32m / (peak32 * 1e12)
    peak_eff = (f64m + f32m) / t_at_peak / 1e12 if t_at_peak > 0 else None
    fp64_achieved = f64d / (t_fp64 / args.steps) / 1e12
    units = {k: int(sum_over_ranks(float(pm[k].astype(np.int64).sum()))) for k in
             ("n_tangent", "n_newton", "n_refine", "n_eval", "n_cond", "n_fp64_retry")}
    units_d = {k: int(sum_over_ranks(float(pd[k].astype(np.int64).sum()))) for k in
               ("n_tangent", "n_newton", "n_refine", "n_eval", "n_cond")}
    pred_corr = units["n_tangent"] + units["n_newton"]
    fp64_share = units["n_fp64_retry"] / pred_corr if pred_corr else None
    counts = {"regular": int(((pd["status"] == 0) & (pd["at_infinity"] == 0) &
                              (pd["singular"] == 0)).sum()),
              "singular": int(((pd["status"] == 0) & (pd["singular"] != 0) &
                               (pd["at_infinity"] == 0)).sum()),
              "infinite": int(((pd["status"] == 0) & (pd["at_infinity"] != 0)).sum()),
              "failed": int((pd["status"] != 0).sum())}
    counts = {k: int(sum_over_ranks(v)) for k, v in counts.items()}

    # end to end through the public ABI, host buffers
    e2e = None
    if not args.no_e2e:
        def pinned(shape, dtype):
            nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
            buf = torch.empty(max(nbytes, 1), dtype=torch.uint8, pin_memory=True)
            arr = buf.numpy().view(dtype)[:int(np.prod(shape))].reshape(shape)
            arr.fill(0)
            pinned.keep.append(buf)
            return arr
        pinned.keep = []
        table_bytes = plan_m.config()["table_bytes"]
        if world == 1 and npaths == npaths_sys:
            bufs = P._result_buffers(n, npaths, alloc=pinned)

            def e2e_step():
                res, _ = P.solve(sysP, gpu=g_mixed, buffers=bufs)
                return res
            how = ("phc_solve_sparse: host table in; each path's results written by the "
                   "kernel to mapped host memory, copied into page-locked caller buffers and "
                   "booked (host bookkeeping in path order) while later paths are tracked")
        else:
            def runner(kk, cc):
                p_, z_, x_, st_ = P.solve_paths(sysP, gpu=g_mixed, k0=kk, count=cc)
                if st_ != 0:
                    raise RuntimeError(f"solve_paths: status {st_}")
                return p_, z_, x_

            def e2e_step():
                return shard.solve_sharded(sysP, rank, world, gpu=g_mixed, runner=runner,
                                           npaths=npaths)
            how = ("phc_solve_paths per rank on its path range (host buffers), records "
                   "gathered to rank 0, phc_finish_solve there")
        for _ in range(2):
            e2e_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            res = e2e_step()
        t_e2e = time.perf_counter() - t0
        barrier()
        t_e2e = max_over_ranks(t_e2e)
        e2e = {"value": npaths * args.steps / t_e2e, "unit": "paths/s",
               "h2d_bytes_per_step": table_bytes * world,
               "d2h_bytes_per_step": npaths * (96 + 16 * (n + 1) + 16 * n),
               "ms_per_step": 1e3 * t_e2e / args.steps, "path": how}
        if rank == 0 and res is not None:
            e2e.update({"nsolutions": int(res.nsolutions), "ninfinite": int(res.ninfinite),
                        "nfailed": int(res.nfailed)})

    # one whole system per rank (weak scaling), beside the split above
    replicas = None
    if world > 1 and args.replica_steps > 0:
        out_r = torch.zeros(npaths * 96, dtype=torch.uint8, device=dev)
        z_r = torch.zeros(npaths * (n + 1) * 2, dtype=torch.float64, device=dev)

        def launch_r():
            plan_m.launch(1, npaths, out_r.data_ptr(), z_r.data_ptr(), sptr)
        launch_r()
        torch.cuda.synchronize()
        barrier()
        t_r = max_over_ranks(time_launches(stream, flush, launch_r, args.replica_steps))
        replicas = {"value": npaths * world * args.replica_steps / t_r, "unit": "paths/s",
                    "steps": args.replica_steps, "ms_per_step": 1e3 * t_r / args.replica_steps,
                    "scaling": "weak",
                    "parallelism": f"{world} replicas (one whole system per GPU)"}
        del out_r, z_r

    n10 = None
    if rank == 0 and not args.no_n10:
        n10 = measure_n10(P, W, dev, stream, flush, args.steps, args.warmup, local)

    serve = None
    if args.serving_systems > 0 and rank == 0:
        serve = serving(P, W, args.serving_systems, local)
        if not args.no_cpu and world == 1:
            serve["cpu_baseline"] = cpu_serving_baseline()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, cores, sample, el = cpu_paths_per_s()
        cpu = {"value": v, "unit": "paths/s", "cores": cores, "kind": "port",
               "sample": sample + " (C++ restatement of the reference, -O3)"}

    if rank == 0:
        cfg = plan_m.config()
        traffic = NCU_DRAM_BYTES["bytes"] * count / NCU_DRAM_BYTES["paths"]
        line = {
            "metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_mixed_max / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32+f64 (complex)",
            "data": "synthetic (seeded reference generator)",
            "config": {"workload": WORKLOAD if npaths == npaths_sys else
                       f"{WORKLOAD}; first {npaths} paths only",
                       "paths": npaths, "paths_per_rank": count, "precision": "mixed",
                       "schedule": SCHED_NAMES[g_mixed.schedule],
                       "warps_per_block": cfg["warps_per_block"], "chunk": g_mixed.chunk,
                       "grid": cfg["grid"], "row_width": cfg["nm"],
                       "tuned_by": ("defaults (--no-tune)" if args.no_tune else "phc_autotune on "
                                    f"{tune_m['sample_paths']} paths, "
                                    f"{len(tune_m['candidates'])} candidates"),
                       "l2": "flushed between timed steps (256 MiB write)",
                       "parallelism": (f"{world} GPUs, contiguous path ranges of one system"
                                       if world > 1 else "one GPU")},
            "fp64_plain": {"value": v_fp64, "unit": "paths/s",
                           "schedule": SCHED_NAMES[g_fp64.schedule],
                           "warps_per_block": plan_d.config()["warps_per_block"],
                           "chunk": g_fp64.chunk,
                           "ms_per_step": 1e3 * t_fp64_max / args.steps,
                           "achieved_tflops": fp64_achieved,
                           "frac_of_fp64_peak": fp64_achieved / peak64,
                           "units": units_d},
            "mixed_vs_fp64": value / v_fp64,
            "endpoint_max_rel_err_mixed_vs_fp64": err,
            "classification_identical_mixed_vs_fp64": bool(same_class),
            "counts": counts,
            "units": dict(units, fp64_share_of_predictor_corrector=fp64_share),
            "roofline": {"bound": "fp64+fp32 CUDA-core pipes (no tensor cores, not HBM)",
                         "achieved": achieved, "peak": peak_eff, "unit": "TFLOP/s",
                         "frac": achieved / peak_eff if peak_eff else None,
                         "traffic": traffic,
                         "traffic_source": (
                             "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                             f"mixed launch on the first {NCU_DRAM_BYTES['paths']} paths of "
                             f"this system, scaled by paths to this launch's {count}"),
                         "peak_fp64_tflops": peak64, "peak_fp32_tflops": peak32,
                         "peak_source": "measured live (phc_measure_fma_peaks FMA loop); "
                                        "blend weighted by the launch's FP64/FP32 flops",
                         "flops_per_launch": {"fp64": f64m, "fp32": f32m},
                         "f_unit": model["F_unit"]},
            "clocks": clocks,
            "gpu_launches": args.steps,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "replicas": replicas,
            "n10": n10,
            "serving": serve,
        }
        print(json.dumps(line), flush=True)
    plan_m.close()
    plan_d.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
