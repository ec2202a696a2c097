#!/usr/bin/env python
"""Benchmark: exact kNN graphs/s (kNN + smooth-kNN, bit-exact to the reference).

One step = one kNN graph (indices, distances) plus its smooth-kNN calibration
(rho, sigma) for one synthetic dataset whose input is already resident in
HBM.  Default workload: embed_50k (N=50,000 x d=384 embedding-like vectors,
cosine, k=30).  Each rank builds its own graph per step (weak scaling; no
collective is on the data path).

    python bench.py [--gpus N --steps K --warmup W] [--workload W] [--path P]
    python bench.py --impl reference ...   # the reference algorithm on host cores

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import csv
import datetime
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
for p in (ROOT, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

import numpy as np  # noqa: E402

METRIC_NAME = "exact kNN graphs/s (kNN + smooth-kNN, bit-exact)"
UNIT = "graphs/s"
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="embed_50k",
                    choices=["embed_50k", "dups_20k", "blobs_1k"])
    ap.add_argument("--path", default="auto")
    ap.add_argument("--rows", type=int, default=None,
                    help="use only the first ROWS points of the workload (a smaller case "
                         "of the same kernels, e.g. for profiling)")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the oracle baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def workload(name, rows=None):
    from holomap_b200.synth import WORKLOADS, Workload
    wl = WORKLOADS[name]()
    if rows:
        wl = Workload(f"{wl.name}[:{rows}]", np.ascontiguousarray(wl.data[:rows]), wl.k, wl.metric)
    return wl


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        rows = [r for r in csv.reader(io.StringIO(self.out.read())) if len(r) >= 9]
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[5 + i].strip().lower() == "active"})
        pw = [float(r[3]) for r in rows if r[3].strip().replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows), "power_w_max": max(pw) if pw else None}


# ---------------------------------------------------------- CPU baselines
def oracle_sample_time(wl, rows: int, threads: int) -> float:
    """Seconds the oracle takes for a block of `rows` query rows (each row
    searches all n points; every row costs the same) plus their smooth-kNN
    rows, on `threads` host threads."""
    import holomap_oracle
    r0 = (wl.n - rows) // 2
    t0 = time.perf_counter()
    _, od = holomap_oracle.exact_knn(wl.data, wl.k, wl.metric, rows=(r0, r0 + rows),
                                     threads=threads)
    holomap_oracle.smooth_knn_rows(od, wl.k, float(np.mean(od)))
    return time.perf_counter() - t0


def cpu_baseline(wl, target_s: float, threads: int = 1) -> dict:
    probe = 4 if threads == 1 else max(4, threads)
    t = oracle_sample_time(wl, probe, threads)
    rows = int(max(probe, min(wl.n, probe * target_s / max(t, 1e-6))))
    t = oracle_sample_time(wl, rows, threads)
    per_graph = t * wl.n / rows
    return {"value": 1.0 / per_graph, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{rows} of {wl.n} query rows (each searching all {wl.n} points) "
                      f"+ their smooth-kNN rows, scaled by {wl.n}/{rows}; "
                      f"C restatement of src/knn.rs + src/metric.rs + src/smooth_knn.rs, "
                      f"gcc -O2 -ffp-contract=off, {threads} thread(s)",
            "seconds": t}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import holomap_oracle
    holomap_oracle.build()
    wl = workload(args.workload, args.rows)
    threads = os.cpu_count() or 1
    # one step = a bounded sample of rows, sized for about 4 s of host work
    probe_rows = max(threads, 4)
    t = oracle_sample_time(wl, probe_rows, threads)
    rows = int(max(probe_rows, min(wl.n, probe_rows * 4.0 / max(t, 1e-6))))
    for _ in range(args.warmup):
        oracle_sample_time(wl, rows, threads)
    times = [oracle_sample_time(wl, rows, threads) for _ in range(args.steps)]
    per_graph = sum(times) / len(times) * wl.n / rows
    value = 1.0 / per_graph
    line = {
        "metric": METRIC_NAME, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_graph * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(wl), "path": "reference (host cores)",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{rows} of {wl.n} query rows per step, scaled by "
                                   f"{wl.n}/{rows}; Rust reference not buildable here (no cargo), "
                                   "timed through its C restatement"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def config_of(wl) -> dict:
    return {"workload": wl.name, "n": wl.n, "d": wl.d, "k": wl.k, "metric": wl.metric,
            "smooth_knn": True, "l2": "flushed before every timed step (256 MiB write)",
            "parallelism": "replicas"}


# ------------------------------------------------------------------ ours
def main():
    args = parse_args()
    if args.impl == "reference":
        return reference_arm(args)

    import torch
    import torch.distributed as dist

    import holomap_b200 as hm
    from holomap_b200 import _lib
    from holomap_b200.device import DeviceKnnProblem

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    wl = workload(args.workload, args.rows)
    path = hm.KnnPath.parse(args.path)
    resolved = hm.autotune_path(wl.n, wl.d, wl.k, wl.metric) if path == hm.KnnPath.AUTO else path
    prob = DeviceKnnProblem(wl.n, wl.d, wl.k, wl.metric, resolved, device=dev)
    x_dev = torch.from_numpy(wl.data).to(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    for _ in range(args.warmup):
        prob.run(x_dev, stream)
    torch.cuda.synchronize(dev)
    st = prob.stats()

    # timed region: K steps, each bracketed by CUDA events on the launching
    # stream, L2 flushed before each step
    _lib.timing_enable(True)
    for cls in _lib.KCLASS:
        _lib.timing_read(cls, reset=True)
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize(dev)
    launches0 = _lib.launch_count()
    evs = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        prob.run(x_dev, stream)
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize(dev)
    launches = _lib.launch_count() - launches0
    barrier()
    clk = clocks.stop()
    _lib.timing_enable(False)
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = sum(step_ms)
    kern = {cls: _lib.timing_read(cls, reset=True) for cls in _lib.KCLASS}
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps / (total_ms / 1e3)

    # end to end through the public host API: pinned host input, H2D, both
    # stages, D2H of indices/dists/sigma/rho, every step
    e2e_steps = args.e2e_steps or max(3, min(args.steps, 10))
    pin_x = torch.from_numpy(wl.data).pin_memory()
    outs = (torch.empty(wl.n * wl.k, dtype=torch.int32).pin_memory(),
            torch.empty(wl.n * wl.k, dtype=torch.float32).pin_memory(),
            torch.empty(wl.n, dtype=torch.float32).pin_memory(),
            torch.empty(wl.n, dtype=torch.float32).pin_memory())
    outs_np = (outs[0].numpy().view(np.uint32), outs[1].numpy(), outs[2].numpy(), outs[3].numpy())
    x_np = pin_x.numpy()
    hm.knn_smooth(x_np, wl.d, wl.k, wl.metric, resolved, out=outs_np)  # warm
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        hm.knn_smooth(x_np, wl.d, wl.k, wl.metric, resolved, out=outs_np)
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * e2e_steps / e2e_s
    # the end-to-end result equals the device-resident result
    same = bool(np.array_equal(outs_np[0], prob.idx.cpu().numpy().view(np.uint32)) and
                np.array_equal(outs_np[2].view(np.uint32), prob.sigma.cpu().numpy().view(np.uint32)))

    line = None
    if rank == 0:
        bulk_ms, bulk_n = kern["bulk"]
        roof = roofline(wl, resolved, bulk_ms, bulk_n, clk)
        line = {
            "metric": METRIC_NAME, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if resolved == hm.KnnPath.PLAIN else "bf16+f64",
            "data": "synthetic", "config": config_of(wl), "path": str(resolved.name).lower(),
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": int(wl.n * wl.d * 4),
                    "d2h_bytes_per_step": int(wl.n * wl.k * 8 + wl.n * 8),
                    "steps": e2e_steps, "matches_device_run": same},
            "gpu_launches": int(launches),
            "roofline": roof,
            "kernels_ms_per_step": {c: kern[c][0] / max(args.steps, 1) for c in kern},
            "clocks": clk,
            "step_ms": {"min": min(step_ms), "median": statistics.median(step_ms),
                        "max": max(step_ms)},
            "stats": {"path_used": int(st.path_used), "col_splits": int(st.col_splits),
                      "candidates_per_row": st.candidates_total / wl.n,
                      "emitted_per_row": st.candidates_emitted / wl.n,
                      "candidates_max_row": int(st.candidates_max_row),
                      "candidate_cap": int(st.candidate_cap),
                      "overflow_rows": int(st.overflow_rows),
                      "zero_rho_rows": int(st.zero_rho_rows),
                      "screen_band": st.screen_band},
        }
        if world == 1 and not args.no_cpu_baseline:
            cb = cpu_baseline(wl, args.cpu_seconds, threads=1)
            cb.pop("seconds", None)
            line["cpu_baseline"] = cb
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


def traffic_table() -> dict:
    p = ROOT / "profiles" / "traffic.json"
    return json.loads(p.read_text()) if p.exists() else {}


def roofline(wl, path, bulk_ms, bulk_launches, clk) -> dict:
    import holomap_b200 as hm
    avg_s = bulk_ms / max(bulk_launches, 1) / 1e3
    peaks = measured_peaks()
    key = f"{wl.name}/{str(path).lower()}"
    traffic = traffic_table().get(key)
    if path == hm.KnnPath.PLAIN:
        # binary64 SIMT pipe: per pair and dimension, euclidean sub+mul+add,
        # cosine mul+add, manhattan sub+add (+abs)
        per_dim = {"euclidean": 3, "cosine": 2, "manhattan": 2}[wl.metric]
        ops = float(wl.n) * wl.n * wl.d * per_dim
        mhz = clk.get("sm_mhz") or 1965.0
        peak = 148 * 64 * mhz * 1e6  # 64 binary64 lanes per SM, one op each per clock
        return {"bound": "fp64", "kernel": "plain_knn_kernel",
                "achieved": ops / avg_s / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
                "frac": ops / avg_s / peak, "traffic": traffic,
                "algorithmic": f"{per_dim} binary64 ops x N^2 x d = {ops:.3e} per launch",
                "peak_source": f"nominal: 148 SMs x 64 FP64 lanes x measured median "
                               f"{mhz:.0f} MHz (no measured FP64 peak available)",
                "launches": bulk_launches, "avg_launch_ms": avg_s * 1e3}
    flops = 2.0 * wl.n * wl.n * wl.d
    peak = peaks.get("bf16_tflops_sustained", 1400.0)
    src = "MEASURED_PEAKS.json bf16_tflops_sustained (of measured)" if peaks else \
        "fallback 1.4 PFLOP/s sustained (of fallback)"
    return {"bound": "tensor", "kernel": "screen_gemm",
            "achieved": flops / avg_s / 1e12, "peak": peak, "unit": "TFLOP/s",
            "frac": flops / avg_s / 1e12 / peak, "traffic": traffic,
            "algorithmic": f"2 x N^2 x d = {flops:.3e} flops per launch",
            "peak_source": src, "launches": bulk_launches, "avg_launch_ms": avg_s * 1e3}


if __name__ == "__main__":
    sys.exit(main())
