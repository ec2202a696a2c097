"""The autotuner: measures every path of the kNN + smooth-kNN pipeline on a
grid of problem shapes on the GPU and writes the table that HM_PATH_AUTO
reads.

For every grid point (N, d, k, metric) it times, with CUDA events on the
launching stream, one full kNN + smooth-kNN run of

* the plain exact binary64 path, and
* each tensor-core screen (BF16, TF32, split-BF16) with the threshold pass
  sampling 1/4, 1/8 and 1/16 of the columns (emission pass over every column
  tile, in the 2-SM form where it applies), and the fastest of those again
  with one CTA per 128-row block instead of the 2-SM form and with the
  symmetric emission pass (tiles on and above the diagonal only),

on seeded data of that shape, checks that every screened result equals the
plain path's bytes, and records the fastest choice.  Up to 8192 points it
also times each path on a batch of 32 jobs of that shape (one CUDA graph per
batch, windows of the same pool), where the screens' fixed per-call costs are
shared: jobs planned in a batch take that choice.  Euclidean points are
Gaussian mixtures (3-20 clusters); cosine points have the shape of text or
image embeddings (a decaying spectrum, N(0, diag(i^-1.2)), a shared offset,
unit norm).  Cosine data made of a few very tight clusters far from the
origin is the screens' hard case: neighbour gaps far below the BF16 band
send most rows to the exact fallback, where TF32 or split-BF16 is faster.
Two files are written:

* ``holomap_b200/autotune_table.json`` -- every measurement, the choice per
  grid point, and the device and command that produced them;
* ``holomap_b200/csrc/autotune_table.inc`` -- the same choices as a C table
  compiled into the library (``hm_autotune_path`` and the screen planner look
  up the nearest grid point).

    python -m holomap_b200.autotune              # sweep on cuda:0, write both files
    python -m holomap_b200.autotune --emit-only  # regenerate the .inc from the JSON

Manhattan (no inner-product form), k > 64 and d > 2048 always take the plain
path: no screen applies.
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import statistics
import time
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
JSON_PATH = PKG / "autotune_table.json"
INC_PATH = PKG / "csrc" / "autotune_table.inc"

GRID_N = [256, 512, 1024, 2048, 4096, 8192, 16384, 32768, 50000]
GRID_D = [16, 32, 50, 64, 128, 300, 384]
GRID_K = [15, 30]
METRICS = ["euclidean", "cosine"]
SCREENS = ["screen_bf16", "screen_tf32", "screen_bf16x3"]
SEED_DIVS = [4, 8, 16]
BATCH_JOBS = 32
BATCH_MAX_N = 8192
# Up to this d a screened job planned in a batch takes the split-BF16 screen
# whatever screen won its shape's batch: a batch of mixed shapes then shares
# one screen launch (three formats cost three pipelines of launches), and
# split-BF16's band (about 2^-16 of the norms) needs no escalation copy.
# Measured on batch_256 (256 datasets, d in {16, 50, 128}): 25,300 graphs/s
# with each job on its shape's batch winner (TF32 for 139 jobs, split-BF16 for
# 72) against 35,900 with every screened job on split-BF16; at these d the
# per-shape batch times of TF32 and split-BF16 are within a few percent.
BATCH_SHARED_MAX_D = 256
PATH_CODE = {"plain": 1, "screen_bf16": 2, "screen_tf32": 3, "screen_bf16x3": 4}


def hand_rule(n: int, d: int, k: int, metric: str) -> tuple[str, int, int, int]:
    """The choice used before any measurement exists (and the shape of the
    table when the sweep has not run): plain below 512 points, split-BF16 up
    to d = 256, then BF16 (cosine) or TF32 (euclidean); an eighth sampled;
    the emission pass over every column tile in the 2-SM form.  Returns
    (path, seed_div, symmetric, pair)."""
    if n < 512:
        return "plain", 8, 0, 1
    if d <= 256:
        return "screen_bf16x3", 8, 0, 1
    return ("screen_bf16" if metric == "cosine" else "screen_tf32"), 8, 0, 1


def _pool(d: int, n: int, metric: str) -> np.ndarray:
    from .synth import _rng, embedding_like, gaussian_mixture
    if metric == "cosine":
        g = _rng(900001 + 10 * d)
        return np.ascontiguousarray(embedding_like(g, n, d).astype(np.float32))
    g = _rng(900000 + 10 * d)
    clusters = int(g.integers(3, 21))
    return np.ascontiguousarray(gaussian_mixture(g, n, d, clusters, 4.0, 0.3, 3.0).astype(np.float32))


def _time_run(prob, x, reps: int) -> float:
    import torch
    s = torch.cuda.current_stream()
    prob.run(x, s)  # warm: workspace first touch, plan
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        prob.run(x, s)
        e1.record(s)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return statistics.median(ms)


def _time_batch(batch, reps: int) -> float:
    import torch
    s = torch.cuda.current_stream()
    batch.run(s, graph=True)  # warm: captures the batch's graph
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        batch.run(s, graph=True)
        e1.record(s)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return statistics.median(ms)


def _batch_measure(xpool, n: int, k: int, metric: str, seed_div: dict, lib) -> dict:
    """Per-batch times of BATCH_JOBS jobs of one shape on each path (None
    where a screened batch's bytes differ from the plain batch's)."""
    from . import _lib
    from .device import DeviceBatch
    span = xpool.shape[0] - n
    xs = [xpool[(j * 1543) % max(span, 1):][:n].contiguous() for j in range(BATCH_JOBS)]
    times, ref = {}, None
    for path in ["plain"] + SCREENS:
        _lib.check(lib.hm_tuning_override(seed_div.get(path, 8)))
        try:
            b = DeviceBatch([(x, k, metric, path) for x in xs])
            t = _time_batch(b, 5)
            got = [b.result(j) for j in range(BATCH_JOBS)]
            del b
        finally:
            _lib.check(lib.hm_tuning_override(0))
        if ref is None:
            ref = got
            times[path] = t
        else:
            same = all(np.array_equal(a.view(np.uint32), r.view(np.uint32))
                       for g, rr in zip(got, ref) for a, r in zip(g, rr))
            times[path] = t if same else None
    return times


def sweep(grid_n=GRID_N, grid_d=GRID_D, grid_k=GRID_K, metrics=METRICS, verbose=True) -> dict:
    import torch

    from . import _lib
    from .device import DeviceKnnProblem
    lib = _lib.lib()
    entries = []
    t_start = time.time()
    for metric in metrics:
        for d in grid_d:
            pool = _pool(d, max(grid_n), metric)
            xpool = torch.from_numpy(pool).cuda()
            for k in grid_k:
                for n in grid_n:
                    x = xpool[:n].contiguous()
                    times, exact = {}, True
                    plain = DeviceKnnProblem(n, d, k, metric, "plain")
                    reps = 2 if n * n * d > 2e11 else 5
                    times["plain"] = _time_run(plain, x, reps)
                    ref = (plain.idx.cpu().numpy(), plain.dist.cpu().numpy().view(np.uint32),
                           plain.sigma.cpu().numpy().view(np.uint32))
                    del plain
                    def measure(path, sd, sym, pair=1):
                        _lib.check(lib.hm_tuning_override(sd))
                        _lib.check(lib.hm_tuning_symmetric(sym))
                        _lib.check(lib.hm_tuning_pair(pair))
                        try:
                            p = DeviceKnnProblem(n, d, k, metric, path)
                            t = _time_run(p, x, 5)
                            got = (p.idx.cpu().numpy(), p.dist.cpu().numpy().view(np.uint32),
                                   p.sigma.cpu().numpy().view(np.uint32))
                            same = all(np.array_equal(a, b) for a, b in zip(got, ref))
                            del p
                        finally:
                            _lib.check(lib.hm_tuning_override(0))
                            _lib.check(lib.hm_tuning_symmetric(-1))
                            _lib.check(lib.hm_tuning_pair(-1))
                        return t if same else None

                    for path in SCREENS:
                        for sd in SEED_DIVS:
                            times[f"{path}/{sd}/full"] = measure(path, sd, 0)
                    screened = {c: t for c, t in times.items() if t is not None and c != "plain"}
                    if screened:
                        c0 = min(screened, key=screened.get)
                        p0, sd0, _ = c0.split("/")
                        times[f"{p0}/{sd0}/single"] = measure(p0, int(sd0), 0, 0)
                        times[f"{p0}/{sd0}/sym"] = measure(p0, int(sd0), 1)
                    exact = all(t is not None for t in times.values())
                    valid = {c: t for c, t in times.items() if t is not None}
                    best = min(valid, key=valid.get)
                    path, sd, form = (best.split("/") + ["8", "full"])[:3]
                    e = {"n": n, "d": d, "k": k, "metric": metric, "times_ms": times, "best": path,
                         "seed_div": int(sd), "symmetric": int(form == "sym"), "pair": int(form != "single"),
                         "all_paths_equal_plain": exact}
                    if n <= BATCH_MAX_N:
                        # each screen at its fastest single-job sample
                        sds = {}
                        for c, t in valid.items():
                            pth, *rest = c.split("/")
                            if rest and rest[1] == "full" and (pth not in sds or t < valid[f"{pth}/{sds[pth]}/full"]):
                                sds[pth] = int(rest[0])
                        bt = _batch_measure(xpool, n, k, metric, sds, lib)
                        bvalid = {c: t for c, t in bt.items() if t is not None}
                        bbest = min(bvalid, key=bvalid.get)
                        e.update({"batch_jobs": BATCH_JOBS, "batch_times_ms": bt, "batch_best": bbest,
                                  "batch_seed_div": sds.get(bbest, 8),
                                  "all_paths_equal_plain": exact and all(t is not None for t in bt.values())})
                    entries.append(e)
                    if verbose:
                        extra = f"  batch {e['batch_best']}" if "batch_best" in e else ""
                        print(f"{metric:9s} d={d:4d} k={k:2d} n={n:6d}  best {best:18s} "
                              f"{valid[best]:9.3f} ms  (plain {times['plain']:9.3f} ms){extra}", flush=True)
    props = torch.cuda.get_device_properties(0)
    return {
        "device": props.name, "sms": props.multi_processor_count,
        "measured": datetime.datetime.now(datetime.timezone.utc).strftime("%Y-%m-%d %H:%M UTC"),
        "command": "python -m holomap_b200.autotune",
        "timing": "median of CUDA-event times of full kNN + smooth-kNN runs on device-resident "
                  "inputs (one warm-up run first)",
        "data": "euclidean: seeded Gaussian mixtures (3-20 clusters, centres N(0, 16 I), sigma U[0.3, 3]); "
                "cosine: embedding-shaped rows (N(0, diag(i^-1.2)) plus an offset of norm 0.3, unit norm); "
                "prefixes of one 50,000-point pool per (d, metric)",
        "sweep_seconds": round(time.time() - t_start, 1),
        "grid": {"n": list(grid_n), "d": list(grid_d), "k": list(grid_k), "metric": list(metrics)},
        "entries": entries,
    }


def _best_seed_div(e: dict, path: str) -> int:
    """The fastest measured threshold sample of a path at a grid point."""
    t = {c: v for c, v in e["times_ms"].items() if v is not None and c.startswith(path + "/")
         and c.endswith("/full")}
    return int(min(t, key=t.get).split("/")[1]) if t else 8


def table_from(doc: dict | None) -> tuple[dict, dict, list, list, list]:
    """(choice, batch_choice, grid n, d, k); choice[(metric, k, d, n)] =
    (path, seed_div, symmetric, pair) for a problem alone, batch_choice the
    same for a job planned in a batch (the single choice where no batch was
    measured)."""
    if doc is None:
        gn, gd, gk = GRID_N, GRID_D, GRID_K
        choice = {(m, k, d, n): hand_rule(n, d, k, m) for m in METRICS for k in gk for d in gd for n in gn}
        return choice, dict(choice), gn, gd, gk
    g = doc["grid"]
    choice, batch = {}, {}
    for e in doc["entries"]:
        key = (e["metric"], e["k"], e["d"], e["n"])
        choice[key] = (e["best"], e["seed_div"], e.get("symmetric", 1), e.get("pair", 1))
        if "batch_best" in e:
            bp, bsd = e["batch_best"], e.get("batch_seed_div", 8)
            if bp != "plain" and e["d"] <= BATCH_SHARED_MAX_D and bp != "screen_bf16x3":
                # a mixed batch shares one split-BF16 screen launch (see
                # BATCH_SHARED_MAX_D)
                bp = "screen_bf16x3"
                bsd = _best_seed_div(e, bp)
            batch[key] = (bp, bsd, 0, 1)
        else:
            batch[key] = choice[key]
    return choice, batch, g["n"], g["d"], g["k"]


def _nearest(grid, v) -> int:
    return min(grid, key=lambda g: abs(math.log(max(v, 1) / g)))


def describe(n: int, d: int, k: int, metric: str) -> dict:
    """The table entry a problem resolves to (the library's lookup: nearest
    grid point by ratio in n, d and k), with its measured times."""
    if metric == "manhattan" or k > 64 or d > 2048:
        return {"choice": "plain", "reason": "no screen applies"}
    doc = json.loads(JSON_PATH.read_text()) if JSON_PATH.exists() else None
    choice, batch, gn, gd, gk = table_from(doc)
    key = (metric, _nearest(gk, k), _nearest(gd, d), _nearest(gn, n))
    path, sd, sym, pair = choice[key]
    out = {"grid_point": {"metric": key[0], "k": key[1], "d": key[2], "n": key[3]},
           "choice": path, "seed_div": sd, "symmetric_emission": bool(sym), "two_sm_emission": bool(pair),
           "batch_choice": batch[key][0],
           "table": f"measured {doc['measured']} on {doc['device']}" if doc else "hand rule (no measurement)"}
    if doc:
        for e in doc["entries"]:
            if (e["metric"], e["k"], e["d"], e["n"]) == key:
                out["times_ms"] = e["times_ms"]
    return out


def emit_inc(doc: dict | None, path: Path = INC_PATH) -> None:
    choice, batch, gn, gd, gk = table_from(doc)
    src = doc["measured"] + " on " + doc["device"] if doc else "no measurement yet (the hand rule)"
    lines = [
        "// autotune_table.inc -- generated by holomap_b200/autotune.py from",
        "// holomap_b200/autotune_table.json; do not edit by hand.",
        f"// Source: {src}.",
        "// kTune[metric][k][d][n] = path | pair << 4 | seed_div << 8 | symmetric << 15 at the grid",
        "// points below, for a problem alone; kTuneBatch the same for a job planned",
        "// in a batch of several (metric 0 euclidean, 1 cosine).",
        "#pragma once",
        f"static const uint32_t kTuneN[{len(gn)}] = {{{', '.join(map(str, gn))}}};",
        f"static const uint32_t kTuneD[{len(gd)}] = {{{', '.join(map(str, gd))}}};",
        f"static const uint32_t kTuneK[{len(gk)}] = {{{', '.join(map(str, gk))}}};",
    ]
    for name, table in (("kTune", choice), ("kTuneBatch", batch)):
        lines.append(f"static const uint16_t {name}[2][{len(gk)}][{len(gd)}][{len(gn)}] = {{")
        for m in METRICS:
            lines.append("    {")
            for k in gk:
                lines.append("        {")
                for d in gd:
                    row = []
                    for n in gn:
                        p, sd, sym, pair = table[(m, k, d, n)]
                        row.append(str(PATH_CODE[p] | (int(pair) << 4) | (int(sd) << 8) | (int(sym) << 15)))
                    lines.append("            {" + ", ".join(row) + "},")
                lines.append("        },")
            lines.append("    },")
        lines.append("};")
    path.write_text("\n".join(lines) + "\n")


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--emit-only", action="store_true",
                    help="regenerate the C table from the committed JSON (no GPU)")
    ap.add_argument("--out", default=str(JSON_PATH))
    a = ap.parse_args()
    if a.emit_only:
        doc = json.loads(Path(a.out).read_text()) if Path(a.out).exists() else None
        emit_inc(doc)
        return 0
    doc = sweep()
    Path(a.out).write_text(json.dumps(doc, indent=1) + "\n")
    emit_inc(doc)
    print(f"wrote {a.out} and {INC_PATH}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
