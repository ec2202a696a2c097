"""JSON-lines front-end on the reference clusterer's wire format.

The reference's clusterer binary (crates/holomap-clusterer/src/main.rs:10-31)
reads one ``Request`` per stdin line and writes one ``Response`` per stdout
line, in order, with errors returned in band (protocol.rs:17-94).  Its
pipeline (pipeline.rs run_pipeline) validates the request, L2-normalises the
vectors in binary32, reduces them with ``Holomap::fit_transform`` (cosine
metric, ``n_neighbors`` from the params) and clusters the embedding with
HDBSCAN.

This front-end accepts the same requests and runs the same validation and
normalisation, then the stage this library replaces -- exact kNN + smooth-kNN
of the normalised vectors (src/api.rs:147-148 with the fit_transform checks of
src/api.rs:114-145) -- through the serving context (``hm_submit``), so
requests that arrive while others are on the GPU are admitted and overlap
there.  Its responses carry that stage's arrays under ``"knn"``; the
reference's ``assignments`` need the SGD and HDBSCAN stages, which are not
part of this library, and stay empty.  Responses leave in request order.

    python -m holomap_b200.frontend < requests.jsonl > responses.jsonl
"""
from __future__ import annotations

import json
import queue
import sys
import threading

import numpy as np

PROTOCOL_VERSION = 1  # protocol.rs:17
PARAM_KEYS = ("n_components", "n_neighbors", "min_cluster_size", "seed")  # protocol.rs:28-50


def l2_normalise(vectors: np.ndarray) -> np.ndarray:
    """pipeline.rs l2_normalise in binary32: norm = sqrt of the sequential sum
    of x*x (each product and add rounded), rows with norm 0 kept as they are,
    others divided element by element."""
    x = np.ascontiguousarray(vectors, dtype=np.float32)
    s = np.zeros(x.shape[0], dtype=np.float32)
    for t in range(x.shape[1]):
        s = s + x[:, t] * x[:, t]
    norm = np.sqrt(s)
    out = x.copy()
    nz = norm != np.float32(0.0)
    out[nz] = x[nz] / norm[nz, None]
    return out


def _error(msg: str) -> dict:
    return {"protocol_version": PROTOCOL_VERSION, "assignments": [], "error": msg}


def parse_request(line: str):
    """(normalised vectors, params) of a valid request, or (None, response)
    with the reference's in-band error for an invalid one."""
    try:
        req = json.loads(line)
    except json.JSONDecodeError as e:
        return None, _error(f"bad request: {e}")
    if not isinstance(req, dict):
        return None, _error("bad request: expected an object")
    for key in ("protocol_version", "vectors", "params"):
        if key not in req:
            return None, _error(f"bad request: missing field `{key}`")
    params = req["params"]
    if not isinstance(params, dict):
        return None, _error("bad request: params is not an object")
    for key in PARAM_KEYS:
        if key not in params:
            return None, _error(f"bad request: missing field `{key}`")
    # run_pipeline's checks, in its order (pipeline.rs)
    if req["protocol_version"] != PROTOCOL_VERSION:
        return None, _error(f"unsupported protocol_version {req['protocol_version']}")
    vectors = req["vectors"]
    if not vectors:
        return None, _error("empty input")
    dims = [len(v) for v in vectors]
    if any(a != b for a, b in zip(dims, dims[1:])):
        return None, _error("vector dimensions inconsistent")
    if dims[0] == 0:
        return None, _error("zero-dimensional vectors")
    x = l2_normalise(np.asarray(vectors, dtype=np.float32))
    if params["n_components"] == 0:
        # the reference clusters the raw vectors: no reduction, no kNN stage
        return None, {"protocol_version": PROTOCOL_VERSION, "assignments": [],
                      "error": "n_components = 0 skips the reduction: no kNN stage to run"}
    # Holomap::fit_transform's validation (src/api.rs:114-145)
    k, n = int(params["n_neighbors"]), x.shape[0]
    if k < 2:
        return None, _error("holomap reduction failed: invalid parameter: n_neighbors must be >= 2")
    if n <= k:
        return None, _error(f"holomap reduction failed: need more than n_neighbors={k} points, got {n}")
    bad = np.flatnonzero(~np.isfinite(x.reshape(-1)))
    if bad.size:
        return None, _error(f"holomap reduction failed: data contains a non-finite value at index {bad[0]}")
    return (x, params), None


def knn_response(ticket) -> dict:
    k = ticket.k
    return {"protocol_version": PROTOCOL_VERSION, "assignments": [], "stage": "knn+smooth_knn",
            "knn": {"n_neighbors": k, "metric": "cosine",
                    "indices": ticket.indices.reshape(-1, k).tolist(),
                    "dists": ticket.dists.reshape(-1, k).tolist(),
                    "sigmas": ticket.sigmas.tolist(), "rhos": ticket.rhos.tolist()}}


def serve(lines, out, server=None, path="auto") -> int:
    """Answer every request line of ``lines`` on ``out`` in order.  Requests
    are submitted as they are read (a reader thread), so they overlap on the
    device; the caller's thread writes each response once its request is
    done.  Returns the number of responses written."""
    from .serve import Server
    own = server is None
    srv = server or Server()
    fifo: queue.Queue = queue.Queue(maxsize=256)

    def reader():
        try:
            for line in lines:
                if not line.strip():
                    continue
                ok, resp = parse_request(line)
                if ok is None:
                    fifo.put(("done", resp))
                    continue
                x, params = ok
                try:
                    fifo.put(("ticket", srv.submit(x, int(params["n_neighbors"]), "cosine", path)))
                except Exception as e:  # an admission or device error answers this line only
                    fifo.put(("done", _error(f"holomap reduction failed: {e}")))
        finally:
            fifo.put(("eof", None))

    th = threading.Thread(target=reader, daemon=True)
    th.start()
    written = 0
    try:
        while True:
            kind, item = fifo.get()
            if kind == "eof":
                break
            if kind == "ticket":
                try:
                    srv.wait(item)
                    resp = knn_response(item)
                except Exception as e:
                    resp = _error(f"holomap reduction failed: {e}")
                if item.info.get("status", 0) != -7:  # finished (HM_ERR_NOT_READY otherwise)
                    srv.release(item)
            else:
                resp = item
            out.write(json.dumps(resp) + "\n")
            out.flush()
            written += 1
    finally:
        th.join()
        if own:
            srv.close()
    return written


def main() -> int:
    serve(sys.stdin, sys.stdout)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
