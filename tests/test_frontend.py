"""The JSON-lines front-end on the reference clusterer's wire format
(crates/holomap-clusterer/src/protocol.rs:17-94, main.rs:10-31,
pipeline.rs run_pipeline): request validation and its in-band errors, the
binary32 L2 normalisation, response order, and (on the GPU) the kNN stage's
arrays against the oracle on the normalised vectors."""
import io
import json

import numpy as np
import pytest

from holomap_b200 import frontend

pytestmark = []


def req(vectors, version=1, n_components=2, n_neighbors=3, min_cluster_size=2, seed=7):
    return json.dumps({"protocol_version": version, "vectors": vectors,
                       "params": {"n_components": n_components, "n_neighbors": n_neighbors,
                                  "min_cluster_size": min_cluster_size, "seed": seed}})


@pytest.mark.parametrize("line,msg", [
    ("{not json", "bad request:"),
    (json.dumps({"vectors": [[1.0]], "params": {}}), "missing field `protocol_version`"),
    (req([[1.0, 2.0]], version=2), "unsupported protocol_version 2"),
    (req([]), "empty input"),
    (req([[1.0, 2.0], [1.0]]), "vector dimensions inconsistent"),
    (req([[], []]), "zero-dimensional vectors"),
    (req([[1.0, 2.0]] * 5, n_neighbors=1), "n_neighbors must be >= 2"),
    (req([[1.0, 2.0]] * 3, n_neighbors=3), "need more than n_neighbors=3 points, got 3"),
    (req([[1.0, 2.0]] * 5, n_components=0), "n_components = 0"),
])
def test_invalid_requests_answer_in_band(line, msg):
    ok, resp = frontend.parse_request(line)
    assert ok is None
    assert resp["protocol_version"] == 1 and resp["assignments"] == []
    assert msg in resp["error"]


def test_l2_normalise_is_binary32_and_keeps_zero_rows():
    g = np.random.default_rng(3)
    x = g.normal(size=(50, 13)).astype(np.float32)
    x[7] = 0.0
    y = frontend.l2_normalise(x)
    assert y.dtype == np.float32
    assert np.array_equal(y[7], x[7])
    # sequential binary32 sum of squares, then one correctly rounded divide
    for i in (0, 11, 49):
        s = np.float32(0.0)
        for v in x[i]:
            s = np.float32(s + np.float32(v * v))
        assert np.array_equal(y[i], x[i] / np.sqrt(s))
    assert np.allclose(np.linalg.norm(y[np.arange(50) != 7], axis=1), 1.0, atol=1e-6)


def test_errors_keep_their_place_in_the_stream_without_a_device():
    lines = [req([]), "", req([[1.0]], version=9), "{bad"]

    class NoServer:  # every line fails validation before any device work
        def submit(self, *a, **k):
            raise AssertionError("no request should reach the device")

    out = io.StringIO()
    assert frontend.serve(iter(lines), out, server=NoServer()) == 3
    got = [json.loads(s) for s in out.getvalue().splitlines()]
    assert [g["error"].split(":")[0] for g in got] == ["empty input", "unsupported protocol_version 9",
                                                       "bad request"]


@pytest.mark.gpu
def test_knn_stage_of_served_requests_matches_the_oracle(oracle):
    g = np.random.default_rng(11)
    sets = [g.normal(size=(n, d)).astype(np.float32) for n, d in ((300, 16), (1200, 50), (40, 8))]
    lines = [req(s.tolist(), n_neighbors=k) for s, k in zip(sets, (15, 30, 5))]
    lines.insert(1, req([[1.0, 2.0]], version=3))  # an error between valid requests
    out = io.StringIO()
    assert frontend.serve(iter(lines), out) == 4
    resp = [json.loads(s) for s in out.getvalue().splitlines()]
    assert resp[1]["error"] == "unsupported protocol_version 3"
    for r, x, k in zip([resp[0], resp[2], resp[3]], sets, (15, 30, 5)):
        assert "error" not in r
        xn = frontend.l2_normalise(x)
        oi, od = oracle.exact_knn(xn, k, "cosine")
        osig, orho = oracle.smooth_knn(od, k)
        kn = r["knn"]
        assert np.array_equal(np.asarray(kn["indices"], dtype=np.uint32), oi)
        assert np.array_equal(np.asarray(kn["dists"], dtype=np.float32).view(np.uint32), od.view(np.uint32))
        assert np.array_equal(np.asarray(kn["sigmas"], dtype=np.float32).view(np.uint32), osig.view(np.uint32))
        assert np.array_equal(np.asarray(kn["rhos"], dtype=np.float32).view(np.uint32), orho.view(np.uint32))
