"""GPU parity of the plain exact path and of smooth-kNN against the oracle
(C restatement of src/knn.rs, src/metric.rs, src/smooth_knn.rs), byte for byte,
and against the reference's golden fixtures."""
import json
from pathlib import Path

import numpy as np
import pytest

import holomap_b200 as hm
from parity import assert_same_bytes, edge_case, rows_sorted_by_key

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def run_both(oracle, x, k, metric, path="plain"):
    n, d = x.shape
    st = hm.HmStats()
    knn, sm = hm.knn_smooth(x, d, k, metric, path, stats=st)
    oi, od = oracle.exact_knn(x, k, metric)
    assert_same_bytes(knn.indices, oi, "indices")
    assert_same_bytes(knn.dists, od, "dists")
    osig, orho = oracle.smooth_knn(od, k)
    assert_same_bytes(sm.rhos, orho, "rho")
    assert_same_bytes(sm.sigmas, osig, "sigma")
    return knn, sm, st


@pytest.mark.parametrize("name", ["blobs_euclidean", "cosine", "duplicates_euclidean"])
def test_golden_fixtures(oracle, name):
    fx = json.loads((GOLDEN / f"stage2_{name}.json").read_text())
    x = np.asarray(fx["data"], dtype=np.float32)
    k = fx["n_neighbors"]
    knn, sm, _ = run_both(oracle, x, k, fx["metric"])
    assert knn.indices.reshape(-1, k).tolist() == fx["knn_indices"]
    tol = lambda e: 1e-5 * (1 + np.abs(np.asarray(e, dtype=np.float64)))
    for got, key in ((knn.dists.reshape(-1, k), "knn_dists"), (sm.rhos, "rhos"),
                     (sm.sigmas, "sigmas")):
        assert (np.abs(got - np.asarray(fx[key])) <= tol(fx[key])).all(), key


def test_reference_unit_cases(oracle):
    # src/knn.rs:64-105 on the device
    line = np.array([[0.0], [1.0], [3.0], [7.0]], np.float32)
    knn = hm.exact_knn(line, 1, 3, "euclidean", "plain")
    assert knn.indices.reshape(4, 3)[1].tolist() == [1, 0, 2]
    assert knn.dists.reshape(4, 3)[3].tolist() == [0.0, 4.0, 6.0]
    dup = np.array([[5.0], [9.0], [5.0]], np.float32)
    knn = hm.exact_knn(dup, 1, 2, "euclidean", "plain")
    assert knn.indices.reshape(3, 2)[2].tolist() == [0, 2]
    cs = np.array([[0.3, 0.7], [0.31, 0.69]], np.float32)
    knn = hm.exact_knn(cs, 2, 2, "cosine", "plain")
    assert knn.dists[0] == 0.0 and knn.dists[2] == 0.0
    assert knn.dists[1] > 0.0 and knn.dists[3] > 0.0
    cs3 = np.array([[1.0, 0.0], [100.0, 1.0], [0.1, 0.1]], np.float32)
    knn = hm.exact_knn(cs3, 2, 2, "cosine", "plain")
    assert knn.indices.reshape(3, 2)[0].tolist() == [0, 1]


@pytest.mark.parametrize("metric", ["euclidean", "cosine", "manhattan"])
@pytest.mark.parametrize("n,d,k", [(40, 1, 2), (97, 5, 7), (300, 50, 15), (1000, 50, 15),
                                   (1500, 33, 30), (700, 128, 64), (520, 20, 129),
                                   (600, 8, 256), (257, 3, 256)])
def test_random_cases(oracle, metric, n, d, k):
    x = edge_case("gauss", n, d, seed=n * 31 + d)
    knn, _, st = run_both(oracle, x, k, metric)
    assert rows_sorted_by_key(knn.indices.reshape(n, k), knn.dists.reshape(n, k))


@pytest.mark.parametrize("kind", ["duplicates", "ulp", "zeros", "huge", "tiny", "grid",
                                  "sorted_line"])
@pytest.mark.parametrize("metric", ["euclidean", "cosine", "manhattan"])
def test_edge_cases(oracle, kind, metric):
    x = edge_case(kind, 611, 6, seed=7)
    run_both(oracle, x, 15, metric)


def test_k_equals_n_minus_one(oracle):
    x = edge_case("gauss", 65, 4, seed=1)
    run_both(oracle, x, 64, "euclidean")


def test_all_zero_rows_use_global_mean_floor(oracle):
    # 40 copies of one point: rows whose k nearest are all at distance 0 take
    # the global-mean floor (src/smooth_knn.rs:70-74)
    g = np.random.default_rng(5)
    x = g.normal(size=(200, 3)).astype(np.float32)
    x[:40] = x[0]
    knn, sm, st = run_both(oracle, x, 15, "euclidean")
    assert st.zero_rho_rows == 40
    assert (sm.rhos[:40] == 0).all()


def test_non_finite_input_reports_first_index():
    x = np.ones((50, 4), np.float32)
    x[7, 2] = np.nan
    x[9, 0] = np.inf
    with pytest.raises(hm.HolomapInvalidInput, match="index 30"):
        hm.exact_knn(x, 4, 5, "euclidean", "plain")


def test_smooth_knn_standalone(oracle):
    g = np.random.default_rng(9)
    for k in (2, 3, 15, 30, 64, 200):
        n = 333
        d = np.sort(g.exponential(size=(n, k)).astype(np.float32), axis=1)
        d[:, 0] = 0.0
        d[::17, : k // 2] = 0.0  # rows whose rho comes later
        d[::29] = 0.0            # rows with no positive distance
        sm = hm.smooth_knn(d, k)
        osig, orho = oracle.smooth_knn(d, k)
        assert_same_bytes(sm.rhos, orho, f"rho k={k}")
        assert_same_bytes(sm.sigmas, osig, f"sigma k={k}")


def test_smooth_knn_reference_literals():
    # src/smooth_knn.rs:104-124
    sm = hm.smooth_knn(np.array([0, 1, 3, 0, 1, 2, 0, 2, 3], np.float32), 3)
    assert sm.sigmas.tolist() == [3.72998046875, 1.864990234375, 1.864990234375]
    assert sm.rhos.tolist() == [1.0, 1.0, 2.0]
    sm = hm.smooth_knn(np.zeros(4, np.float32), 2)
    assert sm.sigmas.tolist() == [1.0, 1.0]


def test_determinism_double_run():
    x = edge_case("duplicates", 3000, 24, seed=3)
    a = hm.knn_smooth(x, 24, 15, "cosine", "plain")
    b = hm.knn_smooth(x, 24, 15, "cosine", "plain")
    for u, v in zip(a[0].__dict__.values(), b[0].__dict__.values()):
        assert np.array_equal(np.asarray(u), np.asarray(v))
    assert np.array_equal(a[1].sigmas.view(np.uint32), b[1].sigmas.view(np.uint32))


def test_device_api_matches_host_api():
    import torch
    from holomap_b200.device import DeviceKnnProblem
    x = edge_case("gauss", 2500, 40, seed=4)
    host = hm.knn_smooth(x, 40, 15, "euclidean", "plain")
    prob = DeviceKnnProblem(2500, 40, 15, "euclidean", "plain")
    prob.run(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    assert np.array_equal(prob.idx.cpu().numpy().view(np.uint32), host[0].indices)
    assert np.array_equal(prob.dist.cpu().numpy().view(np.uint32), host[0].dists.view(np.uint32))
    assert np.array_equal(prob.sigma.cpu().numpy().view(np.uint32), host[1].sigmas.view(np.uint32))
