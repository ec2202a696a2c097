"""The oracle (C restatement of the reference's kNN, smooth-kNN and fuzzy graph
path) pinned against the reference's own known-answer tests and golden
fixtures.

Ports the *assertions* of src/knn.rs:64-105, src/metric.rs:92-102,
src/smooth_knn.rs:104-124, src/fuzzy.rs:97-155 and
src/fixture_parity.rs:42-117."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
FIXTURES = ("blobs_euclidean", "cosine", "duplicates_euclidean")


def f32(x):
    return np.asarray(x, dtype=np.float32)


# --- src/knn.rs tests -------------------------------------------------------

def test_knn_sorted_by_distance_self_first(oracle):
    # src/knn.rs:64-73
    line = f32([0.0, 1.0, 3.0, 7.0]).reshape(4, 1)
    idx, dist = oracle.exact_knn(line, 3, "euclidean")
    assert idx[1].tolist() == [1, 0, 2]
    assert dist[1].tolist() == [0.0, 1.0, 2.0]
    assert idx[3].tolist() == [3, 2, 1]
    assert dist[3].tolist() == [0.0, 4.0, 6.0]


def test_knn_ties_broken_by_lower_index(oracle):
    # src/knn.rs:75-83
    data = f32([5.0, 9.0, 5.0]).reshape(3, 1)
    idx, dist = oracle.exact_knn(data, 2, "euclidean")
    assert idx[0].tolist() == [0, 2]
    assert idx[2].tolist() == [0, 2]
    assert dist[2].tolist() == [0.0, 0.0]


def test_knn_cosine_self_distance_exactly_zero(oracle):
    # src/knn.rs:85-95
    data = f32([0.3, 0.7, 0.31, 0.69]).reshape(2, 2)
    idx, dist = oracle.exact_knn(data, 2, "cosine")
    assert dist[0, 0] == 0.0 and dist[1, 0] == 0.0
    assert dist[0, 1] > 0.0 and dist[1, 1] > 0.0
    # through the metric itself the self distance is not exactly zero
    assert oracle.distance(data[0], data[0], "cosine") >= 0.0


def test_knn_cosine_orders_by_angle_not_magnitude(oracle):
    # src/knn.rs:97-105
    data = f32([1.0, 0.0, 100.0, 1.0, 0.1, 0.1]).reshape(3, 2)
    idx, dist = oracle.exact_knn(data, 3, "cosine")
    assert idx[0].tolist() == [0, 1, 2]
    assert dist[0, 1] < dist[0, 2]


# --- src/metric.rs tests ----------------------------------------------------

def test_euclidean_known_values(oracle):
    # src/metric.rs:92-95
    assert oracle.distance(f32([0, 0]), f32([3, 4]), "euclidean") == 5.0
    assert oracle.distance(f32([1, 2, 3]), f32([1, 2, 3]), "euclidean") == 0.0


def test_cosine_known_values(oracle):
    # src/metric.rs:97-102
    assert oracle.distance(f32([1, 0]), f32([0, 1]), "cosine") == 1.0
    assert oracle.distance(f32([1, 0]), f32([2, 0]), "cosine") == 0.0
    assert oracle.distance(f32([1, 0]), f32([-3, 0]), "cosine") == 2.0


def test_cosine_zero_vector_is_zero_distance(oracle):
    # 0/0 = NaN inside the metric; f64::max(NaN, 0.0) returns 0.0
    assert oracle.distance(f32([0, 0]), f32([1, 2]), "cosine") == 0.0


def test_euclidean_overflow_casts_to_inf(oracle):
    big = f32([3.0e38, -3.0e38])
    assert np.isinf(oracle.distance(big, -big, "euclidean"))


def test_manhattan_extension(oracle):
    assert oracle.distance(f32([0, 0]), f32([3, -4]), "manhattan") == 7.0


# --- src/smooth_knn.rs tests ------------------------------------------------

def test_smooth_knn_matches_reference_on_line_points(oracle):
    # src/smooth_knn.rs:104-112 (exact decimal expansions of the f32 results)
    dists = f32([0.0, 1.0, 3.0, 0.0, 1.0, 2.0, 0.0, 2.0, 3.0])
    sig, rho = oracle.smooth_knn(dists, 3)
    np.testing.assert_allclose(rho, [1.0, 1.0, 2.0], atol=1e-5, rtol=0)
    np.testing.assert_allclose(sig, [3.72998046875, 1.864990234375, 1.864990234375],
                               atol=1e-5, rtol=0)
    # the restatement reproduces the reference's literals bit for bit
    assert sig.tolist() == [3.72998046875, 1.864990234375, 1.864990234375]


def test_all_zero_distances_yield_unit_sigma(oracle):
    # src/smooth_knn.rs:118-124
    sig, rho = oracle.smooth_knn(f32([0.0, 0.0, 0.0, 0.0]), 2)
    assert rho.tolist() == [0.0, 0.0]
    assert sig.tolist() == [1.0, 1.0]


# --- src/fuzzy.rs tests -----------------------------------------------------

def test_fuzzy_line_points_symmetrized_sorted_no_self_edges(oracle):
    # src/fuzzy.rs:97-129: 3 line points, k = 3
    idx = np.array([0, 1, 2, 1, 0, 2, 2, 1, 0], dtype=np.uint32)
    dists = f32([0.0, 1.0, 3.0, 0.0, 1.0, 2.0, 0.0, 2.0, 3.0])
    sig = f32([3.72998046875, 1.864990234375, 1.864990234375])
    rho = f32([1.0, 1.0, 2.0])
    rows, cols, vals = oracle.fuzzy_graph(idx, dists, sig, rho, 3)
    w = oracle.expf(f32([-2.0 / 3.72998046875]))[0]
    fused = np.float32(np.float32(w + w) - np.float32(w * w))
    assert rows.tolist() == [0, 0, 1, 1, 2, 2]
    assert cols.tolist() == [1, 2, 0, 2, 0, 1]
    np.testing.assert_allclose(vals, [1.0, fused, 1.0, 1.0, fused, 1.0], atol=1e-6, rtol=0)


def test_fuzzy_one_directional_edge_becomes_symmetric(oracle):
    # src/fuzzy.rs:131-155
    idx = np.array([0, 1, 1, 2, 2, 1], dtype=np.uint32)
    dists = f32([0.0, 1.0, 0.0, 0.1, 0.0, 0.1])
    rows, cols, vals = oracle.fuzzy_graph(idx, dists, f32([1.0, 1.0, 1.0]), f32([0.5, 0.1, 0.1]), 2)
    w = oracle.expf(f32([-0.5]))[0]
    assert rows.tolist() == [0, 1, 1, 2]
    assert cols.tolist() == [1, 0, 2, 1]
    assert vals.tolist() == [w, w, 1.0, 1.0]


# --- golden fixtures (src/fixture_parity.rs:42-117) -------------------------

def close(actual, expected):
    expected = np.asarray(expected, dtype=np.float64)
    tol = 1e-5 * (1.0 + np.abs(expected))
    return np.abs(np.asarray(actual, dtype=np.float64) - expected) <= tol


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_golden_fixture(oracle, name):
    fx = json.loads((GOLDEN / f"stage2_{name}.json").read_text())
    data = f32(fx["data"])
    k = fx["n_neighbors"]
    idx, dist = oracle.exact_knn(data, k, fx["metric"])
    assert idx.tolist() == fx["knn_indices"], "kNN indices must match exactly"
    assert close(dist, fx["knn_dists"]).all()
    sig, rho = oracle.smooth_knn(dist, k)
    assert close(rho, fx["rhos"]).all()
    assert close(sig, fx["sigmas"]).all()
    # src/fixture_parity.rs:101-117: graph support exact, weights to tolerance
    rows, cols, vals = oracle.fuzzy_graph(idx, dist, sig, rho, k)
    assert rows.tolist() == fx["graph_rows"]
    assert cols.tolist() == fx["graph_cols"]
    assert close(vals, fx["graph_vals"]).all()


# --- expf restatement -------------------------------------------------------

def test_expf_special_values(oracle):
    x = f32([0.0, -0.0, 1.0, -1.0, 88.8, -104.0, -np.inf, np.inf, 1e-8, -1e-8])
    y = oracle.expf(x)
    assert y[0] == 1.0 and y[1] == 1.0
    assert np.isinf(y[4]) and y[5] == 0.0 and y[6] == 0.0 and np.isinf(y[7])
    assert y[8] == np.float32(1.0) + np.float32(1e-8)
    assert np.isnan(oracle.expf(f32([np.nan]))[0])


def _ulp_distance(a, b):
    ia = a.view(np.int32).astype(np.int64)
    ib = b.view(np.int32).astype(np.int64)
    return np.abs(ia - ib)


def test_expf_error_within_one_ulp(oracle):
    # the method's published error bound is below 1 ulp; compare against a
    # binary64 evaluation rounded to binary32 over the range smooth-kNN uses
    rng = np.random.default_rng(3)
    x = np.concatenate([
        -rng.uniform(0, 87.0, 200_000), rng.uniform(-1, 1, 100_000),
        -np.logspace(-7, 1.9, 50_000),
    ]).astype(np.float32)
    y = oracle.expf(x)
    ref = np.exp(x.astype(np.float64)).astype(np.float32)
    assert _ulp_distance(y, ref).max() <= 1
    # the method is not correctly rounded: about 9 in 10 results are
    assert (y == ref).mean() > 0.85


def test_expf_subnormal_range_monotone(oracle):
    x = np.linspace(-103.9, -87.4, 20_001).astype(np.float32)
    y = oracle.expf(x)
    assert (np.diff(y.astype(np.float64)) >= 0).all()
    ref = np.exp(x.astype(np.float64)).astype(np.float32)
    assert _ulp_distance(y, ref).max() <= 1


def test_log2_target_is_platform_log2(oracle):
    for k in (2, 3, 15, 30, 100):
        assert oracle.lib().oracle_log2(float(k)) == math.log2(k)


# --- spectral stage: src/sparse.rs and src/eigen.rs tests -------------------

def p3_graph():
    # src/sparse.rs:105-115: path 0-1-2 with unit weights
    return (np.array([0, 1, 1, 2], dtype=np.uint32), np.array([1, 0, 2, 1], dtype=np.uint32),
            np.ones(4, dtype=np.float32), 3)


def wiggly_graph(n):
    """src/eigen.rs:252-273: a path with hashed weights plus two chords, as a
    (row, col)-sorted COO."""
    coo = []

    def push(a, b, w):
        coo.append((a, b, w))
        coo.append((b, a, w))

    for i in range(n - 1):
        h = (i * 2654435761) & 0xFFFFFFFF
        w = np.float32(np.float32(0.5) + np.float32(0.4) * np.float32(np.float32(h >> 16) / np.float32(65536.0)))
        push(i, i + 1, w)
    push(0, n // 2, np.float32(0.3))
    push(n // 4, 3 * n // 4, np.float32(0.2))
    coo.sort(key=lambda e: (e[0], e[1]))
    return (np.array([e[0] for e in coo], dtype=np.uint32), np.array([e[1] for e in coo], dtype=np.uint32),
            np.array([e[2] for e in coo], dtype=np.float32), n)


def dense_laplacian(indptr, cols, sv, n):
    a = np.eye(n)
    for i in range(n):
        for p in range(int(indptr[i]), int(indptr[i + 1])):
            a[i, cols[p]] -= sv[p]
    return a


def test_laplacian_csr_and_degrees(oracle):
    # src/sparse.rs:117-145
    r, c, v, n = p3_graph()
    indptr, sv, deg = oracle.laplacian(r, c, v, n)
    assert indptr.tolist() == [0, 1, 3, 4]
    assert deg.tolist() == [1.0, 2.0, 1.0]
    y = oracle.laplacian_matvec(indptr, c, sv, [1.0, math.sqrt(2.0), 1.0])
    assert np.abs(y).max() < 1e-12
    y = oracle.laplacian_matvec(indptr, c, sv, [1.0, 0.0, -1.0])
    assert np.abs(y - np.array([1.0, 0.0, -1.0])).max() < 1e-12


def test_laplacian_dense_matches_matvec(oracle):
    # src/sparse.rs:147-160
    r, c, v, n = wiggly_graph(40)
    indptr, sv, _ = oracle.laplacian(r, c, v, n)
    a = dense_laplacian(indptr, c, sv, n)
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        assert np.abs(a[:, j] - oracle.laplacian_matvec(indptr, c, sv, e)).max() < 1e-15


def eigen_close(oracle, indptr, cols, sv, n, vals, vecs, tol):
    # src/eigen.rs:275-299
    assert (np.diff(vals) >= -1e-12).all()
    for j in range(vals.size):
        v = vecs[j]
        assert abs(np.sqrt((v * v).sum()) - 1.0) < 1e-8
        y = oracle.laplacian_matvec(indptr, cols, sv, v)
        assert np.sqrt(((y - vals[j] * v) ** 2).sum()) < tol


def test_lanczos_recovers_p3_spectrum(oracle):
    # src/eigen.rs:300-316
    r, c, v, n = p3_graph()
    indptr, sv, _ = oracle.laplacian(r, c, v, n)
    vals, vecs, _ = oracle.lanczos(indptr, c, sv, n, 3)
    assert np.abs(vals - [0.0, 1.0, 2.0]).max() < 1e-12
    eigen_close(oracle, indptr, c, sv, n, vals, vecs, 1e-10)
    assert abs(vecs[1][1]) < 1e-10 and abs(abs(vecs[1][0]) - 1 / math.sqrt(2)) < 1e-10
    assert abs(vecs[1][0] + vecs[1][2]) < 1e-10


def test_lanczos_matches_dense_on_wiggly_graph(oracle):
    # src/eigen.rs:318-336: numpy's dense eigh stands in for nalgebra
    r, c, v, n = wiggly_graph(120)
    indptr, sv, _ = oracle.laplacian(r, c, v, n)
    k = 4
    vals, vecs, _ = oracle.lanczos(indptr, c, sv, n, k)
    ev, evec = np.linalg.eigh(dense_laplacian(indptr, c, sv, n))
    assert np.abs(vals - ev[:k]).max() < 1e-8
    eigen_close(oracle, indptr, c, sv, n, vals, vecs, 1e-7)
    for j in range(k):
        assert abs(vecs[j] @ evec[:, j]) > 1 - 1e-7


def test_spectral_golden_fixture(oracle):
    # src/fixture_parity.rs:125-185: kNN -> smooth-kNN -> fuzzy graph ->
    # Laplacian -> dim + 1 smallest eigenpairs against scipy's
    fx = json.loads((GOLDEN / "spectral_cloud_connected.json").read_text())
    data = f32(fx["data"])
    k, n, dim = fx["n_neighbors"], fx["n_samples"], fx["dim"]
    idx, dist = oracle.exact_knn(data, k, "euclidean")
    sig, rho = oracle.smooth_knn(dist, k)
    rows, cols, vals = oracle.fuzzy_graph(idx, dist, sig, rho, k)
    indptr, sv, _ = oracle.laplacian(rows, cols, vals, n)
    ev, vecs, _ = oracle.lanczos(indptr, cols, sv, n, dim + 1)
    assert np.abs(ev - np.asarray(fx["eigenvalues"])).max() < 1e-6
    for j, e in enumerate(fx["eigenvectors"][: dim + 1]):
        assert abs(vecs[j] @ np.asarray(e)) > 1 - 1e-6


def fuzzy_by_dict(idx, dist, sig, rho, k):
    """src/fuzzy.rs:25-91 restated once more with Python containers and numpy
    binary32 scalars, to check the C restatement."""
    n = idx.size // k
    a = {}
    for i in range(n):
        for j in range(k):
            c = int(idx[i * k + j])
            if c == i:
                continue
            d = np.float32(dist[i * k + j]) - np.float32(rho[i])
            if d <= 0 or sig[i] == 0:
                w = np.float32(1.0)
            else:
                w = np.float32(oracle_expf_scalar(-(d / np.float32(sig[i]))))
            if w != 0:
                a[(i, c)] = w
    coords = sorted(set(a) | {(c, r) for r, c in a})
    rows, cols, vals = [], [], []
    zero = np.float32(0.0)
    for r, c in coords:
        v, vt = a.get((r, c), zero), a.get((c, r), zero)
        w = np.float32(np.float32(v + vt) - np.float32(v * vt))
        if w != 0:
            rows.append(r)
            cols.append(c)
            vals.append(w)
    return np.array(rows, np.uint32), np.array(cols, np.uint32), np.array(vals, np.float32)


def oracle_expf_scalar(x):
    import holomap_oracle
    return holomap_oracle.expf(np.array([x], np.float32))[0]


@pytest.mark.parametrize("n,k,seed", [(30, 4, 1), (200, 8, 2), (400, 15, 3)])
def test_fuzzy_oracle_against_a_second_restatement(oracle, n, k, seed):
    g = np.random.default_rng(seed)
    idx = np.empty((n, k), np.uint32)
    for i in range(n):
        idx[i, 0] = i
        idx[i, 1:] = g.choice(np.delete(np.arange(n), i), size=k - 1, replace=False)
    dist = np.zeros((n, k), np.float32)
    dist[:, 1:] = np.sort(g.gamma(2.0, 1.0, size=(n, k - 1)).astype(np.float32), axis=1)
    dist, idx = dist.reshape(-1), idx.reshape(-1)
    sig, rho = oracle.smooth_knn(dist, k)
    sig = sig.copy()
    sig[::9] = 0.0
    a = oracle.fuzzy_graph(idx, dist, sig, rho, k)
    b = fuzzy_by_dict(idx, dist, sig, rho, k)
    for x, y, what in zip(a, b, ("rows", "cols", "vals")):
        assert x.shape == y.shape, what
        assert (x.view(np.uint32) == y.view(np.uint32)).all(), what


@pytest.mark.parametrize("n,seed", [(50, 4), (300, 5)])
def test_laplacian_oracle_against_a_second_restatement(oracle, n, seed):
    """src/sparse.rs:21-84 once more in Python floats (binary64, the same
    order; sums start from -0.0), against the C restatement bit for bit."""
    g = np.random.default_rng(seed)
    r, c, v, _ = wiggly_graph(n)
    v = (v * g.uniform(0.5, 1.5, v.size)).astype(np.float32)
    # symmetric weights again (the fuzzy graph is symmetric)
    w = {(int(a), int(b)): v[p] for p, (a, b) in enumerate(zip(r, c))}
    v = np.array([w[(int(min(a, b)), int(max(a, b)))] for a, b in zip(r, c)], np.float32)
    indptr, sv, deg = oracle.laplacian(r, c, v, n)
    ip = [0] * (n + 1)
    for a in r:
        ip[int(a) + 1] += 1
    for i in range(n):
        ip[i + 1] += ip[i]
    d = []
    for i in range(n):
        s = -0.0
        for p in range(ip[i], ip[i + 1]):
            s += float(v[p])
        d.append(s)
    inv = [1.0 / math.sqrt(x) for x in d]
    s2 = [float(v[p]) * (inv[int(r[p])] * inv[int(c[p])]) for p in range(r.size)]
    assert indptr.tolist() == ip
    assert np.array(d).view(np.uint64).tolist() == deg.view(np.uint64).tolist()
    assert np.array(s2).view(np.uint64).tolist() == sv.view(np.uint64).tolist()
    x = g.normal(size=n)
    y = oracle.laplacian_matvec(indptr, c, sv, x)
    for i in range(n):
        acc = -0.0
        for p in range(ip[i], ip[i + 1]):
            acc += s2[p] * x[int(c[p])]
        assert np.float64(x[i] - acc).view(np.uint64) == y[i].view(np.uint64)
