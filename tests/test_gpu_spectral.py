"""GPU parity of the spectral stage: the normalized Laplacian and its matvec
bit for bit against the oracle's restatement of src/sparse.rs, and the
Lanczos eigenpairs of src/eigen.rs against the reference's own tolerances
(its unit tests and the scipy eigenpairs of its spectral fixture)."""
import ctypes
import json
from pathlib import Path

import numpy as np
import pytest

import holomap_b200 as hm
from holomap_b200._lib import check as check_rc
from parity import assert_same_bytes
from test_oracle import dense_laplacian, p3_graph, wiggly_graph

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def device_laplacian(rows, cols, vals, n):
    """hm_laplacian_device on torch memory; returns host (indptr, s, degrees)
    and the device tensors."""
    import torch
    r = torch.from_numpy(np.ascontiguousarray(rows, dtype=np.uint32).view(np.int32)).cuda()
    c = torch.from_numpy(np.ascontiguousarray(cols, dtype=np.uint32).view(np.int32)).cuda()
    v = torch.from_numpy(np.ascontiguousarray(vals, dtype=np.float32)).cuda()
    nnz = r.numel()
    indptr = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    sv = torch.empty(max(nnz, 1), dtype=torch.float64, device="cuda")
    deg = torch.empty(n, dtype=torch.float64, device="cuda")
    check_rc(hm.lib().hm_laplacian_device(r.data_ptr(), c.data_ptr(), v.data_ptr(), n, nnz,
                                          indptr.data_ptr(), sv.data_ptr(), deg.data_ptr(), None))
    torch.cuda.synchronize()
    host = (indptr.cpu().numpy().view(np.uint64), sv.cpu().numpy()[:nnz], deg.cpu().numpy())
    return host, (indptr, c, sv)


def check_laplacian(oracle, rows, cols, vals, n, seed=0):
    import torch
    (ip, sv, deg), (d_ip, d_c, d_sv) = device_laplacian(rows, cols, vals, n)
    oip, osv, odeg = oracle.laplacian(rows, cols, vals, n)
    assert_same_bytes(ip, oip, "indptr")
    assert_same_bytes(sv.view(np.uint64), osv.view(np.uint64), "s")
    assert_same_bytes(deg.view(np.uint64), odeg.view(np.uint64), "degrees")
    x = np.random.default_rng(seed).normal(size=n)
    x[::5] = 0.0
    d_x = torch.from_numpy(x).cuda()
    d_y = torch.empty_like(d_x)
    check_rc(hm.lib().hm_laplacian_matvec_device(d_ip.data_ptr(), d_c.data_ptr(), d_sv.data_ptr(), n,
                                                 d_x.data_ptr(), d_y.data_ptr(), None))
    torch.cuda.synchronize()
    y = oracle.laplacian_matvec(oip, cols, osv, x)
    assert_same_bytes(d_y.cpu().numpy().view(np.uint64), y.view(np.uint64), "L x")
    return oip, osv


def test_laplacian_path_graph(oracle):
    # src/sparse.rs:117-145
    r, c, v, n = p3_graph()
    check_laplacian(oracle, r, c, v, n)
    (ip, _, deg), _ = device_laplacian(r, c, v, n)
    assert ip.tolist() == [0, 1, 3, 4]
    assert deg.tolist() == [1.0, 2.0, 1.0]


@pytest.mark.parametrize("n", [40, 120, 1000])
def test_laplacian_wiggly(oracle, n):
    r, c, v, n = wiggly_graph(n)
    check_laplacian(oracle, r, c, v, n, seed=n)


@pytest.mark.parametrize("n", [130, 3000])
def test_laplacian_hub_rows(oracle, n):
    """Node 0 is joined to every other node (a row of n - 1 entries, summed by
    the long-row kernel) on top of a path with hashed weights."""
    edges = {}
    for j in range(1, n):
        edges[(0, j)] = edges[(j, 0)] = np.float32(0.25 + (j % 7) / 10)
    for j in range(1, n - 1):
        w = np.float32(((j * 2654435761) & 0xFFFF) / 65536.0 + 0.1)
        edges[(j, j + 1)] = edges[(j + 1, j)] = w
    keys = sorted(edges)
    r = np.array([a for a, _ in keys], dtype=np.uint32)
    c = np.array([b for _, b in keys], dtype=np.uint32)
    v = np.array([edges[e] for e in keys], dtype=np.float32)
    check_laplacian(oracle, r, c, v, n, seed=n)


@pytest.mark.parametrize("n,k,metric", [(3000, 15, "euclidean"), (20000, 30, "cosine")])
def test_laplacian_of_fuzzy_graphs(oracle, n, k, metric):
    from parity import edge_case
    x = edge_case("gauss", n, 24, seed=n)
    knn, sm = hm.knn_smooth(x, 24, k, metric)
    g = hm.fuzzy_simplicial_set(knn, sm)
    check_laplacian(oracle, g.rows, g.cols, g.vals, n, seed=k)


def graph_of(rows, cols, vals, n):
    return hm.FuzzyGraph(n, np.asarray(rows, np.uint32), np.asarray(cols, np.uint32),
                         np.asarray(vals, np.float32))


def eigen_close(oracle, ip, cols, sv, pairs, tol):
    # src/eigen.rs:275-299
    assert (np.diff(pairs.values) >= -1e-12).all()
    for j in range(pairs.values.size):
        v = pairs.vectors[j]
        assert abs(np.sqrt((v * v).sum()) - 1.0) < 1e-8
        y = oracle.laplacian_matvec(ip, cols, sv, v)
        assert np.sqrt(((y - pairs.values[j] * v) ** 2).sum()) < tol


def test_eigenpairs_path_graph(oracle):
    # src/eigen.rs:300-316
    r, c, v, n = p3_graph()
    pairs = hm.smallest_eigenpairs(graph_of(r, c, v, n), 3)
    assert np.abs(pairs.values - [0.0, 1.0, 2.0]).max() < 1e-12
    ip, sv, _ = oracle.laplacian(r, c, v, n)
    eigen_close(oracle, ip, c, sv, pairs, 1e-10)
    v1 = pairs.vectors[1]
    assert abs(v1[1]) < 1e-10 and abs(abs(v1[0]) - 1 / np.sqrt(2)) < 1e-10 and abs(v1[0] + v1[2]) < 1e-10


def test_eigenpairs_match_dense_on_wiggly_graph(oracle):
    # src/eigen.rs:318-336 (numpy's dense eigh in place of nalgebra's)
    r, c, v, n = wiggly_graph(120)
    k = 4
    pairs = hm.smallest_eigenpairs(graph_of(r, c, v, n), k)
    ip, sv, _ = oracle.laplacian(r, c, v, n)
    ev, evec = np.linalg.eigh(dense_laplacian(ip, c, sv, n))
    assert np.abs(pairs.values - ev[:k]).max() < 1e-8
    eigen_close(oracle, ip, c, sv, pairs, 1e-7)
    for j in range(k):
        assert abs(pairs.vectors[j] @ evec[:, j]) > 1 - 1e-7


def test_eigenpairs_identical_across_runs():
    # src/eigen.rs:337-344
    r, c, v, n = wiggly_graph(150)
    a = hm.smallest_eigenpairs(graph_of(r, c, v, n), 3)
    b = hm.smallest_eigenpairs(graph_of(r, c, v, n), 3)
    assert_same_bytes(a.values.view(np.uint64), b.values.view(np.uint64), "values")
    assert_same_bytes(a.vectors.view(np.uint64), b.vectors.view(np.uint64), "vectors")


def test_spectral_golden_fixture():
    # src/fixture_parity.rs:125-185, every stage on the GPU
    fx = json.loads((GOLDEN / "spectral_cloud_connected.json").read_text())
    x = np.asarray(fx["data"], dtype=np.float32)
    k, dim = fx["n_neighbors"], fx["dim"]
    knn, sm = hm.knn_smooth(x, x.shape[1], k, "euclidean")
    pairs = hm.smallest_eigenpairs(hm.fuzzy_simplicial_set(knn, sm), dim + 1)
    assert np.abs(pairs.values - np.asarray(fx["eigenvalues"])).max() < 1e-6
    for j, e in enumerate(fx["eigenvectors"][: dim + 1]):
        assert abs(pairs.vectors[j] @ np.asarray(e)) > 1 - 1e-6


def test_eigenpairs_of_a_fuzzy_graph_against_the_oracle(oracle):
    """A 5000-point connected kNN graph: the GPU eigenpairs and the oracle's
    restatement of the reference's Lanczos agree to the reference's
    tolerances."""
    from parity import edge_case
    n, k = 5000, 15
    x = edge_case("gauss", n, 10, seed=8)
    knn, sm = hm.knn_smooth(x, 10, k, "euclidean")
    g = hm.fuzzy_simplicial_set(knn, sm)
    pairs = hm.smallest_eigenpairs(g, 3)
    ip, sv, _ = oracle.laplacian(g.rows, g.cols, g.vals, n)
    ov, ovec, _ = oracle.lanczos(ip, g.cols, sv, n, 3)
    assert pairs.values.size == 3 and ov.size == 3
    assert np.abs(pairs.values - ov).max() < 1e-8
    eigen_close(oracle, ip, g.cols, sv, pairs, 1e-7)
    for j in range(3):
        assert abs(pairs.vectors[j] @ ovec[j]) > 1 - 1e-6


def test_device_entry_points_on_a_stream(oracle):
    import torch
    r, c, v, n = wiggly_graph(150)
    lib = hm.lib()
    s = torch.cuda.Stream()
    d_r = torch.from_numpy(r.view(np.int32)).cuda()
    d_c = torch.from_numpy(c.view(np.int32)).cuda()
    d_v = torch.from_numpy(v).cuda()
    ip = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    sv = torch.empty(r.size, dtype=torch.float64, device="cuda")
    deg = torch.empty(n, dtype=torch.float64, device="cuda")
    s.wait_stream(torch.cuda.current_stream())
    check_rc(lib.hm_laplacian_device(d_r.data_ptr(), d_c.data_ptr(), d_v.data_ptr(), n, r.size, ip.data_ptr(),
                                     sv.data_ptr(), deg.data_ptr(), ctypes.c_void_p(s.cuda_stream)))
    ws_bytes = lib.hm_eigenpairs_workspace_bytes(n, 3)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    vals = np.empty(3)
    vecs = np.empty(3 * n)
    found, cycles = ctypes.c_uint32(0), ctypes.c_uint32(0)
    check_rc(lib.hm_eigenpairs_device(ip.data_ptr(), d_c.data_ptr(), sv.data_ptr(), n, 3, ws.data_ptr(),
                                      ws_bytes, ctypes.c_void_p(s.cuda_stream), vals.ctypes.data,
                                      vecs.ctypes.data, ctypes.byref(found), ctypes.byref(cycles)))
    assert found.value == 3 and cycles.value >= 1
    ref = hm.smallest_eigenpairs(graph_of(r, c, v, n), 3)
    assert_same_bytes(vals.view(np.uint64), ref.values.view(np.uint64), "values")
    assert_same_bytes(vecs.view(np.uint64), ref.vectors.reshape(-1).view(np.uint64), "vectors")
