"""GPU parity of the fuzzy simplicial set (src/fuzzy.rs:25-91) against the
oracle's restatement, entry for entry and bit for bit, and against the
reference's own unit cases and golden fixtures."""
import json
from pathlib import Path

import numpy as np
import pytest

import holomap_b200 as hm
from holomap_b200._lib import check as check_rc
from parity import assert_same_bytes, edge_case

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def f32(x):
    return np.asarray(x, dtype=np.float32)


def check(oracle, idx, dist, sig, rho, k):
    g = hm.fuzzy_simplicial_set(hm.Knn(k, idx, dist), hm.SmoothKnn(sig, rho))
    rows, cols, vals = oracle.fuzzy_graph(idx, dist, sig, rho, k)
    assert g.n == idx.size // k
    assert_same_bytes(g.rows, rows, "rows")
    assert_same_bytes(g.cols, cols, "cols")
    assert_same_bytes(g.vals, vals, "vals")
    return g


def random_knn(n, k, seed):
    """A kNN-shaped graph: self first, then k - 1 distinct other points per
    row with ascending distances."""
    g = np.random.default_rng(seed)
    off = np.sort(g.integers(0, n - k + 1, size=(n, k - 1)), axis=1) + np.arange(k - 1) + 1
    idx = np.empty((n, k), dtype=np.uint32)
    idx[:, 0] = np.arange(n)
    idx[:, 1:] = (np.arange(n)[:, None] + off) % n
    dist = np.zeros((n, k), dtype=np.float32)
    dist[:, 1:] = np.sort(g.gamma(2.0, 1.0, size=(n, k - 1)).astype(np.float32), axis=1)
    return idx.reshape(-1), dist.reshape(-1)


def test_reference_line_points(oracle):
    # src/fuzzy.rs:97-129
    g = check(oracle, np.array([0, 1, 2, 1, 0, 2, 2, 1, 0], dtype=np.uint32),
              f32([0.0, 1.0, 3.0, 0.0, 1.0, 2.0, 0.0, 2.0, 3.0]),
              f32([3.72998046875, 1.864990234375, 1.864990234375]), f32([1.0, 1.0, 2.0]), 3)
    assert g.rows.tolist() == [0, 0, 1, 1, 2, 2]
    assert g.cols.tolist() == [1, 2, 0, 2, 0, 1]


def test_reference_one_directional_edge(oracle):
    # src/fuzzy.rs:131-155
    g = check(oracle, np.array([0, 1, 1, 2, 2, 1], dtype=np.uint32),
              f32([0.0, 1.0, 0.0, 0.1, 0.0, 0.1]), f32([1.0, 1.0, 1.0]), f32([0.5, 0.1, 0.1]), 2)
    w = oracle.expf(f32([-0.5]))[0]
    assert g.rows.tolist() == [0, 1, 1, 2]
    assert g.cols.tolist() == [1, 0, 2, 1]
    assert g.vals.tolist() == [w, w, 1.0, 1.0]


@pytest.mark.parametrize("name", ["blobs_euclidean", "cosine", "duplicates_euclidean"])
def test_golden_fixtures(oracle, name):
    # src/fixture_parity.rs:101-117 on the GPU's own kNN + smooth-kNN output
    fx = json.loads((GOLDEN / f"stage2_{name}.json").read_text())
    x = np.asarray(fx["data"], dtype=np.float32)
    k = fx["n_neighbors"]
    knn, sm = hm.knn_smooth(x, x.shape[1], k, fx["metric"])
    g = check(oracle, knn.indices, knn.dists, sm.sigmas, sm.rhos, k)
    assert g.rows.tolist() == fx["graph_rows"]
    assert g.cols.tolist() == fx["graph_cols"]
    e = np.asarray(fx["graph_vals"], dtype=np.float64)
    assert (np.abs(g.vals - e) <= 1e-5 * (1 + np.abs(e))).all()


@pytest.mark.parametrize("kind", ["gauss", "duplicates", "zeros", "huge", "grid", "sorted_line"])
@pytest.mark.parametrize("metric", ["euclidean", "cosine"])
def test_after_knn_edge_cases(oracle, kind, metric):
    # zero distances (d <= rho), sigma floors, zero vectors, tied neighbours
    x = edge_case(kind, 1500, 6, seed=5)
    knn, sm = hm.knn_smooth(x, 6, 15, metric)
    check(oracle, knn.indices, knn.dists, sm.sigmas, sm.rhos, 15)


@pytest.mark.parametrize("n,k", [(1, 1), (2, 2), (5, 5), (300, 1), (3000, 7), (65535, 4),
                                 (65536, 4), (200000, 15)])
def test_random_graphs(oracle, n, k):
    # the reverse copies are sorted on the bits of n: 16 up to n = 65535, 17
    # (a third radix pass) from n = 65536
    if k > n:
        pytest.skip("k above n")
    idx, dist = random_knn(n, k, seed=n + k) if k > 1 else (np.arange(n, dtype=np.uint32),
                                                            np.zeros(n, np.float32))
    sm = hm.smooth_knn(dist, k)
    g = check(oracle, idx, dist, sm.sigmas, sm.rhos, k)
    if k == 1:
        assert g.rows.size == 0  # only self edges
    key = g.rows.astype(np.uint64) << np.uint64(32) | g.cols
    assert (np.diff(key.astype(np.int64)) > 0).all()


def test_special_calibrations(oracle):
    # sigma == 0 rows, d <= rho, d - rho > 0 so large that expf underflows to
    # zero (dropped), +inf distances (weight 0, or 1 where sigma == 0), and
    # subnormal weights
    n, k = 4000, 8
    idx, dist = random_knn(n, k, seed=3)
    g = np.random.default_rng(4)
    sig = g.uniform(0.05, 2.0, size=n).astype(np.float32)
    rho = dist.reshape(n, k)[:, 1].copy()
    sig[::7] = 0.0
    rho[::11] = np.float32(1e30)
    d2 = dist.reshape(n, k)
    d2[::13, k // 2:] = np.float32(3e38)
    d2[5::17, 1:] = rho[5::17, None] + np.float32(95.0) * sig[5::17, None]
    d2[3::19, k - 1] = np.inf
    check(oracle, idx, dist, sig, rho, k)


def test_hub_rows(oracle):
    """Every row lists the same first points, so their reverse lists hold all
    n rows (in-degree n), next to rows of in-degree 0."""
    n, k = 5000, 6
    idx = np.empty((n, k), dtype=np.uint32)
    idx[:, 0] = np.arange(n)
    for r in range(n):
        others = [c for c in range(k + 1) if c != r][: k - 1]
        idx[r, 1:] = others
    dist = np.zeros((n, k), dtype=np.float32)
    dist[:, 1:] = np.linspace(0.5, 2.0, k - 1, dtype=np.float32)
    sm = hm.smooth_knn(dist.reshape(-1), k)
    g = check(oracle, idx.reshape(-1), dist.reshape(-1), sm.sigmas, sm.rhos, k)
    assert (g.rows == 0).sum() == n - 1


def test_device_entry_point_on_a_stream(oracle):
    """hm_fuzzy_graph_device on torch memory and a side stream equals the
    host entry point."""
    import ctypes
    import torch
    n, k = 20000, 12
    idx, dist = random_knn(n, k, seed=9)
    sm = hm.smooth_knn(dist, k)
    lib = hm.lib()
    ws_bytes = lib.hm_fuzzy_workspace_bytes(n, k)
    assert ws_bytes > 0
    dev = lambda a: torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda()
    d_idx, d_dist, d_sig, d_rho = dev(idx), dev(dist), dev(sm.sigmas), dev(sm.rhos)
    cap = 2 * n * k
    rows = torch.empty(cap, dtype=torch.int32, device="cuda")
    cols = torch.empty(cap, dtype=torch.int32, device="cuda")
    vals = torch.empty(cap, dtype=torch.float32, device="cuda")
    nnz = torch.zeros(1, dtype=torch.int64, device="cuda")
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    for _ in range(2):
        check_rc(lib.hm_fuzzy_graph_device(d_idx.data_ptr(), d_dist.data_ptr(), d_sig.data_ptr(),
                                           d_rho.data_ptr(), n, k, rows.data_ptr(), cols.data_ptr(),
                                           vals.data_ptr(), nnz.data_ptr(), ws.data_ptr(), ws_bytes,
                                           ctypes.c_void_p(s.cuda_stream)))
    s.synchronize()
    m = int(nnz.item())
    r, c, v = oracle.fuzzy_graph(idx, dist, sm.sigmas, sm.rhos, k)
    assert m == r.size
    assert_same_bytes(rows[:m].cpu().numpy().view(np.uint32), r, "rows")
    assert_same_bytes(cols[:m].cpu().numpy().view(np.uint32), c, "cols")
    assert_same_bytes(vals[:m].cpu().numpy(), v, "vals")


def test_device_entry_point_reports_an_index_not_below_n(oracle):
    """hm_fuzzy_graph_device trusts no index: entries at or above n are
    dropped by the rows kernel (so every later access stays in bounds) and
    hm_fuzzy_graph_status reports them; the rest of the graph is the fuzzy
    set of the graph without those entries."""
    import ctypes
    import torch
    n, k = 3000, 10
    idx, dist = random_knn(n, k, seed=17)
    sm = hm.smooth_knn(dist, k)
    bad = idx.copy().reshape(n, k)
    bad[5, 3] = n          # just past the end
    bad[77, 9] = 0xFFFFFFF0  # far past it
    bad = bad.reshape(-1)
    lib = hm.lib()
    ws_bytes = lib.hm_fuzzy_workspace_bytes(n, k)
    dev = lambda a: torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda()
    d_idx, d_dist, d_sig, d_rho = dev(bad), dev(dist), dev(sm.sigmas), dev(sm.rhos)
    cap = 2 * n * k
    rows = torch.empty(cap, dtype=torch.int32, device="cuda")
    cols = torch.empty(cap, dtype=torch.int32, device="cuda")
    vals = torch.empty(cap, dtype=torch.float32, device="cuda")
    nnz = torch.zeros(1, dtype=torch.int64, device="cuda")
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    check_rc(lib.hm_fuzzy_graph_device(d_idx.data_ptr(), d_dist.data_ptr(), d_sig.data_ptr(),
                                       d_rho.data_ptr(), n, k, rows.data_ptr(), cols.data_ptr(),
                                       vals.data_ptr(), nnz.data_ptr(), ws.data_ptr(), ws_bytes,
                                       stream))
    assert lib.hm_fuzzy_graph_status(ws.data_ptr(), n, k, stream) == hm.HM_ERR_INVALID
    assert b"not below n" in lib.hm_last_error()
    m = int(nnz.item())
    assert 0 < m <= cap
    # the same graph with those two entries given strength 0 (dropped) and a
    # valid column, which the oracle drops the same way
    fixed_idx, fixed_dist = idx.copy(), dist.copy()
    r, c, v = oracle.fuzzy_graph(fixed_idx, fixed_dist, sm.sigmas, sm.rhos, k)
    got = set(zip(rows[:m].cpu().numpy().tolist(), cols[:m].cpu().numpy().tolist()))
    want = set(zip(r.tolist(), c.tolist()))
    assert got <= want  # only entries of the valid graph, none invented
    # a valid graph afterwards reports no error on the same workspace
    d_idx.copy_(dev(idx))
    check_rc(lib.hm_fuzzy_graph_device(d_idx.data_ptr(), d_dist.data_ptr(), d_sig.data_ptr(),
                                       d_rho.data_ptr(), n, k, rows.data_ptr(), cols.data_ptr(),
                                       vals.data_ptr(), nnz.data_ptr(), ws.data_ptr(), ws_bytes,
                                       stream))
    assert lib.hm_fuzzy_graph_status(ws.data_ptr(), n, k, stream) == hm.HM_OK
    assert int(nnz.item()) == r.size
