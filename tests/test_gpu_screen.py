"""GPU parity of the screened paths (tcgen05 BF16 / TF32 / split-BF16 screen +
exact rerank): every path must return the oracle's bytes; the screen itself
must stay inside its proven band."""
import numpy as np
import pytest

import holomap_b200 as hm
from parity import assert_same_bytes, edge_case, rows_sorted_by_key

pytestmark = pytest.mark.gpu
PATHS = ["screen_bf16", "screen_tf32", "screen_bf16x3"]


def screened_values(x, metric, path):
    """Run one screened call with the dump hook set; return c^ (n x n)."""
    import torch
    n, d = x.shape
    buf = torch.full((n * n,), float("nan"), dtype=torch.float32, device="cuda")
    hm.lib().hm_debug_set_screen_dump(buf.data_ptr())
    try:
        hm.exact_knn(x, d, 5, metric, path)
    finally:
        hm.lib().hm_debug_set_screen_dump(None)
    return buf.cpu().numpy().reshape(n, n)


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("metric", ["cosine", "euclidean"])
def test_screen_values_track_exact_inner_products(path, metric):
    g = np.random.default_rng(1)
    n, d = 700, 72
    x = g.normal(size=(n, d)).astype(np.float32)
    c = screened_values(x, metric, path)
    xd = x.astype(np.float64)
    if metric == "cosine":
        u = xd / np.linalg.norm(xd, axis=1, keepdims=True)
        exact = 1.0 - u @ u.T
        tol = {"screen_bf16": 2e-2, "screen_tf32": 3e-3, "screen_bf16x3": 1e-4}[path]
    else:
        u = xd - xd.mean(0)
        m = np.sqrt((u * u).sum(1).max())
        u = u * 2.0 ** -np.frexp(m)[1]
        sq = (u * u).sum(1)
        exact = sq[:, None] + sq[None, :] - 2 * u @ u.T
        tol = {"screen_bf16": 2e-2, "screen_tf32": 3e-3, "screen_bf16x3": 1e-4}[path] * 4
    np.fill_diagonal(exact, 0.0)
    assert np.isfinite(c).all(), "screen left entries unwritten"
    err = np.abs(c - exact).max()
    assert err < tol, f"max |c^ - c| = {err}"


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("metric", ["euclidean", "cosine"])
@pytest.mark.parametrize("n,d,k", [(300, 5, 15), (1000, 50, 15), (4500, 130, 30), (2100, 384, 64),
                                   (5000, 16, 2), (1300, 7, 33)])
def test_screened_matches_oracle(oracle, path, metric, n, d, k):
    x = edge_case("gauss", n, d, seed=n + d)
    st = hm.HmStats()
    knn, sm = hm.knn_smooth(x, d, k, metric, path, stats=st)
    oi, od = oracle.exact_knn(x, k, metric)
    assert_same_bytes(knn.indices, oi, "indices")
    assert_same_bytes(knn.dists, od, "dists")
    osig, orho = oracle.smooth_knn(od, k)
    assert_same_bytes(sm.sigmas, osig, "sigma")
    assert_same_bytes(sm.rhos, orho, "rho")
    assert st.path_used == hm.KnnPath.parse(path)
    # every row is either reranked from at least k candidates or sent whole to
    # the exact fallback
    assert st.candidates_total >= (n - st.overflow_rows) * k


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("kind", ["duplicates", "ulp", "zeros", "huge", "tiny", "grid",
                                  "sorted_line"])
@pytest.mark.parametrize("metric", ["euclidean", "cosine"])
def test_screened_edge_cases(oracle, path, kind, metric):
    x = edge_case(kind, 1111, 6, seed=13)
    knn = hm.exact_knn(x, 6, 15, metric, path)
    oi, od = oracle.exact_knn(x, 15, metric)
    assert_same_bytes(knn.indices, oi, "indices")
    assert_same_bytes(knn.dists, od, "dists")


@pytest.mark.parametrize("name", ["blobs_euclidean", "cosine", "duplicates_euclidean"])
@pytest.mark.parametrize("path", PATHS)
def test_screened_golden_fixtures(oracle, name, path):
    import json
    from pathlib import Path
    fx = json.loads((Path(__file__).parent / "golden" / f"stage2_{name}.json").read_text())
    x = np.asarray(fx["data"], dtype=np.float32)
    k = fx["n_neighbors"]
    knn = hm.exact_knn(x, x.shape[1], k, fx["metric"], path)
    assert knn.indices.reshape(-1, k).tolist() == fx["knn_indices"]
    oi, od = oracle.exact_knn(x, k, fx["metric"])
    assert_same_bytes(knn.dists, od, "dists")


def test_screened_equals_plain_on_clustered_duplicates():
    from holomap_b200.synth import dups_20k
    wl = dups_20k(n=12000, d=64)
    a = hm.exact_knn(wl.data, wl.d, wl.k, wl.metric, "plain")
    for path in PATHS:
        st = hm.HmStats()
        b = hm.exact_knn(wl.data, wl.d, wl.k, wl.metric, path, stats=st)
        assert_same_bytes(b.indices, a.indices, f"{path} indices")
        assert_same_bytes(b.dists, a.dists, f"{path} dists")
        assert rows_sorted_by_key(b.indices.reshape(-1, wl.k), b.dists.reshape(-1, wl.k))


@pytest.mark.parametrize("path", PATHS)
def test_device_data_at_a_4_byte_offset(oracle, path):
    """The C ABI takes any 4-byte-aligned device pointer: points given at an
    odd float offset inside a larger buffer (d a multiple of 4, so the
    rerank's 16-byte row loads must not be used) return the oracle's bytes."""
    import torch
    from holomap_b200.device import DeviceKnnProblem
    n, d, k = 1500, 32, 15
    x = edge_case("gauss", n, d, seed=41)
    big = torch.zeros(n * d + 1, dtype=torch.float32, device="cuda")
    big[1:] = torch.from_numpy(x.reshape(-1)).cuda()
    view = big[1:].view(n, d)
    assert view.data_ptr() % 16 != 0
    p = DeviceKnnProblem(n, d, k, "euclidean", path)
    p.run(view)
    torch.cuda.synchronize()
    oi, od = oracle.exact_knn(x, k, "euclidean")
    assert_same_bytes(p.idx.cpu().numpy().view(np.uint32), oi, "indices")
    assert_same_bytes(p.dist.cpu().numpy(), od, "dists")
    assert p.stats().path_used == hm.KnnPath.parse(path)


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("metric", ["euclidean", "cosine"])
@pytest.mark.parametrize("n", [2600, 3000])
def test_full_and_symmetric_emission_agree_with_the_oracle(oracle, path, metric, n):
    """The emission pass over every column tile (hm_tuning_symmetric(0)) and
    over the tiles on and above the diagonal only (hm_tuning_symmetric(1),
    whose rows also take candidates as columns), each with one CTA per
    128-row block and in the 2-SM form, return the oracle's bytes; the zero
    rows under cosine exercise the column side's general (non raw-product)
    test, and n = 3000 ends inside a 256-row block's second half."""
    lib = hm.lib()
    x = edge_case("zeros" if metric == "cosine" else "duplicates", n, 40, seed=5)
    x[::7] += 0.5  # keep most rows non-zero
    oi, od = oracle.exact_knn(x, 15, metric)
    osig, orho = oracle.smooth_knn(od, 15)
    for sym in (0, 1):
        for pair in (0, 1):
            assert lib.hm_tuning_symmetric(sym) == 0
            assert lib.hm_tuning_pair(pair) == 0
            try:
                st = hm.HmStats()
                knn, sm = hm.knn_smooth(x, 40, 15, metric, path, stats=st)
            finally:
                lib.hm_tuning_symmetric(-1)
                lib.hm_tuning_pair(-1)
            what = f"sym={sym} pair={pair}"
            assert_same_bytes(knn.indices, oi, f"{what} indices")
            assert_same_bytes(knn.dists, od, f"{what} dists")
            assert_same_bytes(sm.sigmas, osig, f"{what} sigma")
            assert_same_bytes(sm.rhos, orho, f"{what} rho")


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("n", [200, 1000, 2600])
def test_pair_and_single_cta_emission_agree_with_the_oracle(oracle, path, n):
    """The emission pass in the 2-SM form (hm_tuning_pair(1): a cluster of two
    CTAs shares one 256-row MMA, each loading half of every column tile) and
    with one CTA per 128-row block (hm_tuning_pair(0)) return the oracle's bytes,
    including a last 256-row block that ends inside its first half (n = 200,
    1000) and one whose second half lies past every row (n = 2600)."""
    lib = hm.lib()
    x = edge_case("duplicates", n, 40, seed=n)
    oi, od = oracle.exact_knn(x, 15, "euclidean")
    osig, orho = oracle.smooth_knn(od, 15)
    for pair in (0, 1):
        assert lib.hm_tuning_pair(pair) == 0
        try:
            knn, sm = hm.knn_smooth(x, 40, 15, "euclidean", path)
        finally:
            lib.hm_tuning_pair(-1)
        assert_same_bytes(knn.indices, oi, f"pair={pair} indices")
        assert_same_bytes(knn.dists, od, f"pair={pair} dists")
        assert_same_bytes(sm.sigmas, osig, f"pair={pair} sigma")
        assert_same_bytes(sm.rhos, orho, f"pair={pair} rho")


def _tight_clusters(n, d, seed, sigma=0.05):
    """Eight clusters far tighter than a BF16 or TF32 operand's rounding
    relative to their distance from the origin (the coarse screens' hard case)."""
    g = np.random.default_rng(seed)
    centres = g.normal(0.0, 4.0, size=(8, d))
    labels = g.integers(0, 8, size=n)
    return np.ascontiguousarray((centres[labels] + g.normal(0.0, sigma, size=(n, d))).astype(np.float32))


@pytest.mark.parametrize("metric", ["cosine", "euclidean"])
def test_auto_escalates_on_clusters_tighter_than_the_screen(metric):
    """A job left to the autotuner, whose choice here is the BF16 (cosine) or
    TF32 (euclidean) screen, hands over to its split-BF16 copy when the
    coarse screen's band swamps the rows' thresholds; the bytes equal the
    plain path's either way (escalation off: the coarse screen's own, slow
    but exact, result)."""
    lib = hm.lib()
    n, d, k = 4096, 384, 15
    x = _tight_clusters(n, d, seed=7)
    assert hm.autotune_path(n, d, k, metric) in (hm.KnnPath.SCREEN_BF16, hm.KnnPath.SCREEN_TF32)
    plain, psm = hm.knn_smooth(x, d, k, metric, "plain")
    st = hm.HmStats()
    knn, sm = hm.knn_smooth(x, d, k, metric, "auto", stats=st)
    assert st.path_used == int(hm.KnnPath.SCREEN_BF16X3), st.path_used
    for a, b, what in ((knn.indices, plain.indices, "indices"), (knn.dists, plain.dists, "dists"),
                       (sm.sigmas, psm.sigmas, "sigma"), (sm.rhos, psm.rhos, "rho")):
        assert_same_bytes(a, b, f"escalated {what}")
    assert lib.hm_tuning_escalation(0) == 0
    try:
        st0 = hm.HmStats()
        knn0, sm0 = hm.knn_smooth(x, d, k, metric, "auto", stats=st0)
    finally:
        lib.hm_tuning_escalation(1)
    assert st0.path_used == int(hm.autotune_path(n, d, k, metric))
    assert_same_bytes(knn0.indices, plain.indices, "coarse indices")
    assert_same_bytes(knn0.dists, plain.dists, "coarse dists")


def test_auto_keeps_the_coarse_screen_on_embedding_shaped_data():
    """Embedding-shaped data (the autotuner's cosine family) keeps the BF16
    screen: its band is a few percent of the rows' thresholds."""
    from holomap_b200.synth import embed_50k
    wl = embed_50k(n=8192)
    assert hm.autotune_path(wl.n, wl.d, wl.k, wl.metric) == hm.KnnPath.SCREEN_BF16
    plain, _ = hm.knn_smooth(wl.data, wl.d, wl.k, wl.metric, "plain")
    st = hm.HmStats()
    knn, _ = hm.knn_smooth(wl.data, wl.d, wl.k, wl.metric, "auto", stats=st)
    assert st.path_used == int(hm.KnnPath.SCREEN_BF16)
    assert_same_bytes(knn.indices, plain.indices, "indices")
    assert_same_bytes(knn.dists, plain.dists, "dists")


def test_batch_escalates_only_the_job_that_needs_it():
    """In one batch, the tightly clustered job escalates and the
    embedding-shaped one does not; both return the plain path's bytes."""
    import torch
    from holomap_b200.device import DeviceBatch
    from holomap_b200.synth import embed_50k
    a = _tight_clusters(4096, 384, seed=3)
    b = embed_50k(n=4096).data
    batch = DeviceBatch([(torch.from_numpy(a).cuda(), 15, "cosine"), (torch.from_numpy(b).cuda(), 30, "cosine")])
    batch.run()
    torch.cuda.synchronize()
    for j, (x, k) in enumerate(((a, 15), (b, 30))):
        plain, psm = hm.knn_smooth(x, 384, k, "cosine", "plain")
        idx, dist, sig, rho = batch.result(j)
        assert_same_bytes(idx.reshape(-1), plain.indices, f"job {j} indices")
        assert_same_bytes(dist.reshape(-1), plain.dists, f"job {j} dists")
        assert_same_bytes(sig, psm.sigmas, f"job {j} sigma")
        assert_same_bytes(rho, psm.rhos, f"job {j} rho")
    paths = [batch.stats(j).path_used for j in range(2)]
    assert paths[0] == int(hm.KnnPath.SCREEN_BF16X3), paths
    assert paths[1] != int(hm.KnnPath.SCREEN_BF16X3), paths
