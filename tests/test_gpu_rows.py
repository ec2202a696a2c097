"""Row shards on the device (hm_knn_rows_device): query rows [begin, end) of
the graph of all N points, on every path, must be exactly those rows of the
whole graph; the shards of a split run one after another on this GPU
(holomap_b200.shard.knn_smooth_shards_local) must reassemble the single-call
bytes, smooth-kNN included."""
import numpy as np
import pytest

import holomap_b200 as hm
from parity import assert_same_bytes, edge_case

pytestmark = pytest.mark.gpu

PATHS = ["plain", "screen_bf16", "screen_tf32", "screen_bf16x3"]


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("metric", ["euclidean", "cosine", "manhattan"])
def test_row_ranges_are_rows_of_the_whole_graph(oracle, path, metric):
    import torch
    from holomap_b200.shard import rows_cuda
    if metric == "manhattan" and path != "plain":
        pytest.skip("manhattan runs on the plain path only")
    n, d, k = 1500, 40, 15
    x = edge_case("duplicates", n, d, seed=31)
    oi, od = oracle.exact_knn(x, k, metric)
    oi, od = oi.reshape(n, k), od.reshape(n, k)
    xt = torch.from_numpy(x).cuda()
    for b, e in [(0, n), (0, 1), (n - 1, n), (5, 37), (128, 256), (100, 1300), (1279, 1500)]:
        idx, dist = rows_cuda(xt, k, metric, path, b, e)
        torch.cuda.synchronize()
        assert_same_bytes(idx.cpu().numpy().view(np.uint32), oi[b:e], f"rows [{b},{e}) indices")
        assert_same_bytes(dist.cpu().numpy(), od[b:e], f"rows [{b},{e}) dists")


@pytest.mark.parametrize("world", [2, 3, 7])
@pytest.mark.parametrize("path", ["plain", "screen_bf16x3"])
def test_local_shards_reassemble_the_single_call(world, path):
    import torch
    from holomap_b200.shard import knn_smooth_shards_local
    x = edge_case("gauss", 2100, 24, seed=world)
    whole, sm = hm.knn_smooth(x, 24, 15, "cosine", path)
    idx, dist, sig, rho = knn_smooth_shards_local(torch.from_numpy(x).cuda(), 15, "cosine", path,
                                                  world)
    assert_same_bytes(idx.cpu().numpy().view(np.uint32).reshape(-1), whole.indices, "indices")
    assert_same_bytes(dist.cpu().numpy().reshape(-1), whole.dists, "dists")
    assert_same_bytes(sig.cpu().numpy(), sm.sigmas, "sigma")
    assert_same_bytes(rho.cpu().numpy(), sm.rhos, "rho")


@pytest.mark.parametrize("k", [15, 40])
def test_smooth_rows_equal_rows_of_the_whole_calibration(oracle, k):
    """hm_smooth_knn_rows_device on a row range of the whole distance matrix
    returns those rows of the whole calibration, including rows whose rho is 0
    (their floor is the mean of all n * k distances, src/smooth_knn.rs:26)."""
    import ctypes
    import torch
    g = np.random.default_rng(k)
    n = 3000
    d = np.sort(g.exponential(size=(n, k)).astype(np.float32), axis=1)
    d[:, 0] = 0.0
    d[::13] = 0.0  # rows with no positive distance: the global-mean floor
    osig, orho = oracle.smooth_knn(d, k)
    lib = hm.lib()
    dt = torch.from_numpy(d).cuda()
    ws = torch.empty(lib.hm_smooth_workspace_bytes(n) + 256, dtype=torch.uint8, device="cuda")
    wp = (ws.data_ptr() + 255) // 256 * 256
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for b, e in [(0, n), (0, 1), (1, 14), (1024, 2048), (2999, 3000), (13, 2987)]:
        sig = torch.empty(e - b, dtype=torch.float32, device="cuda")
        rho = torch.empty(e - b, dtype=torch.float32, device="cuda")
        assert lib.hm_smooth_knn_rows_device(dt.data_ptr(), n, k, b, e, sig.data_ptr(), rho.data_ptr(),
                                             wp, stream) == hm.HM_OK, lib.hm_last_error()
        torch.cuda.synchronize()
        assert_same_bytes(sig.cpu().numpy(), osig[b:e], f"rows [{b},{e}) sigma")
        assert_same_bytes(rho.cpu().numpy(), orho[b:e], f"rows [{b},{e}) rho")
    for b, e in [(5, 5), (10, 3), (0, n + 1)]:
        assert lib.hm_smooth_knn_rows_device(dt.data_ptr(), n, k, b, e, sig.data_ptr(), rho.data_ptr(),
                                             wp, stream) == hm.HM_ERR_INVALID


def test_row_ranges_of_an_escalating_job():
    """Row ranges of a job left to the autotuner whose points are clusters far
    tighter than the coarse screen's rounding (the range job carries its
    split-BF16 escalation copy): the rows of the whole plain graph."""
    import torch
    from holomap_b200.shard import rows_cuda
    g = np.random.default_rng(17)
    n, d, k = 4096, 384, 15
    centres = g.normal(0.0, 4.0, size=(8, d))
    x = np.ascontiguousarray((centres[g.integers(0, 8, size=n)] + g.normal(0.0, 0.05, size=(n, d)))
                             .astype(np.float32))
    plain, _ = hm.knn_smooth(x, d, k, "cosine", "plain")
    pi = plain.indices.reshape(n, k)
    pd = plain.dists.reshape(n, k)
    xt = torch.from_numpy(x).cuda()
    for b, e in [(0, n), (100, 1300), (2048, 4096)]:
        idx, dist = rows_cuda(xt, k, "cosine", "auto", b, e)
        torch.cuda.synchronize()
        assert_same_bytes(idx.cpu().numpy().view(np.uint32), pi[b:e], f"rows [{b},{e}) indices")
        assert_same_bytes(dist.cpu().numpy(), pd[b:e], f"rows [{b},{e}) dists")
