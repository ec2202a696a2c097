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
