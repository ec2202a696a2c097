"""Batches: many independent problems of uneven n, d, k and metric in one pass
of the device pipeline (and through a captured CUDA graph); every job must
return the oracle's bytes, the same bytes as when run alone."""
import numpy as np
import pytest

import holomap_b200 as hm
from parity import assert_same_bytes, edge_case

pytestmark = pytest.mark.gpu


def make_problems(seed, count):
    g = np.random.default_rng(seed)
    probs = []
    for i in range(count):
        n = int(g.integers(40, 2500))
        d = int(g.choice([3, 16, 50, 128]))
        k = int(min(n, g.choice([2, 15, 30, 33])))
        metric = str(g.choice(["euclidean", "cosine", "manhattan"]))
        path = "auto"
        if metric != "manhattan" and k <= 64 and i % 3 == 0:
            path = str(g.choice(["screen_bf16", "screen_tf32", "screen_bf16x3"]))
        kind = str(g.choice(["gauss", "duplicates", "grid"]))
        x = edge_case(kind, n, d, seed=seed * 1000 + i)
        probs.append((x, k, metric, path))
    return probs


@pytest.mark.parametrize("graph", [False, True])
def test_batch_matches_oracle_per_job(oracle, graph):
    import torch
    from holomap_b200.device import DeviceBatch
    probs = make_problems(3, 24)
    dev = [(torch.from_numpy(x).cuda(), k, m, p) for x, k, m, p in probs]
    b = DeviceBatch(dev)
    for _ in range(2):  # replays must repeat the bytes
        b.run(graph=graph)
        torch.cuda.synchronize()
        for j, (x, k, metric, path) in enumerate(probs):
            idx, dist, sig, rho = b.result(j)
            oi, od = oracle.exact_knn(x, k, metric)
            assert_same_bytes(idx, oi, f"job {j} indices")
            assert_same_bytes(dist, od, f"job {j} dists")
            osig, orho = oracle.smooth_knn(od, k)
            assert_same_bytes(sig, osig, f"job {j} sigma")
            assert_same_bytes(rho, orho, f"job {j} rho")
            b.stats(j)


def test_batch_job_equals_job_alone():
    import torch
    from holomap_b200.device import DeviceBatch
    probs = make_problems(5, 10)
    dev = [(torch.from_numpy(x).cuda(), k, m, p) for x, k, m, p in probs]
    b = DeviceBatch(dev)
    b.run()
    torch.cuda.synchronize()
    for j, (x, k, metric, path) in enumerate(probs):
        alone, sm = hm.knn_smooth(x, x.shape[1], k, metric, path)
        idx, dist, sig, rho = b.result(j)
        assert_same_bytes(idx, alone.indices, f"job {j}")
        assert_same_bytes(dist, alone.dists, f"job {j}")
        assert_same_bytes(sig, sm.sigmas, f"job {j}")


def test_batch_of_screened_jobs_shares_one_screen():
    import torch
    from holomap_b200.device import DeviceBatch
    g = np.random.default_rng(9)
    xs = [g.normal(size=(int(n), 24)).astype(np.float32) for n in (3000, 4500, 700, 5000)]
    dev = [(torch.from_numpy(x).cuda(), 15, "cosine", "screen_bf16") for x in xs]
    b = DeviceBatch(dev)
    b.run(graph=True)
    torch.cuda.synchronize()
    for j, x in enumerate(xs):
        assert b.path(j) == hm.KnnPath.SCREEN_BF16
        alone = hm.exact_knn(x, 24, 15, "cosine", "plain")
        idx, dist, _, _ = b.result(j)
        assert_same_bytes(idx, alone.indices, f"job {j}")
        assert_same_bytes(dist, alone.dists, f"job {j}")
