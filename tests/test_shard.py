"""Row sharding of one dataset over ranks (holomap_b200.shard): the host logic
(shard bounds, the all-gather, assembly, smooth-kNN over the gathered matrix)
run by world-size-2 gloo ranks on the CPU, with the oracle plugged in as the
per-shard computation.  The assembled arrays must equal the single-process
oracle bytes on every rank, including rho == 0 rows whose sigma floor needs
the mean over all N*k distances."""
import os
import socket

import numpy as np
import pytest

from holomap_b200.shard import row_bounds


def test_row_bounds_cover_rows_once():
    for n in (1, 5, 127, 128, 129, 1000, 50000):
        for world in (1, 2, 3, 8):
            b = row_bounds(n, world)
            assert len(b) == world
            assert b[0][0] == 0 and b[-1][1] == n
            for (b0, e0), (b1, e1) in zip(b, b[1:]):
                assert e0 == b1 and b0 <= e0
            inner = [x for x in b if x[1] > x[0]]
            assert all(x[0] % 128 == 0 for x in inner)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _dataset(kind):
    g = np.random.default_rng(17)
    if kind == "gauss":
        return g.normal(size=(333, 12)).astype(np.float32), 15, "euclidean"
    # heavy duplicates: rows whose k nearest are all at distance 0 (rho == 0)
    base = g.normal(size=(40, 6)).astype(np.float32)
    x = np.repeat(base, 20, axis=0)[:790]
    return np.ascontiguousarray(x), 10, "cosine"


def _rank(rank, world, port, kind, out_dir):
    import torch.distributed as dist

    import holomap_oracle
    from holomap_b200.shard import knn_smooth_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        x, k, metric = _dataset(kind)

        def rows(data, k_, metric_, path_, b, e):
            return holomap_oracle.exact_knn(np.asarray(data), k_, metric_, rows=(b, e))

        idx, dists, sig, rho = knn_smooth_sharded(
            __import__("torch").from_numpy(x), k, metric, compute_rows=rows,
            compute_smooth=holomap_oracle.smooth_knn)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), idx=idx, dists=dists, sig=sig, rho=rho)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["gauss", "dups"])
def test_two_gloo_ranks_assemble_the_single_process_bytes(tmp_path, oracle, kind):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), kind, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    x, k, metric = _dataset(kind)
    oi, od = oracle.exact_knn(x, k, metric)
    osig, orho = oracle.smooth_knn(od, k)
    if kind == "dups":
        assert (orho == 0).any(), "the case must exercise the global-mean floor"
    for r in range(world):
        got = np.load(tmp_path / f"r{r}.npz")
        assert got["idx"].reshape(-1).tobytes() == oi.reshape(-1).tobytes()
        assert got["dists"].reshape(-1).tobytes() == od.reshape(-1).tobytes()
        assert got["sig"].tobytes() == osig.tobytes()
        assert got["rho"].tobytes() == orho.tobytes()
