"""Row-sharded kNN + smooth-kNN of one dataset over the ranks of a process
group (one process per GPU).

Every row's top-k is independent of every other row's (src/knn.rs:31-53 is a
loop over query rows), so rank r computes the query rows of its contiguous
shard against all N points (``hm_knn_rows_device``), and the shards'
indices and distances are all-gathered: the only exchange on the path.
smooth-kNN (src/smooth_knn.rs:23-80) then runs over all N rows on every
rank: a row's sigma depends only on its own distances, except the floor of a
``rho == 0`` row, which uses the mean over all N*k distances (``mean_all``,
src/smooth_knn.rs:26) -- running it on the gathered matrix gives exactly the
single-GPU bytes for any world size.

``compute_rows`` / ``compute_smooth`` default to the CUDA library; they are
parameters so that the host logic (shard bounds, gather, assembly) can be
exercised by CPU ranks with any other exact implementation plugged in.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import HmStats, KnnPath, Metric, check, lib

ROW_ALIGN = 128  # the screen's row block: shards split on block boundaries


def row_bounds(n: int, world: int, align: int = ROW_ALIGN) -> list[tuple[int, int]]:
    """Contiguous [begin, end) query rows per rank, balanced in blocks of
    ``align`` rows; ranks beyond the last block get an empty range."""
    blocks = (n + align - 1) // align
    out = []
    for r in range(world):
        b0 = blocks * r // world
        b1 = blocks * (r + 1) // world
        out.append((min(n, b0 * align), min(n, b1 * align)))
    return out


def rows_cuda(data, k: int, metric="euclidean", path="auto", row_begin: int = 0,
              row_end: int | None = None, stream=None):
    """Query rows [row_begin, row_end) of the exact kNN graph of all points of
    ``data`` (a CUDA float32 tensor n x d), on its device.  Returns
    (indices int32 view of u32, dists) tensors of shape (rows, k)."""
    import torch
    assert data.is_cuda and data.dtype == torch.float32 and data.is_contiguous()
    n, d = data.shape
    row_end = n if row_end is None else row_end
    m, p = int(Metric.parse(metric)), int(KnnPath.parse(path))
    ws = lib().hm_knn_rows_workspace_bytes(n, d, k, m, p, row_begin, row_end)
    if ws == 0:
        check(-1)
    dev = data.device
    work = torch.empty(ws + 256, dtype=torch.uint8, device=dev)
    wptr = (work.data_ptr() + 255) // 256 * 256
    rows = row_end - row_begin
    idx = torch.empty((rows, k), dtype=torch.int32, device=dev)
    dist = torch.empty((rows, k), dtype=torch.float32, device=dev)
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    check(lib().hm_knn_rows_device(data.data_ptr(), n, d, k, m, p, row_begin, row_end,
                                   idx.data_ptr(), dist.data_ptr(), wptr, ws, s.cuda_stream, None))
    st = HmStats()
    check(lib().hm_knn_rows_stats(wptr, n, d, k, m, p, row_begin, row_end, ctypes.byref(st)))
    return idx, dist


def smooth_cuda(dists, k: int, stream=None):
    """smooth-kNN over all rows of a CUDA (n, k) float32 distance tensor."""
    import torch
    n = dists.shape[0]
    dev = dists.device
    ws = lib().hm_smooth_workspace_bytes(n)
    work = torch.empty(ws + 256, dtype=torch.uint8, device=dev)
    wptr = (work.data_ptr() + 255) // 256 * 256
    sigma = torch.empty(n, dtype=torch.float32, device=dev)
    rho = torch.empty(n, dtype=torch.float32, device=dev)
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    check(lib().hm_smooth_knn_device(dists.contiguous().data_ptr(), n, k, sigma.data_ptr(),
                                     rho.data_ptr(), wptr, s.cuda_stream))
    torch.cuda.synchronize(dev)
    return sigma, rho


def knn_smooth_sharded(data, k: int, metric="euclidean", path="auto", group=None,
                       compute_rows=None, compute_smooth=None):
    """kNN + smooth-kNN of one dataset split by query rows over the ranks of
    ``group`` (torch.distributed).  Every rank passes the whole dataset and
    gets back the whole (indices, dists, sigmas, rhos), identical on every
    rank and to a single-GPU run.

    With the defaults, ``data`` is a CUDA tensor on this rank's device and
    the group's backend is NCCL.  Otherwise ``compute_rows(data, k, metric,
    path, begin, end) -> (idx (rows, k) int32/uint32, dists (rows, k) f32)`` and
    ``compute_smooth(dists (n, k), k) -> (sigmas, rhos)`` are used, and the
    tensors go through the group's backend on the CPU."""
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    n = int(data.shape[0])
    on_gpu = compute_rows is None
    compute_rows = compute_rows or rows_cuda
    compute_smooth = compute_smooth or smooth_cuda
    dev = data.device if on_gpu else torch.device("cpu")

    bounds = row_bounds(n, world)
    b0, b1 = bounds[rank]
    most = max(e - b for b, e in bounds)
    idx_pad = torch.zeros((most, k), dtype=torch.int32, device=dev)
    dist_pad = torch.zeros((most, k), dtype=torch.float32, device=dev)
    if b1 > b0:
        li, ld = compute_rows(data, k, metric, path, b0, b1)
        li = torch.as_tensor(np.asarray(li).view(np.int32) if not torch.is_tensor(li) else li)
        ld = torch.as_tensor(ld) if not torch.is_tensor(ld) else ld
        idx_pad[: b1 - b0] = li.reshape(b1 - b0, k).to(dev)
        dist_pad[: b1 - b0] = ld.reshape(b1 - b0, k).to(dev)
    # the one exchange: every rank's shard, padded to the largest
    gi = [torch.empty_like(idx_pad) for _ in range(world)]
    gd = [torch.empty_like(dist_pad) for _ in range(world)]
    dist.all_gather(gi, idx_pad, group=group)
    dist.all_gather(gd, dist_pad, group=group)
    idx = torch.cat([gi[r][: e - b] for r, (b, e) in enumerate(bounds)])
    dists = torch.cat([gd[r][: e - b] for r, (b, e) in enumerate(bounds)])
    if on_gpu:
        sigmas, rhos = compute_smooth(dists, k)
        return idx, dists, sigmas, rhos
    sigmas, rhos = compute_smooth(dists.numpy().reshape(-1), k)
    return idx.numpy().view(np.uint32), dists.numpy(), np.asarray(sigmas), np.asarray(rhos)


def knn_smooth_shards_local(data, k: int, metric="euclidean", path="auto", world: int = 2):
    """The sharded computation with its ``world`` shards run one after another
    on this process's GPU (no process group): the same bytes as the
    multi-rank run, for checking the row shards on a single device."""
    import torch
    n = int(data.shape[0])
    parts_i, parts_d = [], []
    for b, e in row_bounds(n, world):
        if e > b:
            i, d = rows_cuda(data, k, metric, path, b, e)
            parts_i.append(i)
            parts_d.append(d)
    idx = torch.cat(parts_i)
    dists = torch.cat(parts_d)
    sigmas, rhos = smooth_cuda(dists, k)
    return idx, dists, sigmas, rhos
