"""Device-resident runs of the kNN + smooth-kNN path (torch supplies memory and
streams; the work is hm_knn_smooth_device in libholomap_cuda.so)."""
from __future__ import annotations

import ctypes

import torch

from ._lib import HmStats, KnnPath, Metric, check, lib


class DeviceKnnProblem:
    """Output and workspace buffers for one (n, d, k, metric, path) problem,
    allocated once in HBM and reused by every :meth:`run`."""

    def __init__(self, n: int, d: int, k: int, metric="euclidean", path="auto",
                 device: int | torch.device = 0, smooth: bool = True):
        self.n, self.d, self.k = int(n), int(d), int(k)
        self.metric = Metric.parse(metric)
        self.path = KnnPath.parse(path)
        self.device = torch.device("cuda", device) if isinstance(device, int) else device
        ws = lib().hm_workspace_bytes(self.n, self.d, self.k, int(self.metric), int(self.path))
        if ws == 0:
            check(-1)
        self.workspace = torch.empty(ws + 256, dtype=torch.uint8, device=self.device)
        self.ws_ptr = (self.workspace.data_ptr() + 255) // 256 * 256
        self.ws_bytes = ws
        self.idx = torch.empty(self.n * self.k, dtype=torch.int32, device=self.device)
        self.dist = torch.empty(self.n * self.k, dtype=torch.float32, device=self.device)
        self.smooth = smooth
        self.sigma = torch.empty(self.n, dtype=torch.float32, device=self.device) if smooth else None
        self.rho = torch.empty(self.n, dtype=torch.float32, device=self.device) if smooth else None

    def run(self, data: torch.Tensor, stream: torch.cuda.Stream | None = None) -> None:
        """Enqueue both stages on ``stream`` (default: torch's current stream)."""
        assert data.is_cuda and data.dtype == torch.float32 and data.is_contiguous()
        assert data.numel() == self.n * self.d
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        check(lib().hm_knn_smooth_device(
            data.data_ptr(), self.n, self.d, self.k, int(self.metric), int(self.path),
            self.idx.data_ptr(), self.dist.data_ptr(),
            self.sigma.data_ptr() if self.smooth else None,
            self.rho.data_ptr() if self.smooth else None,
            self.ws_ptr, self.ws_bytes, s.cuda_stream, None))

    def stats(self) -> HmStats:
        """Counters of the last finished run (synchronous)."""
        st = HmStats()
        check(lib().hm_stats_from_workspace(self.ws_ptr, self.n, self.d, self.k, int(self.metric),
                                            int(self.path), ctypes.byref(st)))
        return st

    def indices_u32(self) -> torch.Tensor:
        return self.idx


class DeviceBatch:
    """Many independent kNN + smooth-kNN problems run as one batch on the
    device (one pass of the pipeline; screened jobs of one operand format
    share one persistent screen launch).  ``problems`` is a list of
    (data tensor [n, d] float32 on the GPU, k, metric[, path])."""

    def __init__(self, problems, device: int | torch.device = 0, smooth: bool = True):
        from ._lib import HmJob, KnnPath
        self.device = torch.device("cuda", device) if isinstance(device, int) else device
        self.problems = []
        jobs = (HmJob * len(problems))()
        # every job's outputs (indices, distances, sigmas, rhos) live in one
        # 4-byte-element buffer, so a batch's results come back in one copy
        sizes = [int(p[0].shape[0]) * int(p[1]) * 2 + (2 * int(p[0].shape[0]) if smooth else 0)
                 for p in problems]
        self.out = torch.empty(sum(sizes), dtype=torch.float32, device=self.device)
        off = 0
        for i, prob in enumerate(problems):
            data, k, metric = prob[0], int(prob[1]), Metric.parse(prob[2])
            path = KnnPath.parse(prob[3]) if len(prob) > 3 else KnnPath.AUTO
            assert data.is_cuda and data.dtype == torch.float32 and data.is_contiguous()
            n, d = data.shape

            def take(m):
                nonlocal off
                t = self.out[off:off + m]
                off += m
                return t
            idx = take(n * k).view(torch.int32)
            dist = take(n * k)
            sig = take(n) if smooth else None
            rho = take(n) if smooth else None
            self.problems.append((data, idx, dist, sig, rho, k))
            jobs[i] = HmJob(data.data_ptr(), n, d, k, int(metric), int(path), idx.data_ptr(),
                            dist.data_ptr(), sig.data_ptr() if smooth else None,
                            rho.data_ptr() if smooth else None)
        self._jobs = jobs
        h = ctypes.c_void_p()
        check(lib().hm_batch_create(jobs, len(problems), ctypes.byref(h)))
        self.handle = h
        ws = lib().hm_batch_workspace_bytes(h)
        self.workspace = torch.empty(ws + 256, dtype=torch.uint8, device=self.device)
        self.ws_ptr = (self.workspace.data_ptr() + 255) // 256 * 256
        s = torch.cuda.current_stream(self.device)
        check(lib().hm_batch_bind(h, self.ws_ptr, ws, s.cuda_stream))
        s.synchronize()  # the job tables are staged from host memory

    def run(self, stream: torch.cuda.Stream | None = None, graph: bool = False) -> None:
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        fn = lib().hm_batch_graph_launch if graph else lib().hm_batch_run
        check(fn(self.handle, s.cuda_stream))

    def stats(self, job: int) -> HmStats:
        st = HmStats()
        check(lib().hm_batch_job_stats(self.handle, job, ctypes.byref(st)))
        return st

    def path(self, job: int) -> int:
        return lib().hm_batch_job_path(self.handle, job)

    def result(self, job: int):
        """(indices uint32, dists, sigmas, rhos) of one job as numpy arrays."""
        import numpy as np
        _, idx, dist, sig, rho, _ = self.problems[job]
        out = [idx.cpu().numpy().view(np.uint32), dist.cpu().numpy()]
        out += [sig.cpu().numpy(), rho.cpu().numpy()] if sig is not None else [None, None]
        return out

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                lib().hm_batch_destroy(h)
            except Exception:
                pass
