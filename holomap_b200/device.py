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
