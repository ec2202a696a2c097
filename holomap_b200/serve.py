"""Request loop over the C ABI's serving context (``hm_ctx_*``, ``hm_submit``,
``hm_wait``): fit requests are admitted by device footprint and run as
continuously re-formed batches; each request returns the same arrays as
``exact_knn`` + ``smooth_knn`` (src/api.rs:147-148) on its own data.

Host buffers handed to the library must stay alive and unmoved until the
request finishes; :class:`Ticket` keeps them.  Page-locked buffers (the
default here, through torch) let the library's copies overlap the device work.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from ._lib import (HM_ERR_NOT_READY, HM_OK, HmCtxConfig, HmCtxTotals, HmJob, HmRequestInfo,
                   KnnPath, Metric, check, lib)


def host_buffer(shape, dtype, pinned: bool = True) -> np.ndarray:
    """A numpy array, page-locked when ``pinned`` (through torch)."""
    if pinned:
        import torch
        tdt = {np.float32: torch.float32, np.uint32: torch.int32}[np.dtype(dtype).type]
        t = torch.empty(shape, dtype=tdt, pin_memory=True)
        return t.numpy().view(dtype)
    return np.empty(shape, dtype=dtype)


@dataclass
class Ticket:
    id: int
    n: int
    k: int
    data: np.ndarray
    indices: np.ndarray
    dists: np.ndarray
    sigmas: np.ndarray | None
    rhos: np.ndarray | None
    info: dict = field(default_factory=dict)


def _info_dict(info: HmRequestInfo) -> dict:
    return {
        "status": info.status, "path_used": info.path_used, "batch": info.batch,
        "batch_jobs": info.batch_jobs, "submit_ms": info.submit_ms, "admit_ms": info.admit_ms,
        "done_ms": info.done_ms, "stats": info.stats.as_dict(),
    }


class Server:
    """One serving context on the current CUDA device."""

    def __init__(self, memory_bytes: int = 0, max_inflight: int = 0, max_batch_jobs: int = 0,
                 max_batch_work: float = 0.0, small_work: float = 0.0, pinned: bool = True):
        cfg = HmCtxConfig(memory_bytes, max_inflight, max_batch_jobs, max_batch_work, small_work)
        self._ctx = ctypes.c_void_p()
        check(lib().hm_ctx_create(ctypes.byref(cfg), ctypes.byref(self._ctx)))
        self.pinned = pinned

    def submit(self, data: np.ndarray, k: int, metric="euclidean", path="auto",
               smooth: bool = True, outputs: tuple | None = None) -> Ticket:
        """Queue one request; ``data`` is n x d float32 (copied to a
        page-locked buffer unless it already is one of ours)."""
        data = np.ascontiguousarray(data, dtype=np.float32)
        n, d = data.shape
        if outputs is None:
            idx = host_buffer((n, k), np.uint32, self.pinned)
            dist = host_buffer((n, k), np.float32, self.pinned)
            sig = host_buffer(n, np.float32, self.pinned) if smooth else None
            rho = host_buffer(n, np.float32, self.pinned) if smooth else None
        else:
            idx, dist, sig, rho = outputs
        job = HmJob(data.ctypes.data, n, d, k, int(Metric.parse(metric)), int(KnnPath.parse(path)),
                    idx.ctypes.data, dist.ctypes.data,
                    sig.ctypes.data if sig is not None else None,
                    rho.ctypes.data if rho is not None else None)
        t = ctypes.c_uint64()
        check(lib().hm_submit(self._ctx, ctypes.byref(job), ctypes.byref(t)))
        return Ticket(t.value, n, k, data, idx, dist, sig, rho)

    def poll(self, ticket: Ticket) -> bool:
        info = HmRequestInfo()
        rc = lib().hm_poll(self._ctx, ticket.id, ctypes.byref(info))
        ticket.info = _info_dict(info)
        if rc == HM_ERR_NOT_READY:
            return False
        check(rc)
        return True

    def wait(self, ticket: Ticket, timeout_s: float = 600.0) -> Ticket:
        """Block until the request finishes; raises its error, or
        TimeoutError when it is still pending after ``timeout_s``."""
        info = HmRequestInfo()
        rc = lib().hm_wait(self._ctx, ticket.id, int(timeout_s * 1e9), ctypes.byref(info))
        ticket.info = _info_dict(info)
        if rc == HM_ERR_NOT_READY:
            raise TimeoutError(f"request {ticket.id} still pending after {timeout_s} s")
        check(rc)
        return ticket

    def release(self, ticket: Ticket) -> None:
        check(lib().hm_release(self._ctx, ticket.id))

    def totals(self) -> dict:
        t = HmCtxTotals()
        check(lib().hm_ctx_totals_read(self._ctx, ctypes.byref(t)))
        return t.as_dict()

    def close(self) -> None:
        if self._ctx:
            rc = lib().hm_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()
            if rc != HM_OK:
                check(rc)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
