"""The allocation-free entry point, hm_knn_smooth_noalloc.

Some callers of this library cannot call cudaMalloc: a plugin inside a host
engine that has already reserved the card's memory for its own allocator, or
a latency-bound request loop that must not touch the allocator because
cudaMalloc/cudaFree can block and synchronise the device.  For them the
library keeps a fixed scratch array in its own image, and this entry point
takes only the caller's device inputs and outputs.

These tests call it through the C ABI and check that it returns exactly what
the workspace-taking entry point (hm_knn_smooth_device) returns, and what the
oracle (the C restatement of src/knn.rs + src/smooth_knn.rs) returns, on two
calls in a row (the scratch array keeps the previous call's contents, so the
second call must not depend on them).  Because the call does not wait for the
device, an input error (a non-finite point) surfaces through
hm_noalloc_stats, which reads the counters the call left in the scratch
without allocating.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import holomap_b200 as hm
from holomap_b200._lib import Metric

pytestmark = pytest.mark.gpu


def _problem(n, d, seed):
    g = np.random.default_rng(seed)
    x = g.normal(size=(n, d)).astype(np.float32)
    x[n // 2: n // 2 + n // 10] = x[: n // 10]  # exact duplicates: index tie-breaks
    return x


def _outputs(torch, n, k):
    return (torch.empty(n * k, dtype=torch.int32, device="cuda"),
            torch.empty(n * k, dtype=torch.float32, device="cuda"),
            torch.empty(n, dtype=torch.float32, device="cuda"),
            torch.empty(n, dtype=torch.float32, device="cuda"))


def _with_workspace(torch, lib, x_dev, n, d, k, metric):
    """Results of the existing entry point, with a caller-allocated workspace."""
    ws_bytes = lib.hm_workspace_bytes(n, d, k, metric, hm.KnnPath.PLAIN)
    assert ws_bytes > 0
    ws = torch.empty(ws_bytes + 256, dtype=torch.uint8, device="cuda")
    ws_ptr = (ws.data_ptr() + 255) // 256 * 256
    out = _outputs(torch, n, k)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.hm_knn_smooth_device(x_dev.data_ptr(), n, d, k, metric, hm.KnnPath.PLAIN,
                                  out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(),
                                  out[3].data_ptr(), ws_ptr, ws_bytes, stream, None)
    assert rc == hm.HM_OK, lib.hm_last_error()
    torch.cuda.synchronize()
    return [t.cpu().numpy().view(np.uint32) for t in out]


def _launch_no_alloc(torch, lib, x_dev, n, d, k, metric, out):
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.hm_knn_smooth_noalloc(x_dev.data_ptr(), n, d, k, metric, out[0].data_ptr(),
                                   out[1].data_ptr(), out[2].data_ptr(), out[3].data_ptr(),
                                   stream)
    assert rc == hm.HM_OK, lib.hm_last_error()
    return stream


def _no_alloc(torch, lib, x_dev, n, d, k, metric):
    out = _outputs(torch, n, k)
    stream = _launch_no_alloc(torch, lib, x_dev, n, d, k, metric, out)
    st = hm.HmStats()
    rc = lib.hm_noalloc_stats(stream, ctypes.byref(st))
    assert rc == hm.HM_OK, lib.hm_last_error()
    assert st.path_used == hm.KnnPath.PLAIN
    torch.cuda.synchronize()
    return [t.cpu().numpy().view(np.uint32) for t in out]


def _oracle_bits(oracle, x, k, metric):
    oi, od = oracle.exact_knn(x, k, str(metric))
    osig, orho = oracle.smooth_knn(od, k)
    return [np.ascontiguousarray(a).reshape(-1).view(np.uint32) for a in (oi, od, osig, orho)]


def test_no_alloc_matches_workspace_entry_point_on_two_calls_in_a_row(oracle):
    torch = pytest.importorskip("torch")
    lib = hm.lib()
    # a larger problem (two column splits, partial lists in scratch), then a
    # smaller one with another metric and k, so the second call runs over the
    # first call's leftovers
    cases = [(6000, 48, 15, Metric.EUCLIDEAN, 11), (1500, 20, 30, Metric.COSINE, 12)]
    for n, d, k, metric, seed in cases:
        x = _problem(n, d, seed)
        x_dev = torch.from_numpy(x).cuda()
        expected = _with_workspace(torch, lib, x_dev, n, d, k, int(metric))
        got = _no_alloc(torch, lib, x_dev, n, d, k, int(metric))
        want = _oracle_bits(oracle, x, k, metric)
        for name, a, b, c in zip(("indices", "dists", "sigmas", "rhos"), got, expected, want):
            assert np.array_equal(a, b), f"{name} differ for n={n} d={d} k={k} {metric}"
            assert np.array_equal(a, c), f"{name} differ from the oracle for n={n} d={d} k={k}"


def test_no_alloc_reports_a_non_finite_input_through_its_stats():
    torch = pytest.importorskip("torch")
    lib = hm.lib()
    n, d, k = 800, 16, 15
    x = _problem(n, d, 31)
    x[123, 5] = np.nan  # flat index 123 * 16 + 5 = 1973
    x_dev = torch.from_numpy(x).cuda()
    out = _outputs(torch, n, k)
    stream = _launch_no_alloc(torch, lib, x_dev, n, d, k, int(Metric.EUCLIDEAN), out)
    rc = lib.hm_noalloc_stats(stream, None)
    assert rc == hm.HM_ERR_INVALID
    assert b"index 1973" in lib.hm_last_error()
    # the next call clears the counters it inherits from the failed one
    x[123, 5] = 0.0
    x_dev = torch.from_numpy(x).cuda()
    _no_alloc(torch, lib, x_dev, n, d, k, int(Metric.EUCLIDEAN))


def test_no_alloc_repeat_call_is_identical(oracle):
    torch = pytest.importorskip("torch")
    lib = hm.lib()
    n, d, k = 3000, 32, 15
    x = _problem(n, d, 21)
    x_dev = torch.from_numpy(x).cuda()
    first = _no_alloc(torch, lib, x_dev, n, d, k, int(Metric.MANHATTAN))
    second = _no_alloc(torch, lib, x_dev, n, d, k, int(Metric.MANHATTAN))
    expected = _with_workspace(torch, lib, x_dev, n, d, k, int(Metric.MANHATTAN))
    want = _oracle_bits(oracle, x, k, Metric.MANHATTAN)
    for a, b, c, w in zip(first, second, expected, want):
        assert np.array_equal(a, b) and np.array_equal(a, c) and np.array_equal(a, w)


def test_no_alloc_rejects_problems_above_the_static_scratch():
    torch = pytest.importorskip("torch")
    lib = hm.lib()
    limit = lib.hm_noalloc_scratch_bytes()
    n, d, k = 50000, 384, 30  # its binary64 copy alone is ~154 MB
    assert lib.hm_workspace_bytes(n, d, k, int(Metric.COSINE), hm.KnnPath.PLAIN) > limit
    x_dev = torch.empty(n * d, dtype=torch.float32, device="cuda")
    out = _outputs(torch, n, k)
    rc = lib.hm_knn_smooth_noalloc(x_dev.data_ptr(), n, d, k, int(Metric.COSINE),
                                   out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(),
                                   out[3].data_ptr(), None)
    assert rc == hm.HM_ERR_UNSUPPORTED
    assert b"static scratch" in lib.hm_last_error()
