"""The request loop (hm_ctx_*, hm_submit, hm_wait): requests admitted by device
footprint and run as continuously re-formed, overlapping batches must each
return the oracle's bytes and the bytes of the same request run alone, and
the loop must reject what cannot fit and isolate a failing request."""
import threading
import time

import numpy as np
import pytest

import holomap_b200 as hm
from holomap_b200.serve import Server
from parity import assert_same_bytes, edge_case

pytestmark = pytest.mark.gpu


def make_requests(seed, count, n_hi=1800):
    g = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        n = int(g.integers(40, n_hi))
        d = int(g.choice([8, 32, 64, 300]))
        k = int(min(n, g.choice([5, 15, 30])))
        metric = str(g.choice(["euclidean", "cosine", "manhattan"], p=[0.5, 0.4, 0.1]))
        kind = str(g.choice(["gauss", "duplicates", "grid"]))
        reqs.append((edge_case(kind, n, d, seed=seed * 1000 + i), k, metric))
    return reqs


def check_against_oracle(oracle, t, x, k, metric, what):
    oi, od = oracle.exact_knn(x, k, metric)
    assert_same_bytes(t.indices.reshape(-1), oi, f"{what} indices")
    assert_same_bytes(t.dists.reshape(-1), od, f"{what} dists")
    osig, orho = oracle.smooth_knn(od, k)
    assert_same_bytes(t.sigmas, osig, f"{what} sigma")
    assert_same_bytes(t.rhos, orho, f"{what} rho")


def test_mixed_requests_match_oracle_and_alone(oracle):
    reqs = make_requests(21, 28)
    with Server(max_batch_jobs=6, max_inflight=3) as srv:
        tickets = [srv.submit(x, k, m) for x, k, m in reqs]
        for t in tickets:
            srv.wait(t)
        totals = srv.totals()
    assert totals["finished"] == len(reqs) and totals["failed"] == 0
    assert totals["max_batch_jobs_seen"] > 1, "requests were never batched together"
    for j, ((x, k, metric), t) in enumerate(zip(reqs, tickets)):
        check_against_oracle(oracle, t, x, k, metric, f"request {j}")
        alone, sm = hm.knn_smooth(x, x.shape[1], k, metric)
        assert_same_bytes(t.indices.reshape(-1), alone.indices, f"request {j} vs alone")
        assert_same_bytes(t.sigmas, sm.sigmas, f"request {j} sigma vs alone")
        assert t.info["done_ms"] >= t.info["admit_ms"] >= t.info["submit_ms"]


def test_staggered_arrivals_overlap_and_repeat_bytes():
    reqs = make_requests(22, 30, n_hi=6000)
    results = {}
    with Server(max_batch_jobs=4, max_inflight=4) as srv:
        def client(lo, hi, delay):
            for j in range(lo, hi):
                x, k, m = reqs[j]
                results[j] = srv.submit(x, k, m)
                time.sleep(delay)
        threads = [threading.Thread(target=client, args=(i * 10, i * 10 + 10, 0.002 * (i + 1)))
                   for i in range(3)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        for j in range(len(reqs)):
            srv.wait(results[j])
        totals = srv.totals()
    assert totals["finished"] == len(reqs)
    for j, (x, k, metric) in enumerate(reqs):
        alone, sm = hm.knn_smooth(x, x.shape[1], k, metric)
        t = results[j]
        assert_same_bytes(t.indices.reshape(-1), alone.indices, f"request {j}")
        assert_same_bytes(t.dists.reshape(-1), alone.dists, f"request {j}")
        assert_same_bytes(t.rhos, sm.rhos, f"request {j}")


def test_request_larger_than_arena_is_refused_others_run(oracle):
    g = np.random.default_rng(4)
    small = g.normal(size=(300, 16)).astype(np.float32)
    big = g.normal(size=(20000, 300)).astype(np.float32)
    with Server(memory_bytes=64 << 20) as srv:
        t_small = srv.submit(small, 15, "euclidean")
        t_big = srv.submit(big, 15, "euclidean")
        with pytest.raises(hm.HolomapCudaError) as e:
            srv.wait(t_big)
        assert e.value.code == hm.HM_ERR_ADMISSION
        srv.wait(t_small)
    check_against_oracle(oracle, t_small, small, 15, "euclidean", "small request")


def test_small_arena_serialises_but_stays_exact():
    reqs = make_requests(23, 10, n_hi=3000)
    # room for a few of these requests at a time (a screened 3000-point
    # request takes ~100 MB: candidate lists, binary64 copy, operands)
    with Server(memory_bytes=256 << 20, max_batch_jobs=8) as srv:
        tickets = [srv.submit(x, k, m) for x, k, m in reqs]
        for t in tickets:
            srv.wait(t)
        totals = srv.totals()
    assert totals["arena_peak_bytes"] <= totals["arena_bytes"]
    assert totals["batches"] > 1
    for j, ((x, k, metric), t) in enumerate(zip(reqs, tickets)):
        alone, _ = hm.knn_smooth(x, x.shape[1], k, metric)
        assert_same_bytes(t.indices.reshape(-1), alone.indices, f"request {j}")


def test_invalid_request_fails_alone_in_its_batch():
    g = np.random.default_rng(6)
    good = [g.normal(size=(int(n), 12)).astype(np.float32) for n in (200, 500, 900)]
    bad = g.normal(size=(400, 12)).astype(np.float32)
    bad[123, 4] = np.nan
    with Server(max_batch_jobs=8) as srv:
        # hold the loop busy so that all four land in one batch
        tickets = [srv.submit(x, 15, "cosine") for x in good[:1]]
        tickets += [srv.submit(good[1], 15, "cosine"), srv.submit(bad, 15, "cosine"),
                    srv.submit(good[2], 15, "cosine")]
        with pytest.raises(hm.HolomapInvalidInput, match="non-finite"):
            srv.wait(tickets[2])
        for j in (0, 1, 3):
            srv.wait(tickets[j])
    for x, t in zip(good, [tickets[0], tickets[1], tickets[3]]):
        alone = hm.exact_knn(x, 12, 15, "cosine")
        assert_same_bytes(t.indices.reshape(-1), alone.indices, "batch mate of a failing request")


def test_served_tight_clusters_escalate_and_match_the_plain_path():
    """Requests whose points form clusters far tighter than the BF16/TF32
    operands' rounding, batched with ordinary ones: each returns the plain
    path's bytes (the coarse screen hands its rows to the split-BF16 copy
    on the device)."""
    g = np.random.default_rng(41)

    def tight(n, d):
        centres = g.normal(0.0, 4.0, size=(6, d))
        labels = g.integers(0, 6, size=n)
        return np.ascontiguousarray((centres[labels] + g.normal(0.0, 0.05, size=(n, d))).astype(np.float32))

    reqs = [(tight(3000, 384), 15, "cosine"), (edge_case("gauss", 2500, 300, seed=4), 15, "cosine"),
            (tight(2600, 384), 30, "euclidean"), (tight(2048, 300), 15, "cosine")]
    with Server(max_batch_jobs=4, max_inflight=2) as srv:
        tickets = [srv.submit(x, k, m) for x, k, m in reqs]
        for t in tickets:
            srv.wait(t)
    for j, ((x, k, metric), t) in enumerate(zip(reqs, tickets)):
        plain, psm = hm.knn_smooth(x, x.shape[1], k, metric, "plain")
        assert_same_bytes(t.indices.reshape(-1), plain.indices, f"request {j} indices")
        assert_same_bytes(t.dists.reshape(-1), plain.dists, f"request {j} dists")
        assert_same_bytes(t.sigmas, psm.sigmas, f"request {j} sigma")
        assert_same_bytes(t.rhos, psm.rhos, f"request {j} rho")
