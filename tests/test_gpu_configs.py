"""Byte-for-byte oracle parity at the benchmark workloads themselves.

The smaller parity suites check every path on seeded cases the oracle finishes
in a second; these tests check the exact datasets the bench reports on:

* blobs_1k   (1000 x 50, euclidean, k=15): every row, every path, all four
  arrays (indices, distances, sigmas, rhos) against the oracle;
* dups_20k   (20000 x 128, euclidean, k=15, 5% exact duplicates and 2% one-ulp
  copies): every row against the oracle on the plain path and on each screen
  (TF32, BF16, split-BF16); the rows each screen sent to the exact fallback are
  printed as the overflow rate;
* embed_50k  (50000 x 384, cosine, k=30): the whole graph on the device by the
  autotuned (BF16-screened) path and by the plain path, which must agree on all
  1.5 M entries, and 1,024 rows in eight blocks spread over the dataset (row
  block boundaries and the ragged last block included) against the oracle,
  each searching all 50,000 points; rho and sigma of those rows against the
  oracle's smooth_knn with the mean of the device's whole distance matrix
  (src/smooth_knn.rs:26, used only by rows whose rho is 0).

The oracle is the C restatement of src/knn.rs:22-55, src/metric.rs:42-70 and
src/smooth_knn.rs:23-84, run on all host threads.
"""
import os

import numpy as np
import pytest

import holomap_b200 as hm
from parity import assert_same_bytes, rows_sorted_by_key

pytestmark = pytest.mark.gpu
THREADS = max(1, os.cpu_count() or 1)
SCREENS = ["screen_tf32", "screen_bf16", "screen_bf16x3"]


def _check_all(knn, sm, oi, od, osig, orho, what):
    assert_same_bytes(knn.indices, oi, f"{what} indices")
    assert_same_bytes(knn.dists, od, f"{what} dists")
    assert_same_bytes(sm.sigmas, osig, f"{what} sigmas")
    assert_same_bytes(sm.rhos, orho, f"{what} rhos")


@pytest.fixture(scope="module")
def blobs(oracle):
    from holomap_b200.synth import blobs_1k
    wl = blobs_1k()
    oi, od = oracle.exact_knn(wl.data, wl.k, wl.metric, threads=THREADS)
    osig, orho = oracle.smooth_knn(od, wl.k)
    return wl, (oi, od, osig, orho)


@pytest.mark.parametrize("path", ["plain", "auto"] + SCREENS)
def test_blobs_1k_every_row(blobs, path):
    wl, ref = blobs
    st = hm.HmStats()
    knn, sm = hm.knn_smooth(wl.data, wl.d, wl.k, wl.metric, path, stats=st)
    _check_all(knn, sm, *ref, f"blobs_1k/{path}")
    if path == "auto":
        assert st.path_used == hm.autotune_path(wl.n, wl.d, wl.k, wl.metric)


@pytest.fixture(scope="module")
def dups(oracle):
    from holomap_b200.synth import dups_20k
    wl = dups_20k()
    oi, od = oracle.exact_knn(wl.data, wl.k, wl.metric, threads=THREADS)
    osig, orho = oracle.smooth_knn(od, wl.k)
    return wl, (oi, od, osig, orho)


@pytest.mark.parametrize("path", ["plain", "auto"] + SCREENS)
def test_dups_20k_every_row(dups, path):
    wl, ref = dups
    st = hm.HmStats()
    knn, sm = hm.knn_smooth(wl.data, wl.d, wl.k, wl.metric, path, stats=st)
    _check_all(knn, sm, *ref, f"dups_20k/{path}")
    if path != "plain":
        print(f"dups_20k {path} ({hm.KnnPath(st.path_used).name}): overflow rows {st.overflow_rows} of "
              f"{wl.n} ({st.overflow_rows / wl.n:.4%}), candidates/row {st.candidates_total / wl.n:.1f}, "
              f"emitted/row {st.candidates_emitted / wl.n:.1f}, cap {st.candidate_cap}")
    if path == "auto":
        # on the path the autotuner picks, the exact fallback is the
        # exception (BF16's band is wide against this clustered data's
        # distance gaps, and TF32's too at d = 128; both are still exact)
        assert st.overflow_rows <= wl.n // 100


# eight blocks of 128 query rows: the first and last blocks (the last row block
# of the screen holds 50000 - 390 * 128 = 80 rows), blocks on and off the
# 128-row screen boundaries, and the middle
C3_BLOCKS = [0, 6400, 12864, 19217, 25600, 32100, 41033, 50000 - 128]


@pytest.fixture(scope="module")
def embed(oracle):
    import torch

    from holomap_b200.device import DeviceKnnProblem
    from holomap_b200.synth import embed_50k
    wl = embed_50k()
    x = torch.from_numpy(wl.data).cuda()
    out = {}
    for path in ("auto", "plain"):
        p = DeviceKnnProblem(wl.n, wl.d, wl.k, wl.metric, path)
        p.run(x)
        torch.cuda.synchronize()
        st = p.stats()
        out[path] = (p.idx.cpu().numpy().view(np.uint32).reshape(wl.n, wl.k),
                     p.dist.cpu().numpy().reshape(wl.n, wl.k), p.sigma.cpu().numpy(),
                     p.rho.cpu().numpy(), st)
        del p
    return wl, out


def test_embed_50k_screened_equals_plain_on_every_row(embed):
    wl, out = embed
    a, b = out["auto"], out["plain"]
    assert a[4].path_used == hm.KnnPath.SCREEN_BF16
    assert b[4].path_used == hm.KnnPath.PLAIN
    for i, name in enumerate(("indices", "dists", "sigmas", "rhos")):
        assert_same_bytes(a[i], b[i], f"embed_50k screened vs plain {name}")
    assert rows_sorted_by_key(a[0], a[1])
    assert a[4].overflow_rows == 0


@pytest.mark.parametrize("path", ["auto", "plain"])
def test_embed_50k_sampled_rows_against_oracle(oracle, embed, path):
    wl, out = embed
    idx, dist, sig, rho, st = out[path]
    mean_all = oracle.mean(dist)  # src/smooth_knn.rs:26 over the device's n x k distances
    for r0 in C3_BLOCKS:
        r1 = r0 + 128
        oi, od = oracle.exact_knn(wl.data, wl.k, wl.metric, rows=(r0, r1), threads=THREADS)
        assert_same_bytes(idx[r0:r1], oi, f"embed_50k/{path} rows {r0}:{r1} indices")
        assert_same_bytes(dist[r0:r1], od, f"embed_50k/{path} rows {r0}:{r1} dists")
        osig, orho = oracle.smooth_knn_rows(od, wl.k, mean_all)
        assert_same_bytes(sig[r0:r1], osig, f"embed_50k/{path} rows {r0}:{r1} sigmas")
        assert_same_bytes(rho[r0:r1], orho, f"embed_50k/{path} rows {r0}:{r1} rhos")
