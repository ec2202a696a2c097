"""CPU checks of the C ABI: the library loads without a GPU, exports every
symbol include/holomap_cuda.h declares, and rejects bad arguments the way the
reference's validation does (src/api.rs:114-145) before touching a device."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import holomap_b200 as hm
from holomap_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"^HM_API\s+[^(]*?\b(hm_\w+)\s*\(", text, flags=re.M))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"hm_knn", "hm_smooth_knn", "hm_knn_smooth", "hm_last_error"} <= names


def test_library_exports_every_declared_symbol():
    lib = hm.lib()
    for name in sorted(declared_symbols()):
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_python_binding_covers_every_symbol():
    assert declared_symbols() <= set(_lib.SIGNATURES), "binding is missing a declared symbol"


def test_abi_version():
    assert hm.lib().hm_abi_version() == 1


@pytest.mark.parametrize("n_features,k,msg", [
    (0, 3, "not a positive multiple"),     # BadShape (src/api.rs:114-119)
    (3, 3, "not a positive multiple"),     # 10 % 3 != 0
    (1, 0, "n_neighbors must be >= 1"),
    (1, 11, "need at least"),              # TooFewPoints (src/api.rs:135-141)
])
def test_invalid_arguments_are_rejected_without_a_device(n_features, k, msg):
    with pytest.raises(hm.HolomapInvalidInput, match=msg):
        hm.exact_knn(np.zeros(10, np.float32), n_features, k)


def test_unknown_metric_rejected():
    # FromStr rejects anything but euclidean/cosine(/manhattan here) (src/metric.rs:21-30)
    with pytest.raises(ValueError):
        hm.Metric.parse("chebyshev")
    assert hm.Metric.parse("Cosine") is hm.Metric.COSINE
    assert str(hm.Metric.EUCLIDEAN) == "euclidean"
    lib = hm.lib()
    x = np.zeros(12, np.float32)
    rc = lib.hm_knn(x.ctypes.data, 4, 3, 2, 7, 0, None, None, None)
    assert rc == hm.HM_ERR_INVALID
    assert b"metric" in lib.hm_last_error()


def test_k_above_256_is_unsupported_not_wrong():
    lib = hm.lib()
    x = np.zeros(300 * 2, np.float32)
    rc = lib.hm_knn(x.ctypes.data, 300, 2, 257, 0, 1, None, None, None)
    assert rc == hm.HM_ERR_UNSUPPORTED


def test_workspace_sizes_are_plannable_on_cpu():
    b1 = hm.workspace_bytes(1000, 50, 15, "euclidean", "plain")
    b2 = hm.workspace_bytes(20000, 128, 15, "euclidean", "plain")
    assert 0 < b1 < b2
    # the binary64 copy dominates: n_pad x round_up(d, 16) x 8 bytes
    assert b2 >= 20000 * 128 * 8


def test_smooth_workspace_is_small():
    assert hm.lib().hm_smooth_workspace_bytes(50000) < 50000 * 4 + 1024


def test_null_outputs_rejected():
    lib = hm.lib()
    x = np.zeros(40, np.float32)
    rc = lib.hm_knn(x.ctypes.data, 20, 2, 3, 0, 1, None, None, None)
    assert rc == hm.HM_ERR_INVALID


def test_row_shard_ranges_are_validated_on_cpu():
    lib = hm.lib()
    assert lib.hm_knn_rows_workspace_bytes(1000, 8, 5, 0, 1, 0, 1000) > 0
    assert lib.hm_knn_rows_workspace_bytes(1000, 8, 5, 0, 1, 100, 228) > 0
    for b, e in [(0, 0), (10, 5), (0, 1001)]:
        assert lib.hm_knn_rows_workspace_bytes(1000, 8, 5, 0, 1, b, e) == 0
        assert "query rows" in lib.hm_last_error().decode()


def _autotune_doc():
    import json
    from holomap_b200 import autotune
    return json.loads(autotune.JSON_PATH.read_text()) if autotune.JSON_PATH.exists() else None


def test_autotune_table_is_the_committed_measurement():
    """hm_autotune_path returns, at every grid point, the choice recorded in
    holomap_b200/autotune_table.json (the library's C table is generated from
    it), and the generated table is current."""
    from holomap_b200 import autotune
    doc = _autotune_doc()
    choice, batch, gn, gd, gk = autotune.table_from(doc)
    for (metric, k, d, n), (path, *_) in choice.items():
        assert hm.autotune_path(n, d, k, metric) == hm.KnnPath.parse(path), (metric, k, d, n)
    for (metric, k, d, n), (path, *_) in batch.items():
        assert hm.autotune_path(n, d, k, metric, batched=True) == hm.KnnPath.parse(path), (metric, k, d, n)
    import tempfile
    from pathlib import Path
    with tempfile.TemporaryDirectory() as t:
        fresh = Path(t) / "table.inc"
        autotune.emit_inc(doc, fresh)
        assert fresh.read_text() == autotune.INC_PATH.read_text(), "autotune_table.inc is stale"


def test_autotune_covers_the_benchmark_shapes():
    """Every workload shape resolves to a path; where no screen applies the
    path is plain."""
    at = hm.autotune_path
    P = hm.KnnPath
    assert at(50000, 300, 15, "manhattan") == P.PLAIN      # no inner-product form
    assert at(50000, 384, 65, "cosine") == P.PLAIN         # k above the screen's 64
    assert at(50000, 4096, 15, "euclidean") == P.PLAIN     # d above 2048
    shapes = [(1000, 50, 15, "euclidean"), (20000, 128, 15, "euclidean"), (50000, 384, 30, "cosine")]
    shapes += [(n, d, 15, m) for n in (200, 1000, 8000) for d in (16, 50, 128) for m in ("euclidean", "cosine")]
    shapes += [(n, d, k, m) for n in (500, 5000, 50000) for d in (32, 64, 300) for k in (15, 30)
               for m in ("euclidean", "cosine")]
    for n, d, k, m in shapes:
        p = at(n, d, k, m)
        assert p in (P.PLAIN, P.SCREEN_BF16, P.SCREEN_TF32, P.SCREEN_BF16X3)
        assert hm.workspace_bytes(n, d, k, m, "auto") > 0


def test_tuning_override_bounds():
    lib = hm.lib()
    assert lib.hm_tuning_override(8) == 0
    assert lib.hm_tuning_override(0) == 0
    assert lib.hm_tuning_override(-1) == hm.HM_ERR_INVALID
    assert lib.hm_tuning_override(65) == hm.HM_ERR_INVALID
    for hook in (lib.hm_tuning_symmetric, lib.hm_tuning_pair):
        for mode in (0, 1, -1):  # -1 (the table's choice) restores the default
            assert hook(mode) == 0
        assert hook(2) == hm.HM_ERR_INVALID
        assert hook(-2) == hm.HM_ERR_INVALID


def test_symmetric_and_pair_forms_plan_for_the_benchmark_shape():
    """Every emission form plans for the 50,000 x 384 cosine shape (the
    symmetric form's lists: at most 7 column parts, 30 lists per row)."""
    lib = hm.lib()
    try:
        for sym in (0, 1):
            for pair in (0, 1):
                assert lib.hm_tuning_symmetric(sym) == 0
                assert lib.hm_tuning_pair(pair) == 0
                assert hm.workspace_bytes(50000, 384, 30, "cosine", "screen_bf16") > 0
    finally:
        lib.hm_tuning_symmetric(-1)
        lib.hm_tuning_pair(-1)


def test_every_screened_path_plans_for_the_benchmark_shapes():
    for n, d, k, metric in [(1000, 50, 15, "euclidean"), (20000, 128, 15, "euclidean"),
                            (50000, 384, 30, "cosine")]:
        for path in ("auto", "plain", "screen_bf16", "screen_tf32", "screen_bf16x3"):
            assert hm.workspace_bytes(n, d, k, metric, path) > 0


# --- fuzzy graph and spectral stage: host-side checks (no device) ----------

def test_fuzzy_graph_rejects_bad_input_before_the_device():
    lib = hm.lib()
    idx = np.array([0, 5, 1, 0], dtype=np.uint32)  # 5 is not below n = 2
    f = np.zeros(4, np.float32)
    sig = np.ones(2, np.float32)
    out_u = np.zeros(8, np.uint32)
    out_f = np.zeros(8, np.float32)
    nnz = ctypes.c_uint64(0)
    rc = lib.hm_fuzzy_graph(idx.ctypes.data, f.ctypes.data, sig.ctypes.data, sig.ctypes.data, 2, 2,
                            out_u.ctypes.data, out_u.ctypes.data, out_f.ctypes.data, ctypes.byref(nnz))
    assert rc == hm.HM_ERR_INVALID and b"not below n" in lib.hm_last_error()
    idx = np.array([0, 1, 1, 0], dtype=np.uint32)
    neg = np.array([1.0, -0.5], np.float32)
    rc = lib.hm_fuzzy_graph(idx.ctypes.data, f.ctypes.data, neg.ctypes.data, sig.ctypes.data, 2, 2,
                            out_u.ctypes.data, out_u.ctypes.data, out_f.ctypes.data, ctypes.byref(nnz))
    assert rc == hm.HM_ERR_INVALID and b"negative" in lib.hm_last_error()
    rc = lib.hm_fuzzy_graph(idx.ctypes.data, f.ctypes.data, sig.ctypes.data, sig.ctypes.data, 0, 2,
                            out_u.ctypes.data, out_u.ctypes.data, out_f.ctypes.data, ctypes.byref(nnz))
    assert rc == hm.HM_ERR_INVALID
    with pytest.raises(hm.HolomapInvalidInput, match="not below n"):
        hm.fuzzy_simplicial_set(hm.Knn(2, idx * 3, f), hm.SmoothKnn(sig, sig))


def test_spectral_rejects_bad_input_before_the_device():
    lib = hm.lib()
    rows = np.array([1, 0, 1, 2], dtype=np.uint32)  # not sorted
    cols = np.array([0, 1, 2, 1], dtype=np.uint32)
    vals = np.ones(4, np.float32)
    out = np.zeros(16)
    found, cycles = ctypes.c_uint32(0), ctypes.c_uint32(0)

    def call(r, c, n, k):
        return lib.hm_spectral_eigenpairs(r.ctypes.data, c.ctypes.data, vals.ctypes.data, n, r.size, k,
                                          out.ctypes.data, out.ctypes.data, ctypes.byref(found),
                                          ctypes.byref(cycles))

    assert call(rows, cols, 3, 2) == hm.HM_ERR_INVALID and b"not sorted" in lib.hm_last_error()
    rows = np.array([0, 1, 1, 2], dtype=np.uint32)
    assert call(rows, np.array([1, 0, 7, 1], np.uint32), 3, 2) == hm.HM_ERR_INVALID
    assert b"outside" in lib.hm_last_error()
    assert call(rows, cols, 3, 4) == hm.HM_ERR_INVALID  # k above n
    assert call(rows, cols, 3, 0) == hm.HM_ERR_INVALID
    assert lib.hm_eigenpairs_workspace_bytes(5000, 1025) == 0  # k above 1024
    assert lib.hm_eigenpairs_workspace_bytes(50000, 3) > 60 * 50000 * 8
    assert lib.hm_laplacian_device(None, None, None, 3, 4, None, None, None, None) == hm.HM_ERR_INVALID


@pytest.mark.parametrize("m,seed", [(1, 0), (2, 1), (7, 2), (60, 3), (61, 4)])
def test_tridiagonal_eigensolver(m, seed):
    """The implicit QL solver the Lanczos iteration uses for its tridiagonal,
    against numpy's dense eigh (residuals and orthonormality), including a
    matrix with nearly decoupled blocks."""
    g = np.random.default_rng(seed)
    d = g.uniform(0.0, 2.0, m)
    e = g.uniform(0.0, 0.5, max(m - 1, 0))
    if m > 3:
        e[m // 2] = 1e-15
    vals = np.empty(m)
    vecs = np.empty(m * m)
    rc = hm.lib().hm_debug_tridiag_eigen(d.ctypes.data, e.ctypes.data if m > 1 else None, m,
                                         vals.ctypes.data, vecs.ctypes.data)
    assert rc == hm.HM_OK
    z = vecs.reshape(m, m)
    t = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    assert np.abs(t @ z - z * vals).max() < 1e-13
    assert np.abs(z.T @ z - np.eye(m)).max() < 1e-13
    assert np.abs(np.sort(vals) - np.linalg.eigvalsh(t)).max() < 1e-13
