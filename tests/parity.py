"""Shared helpers of the parity tests: byte-level comparison and edge-case
data builders."""
import numpy as np


def bits(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32)).view(np.uint32)


def assert_same_bytes(actual, expected, what: str) -> None:
    a, e = np.asarray(actual).reshape(-1), np.asarray(expected).reshape(-1)
    assert a.shape == e.shape, f"{what}: shape {a.shape} vs {e.shape}"
    if a.dtype == np.float32:
        a, e = bits(a), bits(e)
    bad = np.flatnonzero(a != e)
    assert bad.size == 0, (f"{what}: {bad.size} of {a.size} differ, first at {bad[:5]}: "
                           f"{a[bad[:5]]} vs {e[bad[:5]]}")


def rows_sorted_by_key(idx: np.ndarray, dist: np.ndarray) -> bool:
    key = (bits(dist).astype(np.uint64) << np.uint64(32)) | idx.astype(np.uint64)
    return bool((np.diff(key, axis=1) > 0).all())


def edge_case(kind: str, n: int, d: int, seed: int) -> np.ndarray:
    """Inputs that stress the reference's tie and rounding rules."""
    g = np.random.default_rng(seed)
    if kind == "gauss":
        return g.normal(size=(n, d)).astype(np.float32)
    if kind == "duplicates":  # exact copies: d=0 ties broken by index
        x = g.normal(size=(n, d)).astype(np.float32)
        src = g.integers(0, n // 2, size=n // 3)
        x[n - n // 3:] = x[src]
        return x
    if kind == "ulp":  # one-ulp neighbours
        x = g.normal(size=(n, d)).astype(np.float32)
        half = n // 2
        x[half:2 * half] = x[:half]
        c = g.integers(0, d, size=half)
        x[half + np.arange(half), c] = np.nextafter(x[half + np.arange(half), c], np.float32(np.inf))
        return x
    if kind == "zeros":  # zero vectors and signed zeros
        x = g.normal(size=(n, d)).astype(np.float32)
        x[: n // 4] = 0.0
        x[n // 4: n // 3] = -0.0
        return x
    if kind == "huge":  # distances overflow the f32 cast to +inf
        x = g.normal(size=(n, d)).astype(np.float32)
        x[::3] *= np.float32(3e38) / np.abs(x[::3]).max()
        return x
    if kind == "tiny":  # subnormal-range values
        return (g.normal(size=(n, d)) * 1e-40).astype(np.float32)
    if kind == "grid":  # many exactly equal distances
        return g.integers(-3, 4, size=(n, d)).astype(np.float32)
    if kind == "sorted_line":  # worst case for a streaming select
        return np.sort(g.normal(size=n)).astype(np.float32).reshape(n, 1).repeat(d, axis=1)
    raise ValueError(kind)
