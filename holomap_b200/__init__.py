"""holomap_b200 -- B200-native (sm_100a) exact kNN + smooth-kNN for holomap.

Drop-in for the two calls holomap's ``Holomap::fit_transform`` makes at
src/api.rs:147-148 (``exact_knn`` from src/knn.rs, ``smooth_knn`` from
src/smooth_knn.rs): same arguments, same arrays, bit for bit, computed by
hand-written CUDA kernels behind the C ABI in include/holomap_cuda.h.
"""
from ._lib import (  # noqa: F401
    HM_ERR_ADMISSION, HM_ERR_CUDA, HM_ERR_INVALID, HM_ERR_NOT_READY, HM_ERR_OOM,
    HM_ERR_TIMEOUT, HM_ERR_UNSUPPORTED, HM_OK, HmStats, HolomapCudaError, HolomapInvalidInput,
    EigenPairs, FuzzyGraph, Knn, KnnPath, Metric, SmoothKnn, autotune_path, exact_knn, fuzzy_simplicial_set,
    knn_smooth, lib, smallest_eigenpairs, smooth_knn, workspace_bytes,
)

__all__ = [
    "EigenPairs", "FuzzyGraph", "HmStats", "HolomapCudaError", "HolomapInvalidInput", "Knn", "KnnPath", "Metric",
    "SmoothKnn", "autotune_path", "exact_knn", "fuzzy_simplicial_set", "knn_smooth", "lib",
    "smallest_eigenpairs", "smooth_knn", "workspace_bytes",
]
