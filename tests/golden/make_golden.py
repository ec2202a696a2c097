"""Extract the reference's stage-1/2 golden vectors into tests/golden/.

The reference (mnmal-ai/holomap) pins its kNN and smooth-kNN stages against
umap-learn 0.5.12 fixtures, tests/fixtures/stage2_{blobs_euclidean,cosine,
duplicates_euclidean}.json, produced by its dev/export_stage2_fixtures.py and
asserted in src/fixture_parity.rs:42-99 (kNN indices exact; distances, rho and
sigma within 1e-5 * (1 + |expected|)) and its fuzzy graph at :101-117
(support exact, weights within the same tolerance); the spectral fixture
tests/fixtures/spectral_cloud_connected.json pins the eigenpairs of the
normalized Laplacian (src/fixture_parity.rs:125-185).  This script copies the
keys that the kNN + smooth-kNN path and the fuzzy graph consume or produce
(data, knn_indices, knn_dists, rhos, sigmas, graph_rows, graph_cols,
graph_vals and the shape/metric header) so the tests can run where the
reference checkout is absent.  Run it from the repository root with the
reference checkout path as its only argument:

    python tests/golden/make_golden.py /path/to/holomap
"""
import json
import sys
from pathlib import Path

NAMES = ("blobs_euclidean", "cosine", "duplicates_euclidean")
KEYS = ("name", "metric", "n_neighbors", "n_samples", "n_features", "data",
        "knn_indices", "knn_dists", "rhos", "sigmas", "graph_rows", "graph_cols", "graph_vals")


def main(ref_root: str) -> None:
    out_dir = Path(__file__).resolve().parent
    for name in NAMES:
        src = Path(ref_root) / "tests" / "fixtures" / f"stage2_{name}.json"
        fixture = json.loads(src.read_text())
        slim = {k: fixture[k] for k in KEYS}
        slim["source"] = f"tests/fixtures/stage2_{name}.json (umap-learn 0.5.12 export)"
        (out_dir / f"stage2_{name}.json").write_text(json.dumps(slim) + "\n")
        print(f"stage2_{name}.json: n={slim['n_samples']} d={slim['n_features']} "
              f"k={slim['n_neighbors']} metric={slim['metric']}")
    # the spectral stage: scipy eigsh eigenpairs of the normalized Laplacian of
    # the fuzzy graph of a connected point cloud, asserted in
    # src/fixture_parity.rs:125-185 (eigenvalues within 1e-6, eigenvectors
    # aligned to 1 - 1e-6)
    src = Path(ref_root) / "tests" / "fixtures" / "spectral_cloud_connected.json"
    fixture = json.loads(src.read_text())
    keys = ("name", "metric", "n_neighbors", "n_samples", "n_features", "dim", "data",
            "eigenvalues", "eigenvectors")
    slim = {k: fixture[k] for k in keys}
    slim["source"] = "tests/fixtures/spectral_cloud_connected.json (scipy eigsh export)"
    (out_dir / "spectral_cloud_connected.json").write_text(json.dumps(slim) + "\n")
    print(f"spectral_cloud_connected.json: n={slim['n_samples']} dim={slim['dim']}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <root of the holomap source tree>")
    main(sys.argv[1])
