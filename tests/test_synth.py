"""The synthetic workloads are pinned by the SHA-256 of their bytes
(tests/golden/workload_sha256.json): the benchmark numbers refer to exactly
these datasets (numpy PCG64 streams, float64 draws cast to float32)."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from holomap_b200 import synth

PINS = json.loads((Path(__file__).parent / "golden" / "workload_sha256.json").read_text())


def _sha(arrays) -> str:
    m = hashlib.sha256()
    for a in arrays:
        m.update(np.ascontiguousarray(a).tobytes())
    return m.hexdigest()


@pytest.mark.parametrize("name", ["blobs_1k", "dups_20k", "embed_50k"])
def test_single_dataset_workloads(name):
    wl = synth.WORKLOADS[name]()
    assert wl.data.dtype == np.float32 and wl.data.flags.c_contiguous
    assert _sha([wl.data]) == PINS[name]


def test_batch_256():
    wls = synth.batch_256()
    assert len(wls) == 256
    assert _sha([w.data for w in wls]) == PINS["batch_256"]


def test_serve_pools_and_schedule():
    pools = [synth.serve_pool(d, s) for d in (32, 64, 300) for s in range(synth.SERVE_POOL_SLOTS)]
    assert _sha(pools) == PINS["serve_pool"]
    reqs = synth.serve_2000(100.0)
    key = repr([(r.seq, round(r.arrival_s, 9), r.n, r.d, r.k, r.metric, r.seed) for r in reqs]).encode()
    assert hashlib.sha256(key).hexdigest() == PINS["serve_2000"]
