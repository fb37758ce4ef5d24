"""Digests of the oracle graph of the largest-instance parity subset (test fixture generator).

The largest-instance workload (2^28 points, d = 3, n0 = 4096, k = 32) is checked for bit-exact graphs on its
first 2^20 points. The oracle graph of those points is too large to commit (128 MB of neighbours), so this
script records SHA-256 digests of its arrays; tests/test_gpu_graph.py builds the same graph on the GPU and
compares digests. Run from the repository root: ``python tests/golden/make_largest_subset.py`` (a few
minutes on one core).
"""
import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from bench import largest_points  # noqa: E402
from oracle import graph as og  # noqa: E402

N, N0, K = 1 << 20, 4096, 32


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    pts = largest_points(N)
    t = time.time()
    g = og.build_graph(pts, n0=N0, k=K)
    out = {
        "n": N, "n0": N0, "k": K, "generator": "bench.largest_points(2**20)",
        "points_sha256": digest(pts.astype(np.float32)),
        "indices_sha256": digest(np.asarray(g.indices, np.int32)),
        "neighbors_sha256": digest(np.asarray(g.neighbors, np.int32)),
        "points_graph_sha256": digest(np.asarray(g.points, np.float32)),
        "offsets": [int(x) for x in g.offsets],
        "oracle_seconds": round(time.time() - t, 1),
    }
    (Path(__file__).parent / "largest_subset.json").write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps({k: v for k, v in out.items() if k != "offsets"}), "batches", len(out["offsets"]) - 1)


if __name__ == "__main__":
    main()
