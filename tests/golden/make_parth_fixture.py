"""Writes tests/golden/parth_vamana_1k.json: the reference's own CPU Vamana
(parth/tools/vamana.py, imported from the reference checkout, unmodified) built and
searched on a seeded 1,000 x 128 slice of the plain-Vamana configuration (100-cluster
clipped Gaussian mixture, R=32, L=75, alpha=1.2, 100 queries, k=10), with its recall@10
against FP64 brute force and its top-10 ids.  The reference cannot run where the GPU
tests run, so its results travel as this fixture.

    python tests/golden/make_parth_fixture.py [/path/to/reference]

Its build draws from Python's `random` (seeded 0 here) and takes about two minutes.
"""
import importlib.util
import json
import os
import random
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "cs5013-project_b200"))
from vann import workload  # noqa: E402

N, NQ, DIM, CLUSTERS, R, L, ALPHA, K = 1000, 100, 128, 100, 32, 75, 1.2, 10


def main(ref_root):
    spec = importlib.util.spec_from_file_location("parth_vamana", os.path.join(ref_root, "parth", "tools",
                                                                                "vamana.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    base = workload.mixture(N, DIM, CLUSTERS, seed=1)
    q = workload.mixture(NQ, DIM, CLUSTERS, seed=2)
    random.seed(0)
    idx = mod.VamanaIndex(base, R=R, L=L, alpha=ALPHA)
    t0 = time.time()
    idx.build()
    build_s = time.time() - t0
    t0 = time.time()
    ids = [idx.greedy_search(q[i], K, L)[:K] for i in range(NQ)]
    search_s = time.time() - t0
    d = ((q.astype(np.float64)[:, None, :] - base.astype(np.float64)[None, :, :]) ** 2).sum(-1)
    truth = np.argsort(d, axis=1, kind="stable")[:, :K]
    recall = float(np.mean([len(set(map(int, a)) & set(map(int, b))) / K for a, b in zip(ids, truth)]))
    out = {"source": "parth/tools/vamana.py (VamanaIndex.build, greedy_search), unmodified",
           "n": N, "nq": NQ, "dim": DIM, "clusters": CLUSTERS, "seeds": {"base": 1, "queries": 2, "random": 0},
           "R": R, "L": L, "alpha": ALPHA, "k": K, "recall@10": round(recall, 4), "build_s": round(build_s, 1),
           "search_qps_1_core": round(NQ / search_s, 1), "medoid": int(idx.medoid),
           "ids": [[int(x) for x in row] for row in ids]}
    with open(os.path.join(HERE, "parth_vamana_1k.json"), "w") as f:
        json.dump(out, f)
        f.write("\n")
    print(f"recall@10 {recall:.4f}  build {build_s:.1f} s  search {NQ / search_s:.1f} QPS")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("VANN_REFERENCE_DIR", "/root/reference"))
