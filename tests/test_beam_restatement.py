"""The plain-Python two-parents-per-hop search restatement (beam_restatement.py) at
beam 1 is exactly the oracle's GreedySearch (snapshot bloom filter), ids and
distances, so its beam-2 results are a trustworthy check for the kernel."""
import numpy as np
import pytest

from beam_restatement import beam_search
from vann import workload


@pytest.fixture(scope="module")
def graph(oracle):
    base = workload.mixture(2000, 128, 20, seed=121)
    g, entry = oracle.build_index(base, R=32, L=64, alpha=1.2, seed=121)
    return base, g, entry


def test_restatement_is_greedy_search_at_beam_1(oracle, graph):
    base, g, entry = graph
    q = workload.mixture(12, 128, 20, seed=122)
    st, oids, od, _, _ = g.search(q, 32, 10, entry, bloom_mode=oracle.BLOOM_SNAPSHOT)
    assert st == 0
    for i in range(len(q)):
        ids, ds = beam_search(oracle, base, g.deg, g.adj, q[i], 32, 10, entry, 1)
        assert np.array_equal(ids, oids[i]) and np.array_equal(ds, od[i])
