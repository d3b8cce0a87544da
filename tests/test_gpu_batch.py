"""GPU: batched uneven graphs (many independent graphs decomposed together),
the batch generator (device == host), subgraph extraction, the autotuner."""
import numpy as np
import pytest

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, State, generate_batch_edges_host

pytestmark = pytest.mark.gpu

KW = dict(num_graphs=24, n_min=64, n_max=3000, mean_degree=3.0, rmat_fraction=0.3, seed=77)


def host_batch():
    n, offs, s, d = generate_batch_edges_host(**KW)
    s, d = O.dedup_edges(s, d, n=n)
    return n, offs, s, d


def test_batch_generator_device_matches_host(gpu):
    n, offs, s, d = host_batch()
    g, goffs = Graph.generate_batch(**KW)
    assert np.array_equal(goffs, offs) and g.num_nodes() == n and g.num_edges() == s.size
    for x, y in zip(g.csr(), O.build_csr(n, s, d)):
        assert np.array_equal(x, y)
    # no edge leaves its graph
    assert np.all(np.searchsorted(offs, s, side="right") == np.searchsorted(offs, d, side="right"))


def test_batched_labels_equal_per_graph_labels(gpu):
    n, offs, s, d = host_batch()
    csr = O.build_csr(n, s, d)
    exp = O.tarjan_canonical(csr[0], csr[1])
    g, _ = Graph.generate_batch(**KW)
    st = State(g)
    st.run(2)
    union = st.canonical_labels()
    assert np.array_equal(union, exp)
    for i in range(0, len(offs) - 1, 5):
        sub = g.subgraph(int(offs[i]), int(offs[i + 1]))
        ss = State(sub)
        ss.run(2)
        assert np.array_equal(ss.canonical_labels() + offs[i], union[offs[i]:offs[i + 1]])


def test_subgraph_rejects_open_range(gpu):
    g = Graph.from_edges(4, [0, 1, 2], [1, 2, 3])
    with pytest.raises(Exception):
        g.subgraph(0, 2)


def test_autotune_keeps_labels(gpu):
    n, s, d = 3000, *np.random.default_rng(5).integers(0, 3000, (2, 5000)).astype(np.int32)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    best, ms = st.autotune(max_trials=6)
    assert ms > 0 and st.get_tuning() == best
    st.run(2)
    csr = O.build_csr(n, s, d)
    assert np.array_equal(st.canonical_labels(), O.tarjan_canonical(csr[0], csr[1]))
