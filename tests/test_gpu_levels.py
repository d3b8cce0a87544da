"""GPU: method 7's level analytics through the C ABI against the oracle
(whose FIFO restatement is pinned to the reference's own create_scc_edges on
the CPU): topological levels of condensation DAGs, the levels an inserted
batch affects, and the trim shortcut, whose run must still give the updated
graph's SCCs exactly."""
import numpy as np
import pytest

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, State, affected_levels, condensation_graph, topological_levels

pytestmark = pytest.mark.gpu


def _random(seed, n, deg):
    rng = np.random.default_rng(seed)
    m = int(n * deg)
    return rng, rng.integers(0, n, m).astype(np.int32), rng.integers(0, n, m).astype(np.int32)


@pytest.mark.parametrize("seed,n,deg", [(1, 5000, 1.5), (2, 20000, 2.0), (3, 60000, 1.2)])
def test_levels_of_condensation_match_oracle(gpu, seed, n, deg):
    rng, s, d = _random(seed, n, deg)
    ids, k = O.scc_ids(O.tarjan_canonical(*O.build_csr(n, s, d)[:2]))
    b, a = O.condensation_csr(ids, k, s, d)
    exp, exp_max = O.topo_levels(b, a)
    g = Graph.from_edges(n, s, d)
    dag = condensation_graph(g, ids, k)
    lev, ml = topological_levels(dag)
    assert ml == exp_max and np.array_equal(lev, exp)
    dag.free(); g.free()


def test_levels_when_labels_are_not_sccs(gpu):
    # identity labels on a cyclic graph: nodes on or behind cycles keep what
    # the reference's queue leaves them
    n = 8000
    _, s, d = _random(7, n, 1.3)
    b, a = O.condensation_csr(np.arange(n, dtype=np.int32), n, s, d)
    exp, exp_max = O.topo_levels(b, a)
    g = Graph.from_edges(n, s, d)
    dag = condensation_graph(g, np.arange(n, dtype=np.int32), n)
    lev, ml = topological_levels(dag)
    assert ml == exp_max and np.array_equal(lev, exp)
    dag.free(); g.free()


def test_levels_wide_star_overflows_queues(gpu):
    # one source with 100,000 children, all feeding one sink: the source's
    # warp releases far more nodes than its queue holds
    leaves = 100000
    l = np.arange(1, leaves + 1, dtype=np.int32)
    s = np.concatenate([np.zeros(leaves, np.int32), l])
    d = np.concatenate([l, np.full(leaves, leaves + 1, np.int32)])
    g = Graph.from_edges(leaves + 2, s, d)
    lev, ml = topological_levels(g)
    assert ml == 2 and lev[0] == 0 and (lev[1:leaves + 1] == 1).all() and lev[leaves + 1] == 2
    g.free()


def test_levels_long_chain(gpu):
    n = 200000
    s = np.arange(n - 1, dtype=np.int32)
    g = Graph.from_edges(n, s, s + 1)
    lev, ml = topological_levels(g)
    assert ml == n - 1 and np.array_equal(lev, np.arange(n, dtype=np.int32))
    g.free()


@pytest.mark.parametrize("seed,n_ins", [(11, 0), (12, 1), (13, 5), (14, 40), (15, 2000)])
def test_method7_flow_exact(gpu, seed, n_ins):
    n = 30000
    rng, s, d = _random(seed, n, 1.6)
    ids, k = O.scc_ids(O.tarjan_canonical(*O.build_csr(n, s, d)[:2]))
    isrc = rng.integers(0, n, n_ins).astype(np.int32)
    idst = rng.integers(0, n, n_ins).astype(np.int32)
    g = Graph.from_edges(n, s, d)
    dag = condensation_graph(g, ids, k)
    lev, ml = topological_levels(dag)
    aff, z = affected_levels(dag, lev, ml, ids, isrc, idst)
    b, a = O.condensation_csr(ids, k, s, d)
    exp_aff, exp_z = O.affected_levels(ids, O.topo_levels(b, a)[0], ml, isrc, idst)
    assert z == exp_z and np.array_equal(aff, exp_aff)
    # the trim shortcut, then method 2 on the condensation with the batch
    cond = condensation_graph(g, ids, k, isrc, idst)
    st = State(cond)
    st.reset()
    fin = st.finish_unaffected(lev, aff, ml)
    assert fin == int((aff[lev] == 0).sum())
    r = st.run(2)
    cl = st.canonical_labels()
    upd = O.tarjan_canonical(*O.build_csr(n, np.concatenate([s, isrc]), np.concatenate([d, idst]))[:2])
    assert np.array_equal(O.canonical(cl[ids]), upd)
    assert r["num_sccs"] == len(np.unique(upd))
    st.free(); cond.free(); dag.free(); g.free()


def test_affected_levels_rejects_bad_input(gpu):
    from dynamicgraphs_scc_b200 import SccError
    g = Graph.from_edges(3, np.array([0, 1], np.int32), np.array([1, 2], np.int32))
    lev, ml = topological_levels(g)
    with pytest.raises(SccError):
        affected_levels(g, lev, ml, np.arange(3, dtype=np.int32), [0], [5])      # endpoint outside the graph
    with pytest.raises(SccError):
        affected_levels(g, lev, ml, np.array([0, 1, 9], np.int32), [0], [2])     # label outside [0, 3)
    g.free()


def test_levels_hub_released_by_a_chain(gpu):
    # 0 -> 1 -> 2 (a hub with 50,000 children) -> each child -> a sink: the hub
    # is released by a cascade, then expanded over the whole grid
    k = 50000
    kids = np.arange(3, 3 + k, dtype=np.int32)
    sink = 3 + k
    s = np.concatenate([[0, 1], np.full(k, 2), kids]).astype(np.int32)
    d = np.concatenate([[1, 2], kids, np.full(k, sink)]).astype(np.int32)
    n = sink + 1
    g = Graph.from_edges(n, s, d)
    lev, ml = topological_levels(g)
    b, a = O.condensation_csr(np.arange(n, dtype=np.int32), n, s, d)
    exp, exp_max = O.topo_levels(b, a)
    assert ml == exp_max == 4 and np.array_equal(lev, exp)
    g.free()


def test_method7_flow_with_hubs(gpu):
    # hubs of 200,000 edges in the condensation: the shortcut's pre-finished
    # nodes go through the counting peel, hub items leave the asynchronous
    # drain for the level kernels, and the labels stay exact
    from tests.test_gpu_edge_cases import _hub_graph
    n, s, d = _hub_graph()
    s = np.asarray(s, np.int32); d = np.asarray(d, np.int32)
    rng = np.random.default_rng(61)
    ids, k = O.scc_ids(O.tarjan_canonical(*O.build_csr(n, s, d)[:2]))
    hubs = np.array([10000, 210002, 410003], np.int32)          # the three hubs of the graph
    isrc = np.concatenate([rng.integers(0, n, 20), hubs[[0, 2]]]).astype(np.int32)
    idst = np.concatenate([rng.integers(0, n, 20), [hubs[1], hubs[0]]]).astype(np.int32)
    g = Graph.from_edges(n, s, d)
    dag = condensation_graph(g, ids, k)
    lev, ml = topological_levels(dag)
    aff, z = affected_levels(dag, lev, ml, ids, isrc, idst)
    cond = condensation_graph(g, ids, k, isrc, idst)
    st = State(cond)
    upd = O.tarjan_canonical(*O.build_csr(n, np.concatenate([s, isrc]), np.concatenate([d, idst]))[:2])
    for shortcut in (True, False):
        st.reset()
        if shortcut:
            st.finish_unaffected(lev, aff, ml)
        st.run(2)
        assert np.array_equal(O.canonical(st.canonical_labels()[ids]), upd), shortcut
    st.free(); cond.free(); dag.free(); g.free()
