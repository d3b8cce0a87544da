"""GPU: re-uploading a graph's contents.  With only the forward CSR the
transpose is rebuilt on the device; it must equal the transpose gm_graph's
make_reverse_edges gives (in-lists sorted by source, duplicates and self-loops
kept), and the decomposition must equal Tarjan's."""
import numpy as np
import pytest

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, State
from tests.helpers import random_graph

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("with_transpose", [False, True])
def test_upload_replaces_contents(gpu, with_transpose):
    n, m = 3000, 9000
    s1, d1 = random_graph(n, m, 1)          # duplicates and self-loops kept
    s2, d2 = random_graph(n, m, 2)
    g = Graph.from_edges(n, s1, d1)
    csr2 = O.build_csr(n, s2, d2)
    if with_transpose:
        g.upload_csr(*csr2)
    else:
        g.upload_csr(csr2[0], csr2[1])
    st = State(g)
    st.synchronize()
    b, a, rb, ra = g.csr()
    for got, exp in zip((b, a, rb, ra), csr2):
        assert np.array_equal(got, exp)
    st.reset()
    st.run(2)
    assert np.array_equal(st.canonical_labels(), O.tarjan_canonical(csr2[0], csr2[1]))
    st.free(); g.free()


def test_upload_twice_and_empty_rows(gpu):
    # vertices without in-edges or out-edges at both ends of the id range
    n = 50
    s = np.array([10, 11, 12, 12, 30, 30, 30], np.int32)
    d = np.array([11, 12, 10, 10, 31, 30, 32], np.int32)
    g = Graph.from_edges(n, s, d)
    for rnd in range(2):
        csr = O.build_csr(n, s, d)
        g.upload_csr(csr[0], csr[1])
        st = State(g)
        st.synchronize()
        for got, exp in zip(g.csr(), csr):
            assert np.array_equal(got, exp)
        st.reset()
        st.run(2)
        assert np.array_equal(st.canonical_labels(), O.tarjan_canonical(csr[0], csr[1]))
        st.free()
        d = d[::-1].copy()                    # same m, other edges
    g.free()


def _check_upload(n, s, d):
    csr = O.build_csr(n, s, d)
    g = Graph.from_edges(n, np.zeros(csr[1].size, np.int32), np.zeros(csr[1].size, np.int32))
    g.upload_csr(csr[0], csr[1])                 # forward CSR only: the transpose is rebuilt
    st = State(g)
    st.synchronize()
    for got, exp in zip(g.csr(), csr):
        assert np.array_equal(got, exp)
    st.reset()
    st.run(2)
    assert np.array_equal(st.canonical_labels(), O.tarjan_canonical(csr[0], csr[1]))
    st.free(); g.free()


def test_pipelined_upload_random_multigraph(gpu):
    # above 4 M edges the CSR crosses the bus in chunks whose pairs are sorted
    # while the next chunk is in flight, then merged by one scatter
    n = 1000000
    s, d = random_graph(n, 6000000, 31)           # duplicates and self-loops kept
    _check_upload(n, s, d)


def test_pipelined_upload_hub_spanning_runs(gpu):
    # every vertex points at vertex 7, so its in-list is split over all runs
    # and must come back as one list sorted by source
    rng = np.random.default_rng(32)
    n = 600000
    s = np.concatenate([np.arange(n), rng.integers(0, n, 4000000)]).astype(np.int32)
    d = np.concatenate([np.full(n, 7), rng.integers(0, n, 4000000)]).astype(np.int32)
    _check_upload(n, s, d)


def test_pipelined_upload_giant_out_list_leaves_a_run_empty(gpu):
    # vertex 0 owns half of all edges: runs cut at whole source lists, so one
    # of the four runs is empty
    rng = np.random.default_rng(33)
    n = 300000
    s = np.concatenate([np.zeros(3000000), rng.integers(1, n, 3000000)]).astype(np.int32)
    d = rng.integers(0, n, 6000000).astype(np.int32)
    _check_upload(n, s, d)


def test_offsets_across_long_ranges_without_edges(gpu):
    # edges only among the first and the last 1,000 of 5,000,000 vertices: the
    # offsets of the 4,998,000 ids between them (and of the transpose) come
    # from the gap search, not from one thread walking the range
    rng = np.random.default_rng(34)
    n = 5000000
    ends = np.concatenate([np.arange(1000), np.arange(n - 1000, n)])
    s = ends[rng.integers(0, ends.size, 20000)].astype(np.int32)
    d = ends[rng.integers(0, ends.size, 20000)].astype(np.int32)
    csr = O.build_csr(n, s, d)
    g = Graph.from_edges(n, s, d)
    for got, exp in zip(g.csr(), csr):
        assert np.array_equal(got, exp)
    g.upload_csr(csr[0], csr[1])              # transpose rebuilt by the single sort
    State(g).synchronize()
    for got, exp in zip(g.csr(), csr):
        assert np.array_equal(got, exp)
    g.free()
