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
