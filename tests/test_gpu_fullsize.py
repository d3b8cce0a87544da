"""GPU: the benchmark configurations at their full sizes (hundreds of millions
of edges).  The labels must equal the oracle's Tarjan on the same CSR (read
back from the device), and two size-independent properties must hold: a graph
and its transpose have the same SCCs, and the SCC count is the number of
vertices that label themselves."""
import numpy as np
import pytest

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, State

pytestmark = pytest.mark.gpu

FULL = {
    "R-MAT s24 ef16 U 4096x4096 oriented grid": dict(rmat_scale=24, edge_factor=16, grid_side=4096, seed=2024),
    "R-MAT s24 ef16 + 1,000 planted cycles": dict(rmat_scale=24, edge_factor=16, num_cycles=1000, cycle_min=3,
                                                  cycle_max=100000, seed=2024),
}


@pytest.mark.parametrize("name", sorted(FULL))
def test_full_size_equals_tarjan_and_transpose(gpu, name):
    g = Graph.generate(**FULL[name])
    st = State(g)
    stats = st.run(2)
    lab = st.canonical_labels()
    st.free()
    b, a, rb, ra = g.csr()
    g.free()
    assert np.array_equal(lab, O.tarjan_canonical(b, a)), name
    assert stats["num_sccs"] == int(np.count_nonzero(lab == np.arange(lab.size, dtype=np.int32)))
    gt = Graph.from_csr(rb, ra, b, a)          # the transpose: same strongly connected components
    del b, a, rb, ra
    stt = State(gt)
    stt.run(2)
    assert np.array_equal(stt.canonical_labels(), lab), name
    stt.free(); gt.free()
