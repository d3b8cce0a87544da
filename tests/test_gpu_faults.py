"""GPU: failure paths, injected on the host (no test faults, traps or hangs the
GPU).  An allocation that fails inside an update or a pipelined CSR upload
returns SCC_ERR_OOM and leaves the graph as it was; a bounded device wait that runs out (the drain is handed a
queue slot nobody fills) returns SCC_ERR_TIMEOUT, and the state decomposes
correctly again after a reset."""
import numpy as np
import pytest

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, SccError, State, capi
from tests.helpers import random_graph, seeded_graph
from tests.test_gpu_update import apply_batch

pytestmark = pytest.mark.gpu

SCC_ERR_OOM, SCC_ERR_TIMEOUT = 3, 4
SCC_INJECT_ALLOC, SCC_INJECT_WAIT = 1, 2


def test_update_allocation_failure_leaves_graph_intact(gpu):
    n = 3000
    s, d = random_graph(n, 6000, 7)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    st.run(2)
    before = [a.copy() for a in g.csr()]
    lab_before = st.canonical_labels()
    rng = np.random.default_rng(1)
    ins = (rng.integers(0, n, 200).astype(np.int32), rng.integers(0, n, 200).astype(np.int32))
    capi.call("scc_debug_inject", SCC_INJECT_ALLOC, 1)          # the next scratch allocation fails
    try:
        with pytest.raises(SccError) as ei:
            st.update_batch(*ins, s[:50], d[:50])
        assert ei.value.status == SCC_ERR_OOM
    finally:
        capi.call("scc_debug_inject", SCC_INJECT_ALLOC, 0)
    for a, b in zip(g.csr(), before):
        assert np.array_equal(a, b)
    assert np.array_equal(st.canonical_labels(), lab_before)
    st.update_batch(*ins, s[:50], d[:50])                        # the same batch now goes through
    s2, d2 = apply_batch(s, d, *ins, s[:50], d[:50])
    csr = O.build_csr(n, s2, d2)
    assert np.array_equal(st.canonical_labels(), O.tarjan_canonical(csr[0], csr[1]))
    st.free(); g.free()


def test_drain_wait_limit_reports_timeout_and_recovers(gpu):
    # a long cycle plus a grid: the traversal narrows and the asynchronous drain runs
    n, s, d, csr = seeded_graph(rmat_scale=10, edge_factor=4, grid_side=64, num_cycles=4, cycle_min=500,
                                cycle_max=1000, seed=3)
    g = Graph.from_edges(n, s, d)
    st = State(g)
    capi.call("scc_debug_inject", SCC_INJECT_WAIT, 1)
    try:
        with pytest.raises(SccError) as ei:
            st.reset()
            st.run(2)
        assert ei.value.status == SCC_ERR_TIMEOUT
    finally:
        capi.call("scc_debug_inject", SCC_INJECT_WAIT, 0)
    st.reset()
    st.run(2)
    assert np.array_equal(st.canonical_labels(), O.tarjan_canonical(csr[0], csr[1]))
    st.free(); g.free()


@pytest.mark.parametrize("countdown", [1, 3, 5])
def test_pipelined_upload_allocation_failure(gpu, countdown):
    # above 4 M edges the CSR-only upload sorts chunks on a helper stream; an
    # allocation failing at any of its five scratch buffers returns SCC_ERR_OOM
    # before any copy, leaves the graph as it was, and a retry is exact
    n = 800000
    s1, d1 = random_graph(n, 5000000, 41)
    s2, d2 = random_graph(n, 5000000, 42)
    csr1, csr2 = O.build_csr(n, s1, d1), O.build_csr(n, s2, d2)
    g = Graph.from_edges(n, s1, d1)
    capi.call("scc_debug_inject", SCC_INJECT_ALLOC, countdown)
    try:
        with pytest.raises(SccError) as ei:
            g.upload_csr(csr2[0], csr2[1])
        assert ei.value.status == SCC_ERR_OOM
    finally:
        capi.call("scc_debug_inject", SCC_INJECT_ALLOC, 0)
    for got, exp in zip(g.csr(), csr1):
        assert np.array_equal(got, exp)
    g.upload_csr(csr2[0], csr2[1])
    st = State(g)
    st.synchronize()
    for got, exp in zip(g.csr(), csr2):
        assert np.array_equal(got, exp)
    st.run(2)
    assert np.array_equal(st.canonical_labels(), O.tarjan_canonical(csr2[0], csr2[1]))
    st.free(); g.free()
