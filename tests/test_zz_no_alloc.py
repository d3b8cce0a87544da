"""GPU: the allocation-free Trim1 entry point, scc_trim1_noalloc, called through
the C ABI, gives the same colours, SCC representatives and trimmed count as
scc_do_global_trim1 on the same input -- twice in a row, because every call
reuses the same file-scope scratch array and must not depend on what the
previous call left there.

It exists for callers that cannot call cudaMalloc (a serving process whose
device-memory budget is fixed at start-up and must not fail on an allocation
mid-request, or a host that lends the library a fixed pool).  Integer work:
the comparison is exact.  Kept in its own file, collected last."""
import ctypes as C

import numpy as np
import pytest

from dynamicgraphs_scc_b200 import Graph, State, capi
from tests.helpers import random_graph, seeded_graph

pytestmark = pytest.mark.gpu


def _device_ptrs(graph, state):
    b, a, rb, ra = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    capi.call("scc_graph_device_csr", graph.handle, C.byref(b), C.byref(a), C.byref(rb), C.byref(ra))
    col, scc = C.c_void_p(), C.c_void_p()
    capi.call("scc_state_device_arrays", state.handle, C.byref(col), C.byref(scc))
    return b, a, rb, ra, col, scc


def _check_once(n, s, d, color0):
    g = Graph.from_edges(n, s, d)
    # existing entry point
    ref = State(g)
    ref.set_color(color0)
    t_ref = ref.do_global_trim1()
    # allocation-free entry point on another state's device arrays
    st = State(g)
    st.set_color(color0)
    b, a, rb, ra, col, scc = _device_ptrs(g, st)
    t = C.c_int32(-1)
    capi.call("scc_trim1_noalloc", n, b, a, rb, ra, col, scc, C.byref(t), C.c_void_p(st.stream()))
    assert t.value == t_ref
    assert np.array_equal(st.color(), ref.color())
    assert np.array_equal(st.scc(), ref.scc())
    return t_ref


def test_noalloc_trim1_matches_existing_entry_point_twice(gpu):
    # call 1: an R-MAT + grid graph, every vertex colour -1
    n, s, d, _ = seeded_graph(rmat_scale=16, edge_factor=6, grid_side=128, seed=5)
    t1 = _check_once(n, s, d, np.full(n, -1, np.int32))
    assert t1 > 0
    # call 2: a different graph with mixed colours, reusing the same scratch
    n2 = 40000
    s2, d2 = random_graph(n2, 60000, 17)
    rng = np.random.default_rng(3)
    t2 = _check_once(n2, s2, d2, rng.integers(-1, 4, n2).astype(np.int32))
    assert t2 > 0


def test_noalloc_rejects_oversize(gpu):
    t = C.c_int32(0)
    L = capi.lib()
    rc = L.scc_trim1_noalloc((1 << 20) + 1, None, None, None, None, None, None, C.byref(t), None)
    assert rc == 1
    assert b"at most" in L.scc_last_error()
