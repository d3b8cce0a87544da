"""GPU: the allocation-free Trim1 entry point, scc_trim1_noalloc, called through
the C ABI, gives the same colours, SCC representatives and trimmed count as
scc_do_global_trim1 and as the oracle's Trim1 fixpoint on the same input --
twice in a row, because every call reuses the same file-scope scratch array
and must not depend on what the previous call left there.

It exists for callers that cannot call cudaMalloc (a serving process whose
device-memory budget is fixed at start-up and must not fail on an allocation
mid-request, or a host that lends the library a fixed pool).  Under CUDA's lazy
module loading the scratch array is reserved on a device by the first call
there, so the test makes that call with n = 0 first, as such a caller does at
start-up, and then checks that a later call leaves the device's free memory
unchanged.  Integer work: every comparison is exact.  Kept in its own file,
collected last."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as O
from dynamicgraphs_scc_b200 import Graph, State, capi
from tests.helpers import random_graph, seeded_graph

pytestmark = pytest.mark.gpu


def _device_ptrs(graph, state):
    b, a, rb, ra = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    capi.call("scc_graph_device_csr", graph.handle, C.byref(b), C.byref(a), C.byref(rb), C.byref(ra))
    col, scc = C.c_void_p(), C.c_void_p()
    capi.call("scc_state_device_arrays", state.handle, C.byref(col), C.byref(scc))
    return b, a, rb, ra, col, scc


def _warm_up():
    t = C.c_int32(-1)
    capi.call("scc_trim1_noalloc", 0, None, None, None, None, None, None, C.byref(t), None)
    assert t.value == 0


def _overflow_graph():
    """A graph whose peel must take both overflow routes of the scanning sweep:
    a source hub of 600 out-edges (above the 512-edge limit of a thread's
    cascade, so its neighbours are re-checked by the overflow pass), and a
    vertex whose trim frees 12 children at once (more than the cascade's
    8-entry stack), each at the head of a 10-vertex chain.  Everything drains
    into a 5-vertex cycle, which stays."""
    src, dst = [], []
    z = list(range(5))                                    # the cycle that remains
    src += z; dst += z[1:] + z[:1]
    nxt = 5
    hub = nxt; nxt += 1
    us = list(range(nxt, nxt + 600)); nxt += 600
    for u in us:
        src.append(hub); dst.append(u)
    for u in us[1:]:
        src.append(u); dst.append(z[0])
    for _ in range(12):                                   # us[0] frees 12 children at once
        head = nxt; nxt += 1
        src.append(us[0]); dst.append(head)
        prev = head
        for _ in range(9):
            src.append(prev); dst.append(nxt); prev = nxt; nxt += 1
        src.append(prev); dst.append(z[1])
    n = nxt
    return n, np.asarray(src, np.int32), np.asarray(dst, np.int32)


def _check_once(n, s, d, color0, scc0=None, free_mem_check=False):
    g = Graph.from_edges(n, s, d)
    scc0 = np.full(n, -1, np.int32) if scc0 is None else scc0
    # the existing entry point
    ref = State(g)
    ref.set_color(color0); ref.set_scc(scc0)
    t_ref = ref.do_global_trim1()
    # the oracle's fixpoint
    csr = O.build_csr(n, s, d)
    oc, os_ = color0.copy(), scc0.copy()
    t_orc = O.trim1_fixpoint(csr, oc, os_)
    # the allocation-free entry point on another state's device arrays
    st = State(g)
    st.set_color(color0); st.set_scc(scc0)
    b, a, rb, ra, col, scc = _device_ptrs(g, st)
    t = C.c_int32(-1)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    capi.call("scc_trim1_noalloc", n, b, a, rb, ra, col, scc, C.byref(t), C.c_void_p(st.stream()))
    free1 = torch.cuda.mem_get_info()[0]
    if free_mem_check:
        assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
    assert t.value == t_ref == t_orc
    assert np.array_equal(st.color(), ref.color()) and np.array_equal(st.color(), oc)
    assert np.array_equal(st.scc(), ref.scc()) and np.array_equal(st.scc(), os_)
    st.free(); ref.free(); g.free()
    return t_ref


def test_noalloc_trim1_matches_existing_entry_point_twice(gpu):
    _warm_up()
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


def test_noalloc_overflow_paths_twice_without_allocating(gpu):
    _warm_up()
    n, s, d = _overflow_graph()
    color = np.full(n, -1, np.int32)
    t1 = _check_once(n, s, d, color)
    assert t1 == n - 5
    # the same peel again on the same scratch: free device memory must not move
    t2 = _check_once(n, s, d, color, free_mem_check=True)
    assert t2 == t1
    # within colours: the hub's side in colour 0, the chains in colour 1
    col = np.zeros(n, np.int32)
    col[606:] = 1
    t3 = _check_once(n, s, d, col, free_mem_check=True)
    assert t3 > 0


def test_noalloc_rejects_oversize(gpu):
    t = C.c_int32(0)
    L = capi.lib()
    rc = L.scc_trim1_noalloc((1 << 20) + 1, None, None, None, None, None, None, C.byref(t), None)
    assert rc == 1
    assert b"at most" in L.scc_last_error()
